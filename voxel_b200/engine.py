"""Python view of the backend's Engine (the voxel_engine_* C ABI)."""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np

from . import capi

_DT = {np.dtype(np.float64): capi.F64, np.dtype(np.float32): capi.F32, np.dtype(np.int64): capi.I64,
       np.dtype(np.int32): capi.I32, np.dtype(np.uint64): capi.U64, np.dtype(np.uint32): capi.U32}
NP_OF = {v: k for k, v in _DT.items()}


class VoxelError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"voxel status {status}: {msg}")
        self.status = status


def f64_bits(x: float) -> int:
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def bits_f64(b: int) -> float:
    return struct.unpack("<d", struct.pack("<Q", b & 0xFFFFFFFFFFFFFFFF))[0]


class Engine:
    """One engine over columns of one element type (reference Engine<T>)."""

    def __init__(self, dtype):
        self.dtype = _DT[np.dtype(dtype)] if not isinstance(dtype, int) else dtype
        self._lib = capi.lib()
        self._h = self._lib.voxel_engine_create(self.dtype)
        self._keep = []

    def __del__(self):
        try:
            if self._h:
                self._lib.voxel_engine_destroy(self._h)
        except Exception:
            pass

    @property
    def k_lanes(self) -> int:
        return self._lib.voxel_engine_k_lanes_of(self._h)

    def add_segment(self, arr: np.ndarray) -> int:
        arr = np.ascontiguousarray(arr, dtype=NP_OF[self.dtype])
        self._keep.append(arr)
        return self._lib.voxel_engine_add_segment(self._h, arr.ctypes.data, arr.size)

    def add_segment_device(self, dptr: int, count: int) -> int:
        return self._lib.voxel_engine_add_segment_device(self._h, dptr, count)

    def load_program(self, code) -> None:
        a = np.asarray(code, dtype=np.uint32)
        self._lib.voxel_engine_load_program(self._h, a.ctypes.data, a.size)

    def run(self) -> None:
        st = self._lib.voxel_engine_run_status(self._h)
        if st:
            raise VoxelError(st, capi.last_error())

    def run_parallel(self, seg_id: int, threads: int = 0, result_reg: int = 0) -> None:
        st = self._lib.voxel_engine_run_parallel_status(self._h, seg_id, threads, result_reg)
        if st:
            raise VoxelError(st, capi.last_error())

    def get_scalar(self, r: int) -> int:
        return self._lib.voxel_engine_get_scalar(self._h, r)

    def set_scalar(self, r: int, v: int) -> None:
        self._lib.voxel_engine_set_scalar(self._h, r, v & 0xFFFFFFFFFFFFFFFF)

    def get_scalar_f64(self, r: int) -> float:
        return self._lib.voxel_engine_get_scalar_f64(self._h, r)

    def set_scalar_f64(self, r: int, v: float) -> None:
        self._lib.voxel_engine_set_scalar_f64(self._h, r, v)

    def registers(self, n: int = 64) -> list[int]:
        return [self.get_scalar(i) for i in range(n)]

    def explain(self) -> str:
        n = self._lib.voxel_engine_explain(self._h, None, 0)
        buf = C.create_string_buffer(n + 1)
        self._lib.voxel_engine_explain(self._h, buf, n + 1)
        return buf.value.decode()

    def last_device_ms(self) -> float:
        return self._lib.voxel_engine_last_device_ms(self._h)
