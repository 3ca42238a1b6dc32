"""Serving loop (Python side): a thin handle over the `voxel_server_*` C ABI.

The scheduling itself (arrival queues, admission by device working memory,
continuous batching of programs, concurrent group-by / join execution,
latency percentiles) is in `csrc/serve.cpp`.  This wrapper keeps the host
output arrays of group-by requests alive until their results are read.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi


class ServerError(RuntimeError):
    pass


class Server:
    def __init__(self, budget_bytes: int = 8 << 30, max_batch: int = 4096):
        self.L = capi.lib()
        self.h = self.L.voxel_server_create(budget_bytes, max_batch)
        if not self.h:
            raise ServerError(capi.last_error())
        self._host = {}
        self._outbufs = {}

    def close(self):
        if self.h:
            self.L.voxel_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _check(rid):
        if not rid:
            raise ServerError(capi.last_error())
        return rid

    def prepare_program(self, prog, dcol, n: int | None = None, want_selection: bool = False, capacity: int = 0,
                        dsel=None) -> tuple:
        """The submission arguments of a program over a device column, built
        once (a prepared statement): `submit_prepared` then costs one C call."""
        n = dcol.numel() if n is None else n
        regs = np.array(prog.registers(n), np.uint64)
        code = np.asarray(prog.code, np.uint32)
        return (prog.dtype, code, regs, dcol.data_ptr(), n, int(want_selection), capacity,
                dsel.data_ptr() if dsel is not None else None)

    def submit_prepared(self, p: tuple) -> int:
        dtype, code, regs, col, n, want, cap, sel = p
        return self._check(self.L.voxel_server_submit_program(self.h, dtype, code.ctypes.data, code.size,
                                                              regs.ctypes.data, col, n, want, cap, sel))

    def submit_program(self, prog, dcol, n: int | None = None, want_selection: bool = False, capacity: int = 0,
                       dsel=None) -> int:
        return self.submit_prepared(self.prepare_program(prog, dcol, n, want_selection, capacity, dsel))

    # group-by outputs go to host buffers reused across requests: a fresh
    # array faults its pages in during the device-to-host copy, which then
    # runs at a fraction of the link rate
    def _take_outputs(self, cap: int) -> dict:
        cls = 1 << max(cap - 1, 0).bit_length()
        free = self._outbufs.setdefault(cls, [])
        if free:
            return free.pop()
        out = dict(keys=np.ones(cls, np.uint32), sum=np.ones(cls), min=np.ones(cls), max=np.ones(cls),
                   count=np.ones(cls, np.uint64))  # written once here, so every page is resident
        out["_cls"] = cls
        return out

    def submit_groupby(self, dkeys, dvals, expected_groups: int, capacity: int | None = None) -> int:
        cap = capacity if capacity is not None else max(expected_groups, 1)
        out = self._take_outputs(cap)
        rid = self.L.voxel_server_submit_groupby(self.h, dkeys.data_ptr(), dvals.data_ptr(), dkeys.numel(),
                                                 expected_groups, cap, out["keys"].ctypes.data,
                                                 out["sum"].ctypes.data, out["min"].ctypes.data,
                                                 out["max"].ctypes.data, out["count"].ctypes.data)
        if not rid:
            self._outbufs[out["_cls"]].append(out)
        self._check(rid)
        self._host[rid] = out
        return rid

    def submit_join(self, dbuild, dpayload, dprobe, dleft, dright, capacity: int) -> int:
        rid = self.L.voxel_server_submit_join(self.h, dbuild.data_ptr(),
                                              dpayload.data_ptr() if dpayload is not None else None,
                                              dbuild.numel(), dprobe.data_ptr(), dprobe.numel(), dleft.data_ptr(),
                                              dright.data_ptr(), capacity)
        return self._check(rid)

    def wait(self, rid: int, timeout_s: float = 60.0) -> None:
        st = self.L.voxel_server_wait(self.h, rid, timeout_s)
        if st:
            raise ServerError(capi.last_error())

    def result(self, rid: int) -> dict:
        """Waits for the request and returns its outputs (the request is then forgotten)."""
        try:
            return self._result(rid)
        finally:  # a group-by's host buffers go back to the pool, also after an error
            host = self._host.pop(rid, None)
            if host is not None:
                self._outbufs[host["_cls"]].append(host)

    def _result(self, rid: int) -> dict:
        self.wait(rid)
        regs = np.zeros(64, np.uint64)
        cnt = np.zeros(1, np.uint64)
        aux = np.zeros(1, np.uint64)
        lat = C.c_double(0)
        st = self.L.voxel_server_result(self.h, rid, regs.ctypes.data, cnt.ctypes.data, aux.ctypes.data,
                                        C.byref(lat))
        if st:
            raise ServerError(capi.last_error())
        r = {"registers": [int(x) for x in regs], "count": int(cnt[0]), "aux": int(aux[0]),
             "latency_ms": lat.value}
        host = self._host.get(rid)
        if host is not None:  # group-by: `count` becomes the per-group counts
            g = r["count"]
            r["groups"] = g
            r.update({k: v[:g].copy() for k, v in host.items() if k != "_cls"})
        return r

    def stats(self) -> dict:
        n = C.c_uint64(0)
        p50, p99, mean = C.c_double(0), C.c_double(0), C.c_double(0)
        peak = C.c_uint64(0)
        self.L.voxel_server_stats(self.h, C.byref(n), C.byref(p50), C.byref(p99), C.byref(mean), C.byref(peak))
        return {"completed": n.value, "p50_ms": p50.value, "p99_ms": p99.value, "mean_ms": mean.value,
                "peak_reserved_bytes": peak.value}

    def breakdown(self) -> dict:
        """Mean queue and service milliseconds per request kind."""
        out = {}
        for k, name in enumerate(("program", "groupby", "join")):
            q, sv, n = C.c_double(0), C.c_double(0), C.c_uint64(0)
            if self.L.voxel_server_breakdown(self.h, k, C.byref(q), C.byref(sv), C.byref(n)):
                raise ServerError(capi.last_error())
            if n.value:
                out[name] = {"queue_ms": q.value, "service_ms": sv.value, "n": n.value}
        return out

    def batch_stats(self) -> dict:
        """Program batches: count, programs, largest, host build / wait ms."""
        b, p, m = C.c_uint64(0), C.c_uint64(0), C.c_uint64(0)
        bm, mb, wm = C.c_double(0), C.c_double(0), C.c_double(0)
        self.L.voxel_server_batch_stats(self.h, C.byref(b), C.byref(p), C.byref(m), C.byref(bm), C.byref(mb),
                                        C.byref(wm))
        return {"batches": b.value, "programs": p.value, "max_batch": m.value, "build_ms": bm.value,
                "max_build_ms": mb.value, "wait_ms": wm.value}

    def reset_stats(self) -> None:
        self.L.voxel_server_reset_stats(self.h)
