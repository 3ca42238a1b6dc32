"""ctypes view of ``include/voxel_c.h`` (the backend's C ABI).

The library is the in-tree ``voxel_b200/lib/libvoxel_c.so``.  Loading fails
loudly when it has not been built: there is no Python or CPU stand-in.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "lib", "libvoxel_c.so")
DATAGEN_PATH = os.path.join(HERE, "lib", "libvoxel_datagen.so")
HEADER = os.path.join(ROOT, "include", "voxel_c.h")

F64, F32, I64, I32, U64, U32 = range(6)
EQ, NE, LT, LE, GT, GE, BETWEEN = range(7)

_lib = None
_datagen = None

vp = C.c_void_p
sz = C.c_size_t
u8, u32, u64, i16, i32, i64 = C.c_uint8, C.c_uint32, C.c_uint64, C.c_int16, C.c_int32, C.c_int64
dbl = C.c_double
P = C.POINTER

_SIGS = {
    "voxel_engine_create": (vp, [C.c_int]),
    "voxel_engine_create_f64": (vp, []),
    "voxel_engine_create_f32": (vp, []),
    "voxel_engine_create_i64": (vp, []),
    "voxel_engine_create_i32": (vp, []),
    "voxel_engine_create_u64": (vp, []),
    "voxel_engine_create_u32": (vp, []),
    "voxel_engine_destroy": (None, [vp]),
    "voxel_engine_destroy_i64": (None, [vp]),
    "voxel_engine_dtype": (C.c_int, [vp]),
    "voxel_engine_k_lanes": (sz, []),
    "voxel_engine_k_lanes_of": (sz, [vp]),
    "voxel_engine_add_segment": (sz, [vp, vp, sz]),
    "voxel_engine_add_segment_i64": (sz, [vp, vp, sz]),
    "voxel_engine_add_segment_f32": (sz, [vp, vp, sz]),
    "voxel_engine_add_segment_i32": (sz, [vp, vp, sz]),
    "voxel_engine_add_segment_u32": (sz, [vp, vp, sz]),
    "voxel_engine_add_segment_u64": (sz, [vp, vp, sz]),
    "voxel_engine_add_segment_device": (sz, [vp, vp, sz]),
    "voxel_engine_load_program": (None, [vp, vp, sz]),
    "voxel_engine_load_program_i64": (None, [vp, vp, sz]),
    "voxel_engine_run": (None, [vp]),
    "voxel_engine_run_i64": (None, [vp]),
    "voxel_engine_run_status": (C.c_int, [vp]),
    "voxel_engine_run_parallel": (None, [vp, sz, u32, u8]),
    "voxel_engine_run_parallel_status": (C.c_int, [vp, sz, u32, u8]),
    "voxel_engine_set_scalar": (None, [vp, sz, u64]),
    "voxel_engine_get_scalar": (u64, [vp, sz]),
    "voxel_engine_set_scalar_f64": (None, [vp, sz, dbl]),
    "voxel_engine_get_scalar_f64": (dbl, [vp, sz]),
    "voxel_engine_set_scalar_i64": (None, [vp, sz, u64]),
    "voxel_engine_get_scalar_i64": (u64, [vp, sz]),
    "voxel_engine_explain": (sz, [vp, C.c_char_p, sz]),
    "voxel_engine_reset": (None, [vp]),
    "voxel_engine_plan": (C.c_int, [vp]),
    "voxel_engine_last_device_ms": (dbl, [vp]),
    "voxel_jit_run": (dbl, [vp, sz, vp, sz, dbl]),
    "voxel_last_error": (C.c_char_p, []),
    "voxel_last_status": (C.c_int, []),
    "voxel_instr_vload": (u32, [u8, u8, u8, u8]),
    "voxel_instr_vfilter_gt": (u32, [u8, u8, u8]),
    "voxel_instr_vfilter_ge": (u32, [u8, u8, u8]),
    "voxel_instr_vfilter_lt": (u32, [u8, u8, u8]),
    "voxel_instr_vfilter_le": (u32, [u8, u8, u8]),
    "voxel_instr_vsum": (u32, [u8, u8]),
    "voxel_instr_vred_min": (u32, [u8, u8]),
    "voxel_instr_vred_max": (u32, [u8, u8]),
    "voxel_instr_vcount": (u32, [u8, u8]),
    "voxel_instr_addf": (u32, [u8, u8, u8]),
    "voxel_instr_add": (u32, [u8, u8, u8]),
    "voxel_instr_sub": (u32, [u8, u8, u8]),
    "voxel_instr_mul": (u32, [u8, u8, u8]),
    "voxel_instr_mov": (u32, [u8, i16]),
    "voxel_instr_movr": (u32, [u8, u8]),
    "voxel_instr_cmp": (u32, [u8, u8]),
    "voxel_instr_jnz": (u32, [i16]),
    "voxel_instr_jz": (u32, [i16]),
    "voxel_instr_jmp": (u32, [i16]),
    "voxel_instr_halt": (u32, []),
    "voxel_null_create": (vp, [sz]),
    "voxel_null_destroy": (None, [vp]),
    "voxel_null_is_null": (C.c_int, [vp, sz]),
    "voxel_null_set_null": (None, [vp, sz]),
    "voxel_null_set_valid": (None, [vp, sz]),
    "voxel_null_null_count": (sz, [vp]),
    "voxel_null_valid_count": (sz, [vp]),
    "voxel_agg_create": (vp, []),
    "voxel_agg_destroy": (None, [vp]),
    "voxel_agg_init": (None, [vp, sz]),
    "voxel_agg_accumulate": (None, [vp, vp, vp, sz]),
    "voxel_agg_group_count": (sz, [vp]),
    "voxel_sort_ascending": (None, [vp, sz, vp]),
    "voxel_sort_descending": (None, [vp, sz, vp]),
    "voxel_topk": (None, [vp, sz, sz, vp, C.c_int]),
    "voxel_dict_create": (vp, []),
    "voxel_dict_destroy": (None, [vp]),
    "voxel_dict_build": (None, [vp, vp, sz]),
    "voxel_dict_cardinality": (sz, [vp]),
    "voxel_dict_decode_batch": (None, [vp, vp, sz, sz]),
    "voxel_pool_create": (vp, [u32]),
    "voxel_pool_destroy": (None, [vp]),
    "voxel_pool_wait_all": (None, [vp]),
    "voxel_pool_thread_count": (sz, [vp]),
    "voxel_device_alloc": (vp, [sz]),
    "voxel_device_free": (None, [vp]),
    "voxel_copy_to_device": (C.c_int, [vp, vp, sz, vp]),
    "voxel_copy_to_host": (C.c_int, [vp, vp, sz, vp]),
    "voxel_stream_sync": (C.c_int, [vp]),
    "voxel_host_register": (C.c_int, [vp, sz]),
    "voxel_host_unregister": (C.c_int, [vp]),
    "voxel_vfilter": (sz, [C.c_int, C.c_int, vp, sz, u64, u64, vp]),
    "voxel_bitmap_and": (sz, [vp, sz, sz, vp]),
    "voxel_selection_from_bitmap": (sz, [vp, sz, vp]),
    "voxel_vfilter_dev": (C.c_int, [C.c_int, C.c_int, vp, sz, u64, u64, vp, vp, vp]),
    "voxel_selection_from_bitmap_dev": (C.c_int, [vp, sz, vp, vp, vp]),
    "voxel_bitpack_decode": (C.c_int, [vp, sz, u32, sz, sz, sz, vp]),
    "voxel_dict_bitpack_decode_i32": (C.c_int, [vp, sz, u32, vp, sz, sz, sz, sz, vp]),
    "voxel_dict_decode": (C.c_int, [C.c_int, vp, sz, vp, sz, sz, sz, vp]),
    "voxel_rle_decode_i64": (C.c_int, [vp, vp, sz, sz, sz, vp]),
    "voxel_jit_compile": (C.c_int, [vp, sz, C.POINTER(sz), C.c_char_p, sz]),
    "voxel_window": (sz, [C.c_int, C.c_int, vp, sz, vp, sz, C.c_uint8, dbl]),
    "voxel_window_dev": (C.c_int, [C.c_int, C.c_int, vp, sz, vp, sz, C.c_uint8, dbl, C.POINTER(sz), vp]),
    "voxel_time_window_sum": (sz, [C.c_int, vp, vp, sz, i64, i64, vp, sz]),
    "voxel_time_window_sum_dev": (C.c_int, [C.c_int, vp, vp, sz, i64, i64, vp, sz, C.POINTER(sz), vp]),
    "voxel_merge_join": (sz, [C.c_int, vp, sz, vp, sz, vp, vp, sz, C.c_int]),
    "voxel_join_pairs_swap_order_dev": (C.c_int, [vp, vp, sz, vp, vp, vp]),
    "voxel_groupby_u32_f64_dev": (C.c_int, [vp, vp, sz, sz, C.c_int, vp, vp, vp, vp, vp, C.POINTER(u64), vp]),
    "voxel_merge_join_dev": (C.c_int, [C.c_int, vp, sz, vp, sz, vp, vp, sz, C.c_int, vp, vp]),
    "voxel_semi_join": (sz, [C.c_int, vp, sz, vp, sz, vp, C.c_int]),
    "voxel_semi_join_dev": (C.c_int, [C.c_int, vp, sz, vp, sz, vp, C.c_int, vp, vp]),
    "voxel_delta_decode": (C.c_int, [C.c_int, vp, sz, u64, sz, sz, vp]),
    "voxel_delta_decode_dev": (C.c_int, [C.c_int, vp, sz, u64, sz, sz, vp, vp]),
    "voxel_delta_encode": (C.c_int, [C.c_int, vp, sz, vp]),
    "voxel_delta_encode_dev": (C.c_int, [C.c_int, vp, sz, vp, vp]),
    "voxel_for_decode_f64": (C.c_int, [vp, sz, dbl, dbl, sz, sz, vp]),
    "voxel_for_decode_f64_dev": (C.c_int, [vp, sz, dbl, dbl, sz, sz, vp, vp]),
    "voxel_for_encode_f64": (C.c_int, [vp, sz, vp, C.POINTER(dbl), C.POINTER(dbl)]),
    "voxel_for_encode_f64_dev": (C.c_int, [vp, sz, vp, C.POINTER(dbl), C.POINTER(dbl), vp]),
    "voxel_bitpack_decode_dev": (C.c_int, [vp, sz, u32, sz, sz, sz, vp, vp]),
    "voxel_rle_decode_i64_dev": (C.c_int, [vp, vp, sz, sz, sz, vp, vp]),
    "voxel_dict_bitpack_decode_i32_dev": (C.c_int, [vp, sz, u32, vp, sz, sz, sz, sz, vp, vp]),
    "voxel_dict_decode_dev": (C.c_int, [C.c_int, vp, sz, vp, sz, vp, vp]),
    "voxel_bitmap_and_dev": (C.c_int, [vp, sz, sz, vp, vp, vp]),
    "voxel_scan_groupby": (sz, [vp, sz, u32, vp, sz, vp, vp, sz, dbl, i32, i32, vp, vp, vp, vp, vp]),
    "voxel_scan_groupby_dev": (C.c_int, [vp, sz, u32, vp, sz, vp, vp, sz, dbl, i32, i32,
                                          vp, vp, vp, vp, vp, vp, vp]),
    "voxel_scan_groupby_noalloc_dev": (C.c_int, [vp, sz, u32, vp, sz, vp, vp, sz, dbl, i32, i32,
                                                  vp, vp, vp, vp, vp, vp, vp, vp]),
    "voxel_groupby_i32_f64": (sz, [vp, vp, sz, sz, vp, vp, vp, vp, vp]),
    "voxel_groupby_u32_f64": (sz, [vp, vp, sz, sz, vp, vp, vp, vp, vp]),
    "voxel_grouped_sorted_i32_f64": (sz, [vp, vp, sz, vp, vp, vp, vp, vp]),
    "voxel_radix_sort": (C.c_int, [C.c_int, vp, vp, sz]),
    "voxel_radix_sort_dev": (C.c_int, [C.c_int, vp, vp, sz, vp, sz, vp]),
    "voxel_radix_sort_tmp_bytes": (sz, [C.c_int, sz]),
    "voxel_scan_groupby_tune": (C.c_int, [C.c_int]),
    "voxel_scan_groupby_last_variant": (C.c_int, []),
    "voxel_scan_groupby_tune_state": (C.c_int, []),
    "voxel_scan_groupby_check": (C.c_int, [C.c_void_p]),
    "voxel_scan_groupby_status_code": (C.c_int, [C.c_int]),
    "voxel_agg_accumulate_dev": (C.c_int, [vp, vp, vp, sz, vp]),
    "voxel_agg_results": (sz, [vp, vp, vp, vp, vp, vp]),
    "voxel_dict_values": (sz, [vp, vp]),
    "voxel_batch_create": (vp, []),
    "voxel_batch_destroy": (None, [vp]),
    "voxel_batch_size": (sz, [vp]),
    "voxel_batch_add": (C.c_int, [vp, C.c_int, vp, sz, vp, vp, sz, C.c_int, sz, vp]),
    "voxel_batch_set_capacity": (C.c_int, [vp, sz, sz, vp]),
    "voxel_batch_launch": (C.c_int, [vp, C.c_int, vp]),
    "voxel_batch_fetch": (C.c_int, [vp, vp]),
    "voxel_batch_result": (C.c_int, [vp, sz, vp, vp, vp]),
    "voxel_batch_results_all": (C.c_int, [vp, vp, vp, vp]),
    "voxel_batch_form": (C.c_int, [vp, sz]),
    "voxel_tune_enable": (None, [C.c_int]),
    "voxel_tune_set_cache_path": (None, [C.c_char_p]),
    "voxel_tune_clear": (None, []),
    "voxel_tune_lookup": (C.c_int, [C.c_char_p, C.c_int, sz]),
    "voxel_batch_rerun": (C.c_int, [vp, sz, vp, vp, vp, vp]),
    "voxel_batch_gather_overflow": (C.c_int, [vp, sz, vp, vp, vp]),
    "voxel_batch_set_spill_capacity": (C.c_int, [vp, sz]),
    "voxel_server_create": (vp, [sz, u32]),
    "voxel_server_destroy": (None, [vp]),
    "voxel_server_submit_program": (u64, [vp, C.c_int, vp, sz, vp, vp, sz, C.c_int, sz, vp]),
    "voxel_server_submit_groupby": (u64, [vp, vp, vp, sz, sz, sz, vp, vp, vp, vp, vp]),
    "voxel_server_submit_join": (u64, [vp, vp, vp, sz, vp, sz, vp, vp, sz]),
    "voxel_server_wait": (C.c_int, [vp, u64, dbl]),
    "voxel_server_result": (C.c_int, [vp, u64, vp, vp, vp, vp]),
    "voxel_server_stats": (C.c_int, [vp, vp, vp, vp, vp, vp]),
    "voxel_server_reset_stats": (None, [vp]),
    "voxel_server_breakdown": (C.c_int, [vp, C.c_int, vp, vp, vp]),
    "voxel_server_batch_stats": (C.c_int, [vp, vp, vp, vp, vp, vp, vp]),
    "voxel_hashjoin_i64": (sz, [vp, sz, vp, sz, vp, vp, sz, C.c_int]),
    "voxel_hashjoin_i64_dev": (C.c_int, [vp, vp, sz, vp, sz, vp, vp, sz, C.c_int, vp, vp]),
}


def header_symbols() -> list[str]:
    """Every function name declared in include/voxel_c.h."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(voxel_[a-z0-9_]+)\s*\(", text)))


def lib() -> C.CDLL:
    """The loaded backend library (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"voxel_b200 native library not built ({LIB_PATH}); run __graft_entry__.build()")
        _lib = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(_lib, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
    return _lib


def datagen() -> C.CDLL:
    global _datagen
    if _datagen is None:
        _datagen = C.CDLL(DATAGEN_PATH)
        _datagen.vgen_uniform_f64_mt.restype = None
        _datagen.vgen_uniform_f64_mt.argtypes = [u64, sz, dbl, dbl, vp]
        _datagen.vgen_splitmix64.restype = None
        _datagen.vgen_splitmix64.argtypes = [u64, sz, vp]
        _datagen.vgen_join_probe_i64.restype = None
        _datagen.vgen_join_probe_i64.argtypes = [u64, vp, sz, dbl, dbl, sz, vp, C.c_uint]
    return _datagen


def last_error() -> str:
    msg = lib().voxel_last_error()
    return msg.decode() if msg else ""


def ptr(a) -> int:
    """Address of a numpy array (or 0 for None)."""
    if a is None:
        return 0
    return a.ctypes.data
