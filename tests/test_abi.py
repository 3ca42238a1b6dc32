"""C ABI checks that need no GPU: the library loads, exports every symbol the
header declares, the instruction encoders match the reference's builders, and
the host lowering produces the expected schedules (or rejects programs)."""
import ctypes as C
import os

import numpy as np
import pytest

from voxel_b200 import bytecode as bc
from voxel_b200 import capi
from voxel_b200 import templates as T
from voxel_b200.engine import Engine

REFERENCE_SYMBOLS = """
voxel_engine_create_f64 voxel_engine_destroy voxel_engine_add_segment voxel_engine_load_program
voxel_engine_run voxel_engine_run_parallel voxel_engine_set_scalar voxel_engine_get_scalar
voxel_engine_set_scalar_f64 voxel_engine_get_scalar_f64 voxel_engine_k_lanes voxel_engine_create_i64
voxel_engine_destroy_i64 voxel_engine_add_segment_i64 voxel_engine_load_program_i64 voxel_engine_run_i64
voxel_engine_set_scalar_i64 voxel_engine_get_scalar_i64 voxel_jit_run voxel_instr_vload voxel_instr_vfilter_gt
voxel_instr_vfilter_ge voxel_instr_vfilter_lt voxel_instr_vfilter_le voxel_instr_vsum voxel_instr_vred_min
voxel_instr_vred_max voxel_instr_vcount voxel_instr_addf voxel_instr_add voxel_instr_sub voxel_instr_mul
voxel_instr_mov voxel_instr_movr voxel_instr_cmp voxel_instr_jnz voxel_instr_jz voxel_instr_jmp voxel_instr_halt
voxel_null_create voxel_null_destroy voxel_null_is_null voxel_null_set_null voxel_null_set_valid
voxel_null_null_count voxel_null_valid_count voxel_agg_create voxel_agg_destroy voxel_agg_init
voxel_agg_accumulate voxel_agg_group_count voxel_sort_ascending voxel_sort_descending voxel_topk
voxel_dict_create voxel_dict_destroy voxel_dict_build voxel_dict_cardinality voxel_dict_decode_batch
voxel_pool_create voxel_pool_destroy voxel_pool_wait_all voxel_pool_thread_count voxel_last_error
""".split()


def test_library_exports_every_header_symbol(lib):
    declared = capi.header_symbols()
    assert set(REFERENCE_SYMBOLS) <= set(declared)
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing


def test_instruction_encoders_match_reference_builders(lib):
    assert lib.voxel_instr_vload(0, 1, 2, 0) == bc.vload(0, 1, 2)
    assert lib.voxel_instr_vfilter_gt(1, 0, 3) == bc.vfilter_gt(1, 0, 3)
    assert lib.voxel_instr_vsum(5, 1) == bc.vsum(5, 1)
    assert lib.voxel_instr_addf(0, 0, 5) == bc.addf(0, 0, 5)
    assert lib.voxel_instr_add(1, 1, 4) == bc.add(1, 1, 4)
    assert lib.voxel_instr_cmp(1, 2) == bc.cmp(1, 2)
    assert lib.voxel_instr_jnz(-6) == bc.jnz(-6)
    assert lib.voxel_instr_halt() == bc.halt()
    assert lib.voxel_instr_mov(4, -3) == bc.mov(4, -3)
    assert lib.voxel_engine_k_lanes() == 4
    # 32-bit layout [op:8][rd:4][ra:4][rb:4][imm:12] (instruction.hpp:65-72)
    assert bc.vload(0, 1, 0) == 0x00001070


def test_host_objects(lib):
    nb = lib.voxel_null_create(64)
    for r in (10, 20, 30):
        lib.voxel_null_set_null(nb, r)
    assert lib.voxel_null_null_count(nb) == 3 and lib.voxel_null_valid_count(nb) == 61
    assert lib.voxel_null_is_null(nb, 20) == 1 and lib.voxel_null_is_null(nb, 21) == 0
    lib.voxel_null_set_valid(nb, 20)
    assert lib.voxel_null_null_count(nb) == 2
    lib.voxel_null_destroy(nb)
    p = lib.voxel_pool_create(3)
    assert lib.voxel_pool_thread_count(p) == 3
    lib.voxel_pool_wait_all(p)
    lib.voxel_pool_destroy(p)


def plan(dtype, code, arrays, regs):
    e = Engine(dtype)
    for a in arrays:
        e.add_segment(a)
    for i, v in enumerate(regs):
        e.set_scalar(i, v)
    e.load_program(code)
    st = capi.lib().voxel_engine_plan(e._h)
    return st, e.explain()


def test_plan_fast_path():
    x = np.zeros(1003)
    st, s = plan(0, bc.filter_sum_program(), [x], [0, 0, 1003, T.reg_image(0, 500.0), 4])
    assert st == 0
    assert s.startswith("fast") and "groups=250" in s  # 1003 rows: 250 whole groups, tail dropped


def test_plan_count_loop():
    x = np.zeros(1000)
    st, s = plan(0, bc.filter_sum_count_program(), [x], [0, 0, 1000, T.reg_image(0, 500.0), 4, 0, 0])
    assert st == 0 and s.startswith("loop") and "groups=250" in s
    assert "r0=sum/addf" in s and "r1=count/add" in s
    assert "kernel=fsum" in s  # SUM + COUNT of one compare: the fused filter+sum kernel with its count


def test_plan_multi_aggregate_templates():
    """One predicate set with 2-4 aggregates plans onto the multi-reduction
    range kernel for every element type; one aggregate stays on the
    single-reduction kernels."""
    rng = np.random.default_rng(4)
    for dt in range(6):
        for aggs in (["SUM", "COUNT"], ["SUM", "COUNT", "MIN", "MAX"], ["MIN", "MAX"]):
            base = T.random_program(dt, rng, npreds=int(rng.integers(1, 5)))
            prog = T.build_multi(dt, base.preds, aggs)
            st, s = plan(dt, prog.code, [T.make_column(dt, 64, rng)], prog.registers(64))
            assert st == 0 and "kernel=mrange" in s, (dt, aggs, s)
        prog = T.build_multi(dt, base.preds, ["MAX"])
        st, s = plan(dt, prog.code, [T.make_column(dt, 64, rng)], prog.registers(64))
        assert st == 0 and "kernel=range" in s, s


def test_plan_templates_all_types():
    rng = np.random.default_rng(3)
    for dt in range(6):
        for agg in T.AGGS:
            prog = T.random_program(dt, rng, npreds=4, agg=agg)
            col = T.make_column(dt, 64, rng)
            st, s = plan(dt, prog.code, [col], prog.registers(64))
            assert st == 0, (dt, agg, capi.last_error())
            assert f"groups={64 // T.K_LANES[dt]}" in s


def test_plan_rejects_nonterminating_loop():
    # total not a multiple of kLanes: CMP/JNZ never sees equality (the reference spins)
    code = [bc.mov(7, 1)] + bc.filter_sum_program()  # MOV first defeats the fast-path match
    code[-2] = bc.jnz(-6)
    x = np.zeros(10)
    st, _ = plan(0, code, [x], [0, 0, 10, T.reg_image(0, 1.0), 4])
    assert st == 3  # VOXEL_ENONTERMINATING
    assert "never reaches" in capi.last_error()


def test_plan_rejects_unsupported_shape():
    # vector register carried across iterations (VADD accumulation) is not lowered
    code = [bc.vload(0, 1, 0), bc.enc(0x80, 6, 6, 0), bc.add(1, 1, 4), bc.cmp(1, 2), bc.jnz(-4), bc.halt()]
    st, _ = plan(0, code, [np.zeros(8)], [0, 0, 8, 0, 4])
    assert st == 2  # VOXEL_EUNSUPPORTED


def test_reference_c_example_builds_against_this_library(tmp_path):
    """The reference's own C example (examples/c_test.cpp) compiles and links
    against include/ + libvoxel_c.so with no source change (its
    "bindings/voxel_c.h" include resolves to the forwarding header)."""
    import shutil
    import subprocess

    from oracle import build_oracle

    src = os.path.join(build_oracle.reference_root(), "examples", "c_test.cpp")
    if not os.path.exists(src) or shutil.which("g++") is None:
        pytest.skip("reference sources not present")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib = os.path.join(root, "voxel_b200", "lib")
    out = tmp_path / "c_test"
    r = subprocess.run(["g++", "-std=c++17", src, "-I", os.path.join(root, "include"), "-L", lib, "-lvoxel_c",
                        f"-Wl,-rpath,{lib}", "-o", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_tune_cache_file_round_trip(lib, tmp_path):
    """The autotuner's cache is a JSON object of "<gpu>|<family>|<dtype>|<log2
    n>": choice entries; lookups read it, a malformed file reads as empty, and
    clear() writes an empty object.  Without a GPU the device name is
    "unknown"."""
    import json

    import torch

    if torch.cuda.is_available():
        pytest.skip("keys carry the device name when a GPU is present")
    path = tmp_path / "tune.json"
    path.write_text(json.dumps({"unknown|radix_onesweep|2|20": 1, "unknown|scan_groupby_card10|9|25": 3}))
    try:
        lib.voxel_tune_set_cache_path(str(path).encode())
        assert lib.voxel_tune_lookup(b"radix_onesweep", 2, 1 << 20) == 1
        assert lib.voxel_tune_lookup(b"radix_onesweep", 2, (1 << 21) - 1) == 1  # same log2 bucket
        assert lib.voxel_tune_lookup(b"radix_onesweep", 2, 1 << 21) == -1
        assert lib.voxel_tune_lookup(b"radix_onesweep", 3, 1 << 20) == -1
        assert lib.voxel_tune_lookup(b"scan_groupby_card10", 9, 1 << 25) == 3
        path.write_text('{"unknown|radix_onesweep|2|20": , garbage')
        lib.voxel_tune_set_cache_path(str(path).encode())
        assert lib.voxel_tune_lookup(b"radix_onesweep", 2, 1 << 20) == -1
        lib.voxel_tune_clear()
        assert json.loads(path.read_text()) == {}
    finally:
        lib.voxel_tune_set_cache_path(None)


def test_scan_groupby_variant_selection(lib):
    """The fused scan's variant switch accepts exactly the documented ids
    (-1 autotuned, 0 TMA-fed, 1/2 and 3/5 word table, 6 bulk-copy-fed word
    table, 7 lean word table, 9 prefetching word table, 4/8/16 warp-merged) and
    rejects others; no device work is involved."""
    try:
        for v in (-1, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 16):
            assert lib.voxel_scan_groupby_tune(v) == 0, v
            assert lib.voxel_scan_groupby_tune_state() == v, v
        for v in (-2, 10, 12, 32):
            assert lib.voxel_scan_groupby_tune(v) != 0, v
        # a rejected id leaves the previous choice in place
        assert lib.voxel_scan_groupby_tune(3) == 0
        assert lib.voxel_scan_groupby_tune(10) != 0
        assert lib.voxel_scan_groupby_tune_state() == 3
        assert lib.voxel_scan_groupby_tune(-1) == 0
        assert lib.voxel_scan_groupby_tune(12) != 0
        assert lib.voxel_scan_groupby_tune_state() == -1
    finally:
        lib.voxel_scan_groupby_tune(-1)


def test_scan_groupby_status_words(lib):
    """Status words of the fused scan map to codes and messages on the host:
    the bulk-copy timeout bit wins over the others and is reported as a
    timeout, not an overflow."""
    cases = [(0, 0, None), (1, 7, "not finite"), (2, 1, "dictionary"), (3, 1, "dictionary"),
             (4, 6, "bounded wait"), (5, 6, "bounded wait"), (6, 6, "bounded wait"), (8, 1, "unknown")]
    for word, code, text in cases:
        assert lib.voxel_scan_groupby_status_code(word) == code, word
        if text:
            assert text in capi.last_error(), (word, capi.last_error())
