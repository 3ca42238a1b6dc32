"""Bytecode templates for filter/aggregate programs, and their register setup.

A template program scans one column with 1-4 conjunctive predicates and one
aggregate (SUM, COUNT, MIN or MAX).  It is built only from opcodes the
reference interpreter runs (include/voxel/exec/engine.hpp), so the reference
Engine<T> is the oracle for it:

    VSPLAT thresholds / constant (prologue)
    loop:  VLOAD x; VCMPop_i x, t_i (AND-ed with VAND) -> mask M
           SUM:   VAND M,x            -> VSUM  -> ADD/ADDF acc
           COUNT: VAND M,one          -> VCOUNT-> ADD acc
           MIN:   (M&x)|(~M&sentinel) -> VRED_MIN -> MIN acc
           MAX:   (M&x)|(~M&sentinel) -> VRED_MAX -> MAX acc
           ADD off,kLanes; CMP off,total; JNZ loop
    HALT

For columns whose length is a multiple of kLanes and whose values are
non-negative (and below 2^63 for u64), each template equals the SQL query
``SELECT agg(x) WHERE p_1 AND ... AND p_k`` (MIN/MAX of an empty selection
return the sentinel); tests/test_templates.py checks this against a scalar loop.
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass, field

import numpy as np

from . import bytecode as bc

F64, F32, I64, I32, U64, U32 = range(6)
NP = {F64: np.float64, F32: np.float32, I64: np.int64, I32: np.int32, U64: np.uint64, U32: np.uint32}
K_LANES = {F64: 4, F32: 8, I64: 4, I32: 8, U64: 4, U32: 8}
AGGS = ("SUM", "COUNT", "MIN", "MAX")


def reg_image(dtype: int, value) -> int:
    """The scalar-register image of a T value (f32 registers hold f64)."""
    if dtype in (F64, F32):
        return struct.unpack("<Q", struct.pack("<d", float(value)))[0]
    return int(value) & 0xFFFFFFFFFFFFFFFF


def image_value(dtype: int, bits: int):
    bits &= 0xFFFFFFFFFFFFFFFF
    if dtype in (F64, F32):
        return struct.unpack("<d", struct.pack("<Q", bits))[0]
    if dtype in (I64, I32):
        return bits - (1 << 64) if bits >> 63 else bits
    return bits


def sentinel(dtype: int, agg: str):
    if agg == "MIN":
        return {F64: math.inf, F32: math.inf, I64: 2**63 - 1, I32: 2**31 - 1, U64: 2**63 - 1, U32: 2**32 - 1}[dtype]
    return {F64: -math.inf, F32: -math.inf, I64: -(2**63), I32: -(2**31), U64: 0, U32: 0}[dtype]


@dataclass
class Pred:
    op: int          # 0 EQ 1 NE 2 LT 3 LE 4 GT 5 GE
    value: float


@dataclass
class Program:
    dtype: int
    preds: list
    agg: str
    code: list = field(default_factory=list)
    regs: dict = field(default_factory=dict)   # register -> image before the run
    result_reg: int = 0

    def registers(self, n: int) -> list:
        r = [0] * 64
        for k, v in self.regs.items():
            r[k] = v
        r[2] = n
        return r


def build(dtype: int, preds: list, agg: str, seg: int = 0) -> Program:
    assert 1 <= len(preds) <= 4 and agg in AGGS
    kl = K_LANES[dtype]
    code = []
    regs = {1: 0, 4: kl}
    for i, p in enumerate(preds):
        regs[8 + i] = reg_image(dtype, p.value)
        code.append(bc.vsplat(8 + i, 8 + i))
    if agg == "COUNT":
        regs[12] = reg_image(dtype, 1)
    elif agg in ("MIN", "MAX"):
        regs[12] = reg_image(dtype, sentinel(dtype, agg))
    if agg != "SUM":
        code.append(bc.vsplat(12, 12))
    head = len(code)
    code.append(bc.vload(0, 1, seg))
    code.append(bc.vcmp(preds[0].op, 4, 0, 8))
    for i in range(1, len(preds)):
        code.append(bc.vcmp(preds[i].op, 5, 0, 8 + i))
        code.append(bc.vand(4, 4, 5))
    if agg == "SUM":
        code += [bc.vand(6, 4, 0), bc.vsum(5, 6)]
        code.append(bc.addf(0, 0, 5) if dtype in (F64, F32) else bc.add(0, 0, 5))
        regs[0] = 0
    elif agg == "COUNT":
        code += [bc.vand(6, 4, 12), bc.vcount(5, 6), bc.add(0, 0, 5)]
        regs[0] = 0
    else:
        red = bc.vred_min if agg == "MIN" else bc.vred_max
        fold = bc.smin if agg == "MIN" else bc.smax
        code += [bc.vand(6, 4, 0), bc.vandn(7, 4, 12), bc.vor(6, 6, 7), red(5, 6), fold(0, 0, 5)]
        regs[0] = reg_image(dtype, sentinel(dtype, agg))
    code += [bc.add(1, 1, 4), bc.cmp(1, 2)]
    code.append(bc.jnz(head - len(code)))
    code.append(bc.halt())
    return Program(dtype, preds, agg, code, regs, 0)


# accumulator register of each aggregate in a multi-aggregate program
MULTI_ACC = {"SUM": 0, "MIN": 3, "COUNT": 6, "MAX": 7}


def build_multi(dtype: int, preds: list, aggs: list, seg: int = 0) -> Program:
    """One predicate set, several aggregates of it in one loop: SUM into R0,
    MIN into R3, COUNT into R6, MAX into R7 (the shape of the config-1 program
    `filter x > t; SUM(x); COUNT` and of SUM+COUNT+MIN+MAX queries).  Each
    aggregate is the single-aggregate template's lane formula over the shared
    mask V4."""
    assert 1 <= len(preds) <= 4 and aggs and len(set(aggs)) == len(aggs) and set(aggs) <= set(AGGS)
    kl = K_LANES[dtype]
    code = []
    regs = {1: 0, 4: kl, 12: reg_image(dtype, 1), 13: reg_image(dtype, sentinel(dtype, "MIN")),
            14: reg_image(dtype, sentinel(dtype, "MAX"))}
    for i, p in enumerate(preds):
        regs[8 + i] = reg_image(dtype, p.value)
        code.append(bc.vsplat(8 + i, 8 + i))
    code += [bc.vsplat(12, 12), bc.vsplat(13, 13), bc.vsplat(14, 14)]
    head = len(code)
    code.append(bc.vload(0, 1, seg))
    code.append(bc.vcmp(preds[0].op, 4, 0, 8))
    for i in range(1, len(preds)):
        code.append(bc.vcmp(preds[i].op, 5, 0, 8 + i))
        code.append(bc.vand(4, 4, 5))
    for agg in aggs:
        r = MULTI_ACC[agg]
        if agg == "SUM":
            code += [bc.vand(6, 4, 0), bc.vsum(5, 6)]
            code.append(bc.addf(r, r, 5) if dtype in (F64, F32) else bc.add(r, r, 5))
            regs[r] = 0
        elif agg == "COUNT":
            code += [bc.vand(6, 4, 12), bc.vcount(5, 6), bc.add(r, r, 5)]
            regs[r] = 0
        else:
            red = bc.vred_min if agg == "MIN" else bc.vred_max
            fold = bc.smin if agg == "MIN" else bc.smax
            sv = 13 if agg == "MIN" else 14
            code += [bc.vand(6, 4, 0), bc.vandn(7, 4, sv), bc.vor(6, 6, 7), red(5, 6), fold(r, r, 5)]
            regs[r] = reg_image(dtype, sentinel(dtype, agg))
    code += [bc.add(1, 1, 4), bc.cmp(1, 2)]
    code.append(bc.jnz(head - len(code)))
    code.append(bc.halt())
    return Program(dtype, preds, ",".join(aggs), code, regs, MULTI_ACC[aggs[0]])


def sql_reference(prog: Program, col: np.ndarray):
    """Scalar loop of the equivalent SQL query (Python / numpy)."""
    m = np.ones(col.size, bool)
    for p in prog.preds:
        v = p.value
        if prog.dtype == F32:
            v = np.float32(v)
        else:
            v = NP[prog.dtype](v)
        m &= [np.equal, np.not_equal, np.less, np.less_equal, np.greater, np.greater_equal][p.op](col, v)
    sel = col[m]
    if prog.agg == "COUNT":
        return int(m.sum())
    if prog.agg == "SUM":
        if prog.dtype in (F64, F32):
            return math.fsum(sel.astype(np.float64))
        return int(sel.astype(object).sum()) if sel.size else 0
    if sel.size == 0:
        return sentinel(prog.dtype, prog.agg)
    return (sel.min() if prog.agg == "MIN" else sel.max()).item()


def make_column(dtype: int, n: int, rng: np.random.Generator) -> np.ndarray:
    """Column ~ U[0,1000) cast per element type."""
    x = rng.random(n) * 1000.0
    if dtype in (F64, F32):
        return x.astype(NP[dtype])
    return np.floor(x).astype(NP[dtype])


def random_program(dtype: int, rng: np.random.Generator, selectivity: float | None = None,
                   npreds: int | None = None, agg: str | None = None) -> Program:
    """1-4 conjunctive predicates with selectivity about `selectivity` on U[0,1000)."""
    if selectivity is None:
        selectivity = float(np.exp(rng.uniform(np.log(1e-4), np.log(0.9))))
    if npreds is None:
        npreds = int(rng.integers(1, 5))
    if agg is None:
        agg = AGGS[int(rng.integers(0, 4))]
    integer = dtype not in (F64, F32)
    w = 1000.0 * selectivity
    lo = float(rng.uniform(0, 1000.0 - w))
    hi = lo + w
    if integer:
        lo, hi = math.floor(lo), max(math.floor(lo) + 1, math.floor(hi))
    preds = [Pred(5, lo)] if npreds >= 2 else [Pred(2, w if not integer else max(1, math.floor(w)))]
    if npreds >= 2:
        preds.append(Pred(2, hi))
    for _ in range(npreds - len(preds)):
        c = float(rng.uniform(lo, hi))
        preds.append(Pred(1, math.floor(c) if integer else c))
    return build(dtype, preds, agg)
