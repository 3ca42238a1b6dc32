"""VoxelVM bytecode encoders (the reference's Instruction builders).

32-bit format ``[op:8][rd:4][ra:4][rb:4][imm12:12]`` as in
``include/voxel/bytecode/instruction.hpp:65-72``; opcode numbers from
``include/voxel/bytecode/opcodes.hpp:11-262``.
"""
from __future__ import annotations

OP = dict(
    NOP=0x00, HALT=0x01, MOV=0x10, MOVR=0x11, ADDI=0x12, SUBI=0x13,
    ADD=0x20, SUB=0x21, MUL=0x22, MIN=0x27, MAX=0x28, ADDF=0x2A, SUBF=0x2B, MULF=0x2C,
    CMP=0x40, JMP=0x50, JZ=0x51, JNZ=0x52, JS=0x53, JNS=0x54, JL=0x59, JLE=0x5A, JG=0x5B, JGE=0x5C,
    VLOAD=0x70, VSPLAT=0x78,
    VCMPEQ=0xA0, VCMPNE=0xA1, VCMPLT=0xA2, VCMPLE=0xA3, VCMPGT=0xA4, VCMPGE=0xA5,
    VAND=0xB0, VOR=0xB1, VXOR=0xB2, VNOT=0xB3, VANDN=0xB4,
    VFILTER=0xC0, VFILTER_EQ=0xC1, VFILTER_NE=0xC2, VFILTER_LT=0xC3, VFILTER_LE=0xC4,
    VFILTER_GT=0xC5, VFILTER_GE=0xC6, VBLEND=0xC7,
    VSUM=0xD0, VRED_MIN=0xD5, VRED_MAX=0xD6, VCOUNT=0xD7,
    AGG_COUNT=0xE0, AGG_SUM=0xE1, AGG_MIN=0xE3, AGG_MAX=0xE4,
)

CMP_NAMES = ["EQ", "NE", "LT", "LE", "GT", "GE"]


def enc(op: int, rd: int = 0, ra: int = 0, rb: int = 0, imm: int = 0) -> int:
    return (op & 0xFF) | ((rd & 0xF) << 8) | ((ra & 0xF) << 12) | ((rb & 0xF) << 16) | ((imm & 0xFFF) << 20)


def halt() -> int: return enc(OP["HALT"])
def nop() -> int: return enc(OP["NOP"])
def mov(rd, imm) -> int: return enc(OP["MOV"], rd, 0, 0, imm & 0xFFF)
def movr(rd, ra) -> int: return enc(OP["MOVR"], rd, ra)
def addi(rd, ra, imm) -> int: return enc(OP["ADDI"], rd, ra, 0, imm & 0xFFF)
def add(rd, ra, rb) -> int: return enc(OP["ADD"], rd, ra, rb)
def sub(rd, ra, rb) -> int: return enc(OP["SUB"], rd, ra, rb)
def smin(rd, ra, rb) -> int: return enc(OP["MIN"], rd, ra, rb)
def smax(rd, ra, rb) -> int: return enc(OP["MAX"], rd, ra, rb)
def addf(rd, ra, rb) -> int: return enc(OP["ADDF"], rd, ra, rb)
def cmp(ra, rb) -> int: return enc(OP["CMP"], 0, ra, rb)
def jnz(off) -> int: return enc(OP["JNZ"], 0, 0, 0, off & 0xFFF)
def jz(off) -> int: return enc(OP["JZ"], 0, 0, 0, off & 0xFFF)
def jl(off) -> int: return enc(OP["JL"], 0, 0, 0, off & 0xFFF)
def jle(off) -> int: return enc(OP["JLE"], 0, 0, 0, off & 0xFFF)
def jge(off) -> int: return enc(OP["JGE"], 0, 0, 0, off & 0xFFF)
def jmp(off) -> int: return enc(OP["JMP"], 0, 0, 0, off & 0xFFF)
def vload(vd, ra, seg, count=0) -> int: return enc(OP["VLOAD"], vd, ra, 0, ((seg & 0xF) << 8) | (count & 0xFF))
def vsplat(vd, ra) -> int: return enc(OP["VSPLAT"], vd, ra)
def vcmp(cmp_op: int, vd, va, vb) -> int: return enc(OP["VCMPEQ"] + cmp_op, vd, va, vb)
def vand(vd, va, vb) -> int: return enc(OP["VAND"], vd, va, vb)
def vor(vd, va, vb) -> int: return enc(OP["VOR"], vd, va, vb)
def vandn(vd, va, vb) -> int: return enc(OP["VANDN"], vd, va, vb)
def vfilter(cmp_op: int, vd, va, rb, mask=0) -> int: return enc(OP["VFILTER_EQ"] + cmp_op, vd, va, rb, mask & 7)
def vfilter_gt(vd, va, rb) -> int: return enc(OP["VFILTER_GT"], vd, va, rb)
def vblend(vd, va, vb, mask=0) -> int: return enc(OP["VBLEND"], vd, va, vb, mask & 7)
def vsum(rd, va) -> int: return enc(OP["VSUM"], rd, va)
def vcount(rd, va) -> int: return enc(OP["VCOUNT"], rd, va)
def vred_min(rd, va) -> int: return enc(OP["VRED_MIN"], rd, va)
def vred_max(rd, va) -> int: return enc(OP["VRED_MAX"], rd, va)
def agg(kind: str, rd, seg, rstart, count=0) -> int: return enc(OP["AGG_" + kind], rd, seg, rstart, count)


def filter_sum_program(seg: int = 0, cmp_op: int = 4, k_lanes: int = 4) -> list[int]:
    """The fused filter+sum loop of the reference's benchmarks
    (examples/validate.cpp:40-48): R0 acc, R1 offset, R2 total, R3 threshold."""
    return [vload(0, 1, seg), vfilter(cmp_op, 1, 0, 3), vsum(5, 1), addf(0, 0, 5),
            add(1, 1, 4), cmp(1, 2), jnz(-6), halt()]


def filter_sum_count_program(seg: int = 0, cmp_op: int = 4) -> list[int]:
    """filter x op R3; SUM(x) into R0; COUNT into R6 (VCOUNT of the filtered lanes)."""
    return [vload(0, 1, seg), vfilter(cmp_op, 1, 0, 3), vsum(5, 1), addf(0, 0, 5),
            vcount(7, 1), add(6, 6, 7), add(1, 1, 4), cmp(1, 2), jnz(-8), halt()]
