/*
 * voxel_oracle.c - CPU restatement of the reference VoxelVM hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA backend.  Never linked
 * into, or called by, the product library.  Citations are file:line in the
 * reference project (include/voxel/...).
 *
 * f32 has no reference engine (Engine<f32> does not compile,
 * exec/engine.hpp:398,406).  This restatement defines it as the nearest
 * compilable reading of the same handlers: scalar registers hold f64 values
 * (ScalarAsT narrows to float, SetScalarT widens to double), lane arithmetic
 * is in float exactly as the handlers are written (VSUM sums in T), and the
 * fused fast path accumulates in f64.
 */
#include "voxel_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { DT_F64 = 0, DT_F32 = 1, DT_I64 = 2, DT_I32 = 3, DT_U64 = 4, DT_U32 = 5 };

static size_t esize(int dt) { return (dt == DT_F64 || dt == DT_I64 || dt == DT_U64) ? 8 : 4; }
static int is_float(int dt) { return dt == DT_F64 || dt == DT_F32; }

static double d_of(uint64_t b) { double d; memcpy(&d, &b, 8); return d; }
static uint64_t b_of_d(double d) { uint64_t b; memcpy(&b, &d, 8); return b; }
static float f_of(uint64_t b) { uint32_t u = (uint32_t)b; float f; memcpy(&f, &u, 4); return f; }
static uint64_t b_of_f(float f) { uint32_t u; memcpy(&u, &f, 4); return (uint64_t)u; }

/* ---- typed lane helpers (all values travel as T bits in a u64) ---------- */

static int t_isnan(int dt, uint64_t a) {
    if (dt == DT_F64) return isnan(d_of(a));
    if (dt == DT_F32) return isnan(f_of(a));
    return 0;
}

/* plain C++ comparison operators on T (engine.hpp:456-470, 2896-2923) */
static int t_cmp(int dt, int op, uint64_t a, uint64_t b) {
    switch (dt) {
    case DT_F64: { double x = d_of(a), y = d_of(b);
        switch (op) { case 0: return x == y; case 1: return x != y; case 2: return x < y;
                      case 3: return x <= y; case 4: return x > y; case 5: return x >= y; } break; }
    case DT_F32: { float x = f_of(a), y = f_of(b);
        switch (op) { case 0: return x == y; case 1: return x != y; case 2: return x < y;
                      case 3: return x <= y; case 4: return x > y; case 5: return x >= y; } break; }
    case DT_I64: { int64_t x = (int64_t)a, y = (int64_t)b;
        switch (op) { case 0: return x == y; case 1: return x != y; case 2: return x < y;
                      case 3: return x <= y; case 4: return x > y; case 5: return x >= y; } break; }
    case DT_I32: { int32_t x = (int32_t)(uint32_t)a, y = (int32_t)(uint32_t)b;
        switch (op) { case 0: return x == y; case 1: return x != y; case 2: return x < y;
                      case 3: return x <= y; case 4: return x > y; case 5: return x >= y; } break; }
    case DT_U64: { uint64_t x = a, y = b;
        switch (op) { case 0: return x == y; case 1: return x != y; case 2: return x < y;
                      case 3: return x <= y; case 4: return x > y; case 5: return x >= y; } break; }
    case DT_U32: { uint32_t x = (uint32_t)a, y = (uint32_t)b;
        switch (op) { case 0: return x == y; case 1: return x != y; case 2: return x < y;
                      case 3: return x <= y; case 4: return x > y; case 5: return x >= y; } break; }
    }
    return 0;
}

/* a + b in T (wraps for integers) */
static uint64_t t_add(int dt, uint64_t a, uint64_t b) {
    switch (dt) {
    case DT_F64: return b_of_d(d_of(a) + d_of(b));
    case DT_F32: return b_of_f(f_of(a) + f_of(b));
    case DT_I64: case DT_U64: return a + b;
    default: return (uint64_t)(uint32_t)((uint32_t)a + (uint32_t)b);
    }
}

static int t_is_zero(int dt, uint64_t a) {
    if (dt == DT_F64) return d_of(a) == 0.0;
    if (dt == DT_F32) return f_of(a) == 0.0f;
    if (esize(dt) == 4) return (uint32_t)a == 0;
    return a == 0;
}

/* Engine<T>::ScalarAsT / SetScalarT (engine.hpp:395-409) */
static uint64_t scalar_as_t(int dt, uint64_t reg) {
    switch (dt) {
    case DT_F32: return b_of_f((float)d_of(reg));
    case DT_I32: case DT_U32: return (uint64_t)(uint32_t)reg;
    default: return reg;
    }
}
static uint64_t set_scalar_t(int dt, uint64_t bits) {
    switch (dt) {
    case DT_F32: return b_of_d((double)f_of(bits));
    case DT_I32: return (uint64_t)(int64_t)(int32_t)(uint32_t)bits;
    case DT_U32: return (uint64_t)(uint32_t)bits;
    default: return bits;
    }
}

/* ---- register file (core/registers.hpp:18-164) -------------------------- */

#define F_ZERO 1u
#define F_CARRY 2u
#define F_SIGN 4u
#define F_OVF 8u
#define F_NAN 32u

typedef struct {
    int dt;
    size_t kl, es;
    uint64_t* R;
    uint8_t V[16][32];
    uint32_t M[8];
    uint32_t flags;
    const void* const* segs;
    const size_t* counts;
    size_t nsegs;
} vm_t;

static uint64_t lane(const vm_t* m, int v, size_t i) {
    uint64_t x = 0;
    memcpy(&x, &m->V[v & 15][i * m->es], m->es);
    return x;
}
static void set_lane(vm_t* m, int v, size_t i, uint64_t x) { memcpy(&m->V[v & 15][i * m->es], &x, m->es); }
static uint64_t seg_elem(const vm_t* m, size_t s, size_t i) {
    uint64_t x = 0;
    memcpy(&x, (const uint8_t*)m->segs[s] + i * m->es, m->es);
    return x;
}
static uint64_t bitsplat(const vm_t* m) { return m->es == 8 ? ~(uint64_t)0 : 0xFFFFFFFFull; }

static void arith_flags(vm_t* m, int64_t r) { /* registers.hpp:96-101 */
    m->flags &= ~(F_ZERO | F_SIGN | F_CARRY | F_OVF);
    if (r == 0) m->flags |= F_ZERO;
    if (r < 0) m->flags |= F_SIGN;
}
static void float_flags(vm_t* m, double r) { /* registers.hpp:103-110 */
    m->flags &= ~(F_NAN | 64u | F_OVF | 128u | 256u | 512u);
    if (r == 0.0) { m->flags |= F_ZERO; m->flags &= ~F_SIGN; }
    if (r < 0.0) m->flags |= F_SIGN;
    if (isnan(r)) m->flags |= F_NAN;
}

static int16_t simm12(uint32_t raw) {
    uint16_t v = (raw >> 20) & 0xFFF;
    return (v & 0x800) ? (int16_t)(v | 0xF000) : (int16_t)v;
}

/* ---- fused fast path (engine.hpp:84-141) -------------------------------- */

typedef struct { int ok; int seg, thr, acc, off, tot; int mode; } fast_t;

static fast_t detect_fast(const uint32_t* c, size_t len) {
    fast_t f; memset(&f, 0, sizeof f);
    if (len < 8) return f;
    uint32_t r0 = c[0], r1 = c[1], r2 = c[2], r3 = c[3], r4 = c[4], r5 = c[5], r6 = c[6];
    unsigned o0 = r0 & 0xFF, o1 = r1 & 0xFF, o2 = r2 & 0xFF, o3 = r3 & 0xFF, o4 = r4 & 0xFF,
             o5 = r5 & 0xFF, o6 = r6 & 0xFF;
    unsigned v0rd = (r0 >> 8) & 0xF, v0ra = (r0 >> 12) & 0xF;
    unsigned v1rd = (r1 >> 8) & 0xF, v1ra = (r1 >> 12) & 0xF, v1rb = (r1 >> 16) & 0xF;
    unsigned v2rd = (r2 >> 8) & 0xF, v2ra = (r2 >> 12) & 0xF;
    unsigned v3rd = (r3 >> 8) & 0xF, v3rb = (r3 >> 16) & 0xF;
    unsigned v4ra = (r4 >> 12) & 0xF, v5ra = (r5 >> 12) & 0xF, v5rb = (r5 >> 16) & 0xF;
    int16_t jnz = simm12(r6);
    int isf = (o1 >= 0xC1 && o1 <= 0xC6);
    if (o0 == 0x70 && isf && o2 == 0xD0 && o3 == 0x2A && o4 == 0x20 && o5 == 0x40 && o6 == 0x52 &&
        v1ra == v0rd && v2ra == v1rd && v3rb == v2rd && v4ra == v0ra && v5ra == v0ra && jnz == -6) {
        f.ok = 1;
        f.seg = (r0 >> 28) & 0xF;
        f.thr = (int)v1rb;
        f.acc = (int)v3rd;
        f.off = (int)v0ra;
        f.tot = (int)v5rb;
        f.mode = (int)o1;
    }
    return f;
}

static void run_fast(vm_t* m, const fast_t* f) {
    size_t cnt = (size_t)f->seg < m->nsegs ? m->counts[f->seg] : 0;
    size_t total = (size_t)(int64_t)m->R[f->tot];
    if (cnt < total) total = cnt;
    uint64_t th = scalar_as_t(m->dt, m->R[f->thr]);
    size_t off = (size_t)(int64_t)m->R[f->off];
    int op = f->mode - 0xC1; /* C1 EQ .. C6 GE */
    uint64_t acc = scalar_as_t(m->dt, m->R[f->acc]);
    double accd = d_of(m->R[f->acc]); /* f32: f64 accumulation */
    while (off + m->kl <= total) {
        uint64_t s = 0;
        for (size_t i = 0; i < m->kl; ++i) {
            uint64_t v = seg_elem(m, f->seg, off + i);
            if (!t_cmp(m->dt, op, v, th)) v = 0;
            s = t_add(m->dt, s, v);
        }
        if (m->dt == DT_F32) accd += (double)f_of(s);
        else acc = t_add(m->dt, acc, s);
        off += m->kl;
    }
    m->R[f->acc] = m->dt == DT_F32 ? b_of_d(accd) : set_scalar_t(m->dt, acc);
    m->R[f->off] = (uint64_t)off;
}

/* ---- AGG_* over a segment range (engine.hpp:499-569) --------------------- */

static void handle_agg(vm_t* m, vo_agg_state* st, unsigned rd, unsigned ra, unsigned rb,
                       unsigned imm, int kind) {
    size_t segId = ra;
    size_t start = (size_t)(int64_t)m->R[rb];
    size_t count = imm == 0 ? 0xFFFFFFFFull : (size_t)(imm & 0xFFF);
    vo_agg_state* s = &st[rd & 0xF];
    if (segId >= m->nsegs) return;
    size_t end = start + count;
    if (end > m->counts[segId]) end = m->counts[segId];
    int dt = m->dt;
    switch (kind) {
    case 0: /* COUNT */
        if (!s->init) { s->count = 0; s->init = 1; }
        for (size_t i = start; i < end; ++i) if (!t_is_zero(dt, seg_elem(m, segId, i))) s->count++;
        m->R[rd] = s->count;
        break;
    case 1: /* SUM */
        if (!s->init) { s->sum_f64 = 0; s->sum_i64 = 0; s->init = 1; }
        if (is_float(dt)) {
            for (size_t i = start; i < end; ++i) {
                uint64_t v = seg_elem(m, segId, i);
                s->sum_f64 += dt == DT_F64 ? d_of(v) : (double)f_of(v);
            }
            m->R[rd] = dt == DT_F64 ? b_of_d(s->sum_f64) : b_of_d((double)(float)s->sum_f64);
        } else {
            for (size_t i = start; i < end; ++i) {
                uint64_t v = seg_elem(m, segId, i);
                int64_t x = dt == DT_I32 ? (int64_t)(int32_t)(uint32_t)v
                          : dt == DT_U32 ? (int64_t)(uint32_t)v : (int64_t)v;
                s->sum_i64 = (int64_t)((uint64_t)s->sum_i64 + (uint64_t)x);
            }
            m->R[rd] = (uint64_t)s->sum_i64;
        }
        break;
    case 3: /* MIN */
    case 4: /* MAX */ {
        uint64_t* acc = kind == 3 ? &s->min_bits : &s->max_bits;
        if (!s->init) {
            /* numeric_limits<T>::max() / lowest() */
            uint64_t init;
            switch (dt) {
            case DT_F64: init = b_of_d(kind == 3 ? 1.7976931348623157e308 : -1.7976931348623157e308); break;
            case DT_F32: init = b_of_f(kind == 3 ? 3.40282347e38f : -3.40282347e38f); break;
            case DT_I64: init = kind == 3 ? 0x7FFFFFFFFFFFFFFFull : 0x8000000000000000ull; break;
            case DT_I32: init = kind == 3 ? 0x7FFFFFFFull : 0x80000000ull; break;
            case DT_U64: init = kind == 3 ? ~0ull : 0; break;
            default: init = kind == 3 ? 0xFFFFFFFFull : 0; break;
            }
            *acc = init;
            s->init = 1;
        }
        for (size_t i = start; i < end; ++i) {
            uint64_t v = seg_elem(m, segId, i);
            if (t_cmp(dt, kind == 3 ? 2 : 4, v, *acc)) *acc = v;
        }
        m->R[rd] = set_scalar_t(dt, *acc);
        break;
    }
    }
}

/* ---- interpreter over the restated opcode set (engine.hpp:1113-3111) ---- */

int vo_engine_run(int dtype, const uint32_t* code, size_t len, const void* const* segs,
                  const size_t* counts, size_t nsegs, uint64_t* regs, vo_agg_state* agg,
                  uint64_t max_steps, int* fast_path) {
    vm_t m;
    memset(&m, 0, sizeof m);
    m.dt = dtype;
    m.es = esize(dtype);
    m.kl = 32 / m.es;
    m.R = regs;
    m.segs = segs;
    m.counts = counts;
    m.nsegs = nsegs;
    vo_agg_state local[16];
    if (!agg) { memset(local, 0, sizeof local); agg = local; }

    fast_t f = detect_fast(code, len);
    if (fast_path) *fast_path = f.ok;
    if (f.ok) { run_fast(&m, &f); return 0; }

    size_t pc = 0;
    uint64_t steps = 0;
    while (pc < len) {
        if (++steps > max_steps) return -2;
        uint32_t raw = code[pc];
        unsigned op = raw & 0xFF, rd = (raw >> 8) & 0xF, ra = (raw >> 12) & 0xF,
                 rb = (raw >> 16) & 0xF, imm = (raw >> 20) & 0xFFF;
        int16_t si = simm12(raw);
        uint64_t* R = m.R;
        switch (op) {
        case 0x00: pc++; break;              /* NOP 1117 */
        case 0x01: return 0;                 /* HALT 1120 */
        case 0x10: R[rd] = (uint64_t)(int64_t)si; pc++; break;           /* MOV 1167 */
        case 0x11: R[rd] = R[ra]; pc++; break;                           /* MOVR 1174 */
        case 0x12: R[rd] = (uint64_t)((int64_t)R[ra] + si); pc++; break; /* ADDI 1181 */
        case 0x13: R[rd] = (uint64_t)((int64_t)R[ra] - si); pc++; break; /* SUBI 1189 */
        case 0x20: { int64_t r = (int64_t)(R[ra] + R[rb]); R[rd] = (uint64_t)r; arith_flags(&m, r); pc++; break; } /* ADD 1286 */
        case 0x21: { int64_t r = (int64_t)(R[ra] - R[rb]); R[rd] = (uint64_t)r; arith_flags(&m, r); pc++; break; } /* SUB 1295 */
        case 0x22: { int64_t r = (int64_t)(R[ra] * R[rb]); R[rd] = (uint64_t)r; arith_flags(&m, r); pc++; break; } /* MUL 1304 */
        case 0x27: { int64_t a = (int64_t)R[ra], b = (int64_t)R[rb]; int64_t r = a < b ? a : b; R[rd] = (uint64_t)r; arith_flags(&m, r); pc++; break; } /* MIN 1360 */
        case 0x28: { int64_t a = (int64_t)R[ra], b = (int64_t)R[rb]; int64_t r = a > b ? a : b; R[rd] = (uint64_t)r; arith_flags(&m, r); pc++; break; } /* MAX 1370 */
        case 0x2A: { double r = d_of(R[ra]) + d_of(R[rb]); R[rd] = b_of_d(r); float_flags(&m, r); pc++; break; } /* ADDF 1394 */
        case 0x2B: { double r = d_of(R[ra]) - d_of(R[rb]); R[rd] = b_of_d(r); float_flags(&m, r); pc++; break; } /* SUBF 1403 */
        case 0x2C: { double r = d_of(R[ra]) * d_of(R[rb]); R[rd] = b_of_d(r); float_flags(&m, r); pc++; break; } /* MULF 1412 */
        case 0x40: { int64_t d = (int64_t)(R[ra] - R[rb]); arith_flags(&m, d); pc++; break; } /* CMP 1603 */
        case 0x50: pc += si; break;                                                   /* JMP 1693 */
        case 0x51: if (m.flags & F_ZERO) pc += si; else pc++; break;                  /* JZ 1699 */
        case 0x52: if (!(m.flags & F_ZERO)) pc += si; else pc++; break;               /* JNZ 1706 */
        case 0x53: if (m.flags & F_SIGN) pc += si; else pc++; break;                  /* JS 1713 */
        case 0x54: if (!(m.flags & F_SIGN)) pc += si; else pc++; break;               /* JNS 1720 */
        case 0x59: if (m.flags & F_SIGN) pc += si; else pc++; break;                  /* JL 1771 */
        case 0x5A: if ((m.flags & F_ZERO) || (m.flags & F_SIGN)) pc += si; else pc++; break; /* JLE 1778 */
        case 0x5B: if (!(m.flags & F_ZERO) && !(m.flags & F_SIGN)) pc += si; else pc++; break; /* JG 1755 */
        case 0x5C: if ((m.flags & F_ZERO) || !(m.flags & F_SIGN)) pc += si; else pc++; break; /* JGE 1763 */
        case 0x70: { /* VLOAD 1947-1968 */
            unsigned segId = (imm >> 8) & 0xF, cnt = imm & 0xFF;
            if (cnt == 0) cnt = (unsigned)m.kl;
            size_t off = (size_t)(int64_t)R[ra];
            for (size_t i = 0; i < m.kl; ++i) {
                size_t idx = off + i;
                uint64_t v = 0;
                if (segId < nsegs && i < cnt && idx < counts[segId]) v = seg_elem(&m, segId, idx);
                set_lane(&m, rd, i, v);
            }
            pc++;
            break;
        }
        case 0x78: { uint64_t v = scalar_as_t(dtype, R[ra]); /* VSPLAT 2106 */
            for (size_t i = 0; i < m.kl; ++i) set_lane(&m, rd, i, v);
            pc++; break; }
        case 0xA0: case 0xA1: case 0xA2: case 0xA3: case 0xA4: case 0xA5: { /* VCMP* 2671-2705, HandleVCmp 476-493 */
            uint32_t mask = 0;
            uint64_t out[8];
            for (size_t i = 0; i < m.kl; ++i) {
                int p = t_cmp(dtype, (int)(op - 0xA0), lane(&m, ra, i), lane(&m, rb, i));
                out[i] = p ? bitsplat(&m) : 0;
                if (p) mask |= 1u << i;
            }
            for (size_t i = 0; i < m.kl; ++i) set_lane(&m, rd, i, out[i]);
            m.M[0] = mask;
            pc++;
            break;
        }
        case 0xB0: case 0xB1: case 0xB2: case 0xB4: { /* VAND VOR VXOR VANDN 2757-2804 */
            uint8_t o[32];
            for (int i = 0; i < 32; ++i) {
                uint8_t a = m.V[ra][i], b = m.V[rb][i];
                o[i] = op == 0xB0 ? (a & b) : op == 0xB1 ? (a | b) : op == 0xB2 ? (a ^ b) : (uint8_t)(~a & b);
            }
            memcpy(m.V[rd], o, 32);
            pc++;
            break;
        }
        case 0xB3: { uint8_t o[32]; for (int i = 0; i < 32; ++i) o[i] = (uint8_t)~m.V[ra][i]; /* VNOT 2787 */
            memcpy(m.V[rd], o, 32); pc++; break; }
        case 0xC0: case 0xC1: case 0xC2: case 0xC3: case 0xC4: case 0xC5: case 0xC6: { /* VFILTER 2870-2923 */
            uint64_t th = scalar_as_t(dtype, R[rb]);
            int cop = op == 0xC0 ? (int)(imm & 7) : (int)(op - 0xC1);
            uint32_t mask = 0;
            uint64_t out[8];
            for (size_t i = 0; i < m.kl; ++i) {
                uint64_t v = lane(&m, ra, i);
                int p = cop <= 5 ? t_cmp(dtype, cop, v, th) : 0;
                out[i] = p ? v : 0;
                if (p) mask |= 1u << i;
            }
            for (size_t i = 0; i < m.kl; ++i) set_lane(&m, rd, i, out[i]);
            m.M[imm & 7] = mask;
            pc++;
            break;
        }
        case 0xC7: { uint32_t mask = m.M[imm & 7]; uint64_t out[8]; /* VBLEND 2926-2935 */
            for (size_t i = 0; i < m.kl; ++i) out[i] = (mask >> i) & 1 ? lane(&m, rb, i) : lane(&m, ra, i);
            for (size_t i = 0; i < m.kl; ++i) set_lane(&m, rd, i, out[i]);
            pc++; break; }
        case 0xD0: { uint64_t s = 0; /* VSUM 2980-2987 */
            for (size_t i = 0; i < m.kl; ++i) s = t_add(dtype, s, lane(&m, ra, i));
            R[rd] = set_scalar_t(dtype, s); pc++; break; }
        case 0xD5: case 0xD6: { /* VRED_MIN / VRED_MAX 3071-3094 */
            uint64_t mm = lane(&m, ra, 0);
            for (size_t i = 1; i < m.kl; ++i) {
                uint64_t v = lane(&m, ra, i);
                int take = op == 0xD5 ? (t_cmp(dtype, 2, v, mm) || t_isnan(dtype, v))
                                      : (t_cmp(dtype, 4, v, mm) || t_isnan(dtype, mm));
                if (take) mm = v;
            }
            R[rd] = set_scalar_t(dtype, mm); pc++; break; }
        case 0xD7: { uint64_t c = 0; /* VCOUNT 3097-3110 */
            for (size_t i = 0; i < m.kl; ++i) {
                uint64_t v = lane(&m, ra, i);
                if (!t_isnan(dtype, v) && !t_is_zero(dtype, v)) c++;
            }
            R[rd] = c; pc++; break; }
        case 0xE0: handle_agg(&m, agg, rd, ra, rb, imm, 0); pc++; break; /* AGG_COUNT */
        case 0xE1: handle_agg(&m, agg, rd, ra, rb, imm, 1); pc++; break; /* AGG_SUM */
        case 0xE3: handle_agg(&m, agg, rd, ra, rb, imm, 3); pc++; break; /* AGG_MIN */
        case 0xE4: handle_agg(&m, agg, rd, ra, rb, imm, 4); pc++; break; /* AGG_MAX */
        default: return -1;
        }
    }
    return 0;
}

/* ---- VectorFilter / SelectionVector / ColumnFilter ----------------------- */

size_t vo_vfilter(int dt, int op, const void* data, size_t n, uint64_t a, uint64_t b, uint64_t* bm) {
    size_t es = esize(dt), pass = 0;
    size_t words = (n + 63) / 64;
    memset(bm, 0, words * 8);
    for (size_t i = 0; i < n; ++i) {
        uint64_t v = 0;
        memcpy(&v, (const uint8_t*)data + i * es, es);
        int p = op <= 5 ? t_cmp(dt, op, v, a) : (t_cmp(dt, 5, v, a) && t_cmp(dt, 3, v, b));
        if (p) { bm[i >> 6] |= 1ull << (i & 63); pass++; }
    }
    return pass;
}

size_t vo_selection_from_bitmap(const uint64_t* bm, size_t rows, uint32_t* out) {
    size_t words = (rows + 63) / 64, c = 0;
    for (size_t w = 0; w < words; ++w) {
        uint64_t x = bm[w];
        while (x) {
            out[c++] = (uint32_t)(w * 64 + (size_t)__builtin_ctzll(x));
            x &= x - 1;
        }
    }
    return c;
}

size_t vo_bitmap_and(const uint64_t* const* bms, size_t nbm, size_t rows, uint64_t* out) {
    size_t words = (rows + 63) / 64, c = 0;
    for (size_t w = 0; w < words; ++w) {
        uint64_t x = ~0ull;
        if (w == words - 1 && (rows & 63)) x = (1ull << (rows & 63)) - 1;
        for (size_t k = 0; k < nbm; ++k) x &= bms[k][w];
        out[w] = x;
        c += (size_t)__builtin_popcountll(x);
    }
    return c;
}

/* ---- encodings ----------------------------------------------------------- */

uint32_t vo_bitpack_width(const uint32_t* d, size_t n) {
    uint32_t mx = 0, w = 0;
    for (size_t i = 0; i < n; ++i) if (d[i] > mx) mx = d[i];
    while (mx) { ++w; mx >>= 1; }
    return w ? w : 1;
}

size_t vo_bitpack_build(const uint32_t* d, size_t n, uint32_t w, uint64_t* words) {
    size_t nw = (n * w + 63) / 64;
    memset(words, 0, nw * 8);
    uint64_t mask = w == 64 ? ~0ull : ((1ull << w) - 1);
    for (size_t i = 0; i < n; ++i) {
        uint64_t bit = (uint64_t)i * w, v = (uint64_t)d[i] & mask;
        size_t wi = (size_t)(bit / 64);
        unsigned sh = (unsigned)(bit % 64);
        words[wi] |= v << sh;
        if (sh + w > 64 && wi + 1 < nw) words[wi + 1] |= v >> (64 - sh);
    }
    return nw;
}

void vo_bitpack_decode(const uint64_t* words, size_t nw, uint32_t w, size_t vc, size_t off,
                       size_t cnt, uint32_t* out) {
    uint64_t mask = (1ull << w) - 1;
    for (size_t i = 0; i < cnt && off + i < vc; ++i) {
        uint64_t bit = (uint64_t)(off + i) * w;
        size_t wi = (size_t)(bit / 64);
        unsigned sh = (unsigned)(bit % 64);
        uint64_t r = words[wi] >> sh;
        if (sh + w > 64 && wi + 1 < nw) r |= words[wi + 1] << (64 - sh);
        out[i] = (uint32_t)(r & mask);
    }
}

static int cmp_i32(const void* a, const void* b) {
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return x < y ? -1 : x > y;
}

size_t vo_dict_build_i32(const int32_t* d, size_t n, int32_t* dict, uint32_t* idx) {
    if (n == 0) return 0;
    int32_t* s = (int32_t*)malloc(n * 4);
    memcpy(s, d, n * 4);
    qsort(s, n, 4, cmp_i32);
    size_t card = 0;
    for (size_t i = 0; i < n; ++i) if (i == 0 || s[i] != s[i - 1]) dict[card++] = s[i];
    free(s);
    for (size_t i = 0; i < n; ++i) {
        size_t lo = 0, hi = card;
        while (hi - lo > 1) { size_t mid = (lo + hi) / 2; if (dict[mid] <= d[i]) lo = mid; else hi = mid; }
        idx[i] = (uint32_t)lo;
    }
    return card;
}

void vo_dict_decode_i32(const int32_t* dict, size_t card, const uint32_t* idx, size_t n,
                        size_t off, size_t cnt, int32_t* out) {
    (void)card;
    for (size_t i = 0; i < cnt && off + i < n; ++i) out[i] = dict[idx[off + i]];
}

size_t vo_rle_build_i64(const int64_t* d, size_t n, int64_t* values, uint32_t* runs) {
    if (n == 0) return 0;
    size_t k = 0;
    int64_t cur = d[0];
    uint32_t len = 1;
    for (size_t i = 1; i < n; ++i) {
        if (d[i] == cur) ++len;
        else { values[k] = cur; runs[k++] = len; cur = d[i]; len = 1; }
    }
    values[k] = cur;
    runs[k++] = len;
    return k;
}

/* encoding.hpp:292-306 (DeltaEncoding<T>::Build): deltas[i] = data[i] - data[i-1],
   data[-1] = 0, wrapping in T's width (w = 4 or 8 bytes; T's bits as unsigned). */
void vo_delta_build(int w, const void* data, size_t n, void* deltas) {
    uint64_t prev = 0;
    for (size_t i = 0; i < n; ++i) {
        uint64_t x = w == 8 ? ((const uint64_t*)data)[i] : ((const uint32_t*)data)[i];
        uint64_t d = x - prev;
        if (w == 8) ((uint64_t*)deltas)[i] = d; else ((uint32_t*)deltas)[i] = (uint32_t)d;
        prev = x;
    }
}

/* encoding.hpp:317-330 (DeltaEncoding<T>::DecodeBatch): a running wrapping sum
   from BaseValue over deltas[0..offset), then out[i] = running for the next
   rows while i < cnt and offset + i < n (later outputs are left alone). */
void vo_delta_decode(int w, const void* deltas, size_t n, uint64_t base, size_t off, size_t cnt, void* out) {
    uint64_t run = base;
    for (size_t i = 0; i < off && i < n; ++i)
        run += w == 8 ? ((const uint64_t*)deltas)[i] : ((const uint32_t*)deltas)[i];
    for (size_t i = 0; i < cnt && off + i < n; ++i) {
        run += w == 8 ? ((const uint64_t*)deltas)[off + i] : ((const uint32_t*)deltas)[off + i];
        if (w == 8) ((uint64_t*)out)[i] = run; else ((uint32_t*)out)[i] = (uint32_t)run;
    }
}

/* encoding.hpp:489-500 (FrameOfReferenceEncoding::DecodeBatch):
   BaseValue + (f64)code * Scale, each operation rounded (no contraction). */
void vo_for_decode_f64(const int32_t* code, size_t n, double base, double scale, size_t off, size_t cnt,
                       double* out) {
    for (size_t i = 0; i < cnt && off + i < n; ++i) {
        volatile double prod = (double)code[off + i] * scale;
        out[i] = base + prod;
    }
}

void vo_rle_decode_i64(const int64_t* values, const uint32_t* runs, size_t nruns, size_t off,
                       size_t cnt, int64_t* out) {
    /* encoding.hpp:231-257, including its u32 running total */
    uint32_t cum = 0;
    size_t r = 0;
    while (r < nruns) { cum += runs[r]; if (off < cum) break; ++r; }
    size_t row = off;
    for (size_t i = 0; i < cnt; ++i) {
        if (r >= nruns) { out[i] = 0; continue; }
        out[i] = values[r];
        ++row;
        if (row >= cum) { ++r; if (r < nruns) cum += runs[r]; }
    }
}

/* ---- group-by ------------------------------------------------------------ */

typedef struct { int32_t k; uint32_t row; } kr_t;
static int cmp_kr(const void* a, const void* b) {
    const kr_t* x = (const kr_t*)a; const kr_t* y = (const kr_t*)b;
    if (x->k != y->k) return x->k < y->k ? -1 : 1;
    return x->row < y->row ? -1 : x->row > y->row;
}

size_t vo_groupby_i32_f64(const int32_t* keys, const double* vals, size_t n, int32_t* okeys,
                          double* osum, double* omin, double* omax, uint64_t* ocount) {
    if (n == 0) return 0;
    kr_t* p = (kr_t*)malloc(n * sizeof(kr_t));
    for (size_t i = 0; i < n; ++i) { p[i].k = keys[i]; p[i].row = (uint32_t)i; }
    qsort(p, n, sizeof(kr_t), cmp_kr);
    size_t g = 0;
    for (size_t i = 0; i < n;) {
        int32_t k = p[i].k;
        double v = vals[p[i].row];
        /* AggregateState::Init then Update in row order (aggregate.hpp:85-105) */
        double s = v, mn = v, mx = v;
        uint64_t c = 1;
        size_t j = i + 1;
        for (; j < n && p[j].k == k; ++j) {
            double x = vals[p[j].row];
            s += x;
            if (x < mn) mn = x;
            if (x > mx) mx = x;
            c++;
        }
        okeys[g] = k; osum[g] = s; omin[g] = mn; omax[g] = mx; ocount[g] = c;
        ++g;
        i = j;
    }
    free(p);
    return g;
}

/* ---- radix sort ------------------------------------------------------------ */

void vo_radix_sort(int dt, void* keys, uint32_t* idx, size_t n) {
    if (n <= 1) return;
    size_t es = esize(dt);
    uint8_t* src = (uint8_t*)keys;
    uint8_t* tmp = (uint8_t*)malloc(n * es);
    uint32_t* isrc = idx;
    uint32_t* itmp = (uint32_t*)malloc(n * 4);
    uint8_t* dst = tmp;
    uint32_t* idst = itmp;
    for (size_t byte = 0; byte < es; ++byte) {
        size_t hist[256] = {0}, pre[256];
        for (size_t i = 0; i < n; ++i) hist[src[i * es + byte]]++;
        pre[0] = 0;
        for (int b = 1; b < 256; ++b) pre[b] = pre[b - 1] + hist[b - 1];
        for (size_t i = 0; i < n; ++i) {
            size_t pos = pre[src[i * es + byte]]++;
            memcpy(dst + pos * es, src + i * es, es);
            idst[pos] = isrc[i];
        }
        uint8_t* t = src; src = dst; dst = t;
        uint32_t* ti = isrc; isrc = idst; idst = ti;
    }
    if (dt == DT_I64 || dt == DT_I32) { /* sort.hpp:127-152 */
        size_t neg = 0;
        for (size_t i = 0; i < n; ++i) if (src[i * es + es - 1] & 0x80) ++neg;
        size_t np = 0, pp = neg;
        for (size_t i = 0; i < n; ++i) {
            size_t pos = (src[i * es + es - 1] & 0x80) ? np++ : pp++;
            memcpy(dst + pos * es, src + i * es, es);
            idst[pos] = isrc[i];
        }
        uint8_t* t = src; src = dst; dst = t;
        uint32_t* ti = isrc; isrc = idst; idst = ti;
    }
    if (src != (uint8_t*)keys) memcpy(keys, src, n * es);
    if (isrc != idx) memcpy(idx, isrc, n * 4);
    free(tmp);
    free(itmp);
}

/* ---- hash join --------------------------------------------------------------- */

typedef struct { int64_t k; uint32_t row; } br_t;
static int cmp_br(const void* a, const void* b) {
    const br_t* x = (const br_t*)a; const br_t* y = (const br_t*)b;
    if (x->k != y->k) return x->k < y->k ? -1 : 1;
    return x->row > y->row ? -1 : x->row < y->row; /* newest first within a key */
}

size_t vo_hashjoin_i64(const int64_t* build, size_t nb, const int64_t* probe, size_t np,
                       uint32_t* left, uint32_t* right, size_t maxm, int all) {
    br_t* b = (br_t*)malloc((nb ? nb : 1) * sizeof(br_t));
    for (size_t i = 0; i < nb; ++i) { b[i].k = build[i]; b[i].row = (uint32_t)i; }
    qsort(b, nb, sizeof(br_t), cmp_br);
    size_t m = 0;
    size_t cap = all ? maxm : np;
    for (size_t i = 0; i < np && m < cap; ++i) {
        size_t lo = 0, hi = nb;
        while (lo < hi) { size_t mid = (lo + hi) / 2; if (b[mid].k < probe[i]) lo = mid + 1; else hi = mid; }
        for (size_t j = lo; j < nb && b[j].k == probe[i] && m < cap; ++j) {
            left[m] = (uint32_t)i;
            right[m] = b[j].row;
            ++m;
            if (!all) break;
        }
    }
    free(b);
    return m;
}

/* ---- scan + group-by pipeline --------------------------------------------------- */

size_t vo_scan_groupby(const uint64_t* packed, size_t nwords, uint32_t width, const int32_t* dict,
                       size_t card, const double* price, const int32_t* qty, size_t n,
                       double pthr, int32_t qlo, int32_t qhi, int32_t* okeys, double* osum,
                       double* omin, double* omax, uint64_t* ocount) {
    (void)card;
    size_t sel = 0;
    int32_t* k = (int32_t*)malloc((n ? n : 1) * 4);
    double* v = (double*)malloc((n ? n : 1) * 8);
    double* p = (double*)malloc((n ? n : 1) * 8);
    uint64_t mask = (1ull << width) - 1;
    for (size_t i = 0; i < n; ++i) {
        if (!(price[i] > pthr) || !(qty[i] >= qlo && qty[i] <= qhi)) continue;
        uint64_t bit = (uint64_t)i * width;
        size_t wi = (size_t)(bit / 64);
        unsigned sh = (unsigned)(bit % 64);
        uint64_t r = packed[wi] >> sh;
        if (sh + width > 64 && wi + 1 < nwords) r |= packed[wi + 1] << (64 - sh);
        k[sel] = dict[(uint32_t)(r & mask)];
        v[sel] = price[i] * (double)qty[i];
        p[sel] = price[i];
        ++sel;
    }
    /* SUM/COUNT over (key, price*qty); MIN/MAX over (key, price) */
    size_t g = vo_groupby_i32_f64(k, v, sel, okeys, osum, omin, omax, ocount);
    if (g) {
        int32_t* k2 = (int32_t*)malloc(g * 4);
        double* s2 = (double*)malloc(g * 8);
        uint64_t* c2 = (uint64_t*)malloc(g * 8);
        vo_groupby_i32_f64(k, p, sel, k2, s2, omin, omax, c2);
        free(k2); free(s2); free(c2);
    }
    free(k); free(v); free(p);
    return g;
}

/* join.hpp:218-268 (MergeJoin<TKey>::Join / JoinUnique) over sorted i64 keys:
   two cursors; on equal keys Join emits the whole right run for the left row
   and rewinds the right cursor, JoinUnique emits one pair and advances both.
   Stops writing at cap; returns the pairs written. */
size_t vo_merge_join_i64(const int64_t* l, size_t nl, const int64_t* r, size_t nr, uint32_t* lo, uint32_t* ro,
                         size_t cap, int unique) {
    size_t m = 0, li = 0, ri = 0;
    while (li < nl && ri < nr) {
        if (l[li] < r[ri]) ++li;
        else if (r[ri] < l[li]) ++ri;
        else if (unique) {
            if (m < cap) { lo[m] = (uint32_t)li; ro[m] = (uint32_t)ri; ++m; }
            ++li; ++ri;
        } else {
            size_t start = ri;
            while (ri < nr && r[ri] == l[li]) {
                if (m < cap) { lo[m] = (uint32_t)li; ro[m] = (uint32_t)ri; ++m; }
                ++ri;
            }
            ++li;
            ri = start;
        }
    }
    return m;
}

static int cmp_i64(const void* a, const void* b) {
    int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
    return x < y ? -1 : x > y;
}

/* join.hpp:273-310 (AntiJoin / SemiJoin): left rows in order whose key is
   (anti = 0) / is not (anti = 1) in the set of right keys. */
size_t vo_semi_join_i64(const int64_t* l, size_t nl, const int64_t* r, size_t nr, uint32_t* out, int anti) {
    int64_t* s = (int64_t*)malloc((nr ? nr : 1) * 8);
    memcpy(s, r, nr * 8);
    qsort(s, nr, 8, cmp_i64);
    size_t m = 0;
    for (size_t i = 0; i < nl; ++i) {
        size_t lo = 0, hi = nr;
        while (lo < hi) { size_t mid = (lo + hi) / 2; if (s[mid] < l[i]) lo = mid + 1; else hi = mid; }
        int found = lo < nr && s[lo] == l[i];
        if (found != anti) out[m++] = (uint32_t)i;
    }
    free(s);
    return m;
}

/* exec/engine.hpp:182-300 (Engine<f64>::WindowDelta .. WindowQuantile): each
   window summed left to right, mean = sum / w, ssq = sum of (x - mean)^2,
   quantile from the sorted first min(w, 128) values with linear
   interpolation.  kind 0 delta, 1 sum, 2 mean, 3 stddev, 4 variance, 5
   quantile.  Returns the outputs written. */
static int cmp_f64(const void* a, const void* b) {
    double x = *(const double*)a, y = *(const double*)b;
    return x < y ? -1 : x > y;
}

size_t vo_window_f64(int kind, const double* d, size_t n, double* out, size_t out_len, unsigned w, double q) {
    if (kind == 0) {
        if (n < 2) return 0;
        size_t m = n - 1 < out_len ? n - 1 : out_len;
        for (size_t i = 0; i < m; ++i) out[i] = d[i + 1] - d[i];
        return m;
    }
    if (w == 0 || n < w) return 0;
    if (kind >= 3 && w < 2) return 0;
    if (kind == 5 && !(q >= 0.0 && q <= 1.0)) return 0;
    size_t m = n - w + 1 < out_len ? n - w + 1 : out_len;
    for (size_t j = 0; j < m; ++j) {
        if (kind == 5) {
            double buf[128];
            size_t ww = w < 128 ? w : 128;
            for (size_t k = 0; k < ww; ++k) buf[k] = d[j + k];
            qsort(buf, ww, 8, cmp_f64);
            double pos = q * (double)(ww - 1);
            size_t lo = (size_t)pos;
            if (lo >= ww) lo = ww - 1;
            size_t hi = lo + 1;
            if (hi >= ww) hi = lo;
            if (lo == hi) { out[j] = buf[lo]; continue; }
            volatile double t = (buf[hi] - buf[lo]) * (pos - (double)lo);
            out[j] = buf[lo] + t;
            continue;
        }
        double sum = 0.0;
        for (size_t k = 0; k < w; ++k) sum += d[j + k];
        if (kind == 1) { out[j] = sum; continue; }
        double mean = sum / (double)w;
        if (kind == 2) { out[j] = mean; continue; }
        double ssq = 0.0;
        for (size_t k = 0; k < w; ++k) { volatile double dd = d[j + k] - mean; volatile double p = dd * dd; ssq += p; }
        out[j] = kind == 4 ? ssq / (double)w : sqrt(ssq / (double)w);
    }
    return m;
}

/* exec/engine.hpp:228-241 (TimeWindowSum): out[(ts - start) / dur] += v for
   buckets in [0, out_len), in row order; returns the largest bucket + 1. */
size_t vo_time_window_sum_f64(const int64_t* ts, const double* v, size_t n, int64_t start, int64_t dur, double* out,
                              size_t out_len) {
    if (dur <= 0 || n == 0 || out_len == 0) return 0;
    size_t maxb = 0;
    for (size_t i = 0; i < n; ++i) {
        int64_t b = (ts[i] - start) / dur;
        if (b >= 0 && (size_t)b < out_len) {
            out[b] += v[i];
            if ((size_t)b > maxb) maxb = (size_t)b;
        }
    }
    return maxb + 1;
}
