// Range form of a lowered single-column filter/aggregate program: the
// conjunction of its predicate atoms rewritten as one interval plus up to two
// excluded values, so a kernel tests lo <= x <= hi (x != ne[0], x != ne[1])
// with the reduction kind fixed at compile time.  Host code; shared by the
// single-program scan and the batched executor.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <type_traits>

#include "vx_types.h"

namespace vx {

// The accumulator fold a range-form program uses for each reduction kind
// (SUM: ADDF on floats, ADD on integers; COUNT: ADD; MIN / MAX: MIN / MAX).
#ifdef __CUDACC__
__host__ __device__
#endif
constexpr uint8_t range_acc(int rk, bool is_float) {
    return rk == kRedSum ? (is_float ? kAccAddF : kAccAdd) : rk == kRedCount ? kAccAdd : rk == kRedMin ? kAccMin : kAccMax;
}

struct RangeForm {
    uint32_t fast;  // 0: none; else 1 + 2 * reduction kind + (excluded values present)
    uint32_t pad;
    uint64_t lo, hi;  // T bits
    uint64_t ne[2];
};

// The range form of a lowered single-column program, when it has one.  The
// conjunction of ordered atoms (EQ LT LE GT GE) on column 0 is the interval
// [lo, hi] in T's order (x < t is x <= the next value below t, and so on; an
// empty set is lo > hi); NE atoms stay as up to two excluded values (an NE
// against a NaN threshold holds for every x and is dropped).  A program
// qualifies with one column, one reduction whose predicate is all atoms and
// whose false value is a constant, and at least one ordered atom.
template <typename T>
inline T host_from_bits(uint64_t b) {
    T v;
    if constexpr (sizeof(T) == 8) {
        std::memcpy(&v, &b, 8);
    } else {
        const uint32_t w = static_cast<uint32_t>(b);
        std::memcpy(&v, &w, 4);
    }
    return v;
}

template <typename T>
inline uint64_t host_to_bits(T v) {
    if constexpr (sizeof(T) == 8) {
        uint64_t b;
        std::memcpy(&b, &v, 8);
        return b;
    } else {
        uint32_t w;
        std::memcpy(&w, &v, 4);
        return w;
    }
}

// count_col: also accept a COUNT of the column's lanes (VCOUNT of a VFILTER
// output: passing nonzero values), which the single-program scan kernel
// evaluates; the batched executor's kernels count constants only.
template <typename T>
inline bool range_form_t(const ScanParams& p, RangeForm* out, bool count_col = false) {
    if (p.ncols != 1 || p.nred != 1 || p.natoms < 1 || p.natoms > kMaxAtoms) return false;
    const uint32_t all = (1u << p.natoms) - 1u;
    const Red& r = p.red[0];
    if (r.pmask != all || r.kind > kRedMax) return false;
    constexpr bool kFloat = std::is_floating_point<T>::value;
    if (r.acc != range_acc(r.kind, kFloat)) return false;
    // COUNT counts a constant (the VCOUNT of M & one); the others reduce the column
    const bool acol = r.a.kind == kOpCol && r.a.col == 0;
    if (r.kind == kRedCount ? !(r.a.kind == kOpConst || r.a.kind == kOpZero || (count_col && acol)) : !acol)
        return false;
    if (r.b.kind != kOpConst && r.b.kind != kOpZero) return false;
    const T lowest = kFloat ? -std::numeric_limits<T>::infinity() : std::numeric_limits<T>::lowest();
    const T highest = kFloat ? std::numeric_limits<T>::infinity() : std::numeric_limits<T>::max();
    T lo = lowest, hi = highest, ne[2] = {T(0), T(0)};
    int nne = 0;
    bool ordered = false, empty = false;
    for (int a = 0; a < p.natoms; ++a) {
        const Atom& at = p.atom[a];
        if (at.col != 0 || at.op > 5) return false;
        const T t = host_from_bits<T>(at.thr);
        const bool nan = t != t;
        if (at.op == 1) {  // NE
            if (nan) continue;
            if (nne == 2) return false;
            ne[nne++] = t;
            continue;
        }
        ordered = true;
        if (nan) {
            empty = true;
            continue;
        }
        T l = lowest, h = highest;
        switch (at.op) {
        case 0: l = h = t; break;  // EQ
        case 2:                    // LT
            if (t == lowest) empty = true;
            else if constexpr (kFloat) h = std::nextafter(t, lowest);
            else h = static_cast<T>(t - 1);
            break;
        case 3: h = t; break;  // LE
        case 4:                // GT
            if (t == highest) empty = true;
            else if constexpr (kFloat) l = std::nextafter(t, highest);
            else l = static_cast<T>(t + 1);
            break;
        default: l = t; break;  // GE
        }
        if (l > lo) lo = l;
        if (h < hi) hi = h;
    }
    if (!ordered) return false;
    if (empty || lo > hi) {
        lo = highest;
        hi = lowest;
    }
    if (nne == 1) ne[1] = ne[0];
    out->lo = host_to_bits(lo);
    out->hi = host_to_bits(hi);
    out->ne[0] = host_to_bits(ne[0]);
    out->ne[1] = host_to_bits(ne[1]);
    out->fast = 1u + 2u * r.kind + (nne ? 1u : 0u);
    return true;
}


inline bool range_form_of(const ScanParams& p, RangeForm* out, bool count_col = false) {
    switch (p.dtype) {
    case F64: return range_form_t<double>(p, out, count_col);
    case F32: return range_form_t<float>(p, out, count_col);
    case I64: return range_form_t<int64_t>(p, out, count_col);
    case I32: return range_form_t<int32_t>(p, out, count_col);
    case U64: return range_form_t<uint64_t>(p, out, count_col);
    default: return range_form_t<uint32_t>(p, out, count_col);
    }
}

// Most reductions a multi-reduction range form carries.
constexpr int kMaxRangeRed = 4;

// Range form of a program with 2..kMaxRangeRed reductions over one column that
// all share the conjunction of every atom (the config-1 program's SUM and
// COUNT of one VFILTER output; SUM + COUNT + MIN + MAX of one predicate).
// Each reduction keeps its own kind, operands and canonical fold; the interval
// and excluded values are those of range_form_t.  COUNT may count the column's
// lanes (VCOUNT of a VFILTER output: passing nonzero values) or a constant.
template <typename T>
inline bool multi_range_form_t(const ScanParams& p, RangeForm* out) {
    if (p.ncols != 1 || p.nred < 2 || p.nred > kMaxRangeRed || p.natoms < 1 || p.natoms > kMaxAtoms) return false;
    const uint32_t all = (1u << p.natoms) - 1u;
    constexpr bool kFloat = std::is_floating_point<T>::value;
    for (int i = 0; i < p.nred; ++i) {
        const Red& r = p.red[i];
        if (r.pmask != all || r.kind > kRedMax) return false;
        if (r.acc != range_acc(r.kind, kFloat)) return false;
        const bool acol = r.a.kind == kOpCol && r.a.col == 0;
        const bool aconst = r.a.kind == kOpConst || r.a.kind == kOpZero;
        if (r.kind == kRedCount ? !(acol || aconst) : !acol) return false;
        if (r.b.kind != kOpConst && r.b.kind != kOpZero) return false;
    }
    // the interval: the single-reduction rewrite of the atoms with reduction 0
    // (every reduction has the same predicate, so its interval is shared)
    ScanParams q = p;
    q.nred = 1;
    q.red[0].kind = kRedSum;
    q.red[0].acc = range_acc(kRedSum, kFloat);
    q.red[0].a.kind = kOpCol;
    q.red[0].a.col = 0;
    q.red[0].b.kind = kOpZero;
    if (!range_form_t<T>(q, out)) return false;
    // range_form_t's code is 1 + 2 * kind + (excluded values present)
    out->fast = (out->fast & 1u) ? 1u : 2u;  // 1: interval only, 2: with excluded values
    out->pad = static_cast<uint32_t>(p.nred);
    return true;
}

inline bool multi_range_form_of(const ScanParams& p, RangeForm* out) {
    switch (p.dtype) {
    case F64: return multi_range_form_t<double>(p, out);
    case F32: return multi_range_form_t<float>(p, out);
    case I64: return multi_range_form_t<int64_t>(p, out);
    case I32: return multi_range_form_t<int32_t>(p, out);
    case U64: return multi_range_form_t<uint64_t>(p, out);
    default: return multi_range_form_t<uint32_t>(p, out);
    }
}

}  // namespace vx
