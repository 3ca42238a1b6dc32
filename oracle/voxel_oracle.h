/*
 * voxel_oracle.h - CPU restatement of the reference VoxelVM hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA backend is checked
 * against; it is never linked into the product library.  Each function cites
 * the reference file:line it restates (paths relative to the reference root).
 * Its outputs are pinned against the reference's own compiled operators
 * (oracle/_ref) and the reference's known-answer tests (tests/golden).
 *
 * Element type codes (shared with include/voxel_c.h):
 *   0 f64, 1 f32, 2 i64, 3 i32, 4 u64, 5 u32
 * A scalar "bits" argument carries a T value in the low bytes of a u64
 * (f64: IEEE bits; f32: IEEE bits in the low 32; integers: two's complement).
 */
#ifndef VOXEL_ORACLE_H
#define VOXEL_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Per-slot state of the AGG_* opcodes (engine.hpp:499-569, AggState). */
typedef struct {
    int32_t init;
    uint64_t count;
    double sum_f64;
    int64_t sum_i64;
    uint64_t min_bits;
    uint64_t max_bits;
} vo_agg_state;

/* Run one program like Engine<T>::LoadProgram + Run (engine.hpp:43-141, 3370-3451).
 * regs[64] are read and written.  agg[16] persists AGG_* state across runs.
 * Returns 0 on success, -1 on an opcode outside the restated set, -2 when
 * max_steps instructions were executed without halting.  *fast_path gets 1 when
 * the fused filter+sum pattern (engine.hpp:84-107) was taken. */
int vo_engine_run(int dtype, const uint32_t* code, size_t len, const void* const* segs,
                  const size_t* counts, size_t nsegs, uint64_t* regs, vo_agg_state* agg,
                  uint64_t max_steps, int* fast_path);

/* VectorFilter<T>::Apply{EQ,NE,LT,LE,GT,GE,Between} (filter.hpp:42-288).
 * op: 0 EQ 1 NE 2 LT 3 LE 4 GT 5 GE 6 BETWEEN(lo=a, hi=b).  Returns PassCount. */
size_t vo_vfilter(int dtype, int op, const void* data, size_t n, uint64_t a_bits,
                  uint64_t b_bits, uint64_t* bitmap);
/* SelectionVector::BuildFromBitmap (filter.hpp:378-399). */
size_t vo_selection_from_bitmap(const uint64_t* bm, size_t rows, uint32_t* out);
/* ColumnFilter::Init + AndWith (filter.hpp:526-547); returns the active count. */
size_t vo_bitmap_and(const uint64_t* const* bms, size_t nbm, size_t rows, uint64_t* out);

/* BitPackedEncoding (encoding.hpp:370-449). */
uint32_t vo_bitpack_width(const uint32_t* data, size_t n);
size_t vo_bitpack_build(const uint32_t* data, size_t n, uint32_t width, uint64_t* words);
void vo_bitpack_decode(const uint64_t* words, size_t nwords, uint32_t width, size_t value_count,
                       size_t offset, size_t count, uint32_t* out);
/* DictionaryEncoding<i32> (encoding.hpp:113-167); returns the cardinality. */
size_t vo_dict_build_i32(const int32_t* data, size_t n, int32_t* dict, uint32_t* idx);
void vo_dict_decode_i32(const int32_t* dict, size_t card, const uint32_t* idx, size_t n,
                        size_t offset, size_t count, int32_t* out);
/* RLEEncoding<i64> (encoding.hpp:202-257); returns the run count. */
size_t vo_rle_build_i64(const int64_t* data, size_t n, int64_t* values, uint32_t* runs);
void vo_delta_build(int w, const void* data, size_t n, void* deltas);
size_t vo_window_f64(int kind, const double* d, size_t n, double* out, size_t out_len, unsigned w, double q);
size_t vo_time_window_sum_f64(const int64_t* ts, const double* v, size_t n, int64_t start, int64_t dur, double* out,
                              size_t out_len);
size_t vo_merge_join_i64(const int64_t* l, size_t nl, const int64_t* r, size_t nr, uint32_t* lo, uint32_t* ro,
                         size_t cap, int unique);
size_t vo_semi_join_i64(const int64_t* l, size_t nl, const int64_t* r, size_t nr, uint32_t* out, int anti);
void vo_delta_decode(int w, const void* deltas, size_t n, uint64_t base, size_t off, size_t cnt, void* out);
void vo_for_decode_f64(const int32_t* code, size_t n, double base, double scale, size_t off, size_t cnt,
                       double* out);
void vo_rle_decode_i64(const int64_t* values, const uint32_t* runs, size_t nruns, size_t offset,
                       size_t count, int64_t* out);

/* HashAggregator<i32,f64> per-group state (aggregate.hpp:85-105, 168-239):
 * Sum in row order, Min/Max by < and >, Count.  Groups come out sorted by key
 * (the reference emits slot order, aggregate.hpp:249-261).  Returns #groups. */
size_t vo_groupby_i32_f64(const int32_t* keys, const double* vals, size_t n, int32_t* okeys,
                          double* osum, double* omin, double* omax, uint64_t* ocount);

/* RadixSort<T>::Sort(keys, idx, n) (sort.hpp:83-160): stable LSD, 8-bit digits,
 * negatives-first pass for signed T.  dtype in {2,3,4,5}. */
void vo_radix_sort(int dtype, void* keys, uint32_t* idx, size_t n);

/* HashJoin<i64> Build + Probe / ProbeAllMatches (join.hpp:50-102): pairs in
 * probe order; equal build keys come out newest-first (LIFO chains). */
size_t vo_hashjoin_i64(const int64_t* build, size_t nb, const int64_t* probe, size_t np,
                       uint32_t* left, uint32_t* right, size_t maxm, int all);

/* Scan + group-by: key = dict[unpack(packed)] WHERE price > pthr AND qty BETWEEN
 * qlo AND qhi GROUP BY key -> SUM(price*qty), COUNT, MIN(price), MAX(price),
 * composed as in the reference operators; groups sorted by key. */
size_t vo_scan_groupby(const uint64_t* packed, size_t nwords, uint32_t width, const int32_t* dict,
                       size_t card, const double* price, const int32_t* qty, size_t n,
                       double pthr, int32_t qlo, int32_t qhi, int32_t* okeys, double* osum,
                       double* omin, double* omax, uint64_t* ocount);

#ifdef __cplusplus
}
#endif
#endif
