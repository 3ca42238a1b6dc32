/*
 * voxel_c.h - C ABI of the VoxelVM B200 backend (libvoxel_c.so).
 *
 * Drop-in replacement for the reference's bindings/voxel_c.h: every symbol the
 * reference exports is declared here with the same signature (the comment
 * gives the reference line it replaces), so existing callers (the Go cgo
 * wrapper, the Java FFM wrapper, c_test.cpp) link unchanged.  Data work runs on
 * the GPU; there is no CPU path, and calls that cannot run fail loudly through
 * voxel_last_error().
 *
 * Additive symbols follow.  They never change a reference signature:
 *   - engines for f32 / i32 / u32 / u64 columns, named like the _i64 set;
 *   - status-returning variants (return 0 on success, a VOXEL_E* code otherwise);
 *   - operator entry points for the hot path with host buffers, and "_dev"
 *     variants that take device pointers and a cudaStream_t (as void*).
 *
 * Element-type codes: 0 f64, 1 f32, 2 i64, 3 i32, 4 u64, 5 u32.
 * Comparison codes:   0 EQ, 1 NE, 2 LT, 3 LE, 4 GT, 5 GE, 6 BETWEEN.
 */
#pragma once

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define VOXEL_OK 0
#define VOXEL_EINVAL 1
#define VOXEL_EUNSUPPORTED 2
#define VOXEL_ENONTERMINATING 3
#define VOXEL_ECUDA 4
#define VOXEL_ENOMEM 5
#define VOXEL_ETIMEOUT 6
#define VOXEL_EOVERFLOW 7
#define VOXEL_ENODEVICE 8
#define VOXEL_ECAPACITY 9

/* ================================================================
 * Engine (f64) - reference bindings/voxel_c.h:14-24
 * ================================================================ */
void*     voxel_engine_create_f64(void);                                             /* voxel_c.h:14 */
void      voxel_engine_destroy(void* engine);                                        /* voxel_c.h:15 */
size_t    voxel_engine_add_segment(void* engine, const double* data, size_t count);  /* voxel_c.h:16 */
void      voxel_engine_load_program(void* engine, const uint32_t* code, size_t len); /* voxel_c.h:17 */
void      voxel_engine_run(void* engine);                                            /* voxel_c.h:18 */
void      voxel_engine_run_parallel(void* engine, size_t seg_id, uint32_t threads,
                                    uint8_t result_reg);                             /* voxel_c.h:19 */
void      voxel_engine_set_scalar(void* engine, size_t reg, uint64_t value);         /* voxel_c.h:20 */
uint64_t  voxel_engine_get_scalar(void* engine, size_t reg);                         /* voxel_c.h:21 */
void      voxel_engine_set_scalar_f64(void* engine, size_t reg, double value);       /* voxel_c.h:22 */
double    voxel_engine_get_scalar_f64(void* engine, size_t reg);                     /* voxel_c.h:23 */
size_t    voxel_engine_k_lanes(void);                                                /* voxel_c.h:24 */

/* ================================================================
 * Engine (i64) - reference bindings/voxel_c.h:29-35
 * ================================================================ */
void*     voxel_engine_create_i64(void);                                                 /* voxel_c.h:29 */
void      voxel_engine_destroy_i64(void* engine);                                        /* voxel_c.h:30 */
size_t    voxel_engine_add_segment_i64(void* engine, const int64_t* data, size_t count); /* voxel_c.h:31 */
void      voxel_engine_load_program_i64(void* engine, const uint32_t* code, size_t len); /* voxel_c.h:32 */
void      voxel_engine_run_i64(void* engine);                                            /* voxel_c.h:33 */
void      voxel_engine_set_scalar_i64(void* engine, size_t reg, uint64_t value);         /* voxel_c.h:34 */
uint64_t  voxel_engine_get_scalar_i64(void* engine, size_t reg);                         /* voxel_c.h:35 */

/* ================================================================
 * JIT - reference bindings/voxel_c.h:40-41 (fused filter+sum over one f64
 * column with R0=0, R1=0, R2=data_len, R3=threshold; returns R0).
 * ================================================================ */
double    voxel_jit_run(const uint32_t* code, size_t code_len,
                        const double* data, size_t data_len, double threshold);      /* voxel_c.h:40 */
/* Additive (the reference's pybind jit_compile, bindings/voxel_bindings.cpp:329-340):
 * 0 when the program lowers, with jit_run's registers, onto one fused GPU
 * kernel schedule (host code only); *schedule_bytes = the schedule's size and
 * kernel (cap bytes) = the kernel's name; else a VOXEL_E* code. */
int       voxel_jit_compile(const uint32_t* code, size_t code_len, size_t* schedule_bytes, char* kernel,
                            size_t cap);

/* ================================================================
 * Instruction encoding - reference bindings/voxel_c.h:46-65
 * ================================================================ */
uint32_t  voxel_instr_vload(uint8_t vd, uint8_t ra, uint8_t seg_id, uint8_t count);  /* voxel_c.h:46 */
uint32_t  voxel_instr_vfilter_gt(uint8_t vd, uint8_t va, uint8_t rb);                /* voxel_c.h:47 */
uint32_t  voxel_instr_vfilter_ge(uint8_t vd, uint8_t va, uint8_t rb);                /* voxel_c.h:48 */
uint32_t  voxel_instr_vfilter_lt(uint8_t vd, uint8_t va, uint8_t rb);                /* voxel_c.h:49 */
uint32_t  voxel_instr_vfilter_le(uint8_t vd, uint8_t va, uint8_t rb);                /* voxel_c.h:50 */
uint32_t  voxel_instr_vsum(uint8_t rd, uint8_t va);                                  /* voxel_c.h:51 */
uint32_t  voxel_instr_vred_min(uint8_t rd, uint8_t va);                              /* voxel_c.h:52 */
uint32_t  voxel_instr_vred_max(uint8_t rd, uint8_t va);                              /* voxel_c.h:53 */
uint32_t  voxel_instr_vcount(uint8_t rd, uint8_t va);                                /* voxel_c.h:54 */
uint32_t  voxel_instr_addf(uint8_t rd, uint8_t ra, uint8_t rb);                      /* voxel_c.h:55 */
uint32_t  voxel_instr_add(uint8_t rd, uint8_t ra, uint8_t rb);                       /* voxel_c.h:56 */
uint32_t  voxel_instr_sub(uint8_t rd, uint8_t ra, uint8_t rb);                       /* voxel_c.h:57 */
uint32_t  voxel_instr_mul(uint8_t rd, uint8_t ra, uint8_t rb);                       /* voxel_c.h:58 */
uint32_t  voxel_instr_mov(uint8_t rd, int16_t imm);                                  /* voxel_c.h:59 */
uint32_t  voxel_instr_movr(uint8_t rd, uint8_t ra);                                  /* voxel_c.h:60 */
uint32_t  voxel_instr_cmp(uint8_t ra, uint8_t rb);                                   /* voxel_c.h:61 */
uint32_t  voxel_instr_jnz(int16_t offset);                                           /* voxel_c.h:62 */
uint32_t  voxel_instr_jz(int16_t offset);                                            /* voxel_c.h:63 */
uint32_t  voxel_instr_jmp(int16_t offset);                                           /* voxel_c.h:64 */
uint32_t  voxel_instr_halt(void);                                                    /* voxel_c.h:65 */

/* ================================================================
 * NullBitmap - reference bindings/voxel_c.h:70-76 (1 = null)
 * ================================================================ */
void*     voxel_null_create(size_t count);                      /* voxel_c.h:70 */
void      voxel_null_destroy(void* bitmap);                     /* voxel_c.h:71 */
int       voxel_null_is_null(const void* bitmap, size_t row);   /* voxel_c.h:72 */
void      voxel_null_set_null(void* bitmap, size_t row);        /* voxel_c.h:73 */
void      voxel_null_set_valid(void* bitmap, size_t row);       /* voxel_c.h:74 */
size_t    voxel_null_null_count(const void* bitmap);            /* voxel_c.h:75 */
size_t    voxel_null_valid_count(const void* bitmap);           /* voxel_c.h:76 */

/* ================================================================
 * HashAggregator<u32,f64> - reference bindings/voxel_c.h:81-85
 * ================================================================ */
void*     voxel_agg_create(void);                                                       /* voxel_c.h:81 */
void      voxel_agg_destroy(void* agg);                                                 /* voxel_c.h:82 */
void      voxel_agg_init(void* agg, size_t expected_groups);                            /* voxel_c.h:83 */
void      voxel_agg_accumulate(void* agg, const uint32_t* keys, const double* values,
                               size_t count);                                           /* voxel_c.h:84 */
size_t    voxel_agg_group_count(const void* agg);                                       /* voxel_c.h:85 */

/* ================================================================
 * Sort & TopK - reference bindings/voxel_c.h:90-92
 * ================================================================ */
void      voxel_sort_ascending(const double* data, size_t count, uint32_t* indices_out);  /* voxel_c.h:90 */
void      voxel_sort_descending(const double* data, size_t count, uint32_t* indices_out); /* voxel_c.h:91 */
void      voxel_topk(const double* data, size_t count, size_t k, double* out, int largest);/* voxel_c.h:92 */

/* ================================================================
 * DictionaryEncoding<f64> - reference bindings/voxel_c.h:97-101
 * ================================================================ */
void*     voxel_dict_create(void);                                                    /* voxel_c.h:97 */
void      voxel_dict_destroy(void* dict);                                             /* voxel_c.h:98 */
void      voxel_dict_build(void* dict, const double* data, size_t count);             /* voxel_c.h:99 */
size_t    voxel_dict_cardinality(const void* dict);                                   /* voxel_c.h:100 */
void      voxel_dict_decode_batch(void* dict, double* out, size_t offset, size_t count); /* voxel_c.h:101 */

/* ================================================================
 * ThreadPool - reference bindings/voxel_c.h:106-109 (host worker pool)
 * ================================================================ */
void*     voxel_pool_create(uint32_t threads);           /* voxel_c.h:106 */
void      voxel_pool_destroy(void* pool);                /* voxel_c.h:107 */
void      voxel_pool_wait_all(void* pool);               /* voxel_c.h:108 */
size_t    voxel_pool_thread_count(const void* pool);     /* voxel_c.h:109 */

/* ================================================================
 * Error handling - reference bindings/voxel_c.h:114.  Unlike the reference
 * (whose buffer is never written, voxel_c.cpp:7,227) this returns the calling
 * thread's last failure message, or "" after a success.
 * ================================================================ */
const char* voxel_last_error(void);                      /* voxel_c.h:114 */

/* ================================================================
 * Additive: engines for the other column types (north-star EngineF32/I32/
 * U32/U64), following the _i64 naming.  voxel_engine_destroy accepts any
 * engine handle.  f32 engines keep scalar registers as f64 values.
 * ================================================================ */
void*     voxel_engine_create(int dtype);
int       voxel_engine_dtype(const void* engine);
size_t    voxel_engine_k_lanes_of(const void* engine);
void*     voxel_engine_create_f32(void);
void*     voxel_engine_create_i32(void);
void*     voxel_engine_create_u32(void);
void*     voxel_engine_create_u64(void);
size_t    voxel_engine_add_segment_f32(void* engine, const float* data, size_t count);
size_t    voxel_engine_add_segment_i32(void* engine, const int32_t* data, size_t count);
size_t    voxel_engine_add_segment_u32(void* engine, const uint32_t* data, size_t count);
size_t    voxel_engine_add_segment_u64(void* engine, const uint64_t* data, size_t count);
/* a column already resident in device memory (not copied; must outlive runs) */
size_t    voxel_engine_add_segment_device(void* engine, const void* device_data, size_t count);
int       voxel_engine_run_status(void* engine);
int       voxel_engine_run_parallel_status(void* engine, size_t seg_id, uint32_t threads,
                                           uint8_t result_reg);
/* the schedule the last run executed, as text (for diagnostics and tests) */
size_t    voxel_engine_explain(void* engine, char* buf, size_t cap);
/* lower the loaded program without running it (no device needed); the
 * schedules are then available from voxel_engine_explain */
int       voxel_engine_plan(void* engine);
void      voxel_engine_reset(void* engine);
/* milliseconds of device time of the last run's kernels (CUDA events) */
double    voxel_engine_last_device_ms(const void* engine);
int       voxel_last_status(void);

/* ================================================================
 * Additive: memory helpers for callers that keep columns resident
 * ================================================================ */
void*     voxel_device_alloc(size_t bytes);
void      voxel_device_free(void* d_ptr);
int       voxel_copy_to_device(void* d_dst, const void* src, size_t bytes, void* stream);
int       voxel_copy_to_host(void* dst, const void* d_src, size_t bytes, void* stream);
int       voxel_stream_sync(void* stream);
/* page-lock an existing host buffer so the H2D copies of host entry points run at full speed */
int       voxel_host_register(void* ptr, size_t bytes);
int       voxel_host_unregister(void* ptr);

/* ================================================================
 * Additive: VectorFilter / ColumnFilter / SelectionVector on the GPU
 * (reference include/voxel/ops/filter.hpp:42-399).  Host buffers.
 * ================================================================ */
/* bitmap: ceil(n/64) words, bit i&63 of word i>>6 set iff row i passes.
 * Returns PassCount, or (size_t)-1 on failure. */
size_t    voxel_vfilter(int dtype, int op, const void* data, size_t n, uint64_t lo_bits,
                        uint64_t hi_bits, uint64_t* bitmap);
size_t    voxel_bitmap_and(const uint64_t* const* bitmaps, size_t nbitmaps, size_t rows,
                           uint64_t* out);
size_t    voxel_selection_from_bitmap(const uint64_t* bitmap, size_t rows, uint32_t* out);
/* device variants: asynchronous on `stream` (NULL = the CUDA default stream) */
int       voxel_vfilter_dev(int dtype, int op, const void* d_data, size_t n, uint64_t lo_bits,
                            uint64_t hi_bits, uint64_t* d_bitmap, uint64_t* d_count, void* stream);
int       voxel_selection_from_bitmap_dev(const uint64_t* d_bitmap, size_t rows, uint32_t* d_out,
                                          uint64_t* d_count, void* stream);
/* ColumnFilter::AndWith over device bitmaps: d_bitmaps is a host array of nbm
 * device pointers; *d_count receives the popcount of the result */
int       voxel_bitmap_and_dev(const uint64_t* const* d_bitmaps, size_t nbm, size_t rows, uint64_t* d_out,
                               uint64_t* d_count, void* stream);

/* ================================================================
 * Additive: decoders (reference include/voxel/data/encoding.hpp)
 * ================================================================ */
/* BitPackedEncoding::DecodeBatch (encoding.hpp:397-422) */
int       voxel_bitpack_decode(const uint64_t* words, size_t nwords, uint32_t width,
                               size_t value_count, size_t offset, size_t count, uint32_t* out);
/* DictionaryEncoding<i32>::DecodeBatch over packed indices: out[i] = dict[unpack(i)] */
int       voxel_dict_bitpack_decode_i32(const uint64_t* words, size_t nwords, uint32_t width,
                                        const int32_t* dict, size_t card, size_t value_count,
                                        size_t offset, size_t count, int32_t* out);
/* DictionaryEncoding<T>::DecodeBatch (encoding.hpp:156-167), dtype 0 or 3 */
int       voxel_dict_decode(int dtype, const void* dict, size_t card, const uint32_t* indices,
                            size_t n, size_t offset, size_t count, void* out);
/* RLEEncoding<i64>::DecodeBatch (encoding.hpp:231-257) */
int       voxel_rle_decode_i64(const int64_t* values, const uint32_t* runs, size_t nruns,
                               size_t offset, size_t count, int64_t* out);
int       voxel_bitpack_decode_dev(const uint64_t* d_words, size_t nwords, uint32_t width,
                                   size_t value_count, size_t offset, size_t count, uint32_t* d_out,
                                   void* stream);
int       voxel_rle_decode_i64_dev(const int64_t* d_values, const uint32_t* d_runs, size_t nruns,
                                   size_t offset, size_t count, int64_t* d_out, void* stream);
/* device variants of the dictionary decoders; they return after the kernel
 * (an index outside the dictionary is reported as VOXEL_EINVAL) */
/* ================================================================
 * Additive: window functions of Engine<T> (reference exec/engine.hpp:176-300)
 * for dtype 0 f64, 2 i64, 3 i32, 4 u64, 5 u32.  kind: 0 WindowDelta, 1
 * WindowSum, 2 WindowMean, 3 WindowStdDev, 4 WindowVariance, 5
 * WindowQuantile (quantile in [0, 1]; the first min(window, 128) values of
 * each window).  Every window is evaluated in the reference's operation
 * order (left-to-right sums in T, one rounding per operation), so outputs are
 * bit-identical.  Returns the number of outputs written, as the reference
 * does (0 for an empty or invalid request); the _dev form stores it in
 * *n_out and returns a status.
 * voxel_time_window_sum: TimeWindowSum (228-241): out[(ts[i] - start) /
 * duration] += values[i] for buckets in [0, out_len) (out is added to, not
 * cleared); returns the largest bucket touched + 1.  f64 bucket sums are
 * added in parallel (within 1e-12 of the reference's row order); integers
 * are exact.
 * ================================================================ */
size_t    voxel_window(int dtype, int kind, const void* data, size_t count, void* out, size_t out_len,
                       uint8_t window, double quantile);
int       voxel_window_dev(int dtype, int kind, const void* d_data, size_t count, void* d_out, size_t out_len,
                           uint8_t window, double quantile, size_t* n_out, void* stream);
size_t    voxel_time_window_sum(int dtype, const int64_t* timestamps, const void* values, size_t count,
                                int64_t start_time, int64_t duration, void* out, size_t out_len);
int       voxel_time_window_sum_dev(int dtype, const int64_t* d_timestamps, const void* d_values, size_t count,
                                    int64_t start_time, int64_t duration, void* d_out, size_t out_len,
                                    size_t* n_out, void* stream);

/* ================================================================
 * Additive: delta and frame-of-reference codecs.
 * DeltaEncoding<T> (reference data/encoding.hpp:281-354), T an integer type
 * (dtype 2 i64, 3 i32, 4 u64, 5 u32; base_bits = BaseValue's bits):
 *   decode: out[i] = base + deltas[0] + ... + deltas[offset + i], wrapping in
 *   T, for i < count and offset + i < n (DecodeBatch, 317-330); outputs past n
 *   are not written.  encode: deltas[i] = data[i] - data[i-1], data[-1] = 0
 *   (Build, 292-306; BaseValue 0).
 * FrameOfReferenceEncoding (encoding.hpp:456-521), f64 values as i32 codes:
 *   decode: out[i] = base + (double)code[offset + i] * scale, one rounding per
 *   operation, for offset + i < n (DecodeBatch, 489-500).  encode: base = min,
 *   scale = (max - min) / INT32_MAX (1 when max == min), code =
 *   (int32)llround((x - base) / scale) (Build, 461-482); NaN-free columns.
 * Return 0 or a VOXEL_E* code.
 * ================================================================ */
int       voxel_delta_decode(int dtype, const void* deltas, size_t n, uint64_t base_bits, size_t offset,
                             size_t count, void* out);
int       voxel_delta_decode_dev(int dtype, const void* d_deltas, size_t n, uint64_t base_bits, size_t offset,
                                 size_t count, void* d_out, void* stream);
int       voxel_delta_encode(int dtype, const void* data, size_t n, void* deltas);
int       voxel_delta_encode_dev(int dtype, const void* d_data, size_t n, void* d_deltas, void* stream);
int       voxel_for_decode_f64(const int32_t* code, size_t n, double base, double scale, size_t offset,
                               size_t count, double* out);
int       voxel_for_decode_f64_dev(const int32_t* d_code, size_t n, double base, double scale, size_t offset,
                                   size_t count, double* d_out, void* stream);
int       voxel_for_encode_f64(const double* data, size_t n, int32_t* code, double* base, double* scale);
/* base / scale are host outputs; the call synchronises `stream` once (min / max) */
int       voxel_for_encode_f64_dev(const double* d_data, size_t n, int32_t* d_code, double* base, double* scale,
                                   void* stream);
int       voxel_dict_bitpack_decode_i32_dev(const uint64_t* d_words, size_t nwords, uint32_t width,
                                            const int32_t* d_dict, size_t card, size_t value_count,
                                            size_t offset, size_t count, int32_t* d_out, void* stream);
int       voxel_dict_decode_dev(int dtype, const void* d_dict, size_t card, const uint32_t* d_indices,
                                size_t count, void* d_out, void* stream);

/* ================================================================
 * Additive: fused scan + group-by (decode key, two predicates, group SUM of a
 * product, COUNT, MIN, MAX).  Groups come out sorted by key; returns the
 * group count or (size_t)-1.  Dictionaries of up to 4,096 entries aggregate
 * in shared-memory tables; larger ones (up to 2^26 entries) keep their
 * frequent groups in per-block shared-memory slot caches, send the other rows
 * to an HBM table with reductions, and compact the groups with a second
 * kernel (the same exact integers: identical results).
 *   key = dict[unpack(packed_key)], WHERE price > price_gt AND
 *   qty BETWEEN qty_lo AND qty_hi, GROUP BY key:
 *   SUM(price*qty) (one rounded multiply), COUNT(*), MIN(price), MAX(price)
 * ================================================================ */
size_t    voxel_scan_groupby(const uint64_t* packed_key, size_t nwords, uint32_t width,
                             const int32_t* dict, size_t card, const double* price,
                             const int32_t* qty, size_t n, double price_gt, int32_t qty_lo,
                             int32_t qty_hi, int32_t* out_keys, double* out_sum, double* out_min,
                             double* out_max, uint64_t* out_count);
/* kernel variant of the calling thread's fused scan:
 *   -1 = default: the autotuner times variants 1, 2, 3, 5, 7 and 9 on the first
 *        call of each (dictionary size, row count) of 65,536 rows or more and
 *        keeps the fastest (1 for smaller scans and when tuning is off);
 *    1 / 2 = 32-bit-word group table fed by a per-warp row queue, 4 / 8 rows
 *        per thread (1 is the default);
 *    3 / 5 = 32-bit-word group table, rows added where read, 4 / 8 rows per thread;
 *    6 = 32-bit-word group table fed by bulk copies into shared-memory stages
 *        (a producer warp keeps them in flight while 16 warps aggregate); needs
 *        16-byte-aligned packed keys, at least 2048 rows, at most 2^19 rows per
 *        SM and a table that fits beside two stages, else runs variant 1;
 *    7 = lean word table: 16-byte queue entries, MIN / MAX screened by the
 *        high 32 bits of the order keys (scans of fewer than 2^32 rows; else 1);
 *    9 = variant 1 with each block's next tile of price / qty loaded into
 *        registers while the current one is filtered and aggregated (two
 *        blocks per SM);
 *    4 / 8 / 16 = warp-merged rows, 192-bit shared atomics, that many rows per thread;
 *    0 = TMA-fed private warp tables (dictionaries up to 1024 entries).
 * All but 0 give bit-identical results; the autotuner also times 7.
 * voxel_scan_groupby_last_variant reports the kernel the last call ran: 0
 * warp-merged, 1 TMA-fed, 2 word table with queue, 3 word table direct, 4
 * word table fed by bulk copies, 5 lean word table, 6 the slot caches and
 * HBM table of dictionaries above 4096 entries, 7 the prefetching word table. */
int       voxel_scan_groupby_tune(int variant);
int       voxel_scan_groupby_last_variant(void);
/* the calling thread's current variant id (as passed to voxel_scan_groupby_tune) */
int       voxel_scan_groupby_tune_state(void);
/* Errors of the device-pointer fused scan.  The kernels OR bits into a device
 * status word: 1 = a price*qty product not finite or beyond 2^63, 2 = a packed
 * key index outside the dictionary, 4 = a bounded wait ran out (the bulk
 * copies of variants 0 and 6, the tile look-back of the large-dictionary
 * path; the group rows are then partial).
 * voxel_scan_groupby_check synchronises `stream`, reads and clears the calling
 * thread's status word of voxel_scan_groupby_dev and returns VOXEL_OK, or
 * VOXEL_ETIMEOUT (bit 4), VOXEL_EINVAL (bit 2), VOXEL_EOVERFLOW (bit 1), with
 * voxel_last_error() set.  voxel_scan_groupby_status_code maps a status word
 * the caller read itself (the *d_status of voxel_scan_groupby_noalloc_dev) the
 * same way. */
int       voxel_scan_groupby_check(void* stream);
int       voxel_scan_groupby_status_code(int status_word);
/* Autotuner (no reference counterpart): kernel families with several
 * equivalent configurations (the fused scan's variants, the radix sort's
 * keys per thread) time them on the first call of each (GPU, element type,
 * log2 size) and cache the fastest in a JSON file: $VOXEL_TUNE_CACHE, else
 * tune_cache.json beside this library.  VOXEL_TUNE=0 (or enable(0)) uses
 * each family's default.  lookup returns the cached choice or -1. */
void      voxel_tune_enable(int on);
void      voxel_tune_set_cache_path(const char* path);
void      voxel_tune_clear(void);
int       voxel_tune_lookup(const char* family, int dtype, size_t n);
int       voxel_scan_groupby_dev(const uint64_t* d_packed_key, size_t nwords, uint32_t width,
                                 const int32_t* d_dict, size_t card, const double* d_price,
                                 const int32_t* d_qty, size_t n, double price_gt, int32_t qty_lo,
                                 int32_t qty_hi, int32_t* d_keys, double* d_sum, double* d_min,
                                 double* d_max, uint64_t* d_count, uint64_t* d_ngroups,
                                 void* stream);

/*
 * Allocation-free variant of voxel_scan_groupby_dev (no counterpart in the
 * reference; added for callers that must not allocate device memory, e.g. a
 * host that has handed all device memory to its own pool and forbids the
 * library from calling cudaMalloc/cudaFree, or a caller on a latency-critical
 * path where an allocation could block).  Same inputs, outputs and results as
 * voxel_scan_groupby_dev (bit-identical), always with the shared-atomic kernel.
 *
 * - Allocates nothing: the group table (the only scratch) is a fixed
 *   196,864-byte device array inside libvoxel_c.so, sized for the largest
 *   dictionary, card <= 4096 groups.  A larger card returns VOXEL_EINVAL with
 *   a message; nothing is launched.
 * - The first call on each device does a one-time setup (finds the array's
 *   address, sets its min keys, waits for that on `stream`); make the first
 *   call before any stream capture.  Later calls only enqueue the kernel.
 * - *d_status is caller-owned device memory that must be 0 before the call;
 *   the kernel ORs in 1 (a price*qty product not finite or beyond 2^63) or 2
 *   (a packed key index outside the dictionary).  Output buffers need no
 *   clearing.
 * - The table is shared by every call on a device: calls that overlap in time
 *   (different streams or threads, same device) race and give wrong results;
 *   calls queued on one stream are fine.  Each launch leaves the table ready
 *   for the next.
 */
int       voxel_scan_groupby_noalloc_dev(const uint64_t* d_packed_key, size_t nwords, uint32_t width,
                                         const int32_t* d_dict, size_t card, const double* d_price,
                                         const int32_t* d_qty, size_t n, double price_gt,
                                         int32_t qty_lo, int32_t qty_hi, int32_t* d_keys,
                                         double* d_sum, double* d_min, double* d_max,
                                         uint64_t* d_count, uint64_t* d_ngroups, int* d_status,
                                         void* stream);

/* ================================================================
 * Additive: GROUP BY over explicit keys (HashAggregator semantics,
 * aggregate.hpp:159-301): per key SUM (compensated f64), MIN, MAX, COUNT,
 * groups sorted by key.  Returns the group count or (size_t)-1.
 * ================================================================ */
size_t    voxel_groupby_i32_f64(const int32_t* keys, const double* values, size_t n,
                                size_t expected_groups, int32_t* out_keys, double* out_sum,
                                double* out_min, double* out_max, uint64_t* out_count);
size_t    voxel_groupby_u32_f64(const uint32_t* keys, const double* values, size_t n,
                                size_t expected_groups, uint32_t* out_keys, double* out_sum,
                                double* out_min, double* out_max, uint64_t* out_count);
/* GROUP BY over device columns with a chosen plan: method 0 = HashAggregator
 * sized for expected_groups (grown if too small), 1 = sort-based
 * (GroupedAggregator over radix-sorted keys).  Outputs are bit-identical
 * either way (groups in key order); *ngroups (host) = the group count. */
int       voxel_groupby_u32_f64_dev(const uint32_t* d_keys, const double* d_values, size_t n,
                                    size_t expected_groups, int method, uint32_t* d_keys_out, double* d_sum,
                                    double* d_min, double* d_max, uint64_t* d_count, uint64_t* ngroups,
                                    void* stream);
/* the voxel_agg_* object: device-pointer accumulate, and its groups sorted by key */
int       voxel_agg_accumulate_dev(void* agg, const uint32_t* d_keys, const double* d_values, size_t count,
                                   void* stream);
size_t    voxel_agg_results(void* agg, uint32_t* keys, double* sum, double* min, double* max,
                            uint64_t* count);
/* the voxel_dict_* object's sorted dictionary (returns the cardinality) */
size_t    voxel_dict_values(const void* dict, double* out);
/* GroupedAggregator over pre-sorted keys (aggregate.hpp:665-706) */
size_t    voxel_grouped_sorted_i32_f64(const int32_t* sorted_keys, const double* values,
                                       size_t n, int32_t* out_keys, double* out_sum,
                                       double* out_min, double* out_max, uint64_t* out_count);

/* ================================================================
 * Additive: stable LSD radix sort of keys with a u32 payload
 * (RadixSort<T>::Sort, sort.hpp:83-160).  keys and idx are sorted in place.
 * dtype in {2 i64, 3 i32, 4 u64, 5 u32}.
 * ================================================================ */
int       voxel_radix_sort(int dtype, void* keys, uint32_t* idx, size_t n);
int       voxel_radix_sort_dev(int dtype, void* d_keys, uint32_t* d_idx, size_t n,
                               void* d_tmp, size_t tmp_bytes, void* stream);
size_t    voxel_radix_sort_tmp_bytes(int dtype, size_t n);

/* ================================================================
 * Additive: merge, semi and anti joins (reference ops/join.hpp:216-310) over
 * integer keys (dtype 2 i64, 3 i32, 4 u64, 5 u32); row ids are u32.
 * voxel_merge_join: MergeJoin<TKey> over keys sorted ascending.  unique = 0:
 *   Join (218-244), every (left, right) pair of equal keys, left-major with
 *   right rows ascending; unique = 1: JoinUnique (246-268), the t-th left row
 *   of a key pairs with the t-th right row of that key.  Writes at most
 *   max_matches pairs and returns how many it wrote ((size_t)-1 on error);
 *   the _dev form writes {written, all matches} to d_count2.
 * voxel_semi_join: SemiJoin (294-310, anti = 0) / AntiJoin (273-290, anti =
 *   1): the ascending left row ids whose key is / is not among the right keys
 *   (no order assumed); out holds nl entries; returns the count.
 * ================================================================ */
size_t    voxel_merge_join(int dtype, const void* left, size_t nl, const void* right, size_t nr,
                           uint32_t* left_out, uint32_t* right_out, size_t max_matches, int unique);
int       voxel_merge_join_dev(int dtype, const void* d_left, size_t nl, const void* d_right, size_t nr,
                               uint32_t* d_left_out, uint32_t* d_right_out, size_t max_matches, int unique,
                               uint64_t* d_count2, void* stream);
/* the pairs of a join built on the left side (d_probe = right rows, d_build =
 * left rows) in the order of the join built on the right: left rows
 * ascending, each one's right rows descending (ProbeAllMatches order) */
int       voxel_join_pairs_swap_order_dev(const uint32_t* d_probe, const uint32_t* d_build, size_t m,
                                          uint32_t* d_left, uint32_t* d_right, void* stream);
size_t    voxel_semi_join(int dtype, const void* left, size_t nl, const void* right, size_t nr, uint32_t* out,
                          int anti);
int       voxel_semi_join_dev(int dtype, const void* d_left, size_t nl, const void* d_right, size_t nr,
                              uint32_t* d_out, int anti, uint64_t* d_count, void* stream);

/* ================================================================
 * Additive: hash join on i64 keys (HashJoin<TKey>, join.hpp:36-165).
 * Pairs (probe_idx, build_idx) in ascending probe order; for equal build
 * keys the newest build row comes first (the reference's LIFO chains).
 * all=0 keeps the first match only (Probe), all=1 every match
 * (ProbeAllMatches).  Returns the pair count or (size_t)-1.
 * ================================================================ */
size_t    voxel_hashjoin_i64(const int64_t* build, size_t nb, const int64_t* probe, size_t np,
                             uint32_t* left, uint32_t* right, size_t max_matches, int all);
/* count + u64 SUM(build payload) + pairs, device pointers */
int       voxel_hashjoin_i64_dev(const int64_t* d_build, const uint64_t* d_payload, size_t nb,
                                 const int64_t* d_probe, size_t np, uint32_t* d_left,
                                 uint32_t* d_right, size_t max_matches, int all,
                                 uint64_t* d_count_sum, void* stream);

/* ================================================================
 * Additive: batched persistent executor.  Many single-column filter /
 * aggregate programs over device-resident columns run in ONE persistent
 * launch (a device work queue of (program, tile) items), optionally replayed
 * from a captured CUDA graph.  Each program can also emit its selection
 * vector (ascending row ids satisfying all of its predicates) into a caller
 * buffer of a given capacity; a program whose selection does not fit is
 * flagged (its exact count is still reported) and can be re-run.
 * ================================================================ */
void*     voxel_batch_create(void);
void      voxel_batch_destroy(void* batch);
size_t    voxel_batch_size(const void* batch);
/* regs64: the 64 registers before the run; returns a status */
int       voxel_batch_add(void* batch, int dtype, const uint32_t* code, size_t len, const uint64_t* regs64,
                          const void* d_col, size_t count, int want_selection, size_t sel_capacity,
                          uint32_t* d_sel);
int       voxel_batch_set_capacity(void* batch, size_t prog, size_t capacity, uint32_t* d_sel);
int       voxel_batch_launch(void* batch, int use_graph, void* stream);
int       voxel_batch_fetch(void* batch, void* stream);
/* after fetch: the program's 64 registers, exact selected-row count, overflow
 * flag (0: the selection fit; 1: rows past the capacity went to the spill
 * arena, voxel_batch_gather_overflow assembles them; 2: some did not fit the
 * arena either, re-run the program) */
int       voxel_batch_result(const void* batch, size_t prog, uint64_t* regs64, uint64_t* sel_count,
                             int* overflow);
/* after fetch: every program at once (regs64: 64 per program; any pointer may be NULL) */
int       voxel_batch_results_all(const void* batch, uint64_t* regs64, uint64_t* sel_counts, int* overflows);
/* how the executor runs program `prog`: 0 = interpreted atoms, 1..8 = range
 * form (predicate rewritten as lo <= x <= hi with up to two excluded values;
 * 1 + 2 * reduction kind SUM/COUNT/MIN/MAX + excluded values present);
 * -1 for an invalid index */
int       voxel_batch_form(const void* batch, size_t prog);
/* rows past a program's selection capacity go to a spill arena of `rows`
 * entries (default 2^24); takes effect at the next launch */
int       voxel_batch_set_spill_capacity(void* batch, size_t rows);
/* after fetch: the whole selection of each overflowed program progs[k] (its
 * exact count of rows) into d_pool at offset count[progs[0]] + ... +
 * count[progs[k-1]], from its buffer and its spilled rows; VOXEL_ECAPACITY if
 * a listed program's rows did not all fit the spill arena (re-run those) */
int       voxel_batch_gather_overflow(void* batch, size_t n, const size_t* progs, uint32_t* d_pool,
                                      void* stream);
/* after fetch: re-run programs progs[0..n) (e.g. those that overflowed) with
 * selection capacities capacities[k], writing program k's row ids at
 * d_pool + capacities[0] + ... + capacities[k-1]; one launch from the
 * programs' already-lowered descriptors; their results then replace the
 * fetched ones (voxel_batch_result / _results_all) */
int       voxel_batch_rerun(void* batch, size_t n, const size_t* progs, const size_t* capacities,
                            uint32_t* d_pool, void* stream);

/* ================================================================
 * Additive: serving loop (no reference counterpart).  Requests arrive from
 * any thread; programs are batched continuously (each batch is one launch of
 * the batched executor, prepared while the previous one runs), group-by and
 * join requests run concurrently on a second stream, and every request is
 * admitted only when its estimated device working memory fits what is left
 * of `budget_bytes`.  Columns, keys, values and output buffers are caller
 * device memory that must stay valid until the request completes.
 * submit_* return a request id (0 on error: voxel_last_error says why, e.g.
 * VOXEL_ECAPACITY for a request larger than the whole budget).  result()
 * copies a completed request's outputs and forgets it:
 *   program:  regs64 = the 64 registers after the run, *count = selected
 *             rows, *aux = 1 if the selection overflowed its capacity;
 *   group-by: *count = groups written (sorted by key) to the host arrays;
 *   join:     *count = pairs written, *aux = u64 SUM of payload over them.
 * stats(): requests completed since the last reset, latency percentiles
 * (submission to completion, ms) and the peak reserved working memory.
 * ================================================================ */
void*     voxel_server_create(size_t budget_bytes, uint32_t max_batch);
void      voxel_server_destroy(void* server);
uint64_t  voxel_server_submit_program(void* server, int dtype, const uint32_t* code, size_t len,
                                      const uint64_t* regs64, const void* d_col, size_t count,
                                      int want_selection, size_t sel_capacity, uint32_t* d_sel);
uint64_t  voxel_server_submit_groupby(void* server, const uint32_t* d_keys, const double* d_values,
                                      size_t n, size_t expected_groups, size_t out_capacity,
                                      uint32_t* out_keys, double* out_sum, double* out_min,
                                      double* out_max, uint64_t* out_count);
uint64_t  voxel_server_submit_join(void* server, const int64_t* d_build, const uint64_t* d_payload,
                                   size_t nb, const int64_t* d_probe, size_t np, uint32_t* d_left,
                                   uint32_t* d_right, size_t capacity);
int       voxel_server_wait(void* server, uint64_t id, double timeout_s);
int       voxel_server_result(void* server, uint64_t id, uint64_t* regs64, uint64_t* count,
                              uint64_t* aux, double* latency_ms);
int       voxel_server_stats(void* server, uint64_t* completed, double* p50_ms, double* p99_ms,
                             double* mean_ms, uint64_t* peak_bytes);
void      voxel_server_reset_stats(void* server);
/* Mean milliseconds a completed request of `kind` (0 program, 1 group-by,
 * 2 join) spent in the arrival queue and in service since the last reset. */
int       voxel_server_breakdown(void* server, int kind, double* queue_ms, double* service_ms,
                                 uint64_t* completed);
/* Program batches since the last reset: how many, their programs, the largest,
 * the host milliseconds spent lowering + uploading + launching them (total and
 * the longest) and waiting for their results. */
int       voxel_server_batch_stats(void* server, uint64_t* batches, uint64_t* programs, uint64_t* max_batch,
                                   double* build_ms, double* max_build_ms, double* wait_ms);

/* ================================================================
 * Additive: learned cardinality / selectivity estimator.
 * Column sketches are computed on the device (min / max, 64-bucket
 * equi-width histogram, HyperLogLog p = 12); the FP32 MLP
 * (48 -> 64 -> 64 -> 64 -> 2, 11,586 parameters) is trained and evaluated by
 * the backend's own kernels.  Estimates only size buffers and pick plans.
 * ================================================================ */
typedef struct {
    uint64_t n;
    double min, max;
    uint64_t hist[64];
    uint8_t hll[4096];
} voxel_column_sketch;

/* up to 4 conjunctive "value op threshold" atoms (threshold as T bits) */
typedef struct {
    int32_t natoms;
    int32_t op[4];
    int32_t pad;
    uint64_t thr[4];
} voxel_pred_set;

int       voxel_sketch_column_dev(int dtype, const void* d_col, size_t n, voxel_column_sketch* out);
/* exact selected-row and distinct-selected-value counts for each predicate set */
int       voxel_exact_labels_dev(int dtype, const void* d_col, size_t n, const voxel_pred_set* sets,
                                 uint32_t nsets, uint64_t* rows, uint64_t* distinct);
size_t    voxel_mlp_param_count(void);
void*     voxel_mlp_create(uint64_t seed);
void      voxel_mlp_destroy(void* mlp);
int       voxel_mlp_set_params(void* mlp, const float* params);
int       voxel_mlp_get_params(const void* mlp, float* params);
/* gradient (summed over the samples) of the squared error and the loss, on the host */
int       voxel_mlp_grad(void* mlp, const float* d_x, const float* d_y, const uint32_t* d_idx, uint32_t count,
                         float* grad, float* loss);
/* one Adam step on the minibatch d_idx[0..count) of (d_x [N x 48], d_y [N x 2]) */
int       voxel_mlp_train_step(void* mlp, const float* d_x, const float* d_y, const uint32_t* d_idx,
                               uint32_t count, float lr);
int       voxel_mlp_infer(void* mlp, const float* d_x, size_t n, float* d_y, void* stream);

#ifdef __cplusplus
}
#endif
