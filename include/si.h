/*
 * si.h -- C ABI of the B200 set-intersection engine (libsi_b200.so).
 *
 * The reference (chribell/set_intersection) exposes no library: each technique
 * is a standalone executable whose hot path is a host loop that launches
 * sm_61 kernels on a dataset already copied to the device.  Each entry point
 * below replaces one such hot path and is what a per-technique executable (or
 * any other host code) calls instead of the reference's kernels; the cited
 * file:line ranges are the reference code each one replaces.
 *
 * Conventions
 *  - All set pointers are DEVICE pointers to ascending, duplicate-free uint32
 *    arrays (the reference assumes this and never checks it; si_validate_sorted
 *    checks it on the device).  They must be 4-byte aligned.
 *  - Everything is stream-ordered on the given stream (NULL = legacy default
 *    stream) and asynchronous; nothing synchronises unless documented.
 *  - The library never allocates device memory on these paths: scratch comes
 *    from the caller as a workspace of the size the matching *_workspace_size
 *    function returns.  It never calls exit().
 *  - Device-detected problems (unsorted input, a bounded wait that gave up,
 *    output overflow) are recorded in the workspace's error word;
 *    si_workspace_check reads it back.
 *  - Counts of one pair are uint32 as in the reference, except the single-pair
 *    (SISI) count, which is uint64.
 */
#ifndef SI_B200_H
#define SI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same handle as cudaStream_t. */
typedef struct CUstream_st* si_stream_t;

typedef enum si_status {
    SI_OK = 0,
    SI_ERR_INVALID_ARGUMENT = 1,   /* bad pointer, size or enum value (host-side check) */
    SI_ERR_WORKSPACE_TOO_SMALL = 2,
    SI_ERR_CUDA = 3,               /* a CUDA runtime call failed; see si_last_error_string */
    SI_ERR_UNSUPPORTED = 4,        /* technique not available for this entry point */
    SI_ERR_TIMEOUT = 5,            /* a bounded device-side wait gave up (device error word) */
    SI_ERR_INVALID_INPUT = 6,      /* a set is not strictly increasing (device error word) */
    SI_ERR_OUTPUT_OVERFLOW = 7     /* materialised output exceeded out_cap (device error word) */
} si_status;

/* Techniques: one per reference executable (CMakeLists.txt:56-160). */
typedef enum si_technique {
    SI_TECH_IP = 0,            /* intersect-path merge partitioning      (src/ip.cu) */
    SI_TECH_OBS = 1,           /* optimized binary search, cached tree   (src/obs.cu) */
    SI_TECH_HI = 2,            /* hash intersection                      (src/hi.cu) */
    SI_TECH_BITMAP = 3,        /* dynamic bitmap probe                   (src/bitmap_dynamic.cu) */
    SI_TECH_BITMAP_NAIVE = 4,  /* all-set bitmaps, plain AND-popcount    (src/bitmap_naive.cu) */
    SI_TECH_MM = 5,            /* incidence-matrix product               (src/matrix_multiplication.cu) */
    SI_TECH_AUTO = 6           /* the engine picks per input */
} si_technique;

const char* si_version(void);
const char* si_status_string(si_status s);
/* Text of the last CUDA error seen by this thread (empty if none). */
const char* si_last_error_string(void);

/* ------------------------------------------------------------------ SISI --
 * One pair: count |A ∩ B| and optionally write the sorted elements of A ∩ B.
 *
 * Replaces the single-instance path of the GPU executables: src/ip.cu:141-177
 * (findDiagonals + intersectPath for the one pair of a 2-set file),
 * src/obs.cu:180-229 and src/hi.cu:205-245 with --path (intersectPathOBS,
 * intersectPathHI), src/bitmap_dynamic.cu:168-176 (constructBitmap +
 * singleInstanceIntersect + thrust::reduce).  The reference writes only the
 * count; element output is this engine's addition, ordered as
 * std::set_intersection orders it.
 *
 * Techniques: IP merges the two sets tile by tile (value-pivot tiles of <= 6144
 * elements per set, both sets streamed once); HI streams them like BITMAP
 * below, but each window of 512 elements of the smaller set goes into a
 * warp-private hash table that the larger set's elements probe; BITMAP streams
 * the larger set in equal ranges, one warp per range, with the matching part
 * of the smaller set, through windows of 32768 values (two bitmaps per warp,
 * AND and popcount), and orders the output by a scan of the range counts,
 * through a scratch array as long as the smaller set (so its workspace is
 * about 4 min(nA, nB) bytes larger); OBS searches every element of the smaller set in the larger one
 * (cached top levels in shared memory); AUTO takes OBS when one set is more
 * than 64 times larger than the other, else BITMAP.
 *
 * d_count: device uint64, receives |A ∩ B|.
 * d_out:   device uint32[out_cap] or NULL (count only).  When non-NULL,
 *          out_cap must be >= min(nA, nB).
 */
size_t si_sisi_workspace_size(uint64_t nA, uint64_t nB, si_technique t);
si_status si_sisi(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB,
                  si_technique t, uint64_t* d_count, uint32_t* d_out, uint64_t out_cap,
                  void* d_workspace, size_t workspace_bytes, si_stream_t stream);

/* Single pair from HOST buffers: copies A and B to the device, intersects
 * them and copies the count and (when h_out is non-NULL) the sorted elements
 * back; returns when *count and h_out are final.  The path of the reference's
 * executables for a 2-set file (src/ip.cu:129-177: the dataset copied with
 * cudaMemcpy, the kernels, the count copied back), as one call.
 *
 * The pair is cut into `chunks` value ranges (0: 8 for pairs of 2^22 elements
 * or more, else 1; at most 64) that are pipelined: one range's sets are copied
 * up while the previous range is intersected and the elements of earlier
 * ranges are copied down, so with pinned host buffers the call costs about the
 * host-to-device copy.  A pageable input is staged through pinned buffers of
 * the context: host threads copy 16 MiB pieces into them while the DMA engine
 * moves the previous pieces up.
 *
 * d_workspace: device, 256-byte aligned, of si_sisi_host_workspace_size bytes
 * (it holds the device copies of both sets, the output and the per-range
 * si_sisi workspace).  h_out: host uint32[out_cap], out_cap >= min(nA, nB).
 * Technique t as in si_sisi (AUTO picks per range). */
size_t si_sisi_host_workspace_size(const uint32_t* hA, uint64_t nA, const uint32_t* hB, uint64_t nB,
                                   si_technique t, uint32_t chunks);
si_status si_sisi_host(const uint32_t* hA, uint64_t nA, const uint32_t* hB, uint64_t nB, si_technique t,
                       uint32_t chunks, uint64_t* count, uint32_t* h_out, uint64_t out_cap,
                       void* d_workspace, size_t workspace_bytes, si_stream_t stream);

/* The same call with its host-side resources made once: a si_host_ctx holds
 * the two copy streams, the per-range events and the pinned words that each
 * range's count and error word land in.  si_sisi_host creates and destroys one
 * per call; a caller that intersects many pairs creates one
 * (si_host_ctx_create, on the device that is current then) and passes it to
 * every si_sisi_host_ctx call on that device, which then creates, allocates
 * and frees nothing (the staging buffers for pageable inputs, 64 MiB of pinned
 * memory and a pool of up to 8 copy threads, are made at the first call that
 * needs them and kept).  Calls sharing a context must not overlap (one host
 * thread at a time).  Errors recorded on the device by any range are reported
 * (the first one); a set that descends across a range boundary is reported as
 * SI_ERR_INVALID_INPUT before anything is launched. */
typedef struct si_host_ctx si_host_ctx;
si_status si_host_ctx_create(si_host_ctx** out);
void si_host_ctx_destroy(si_host_ctx* ctx);
si_status si_sisi_host_ctx(si_host_ctx* ctx, const uint32_t* hA, uint64_t nA, const uint32_t* hB, uint64_t nB,
                           si_technique t, uint32_t chunks, uint64_t* count, uint32_t* h_out, uint64_t out_cap,
                           void* d_workspace, size_t workspace_bytes, si_stream_t stream);

/* Single pair without any caller-provided scratch.  No counterpart in the
 * reference (whose executables cudaMalloc everything themselves).
 *
 * For callers that cannot allocate device memory: FFI hosts (cgo, JNI, ctypes)
 * that receive device buffers from another runtime and have no CUDA allocator
 * of their own, engines whose memory manager already owns the whole HBM
 * budget, and paths where cudaMalloc/cudaFree would synchronise the device.
 * Same kernels and results as si_sisi with SI_TECH_IP; the caller passes only
 * inputs and outputs, and the call allocates nothing.
 *
 * Scratch is a fixed 4 MiB array in device memory owned by the library (held
 * by every GPU that loads it, until the process exits), enough for any pair
 * with |A| + |B| <= 2^29 elements; larger pairs are rejected with
 * SI_ERR_WORKSPACE_TOO_SMALL before anything is launched.  The first call on a
 * device looks up the array's device address (issue it before any stream
 * capture).  All calls share the array: calls that may overlap on the GPU
 * (e.g. on unordered streams) race and must not be issued.  A call returns
 * only the host-side status; what its kernels record on the device (input
 * that is not strictly increasing, a bounded wait that gave up) stays in the
 * array's error word until the next call clears it: si_sisi_noalloc_check
 * reads it. */
si_status si_sisi_noalloc(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB,
                          uint64_t* d_count, uint32_t* d_out, uint64_t out_cap, si_stream_t stream);
/* Synchronises the stream and returns the error that the last si_sisi_noalloc
 * call on this device recorded on the device (SI_OK if none).  Allocates
 * nothing.  No counterpart in the reference. */
si_status si_sisi_noalloc_check(si_stream_t stream);

/* Synchronises the stream and returns the error recorded in a workspace by the
 * last call that used it (SI_OK if none). */
si_status si_workspace_check(const void* d_workspace, si_stream_t stream);

/* Same, plus where on the device the error was recorded (site: an id of the
 * bounded wait or check that gave up; detail: site-specific, e.g. a tile). */
si_status si_workspace_diagnostic(const void* d_workspace, si_stream_t stream, uint32_t* site, uint32_t* detail);

/* Self-test of the engine's bounded device waits (every wait of every kernel
 * gives up after a time limit, records SI_ERR_TIMEOUT with a site id in the
 * workspace's error word and lets its kernel end).  One thread waits on an
 * mbarrier phase that nothing completes, for limit_ns (<= 4 s); synchronises
 * the stream and returns the error word: SI_ERR_TIMEOUT when the wait gave up
 * as it should.  d_workspace: >= 16 bytes, 16-byte aligned. */
si_status si_wait_selftest(void* d_workspace, uint64_t limit_ns, si_stream_t stream);

/* Device-side check that x[0..n) is strictly increasing.  Writes 1 (ok) or 0
 * to d_flag (device uint32).  No workspace. */
si_status si_validate_sorted(const uint32_t* d_x, uint64_t n, uint32_t* d_flag, si_stream_t stream);

/* ------------------------------------------------------------------ MISI --
 * All pairs between two ranges of sets of a collection (one tile pair of the
 * reference's MISI loop, include/util.hpp:24-52).
 *
 * d_elements / d_offsets: the collection in CSR form on the device (set i is
 * d_elements[d_offsets[i] .. d_offsets[i+1]), sets ascending and duplicate
 * free, each below 2^32 elements).  A, B: set ranges [start, end).
 *  - A == B (self-join tile): every pair a < b of the range;
 *    counts[tri(stride, a - A.start, b - A.start)], tri = include/util.hpp:68-70.
 *  - A != B (cross tile, disjoint ranges): every pair (a in A, b in B);
 *    counts[(a - A.start) * stride + (b - B.start)] (include/util.hpp:72-74).
 * stride is the reference's numOfSets: the cardinality for the single-tile
 * run (A = B = {0, k}), else the partition size.  Every count of the tile is
 * written (zero for pairs with an empty set).
 *
 * Replaces the per-run kernels of src/ip.cu:141-177 (findDiagonals +
 * intersectPath), src/obs.cu:275-438 (warpBasedOBS / blockBasedOBS),
 * src/hi.cu:295-420 (warpBasedHI / blockBasedHI) and
 * src/bitmap_dynamic.cu:240-319.  t: IP, OBS, HI, BITMAP or AUTO (= BITMAP).
 * MM and BITMAP_NAIVE are served by si_misi_dense (single-tile run only).
 */
typedef struct si_set_range { uint32_t start, end; } si_set_range;
size_t si_misi_workspace_size(si_set_range A, si_set_range B, si_technique t);
si_status si_misi(const uint32_t* d_elements, const uint64_t* d_offsets, si_set_range A, si_set_range B,
                  uint64_t stride, si_technique t, uint32_t* d_counts, void* d_workspace, size_t workspace_bytes,
                  si_stream_t stream);

/* --------------------------------------------------------- batched pairs --
 * Counts of a list of pairs of one collection, in one persistent launch.  No
 * counterpart in the reference, which launches kernels per pair
 * (src/ip.cu:141-177); this is the batched form of the single-pair count.
 *
 * d_pairs: device uint32[2 * npairs], pair p = (d_pairs[2p], d_pairs[2p+1]),
 * set indices < k.  d_counts: device uint32[npairs], counts[p] = |S_a ∩ S_b|.
 * One technique for every pair: t = SI_TECH_IP (streaming merge), SI_TECH_OBS
 * (binary search of the smaller set in the larger), SI_TECH_HI (the smaller
 * set hashed in windows of 1024 elements, the larger probing) or
 * SI_TECH_BITMAP (AND of two bitmaps per window of 16384 values).
 * SI_TECH_AUTO: per bucket from `table` (host uint8[SI_BATCH_TABLE_SIZE] of
 * SI_BATCH_* codes; a code >= SI_BATCH_CODES counts as merge), or, with
 * table == NULL, search when l >= 16 s and hash otherwise.
 *   bucket = (d << 8) | (min(15, log2 s) << 4) | min(15, log2(l / s)),
 * s <= l the two sizes, d the larger set's density class: its mean gap
 * (last - first) / (l - 1) below 4, 32, 256 or larger (d = 0..3; 3 when
 * l < 2).  The hash and bitmap techniques run a pair whose larger set has
 * 2^32 - 1024 elements or more by merge.  npairs < 2^32.
 */
#define SI_BATCH_TABLE_SIZE 1024
enum {
    SI_BATCH_MERGE = 0,       /* streaming merge                              (src/ip.cu) */
    SI_BATCH_SEARCH = 1,      /* binary search of the smaller set             (src/obs.cu) */
    SI_BATCH_HASH_1024 = 2,   /* smaller set hashed, windows of 1024 elements (src/hi.cu) */
    SI_BATCH_HASH_512 = 3,    /* the same, windows of 512 elements */
    SI_BATCH_BITMAP_16K = 4,  /* window bitmaps of 16384 values               (src/bitmap_dynamic.cu) */
    SI_BATCH_BITMAP_32K = 5,  /* window bitmaps of 32768 values */
    SI_BATCH_CODES = 6
};
size_t si_batch_workspace_size(uint64_t npairs);
si_status si_batch_count(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, const uint32_t* d_pairs,
                         uint64_t npairs, si_technique t, const uint8_t* table, uint32_t* d_counts,
                         void* d_workspace, size_t workspace_bytes, si_stream_t stream);

/* The autotuner: times every SI_BATCH_* technique on up to `sample` pairs of
 * every bucket that holds at least 32 pairs of this batch and writes the
 * fastest per bucket to table_out (host uint8[SI_BATCH_TABLE_SIZE]; the
 * default rule's choice stays unless another is 3 % faster; buckets with
 * fewer pairs keep the default).  Synchronises the stream; overwrites
 * d_counts. */
si_status si_batch_tune(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, const uint32_t* d_pairs,
                        uint64_t npairs, uint32_t sample, uint32_t* d_counts, void* d_workspace,
                        size_t workspace_bytes, si_stream_t stream, uint8_t* table_out);

/* The same batch captured once into a CUDA graph (all of si_batch_count's
 * launches for these pointers and sizes), replayed by si_batch_graph_launch on
 * any stream.  The buffers must stay valid while the graph exists. */
typedef struct si_batch_graph si_batch_graph;
si_status si_batch_graph_create(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k,
                                const uint32_t* d_pairs, uint64_t npairs, si_technique t, const uint8_t* table,
                                uint32_t* d_counts, void* d_workspace, size_t workspace_bytes,
                                si_batch_graph** out);
si_status si_batch_graph_launch(si_batch_graph* graph, si_stream_t stream);
void si_batch_graph_destroy(si_batch_graph* graph);

/* ------------------------------------------------------ degree statistics --
 * The per-value and per-set figures of the reference's degree_cdf tool
 * (src/degree_cdf.cpp:19-62), on the device, for a collection of k sets
 * holding n_elements elements (d_offsets[k] == n_elements):
 *   d_inv[v]     = number of sets that hold value v, v < slots (uint32[slots]);
 *   d_set_sum[s] = sum over the values of set s of d_inv[value] (uint64[k]).
 * A value >= slots is reported as SI_ERR_INVALID_INPUT in the workspace's
 * error word.  The sorted lists and running sums of the tool's four files
 * are formed from these on the host. */
size_t si_degree_stats_workspace_size(void);
si_status si_degree_stats(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, uint64_t n_elements,
                          uint64_t slots, uint32_t* d_inv, uint64_t* d_set_sum, void* d_workspace,
                          size_t workspace_bytes, si_stream_t stream);

/* --------------------------------------------------- MISI, dense form --
 * All pairs a < b of a collection of k sets over values 0..universe:
 * counts[tri(k, a, b)] = |S_a ∩ S_b|, tri = include/util.hpp:68-70 (the
 * reference's single-run result order, src/bitmap_naive.cu:443-447).
 *
 * d_elements / d_offsets: the collection in CSR form on the device (set a is
 * d_elements[d_offsets[a] .. d_offsets[a+1]), k + 1 offsets).
 * t = SI_TECH_MM: tensor-core product of the 0/1 incidence matrix, dtype
 *     INT8 (s32 accumulation) or FP8-e4m3 (f32 accumulation), both exact.
 *     Replaces the mm tile loop, src/matrix_multiplication.cu:139-184
 *     (host-built FP32 matrix + cublasSgemm per tile pair).
 * t = SI_TECH_BITMAP_NAIVE: bitmaps + AND-popcount on CUDA cores, the plain
 *     comparison.  Replaces src/bitmap_naive.cu:433-441 (generateBitmaps +
 *     intersectPerPair).
 * d_counts: device uint32[k*(k-1)/2].
 * Range: MM needs universe < 2^24 (every count exact in f32), BITMAP_NAIVE a
 * universe whose bitmap fits 200 KiB (< 6.5M values); outside it the call
 * returns SI_ERR_UNSUPPORTED and si_misi_dense_workspace_size returns 0.
 */
typedef enum si_dense_dtype { SI_DENSE_INT8 = 0, SI_DENSE_FP8_E4M3 = 1 } si_dense_dtype;
size_t si_misi_dense_workspace_size(uint32_t k, uint32_t universe, si_technique t);
si_status si_misi_dense(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, uint32_t universe,
                        si_technique t, si_dense_dtype dtype, uint32_t* d_counts, void* d_workspace,
                        size_t workspace_bytes, si_stream_t stream);

/* ---------------------------------------------------------- phase timer --
 * Named cudaEvent pairs around the engine's own kernel launches, recorded on
 * the launching stream while enabled -- the counterpart of the reference's
 * DeviceTimer (include/device_timer.cuh:20-78), which wraps every phase of
 * every executable the same way.  Phase names: single pair "sisi_prepare",
 * "sisi_split", "sisi_tile", and for BITMAP with elements "sisi_scan",
 * "sisi_copy"; dense all pairs "mm_incidence", "mm_gemm",
 * "naive_bitmaps", "naive_popcount"; all pairs of a tile "misi_plan",
 * "misi_probe"; single pair by search "obs_sample", "obs_search" (with the
 * offsets scan when elements are written), "obs_compact"; batched pairs
 * "batch_plan", "batch_count".  The events come from a pool that
 * si_timer_reset refills, so a timed launch costs two event records.
 * si_timer_read synchronises on the recorded events and returns the summed
 * milliseconds and the number of launches of one phase.
 */
void si_timer_enable(int on);
void si_timer_reset(void);
si_status si_timer_read(const char* phase, double* total_ms, uint64_t* launches);

/* ------------------------------------------------------- data generators --
 * Seeded, deterministic host generators for the benchmark configurations
 * (stand-in for src/generate_dataset.cpp, whose std::random_device seed is not
 * reproducible).  threads <= 0 uses all cores.
 *
 * si_gen_uniform: n distinct values drawn uniformly without replacement from
 * [lo, hi), written ascending to out[n].  hi - lo <= 2^32.
 */
si_status si_gen_uniform(uint64_t seed, uint64_t n, uint64_t lo, uint64_t hi, uint32_t* out, int threads);

/* si_gen_bernoulli: k sets over values [0, n_values), value v in set a with
 * probability p, independently.  Call once with elements == NULL to fill
 * offsets[k + 1] (CSR offsets), then again with elements[offsets[k]] and the
 * same offsets to fill the sets (each ascending). */
si_status si_gen_bernoulli(uint64_t seed, uint32_t k, uint32_t n_values, double p, uint64_t* offsets,
                           uint32_t* elements, int threads);

/* si_gen_powerlaw: k sets with sizes from the power law P(n) ~ n^-size_exp on
 * [n_min, n_max] and distinct values of [1, universe] drawn with Zipf
 * popularity P(v) ~ v^-value_exp.  Same two-call protocol as
 * si_gen_bernoulli.  n_max <= universe. */
/* si_gen_loguniform: k sets with sizes log-uniform on [n_min, n_max] and
 * distinct values of [0, universe) drawn uniformly.  Same two-call protocol as
 * si_gen_bernoulli.  n_max <= universe / 2. */
si_status si_gen_loguniform(uint64_t seed, uint32_t k, uint32_t n_min, uint32_t n_max, uint32_t universe,
                            uint64_t* offsets, uint32_t* elements, int threads);
si_status si_gen_powerlaw(uint64_t seed, uint32_t k, uint32_t n_min, uint32_t n_max, double size_exp,
                          uint32_t universe, double value_exp, uint64_t* offsets, uint32_t* elements, int threads);

#ifdef __cplusplus
}
#endif

#endif /* SI_B200_H */
