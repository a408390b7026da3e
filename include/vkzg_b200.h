/*
 * Extensions of the vkzg C API exported by this library.  None of these
 * replaces a reference function; each says what in the reference it relates to.
 */
#ifndef VKZG_B200_H
#define VKZG_B200_H

#include "vkzg.h"

#ifdef __cplusplus
extern "C" {
#endif

/*
 * Generates the FK20 setup tables on the GPU from 4096 compressed G1 monomial
 * points ([tau^i]G1, 48 bytes each) and writes them to `out_path` in the
 * reference's precomputed_tables.bin format (src/precomputed_tables.cpp:16-58),
 * which the reference ships prebuilt and its Java binding extracts to
 * $VKZG_TABLES_PATH (Vkzg.java:80-93).  A synthetic setup is selected the same
 * way: generate its file, point VKZG_TABLES_PATH at it.
 */
vkzg_result vkzg_b200_write_tables(const uint8_t *g1_monomial_compressed, const char *out_path);

/* Where the prover's tables came from: "file:<path>" or "generated:<setup path>". */
const char *vkzg_b200_prover_tables_source(const vkzg_prover *p);

/*
 * Per-stage device time of the last proof or recovery chunk, in milliseconds,
 * from CUDA events (the reference's bench/profile.cpp wall-clocks each stage by
 * flushing the queue between dispatches, src/profile.h:12-28).  Fills up to
 * `cap` entries and returns the number of stages; names via
 * vkzg_b200_stage_name.  Timing is recorded only while enabled.  The fold runs
 * inside the ladder's launch, so "fold" reads ~0 and "ladder" holds both; on
 * plans 3-4 the finish runs inside phase B's reduction (its Horner step and the
 * finish share a launch), so "finish" reads ~0 and "reduce_b" holds both.
 */
void vkzg_b200_set_stage_timing(vkzg_prover *p, int enabled);
int vkzg_b200_last_stage_times(const vkzg_prover *p, int recovery, double *ms, int cap);
const char *vkzg_b200_stage_name(int recovery, int i);

/*
 * Device-resident forms of vkzg_compute_proofs_batch / vkzg_recover_cells_batch
 * (include/vkzg.h:103-104, 120-121) for callers whose data already lives in
 * device memory: same layouts, device pointers, no host copies.  The work is
 * ordered after everything already enqueued on `stream` (a cudaStream_t; NULL
 * = the legacy default stream) and everything enqueued on `stream` afterwards
 * is ordered after it; the call returns once the work is enqueued.
 * d_err (num_blobs words) receives a nonzero word for each blob with a
 * non-canonical element (proofs) or more than 64 missing cells (recovery);
 * those blobs' outputs are unspecified.  Bit 31 of every word of a proof chunk
 * (VKZG_B200_DEVICE_FAILED) means a grid barrier of the chunk's cooperative
 * launches gave up waiting (the host entry points return VKZG_ERR_GPU then).
 */
#define VKZG_B200_DEVICE_FAILED 0x80000000u
vkzg_result vkzg_b200_compute_proofs_device(vkzg_prover *p, uint8_t *d_proofs, const uint8_t *d_blobs,
                                            uint32_t *d_err, size_t num_blobs, void *stream);
vkzg_result vkzg_b200_recover_cells_device(vkzg_prover *p, uint8_t *d_cells_out, const uint8_t *d_cells,
                                           const uint8_t *d_cell_present, uint32_t *d_err, size_t num_blobs,
                                           void *stream);

/*
 * Allocation-free form of vkzg_b200_recover_cells_device.  No counterpart in
 * the reference.
 *
 * For callers that must not allocate device memory at call time: code running
 * where a framework's pool owns nearly all of HBM (an extra cudaMalloc would
 * fail), latency-critical loops that cannot absorb the device-wide
 * synchronisation a cudaMalloc/cudaFree can imply, and code that enqueues work
 * on a stream it does not own.  This call allocates nothing and frees nothing,
 * and uses no scratch: one cluster of four blocks per blob keeps its working
 * state in shared memory.  Inputs and outputs are the caller's device buffers,
 * laid out as for vkzg_b200_recover_cells_device; the work is enqueued on
 * `stream` (a cudaStream_t, NULL = legacy default stream) and the call returns
 * after enqueueing.  The prover's device must be current.  Calls on different
 * streams or threads may overlap on the GPU: they share nothing but the
 * prover's read-only tables.
 *
 * Limits: at most VKZG_B200_NOALLOC_MAX_BLOBS blobs per call; more returns
 * VKZG_ERR_BADARGS without enqueueing anything.
 */
#define VKZG_B200_NOALLOC_MAX_BLOBS 16
vkzg_result vkzg_b200_recover_cells_device_noalloc(vkzg_prover *p, uint8_t *d_cells_out, const uint8_t *d_cells,
                                                   const uint8_t *d_cell_present, uint32_t *d_err,
                                                   size_t num_blobs, void *stream);

/*
 * The 128 cells of each blob (the 2x Reed-Solomon extension, 128 x 2048 bytes
 * per blob in cell order), and cells plus proofs in one call sharing one upload
 * (the consensus specs' compute_cells_and_kzg_proofs).  The reference computes
 * proofs only and leaves cells out (include/vkzg.h:16-18).  Same blob format and
 * error rules as vkzg_compute_proofs_batch; a chunk with an invalid blob leaves
 * its outputs untouched, except in vkzg_b200_compute_cells_batch from
 * page-locked buffers with 16 blobs or more in the chunk: that form copies
 * each part's cells out as the part finishes, before the error words are read,
 * and zeroes the chunk's cells when one of its blobs is invalid.
 */
vkzg_result vkzg_b200_compute_cells_batch(vkzg_prover *p, uint8_t *cells, const uint8_t *blobs, size_t num_blobs);
vkzg_result vkzg_b200_compute_cells_and_proofs_batch(vkzg_prover *p, uint8_t *cells, uint8_t *proofs,
                                                     const uint8_t *blobs, size_t num_blobs);

/*
 * Recovered cells and the proofs of the recovered blob in one call (the
 * consensus specs' recover_cells_and_kzg_proofs; the reference recovers cells
 * only, include/vkzg.h:106-121).  Same inputs and error rules as
 * vkzg_recover_cells_batch; proofs_out receives num_blobs x 128 x 48 bytes.
 */
vkzg_result vkzg_b200_recover_cells_and_proofs_batch(vkzg_prover *p, uint8_t *cells_out, uint8_t *proofs_out,
                                                     const uint8_t *cells, const uint8_t *cell_present,
                                                     size_t num_blobs);

/*
 * Autotuner.  Proof chunks run under one of VKZG_B200_PLANS plans that compute
 * identical bytes: 0 = serial Jacobian bucket accumulation and reduction (one
 * output per block, the reference's scheme, k_phase_a.comp /
 * k_bucket_reduce.comp); 1 = batch-affine bucket accumulation and a
 * binary-split batch-affine reduction; 2 = batch-affine accumulation with the
 * serial reduction; 3 = phase A as plain sums over a precomputed digit table
 * (every signed digit multiple of every base in each of D windows, sized by a
 * byte budget as described below, built on first use and shared by the
 * process's provers with the same setup; a smaller table is used when free
 * memory is short) summed in grid-wide batch-affine rounds, phase B also in
 * grid-wide rounds; 4 = phase A as plan 1, phase B as plan 3 (no digit
 * table).  The first chunk of each
 * power-of-two size class is timed under all plans and the fastest is kept
 * (also in $VKZG_TUNE_CACHE when set; $VKZG_PLAN forces a plan).  Plan 3 is
 * timed at every size class of a prover whose max_batch_size is 16 or more
 * (below 16 blobs with the fewest windows the budget allows); for a smaller
 * prover the tuner leaves the digit table out ($VKZG_PLAN=3 still forces it).
 * vkzg_b200_autotune tunes every size class up to max_blobs (0 = the prover's
 * max_batch_size) on seeded synthetic blobs; vkzg_b200_tuning_table reports the
 * decisions (size class, plan, and VKZG_B200_PLANS times in ms per class, -1
 * where a plan was not timed) and returns how many classes are tuned.
 * vkzg_b200_digit_table returns the digit table's windows per scalar D (0 =
 * none built), its build time and size.
 *
 * Plan 3's digit table cuts a scalar's 256 bits into D signed windows of
 * widths W + 1 (the first 256 mod D of them) and W = floor(256 / D), and holds
 * m 2^(b_k) X[j][i] for every window k (at bit b_k) and m = 1..2^(width - 1):
 * points of 96 bytes, 128 x 64 x that many per base (D = 32: 8-bit windows,
 * 3.2 GB; 26: 9.7 GB; 24: 16.1 GB; 23: 20.9 GB; 22: 29.0 GB; 21: 40.3 GB; 20:
 * 58.0 GB; 19: 90.2 GB; 18: 141.7 GB); fewer windows mean fewer additions per
 * output (64 D - 1).  Its size is bounded by a budget: $VKZG_COMB_BUDGET_GB
 * (GiB, default 20, so D >= 23 unless raised); a serving loop uses its
 * table_budget_bytes.  When plan 3 is tuned at 16 blobs or more, the fewest
 * windows whose table fits the budget and the next two counts are each built
 * and timed, and the
 * fastest is kept (and remembered in $VKZG_TUNE_CACHE); $VKZG_COMB_WINDOWS pins
 * D (18..32), $VKZG_COMB_BITS pins the widest window instead (D =
 * ceil(256 / bits)), and 0 in either means no digit table.
 * vkzg_b200_window_trials reports those trials for a size class (windows,
 * table bytes, build ms, proof-chunk ms) and returns their count.  vkzg_b200_prover_device_bytes reports the device
 * memory a prover holds: its working set, its setup tables, and the digit
 * table it uses (shared by all provers of the process with the same setup).
 */
#define VKZG_B200_PLANS 5
vkzg_result vkzg_b200_autotune(vkzg_prover *p, uint32_t max_blobs);
int vkzg_b200_tuning_table(const vkzg_prover *p, uint32_t *size_class, int *plan, double *ms, int cap);
int vkzg_b200_digit_table(const vkzg_prover *p, double *build_ms, uint64_t *bytes);
int vkzg_b200_window_trials(const vkzg_prover *p, uint32_t size_class, int *windows, uint64_t *table_bytes,
                            double *build_ms, double *ms, int cap);
void vkzg_b200_prover_device_bytes(const vkzg_prover *p, uint64_t *working, uint64_t *tables, uint64_t *digit_table);

/*
 * Number of CUDA kernels this library has launched in this process (proof,
 * recovery, cells and table-generation launchers; the diagnostics below are not
 * counted).  No counterpart in the reference.
 */
uint64_t vkzg_b200_kernel_launches(void);

/*
 * Serving loop with continuous batching (the reference has none: one blocking
 * batch call per caller, serialised per prover, src/vkzg.cpp:1183-1218).
 *
 * Requests of any blob count are submitted without blocking and identified by
 * a ticket; their buffers must stay valid until vkzg_b200_server_wait returns
 * the ticket's final status (not its timeout).  A dispatcher cuts pending requests into batches (one kind
 * per batch, first come first served, at most max_blobs_per_batch blobs;
 * larger requests are split) and hands each batch to a free lane: a prover with
 * its own CUDA stream and buffers, so batches on different lanes run
 * concurrently on the GPU and requests that arrive while lanes are busy join
 * the next batch.  A batch is admitted only while the device working set of
 * all batches in flight stays within hbm_budget_bytes (a batch is always admitted
 * when none is in flight, so a budget below one batch serialises batches; the
 * dispatcher sleeps until a batch completes).  A batch is charged its blobs
 * times the device working set per blob that the lanes hold (measured from
 * their allocations at creation: a lane prover's working set over its
 * capacity, plus the lane's I/O buffers); the setup tables and the shared
 * digit table are resident and reported apart (resident_bytes).  The lanes'
 * digit table is bounded by table_budget_bytes (0 = 20 GiB).  Stats also count
 * the batches admission deferred and the peak in-flight charge.  Each blob is computed
 * independently, so a request's output is the same alone and in any mix.
 * vkzg_b200_server_new tunes the proof plan of every batch size class up to
 * max_blobs_per_batch on one lane and gives the choices to all lanes, so that
 * no request waits for a tuning run.  vkzg_b200_server_wait returns the request's final status
 * (VKZG_ERR_INVALID_BLOB / VKZG_ERR_BADARGS / VKZG_ERR_GPU as the batch calls would), after
 * which the ticket is spent; or VKZG_B200_PENDING when timeout_ms ran out first, in which case
 * the request is still in flight, its buffers are still in use and the ticket stays valid.
 * Stats cover requests completed since the last reset: latency from submit to completion.
 */
/* Status of vkzg_b200_server_wait only: the wait timed out before the request
 * finished.  Outside the reference's vkzg_result values 0..6. */
#define VKZG_B200_PENDING ((vkzg_result)7)
typedef struct vkzg_server vkzg_server;
typedef struct {
    uint32_t max_blobs_per_batch; /* 0 = 128 */
    uint32_t lanes;               /* concurrent device batches; 0 = 3 */
    uint64_t hbm_budget_bytes;    /* admission cap on the in-flight working set; 0 = 8 GiB */
    uint64_t table_budget_bytes;  /* cap on the lanes' digit table; 0 = 20 GiB */
} vkzg_server_options;
typedef struct {
    uint64_t requests, blobs;
    double p50_ms, p99_ms, p999_ms, mean_ms, max_ms, seconds;
    uint64_t deferrals;            /* times admission held a batch back for the budget */
    uint64_t peak_in_flight_bytes; /* largest in-flight charge */
    uint64_t resident_bytes;       /* setup tables of the lanes + the shared digit table */
    uint64_t proof_bytes_per_blob, recover_bytes_per_blob; /* admission charges */
} vkzg_server_stats;
void vkzg_b200_server_options_default(vkzg_server_options *opts);
vkzg_result vkzg_b200_server_new(vkzg_server **out, const vkzg_server_options *opts);
void vkzg_b200_server_free(vkzg_server *s);
vkzg_result vkzg_b200_server_submit_proofs(vkzg_server *s, uint8_t *proofs, const uint8_t *blobs, size_t num_blobs,
                                           uint64_t *ticket);
vkzg_result vkzg_b200_server_submit_recovery(vkzg_server *s, uint8_t *cells_out, const uint8_t *cells,
                                             const uint8_t *cell_present, size_t num_blobs, uint64_t *ticket);
vkzg_result vkzg_b200_server_wait(vkzg_server *s, uint64_t ticket, int64_t timeout_ms);
vkzg_result vkzg_b200_server_stats(vkzg_server *s, vkzg_server_stats *out, int reset);

/*
 * Throughput probes on the current device, for roofline denominators (the
 * reference has none).  which = 0: 32-bit integer multiply-add issue rate in
 * tera-ops/s; 1: this library's Fp (381-bit) Montgomery multiplies in giga-ops/s;
 * 2: Fr (255-bit) multiplies in giga-ops/s; 3: Fp squares; 4: Fp multiplies through
 * one Karatsuba level; 5: Fr multiplies through one Karatsuba level; 6: Fp
 * squares through one Karatsuba level; 7: Fp multiplies through two Karatsuba
 * levels (all giga-ops/s); 8: mad.wide.u32 (32x32+64-bit) issue rate and 9:
 * fma.rn.f64 issue rate, in tera-ops/s; 10 and 11: the time in microseconds of
 * one launch inverting 16 Fp values per SM, one per thread (the inversion
 * between the passes of a batch-affine round), with variable-time and with
 * fixed 30-divstep batches; 12: Fp multiplies with the partial products on the
 * FP64 pipe, 13: Fp squares on the FP64 pipe, 14: Fp multiplies with half the
 * warps on each pipe, 15 and 16: Fp multiplies on the FP64 pipe and through one
 * Karatsuba level with four independent chains per thread instead of two
 * (giga-ops/s); 17: as 11, each value inverted by four lanes (the form the
 * proof rounds use), in microseconds.  Best of three timed launches.
 */
vkzg_result vkzg_b200_microbench(int which, double *result);

/*
 * Self-test of the batched-affine bucket summation the proof kernels use (the
 * reference sums buckets serially, k_phase_a.comp:37-42): sums n <= 2048 affine
 * points (96 bytes each, x || y canonical big-endian, all-zero = infinity) into
 * 128 buckets (bucket_of[i] < 128) on the current device and writes the 128
 * sums in the same encoding.  For tests of the doubling, cancellation and
 * infinity cases that random inputs never reach.
 */
vkzg_result vkzg_b200_bucket_sums_selftest(const uint8_t *points_xy, const uint32_t *bucket_of, size_t n,
                                           uint8_t *sums_xy);

/*
 * Self-test of the grid barrier that the cooperative launches of plans 3-4 use
 * between their passes.  No counterpart in the reference.  One cooperative
 * launch of two blocks per SM crosses `rounds` barriers; *barriers_passed is
 * the sum over blocks of the barriers each passed, *failed_flag the barrier's
 * failure flag, *error_words_marked how many of the launch's 8 error words got
 * VKZG_B200_DEVICE_FAILED.  With extra_arrivals > 0 every barrier waits for
 * blocks that do not exist: each wait gives up after spin_limit polls (about
 * 100 ns each), so the launch ends with the flag set instead of waiting forever.
 */
vkzg_result vkzg_b200_grid_sync_selftest(uint32_t extra_arrivals, uint32_t spin_limit, int rounds,
                                         uint32_t *barriers_passed, uint32_t *failed_flag,
                                         uint32_t *error_words_marked);

/*
 * Self-test of the inversion used between the passes of the proof path's
 * grid-wide rounds (four lanes per value, divsteps in table-driven groups)
 * against the one-lane divstep inversion, on n seeded pseudo-random Fp values
 * (the first four: 0, 1, 2, p - 1).  *mismatched_words: how many 32-bit words
 * of the n results differ (0 when the two agree).  No counterpart in the
 * reference.
 */
vkzg_result vkzg_b200_inverse_selftest(int n, uint32_t seed, uint32_t *mismatched_words);

/*
 * Sums n_lists lists of m affine points each (points_xy: n_lists * m x 96
 * bytes, list o first; all zero = infinity) with the grid-wide batch-affine
 * tree rounds of the proof path's plan 3.  points_xy NULL: seeded pseudo-random
 * coordinates generated on the device instead (a timing workload, not curve
 * points).  sums_xy (may be NULL): n_lists x 96 bytes; *ms (may be NULL): the
 * rounds' device time.  At most 2^27 points.  No counterpart in the reference.
 */
vkzg_result vkzg_b200_tree_sums_selftest(const uint8_t *points_xy, size_t n_lists, uint32_t m, uint64_t seed,
                                         uint8_t *sums_xy, double *ms);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* VKZG_B200_H */
