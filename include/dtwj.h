/* dtwj — top-1 z-normalised DTW subsequence self-join on one NVIDIA B200.
 *
 * C ABI of libdtwj.so.  Plain pointers and sizes; no C++ or framework types.
 *
 * The reference (QW1k0YA/Scaling-Subsequence-Similarity-Join-Based-on-Dynamic-
 * Time-Warping-CPU-GPU) ships two executables and no library; its in-process
 * seam for this path is
 *     void DTWMotifDiscoveryGUI(const vector<T>& TS, int subseqlen, int maxwarp,
 *                               const char* output_time_file_path)
 * (CPU_version1/DTWMotifDiscoveryGUI.cpp:12, GPU_version1/src/DTWMotifDiscoveryGUI.cu:12),
 * which runs mpx_v2 and then new_dtw_motifGUI[_malloc]
 * (CPU_version1/new_dtw_motifGUI.cpp:21, GPU_version1/src/new_dtw_motifGUI_malloc.cu:30)
 * and prints the result.  dtwj_join() replaces that seam and returns the
 * result instead of printing it; the `dtwj` CLI replaces the executables'
 * argv interface (README.md:15-34, GPU_version1/src/AAAA.cu:17-36).
 *
 * Semantics shared by every entry point:
 *   n series length, m subsequence length, w Sakoe-Chiba band (cells with
 *   |r - c| <= w), s = n - m + 1 subsequences, each z-normalised with its own
 *   mean and population standard deviation.  Candidate pairs are (i, j) with
 *   j - i >= m (the reference's exclusion zone, minlag = m,
 *   CPU_version1/new_dtw_motifGUI.cpp:182).  Windows with zero deviation are
 *   excluded.  Indices are 0-based.  The top-1 pair minimises
 *   (dist, i, j) lexicographically, so exact ties go to the lowest index.
 *
 * Errors: every function returns DTWJ_OK (0) or a negative DTWJ_ERR_* code;
 * dtwj_strerror() names it.  Nothing calls exit().  Inputs are read-only and
 * owned by the caller; the library owns all device memory it allocates.
 * Calls on one dtwj_ctx must not overlap; distinct contexts may be used from
 * distinct host threads.
 */
#ifndef DTWJ_H
#define DTWJ_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DTWJ_OK 0
#define DTWJ_ERR_ARG (-1)       /* invalid n, m, w, pointer or flags          */
#define DTWJ_ERR_NAN (-2)       /* input contains NaN or infinity             */
#define DTWJ_ERR_CUDA (-3)      /* a CUDA call failed                         */
#define DTWJ_ERR_OOM (-4)       /* device allocation failed                   */
#define DTWJ_ERR_BAND (-5)      /* 2w+1 exceeds the register band (w <= 255)  */
#define DTWJ_ERR_OVERFLOW (-6)  /* candidate list overflowed                  */
#define DTWJ_ERR_TIMEOUT (-7)   /* a bounded device-side wait ran out         */
#define DTWJ_ERR_NODEVICE (-8)  /* no CUDA device                             */
#define DTWJ_ERR_IO (-9)        /* file could not be read or written          */
#define DTWJ_ERR_NOMODEL (-10)  /* learned ordering requested, no model loaded */
#define DTWJ_ERR_SCRATCH (-11)  /* size exceeds the fixed scratch of dtwj_pair_dtw_noalloc */

/* longest subsequence the joins accept (62 blocks of 1024 samples); longer m
 * returns DTWJ_ERR_ARG */
#define DTWJ_MAX_M 63488

/* flags */
#define DTWJ_F_NO_MASKED 0x1u   /* with DTWJ_F_MASKED_CASCADE: skip the masked
                                   diagonal bound (endpoint bound only)       */
#define DTWJ_F_NO_SEED 0x2u     /* no ED-profile seeding of the best-so-far   */
#define DTWJ_F_NO_DIAG 0x4u     /* skip all diagonal bounds (LB_Keogh + DTW)  */
#define DTWJ_F_LEARNED 0x8u     /* sweep tiles in the order the context's MLP
                                   scores them (dtwj_ctx_set_model)           */
#define DTWJ_F_VERBOSE 0x10u    /* phase timings on stderr                    */
#define DTWJ_F_PROFILE 0x20u    /* per-phase device times (CUDA events)       */
#define DTWJ_F_NO_GRAPH 0x40u   /* launch the sweep directly, not as a CUDA graph
                                   (by default a context captures the sweep once and
                                   replays it while its launches are unchanged) */
#define DTWJ_F_MASKED_CASCADE 0x80u /* run filter = the reference's masked diagonal
                                   bound and endpoint bound (diag_mask_global,
                                   CPU_version1/diag_mask_global.cpp:11-311) on
                                   runs of the fast bound's survivors, instead of
                                   the default block-mean LB_Keogh bound; the
                                   same result, more pairs reach LB_Keogh      */
#define DTWJ_F_PETITJEAN 0x100u /* LB_Petitjean (lbPetitjean_new,
                                   CPU_version1/LB_PETITJEAN.cpp:10-123) on the
                                   pairs that pass LB_Keogh, before DTW, where
                                   2 (m + 2 min(w, m - 1)) doubles fit 200 KiB
                                   (no effect beyond); the same result         */

/* phases reported in dtwj_result.phase_seconds / phase_launches */
#define DTWJ_PHASE_PREP 0       /* statistics, envelopes, mask, row terms     */
#define DTWJ_PHASE_PROFILE 1    /* ED matrix profile                          */
#define DTWJ_PHASE_SEEDS 2      /* seed selection and seed DTWs               */
#define DTWJ_PHASE_DIAG 3       /* diagonal bound sweep                       */
#define DTWJ_PHASE_PAIRS 4      /* LB_Keogh with cumulative bound + DTW       */
#define DTWJ_PHASE_VERIFY 5     /* FP64 re-verification                       */
#define DTWJ_PHASE_RUNS 6       /* run filter: block-mean bound + endpoint bound
                                   (or the masked cascade) on the fast bound's
                                   survivors                                  */
#define DTWJ_PHASE_KEOGH 7      /* LB_Keogh on the run filter's survivors     */
#define DTWJ_NUM_PHASES 8

typedef struct {
  int64_t i, j;            /* top-1 pair, 0-based, j - i >= m                */
  double dist;             /* its DTW distance, recomputed in FP64           */
  double dist_fp32;        /* the FP32 distance the device search found      */
  double seed_bsf;         /* best-so-far after the ED-profile seeds         */
  uint64_t pairs;          /* candidate pairs (non-flat, j - i >= m)         */
  uint64_t pruned_fast;    /* pruned by the O(1) diagonal ED/LB_Keogh bound  */
  uint64_t pruned_kim;     /* pruned by the endpoint bound                   */
  uint64_t pruned_masked;  /* pruned by the masked diagonal bound            */
  uint64_t pruned_keogh;   /* pruned by LB_Keogh (either direction)          */
  uint64_t dtw_calls;      /* banded DTW evaluations (FP32)                  */
  uint64_t dtw_abandoned;  /* of which abandoned early                       */
  uint64_t dtw_cells;      /* DTW cells swept                                */
  uint64_t candidates;     /* pairs re-verified in FP64                      */
  double seconds_join;     /* device time of the join, inputs resident       */
  double seconds_total;    /* wall time of the call                          */
  int64_t n;
  int32_t m, w;
  double phase_seconds[8];   /* with DTWJ_F_PROFILE: device time per phase   */
  uint64_t phase_launches[8];/* kernel launches per phase                    */
  uint64_t pruned_paa;     /* pruned by the block-mean LB_Keogh bound (LB_PAA) */
  uint64_t pruned_petitjean; /* pruned by LB_Petitjean (DTWJ_F_PETITJEAN)    */
} dtwj_result;

typedef struct dtwj_ctx dtwj_ctx;

/* One-shot join of a host series (DTWMotifDiscoveryGUI's seam). */
int dtwj_join(const double* x, int64_t n, int32_t m, int32_t w, uint32_t flags,
              dtwj_result* out);

/* Many independent series, each with its own m and w; outs[k] is identical to
 * dtwj_join(xs[k], ns[k], ms[k], ws[k], flags).  Series of one (m, w) are
 * joined together in one pass; up to four such groups run at the same time,
 * each on its own host thread and device context (about 4 GB of device
 * buffers each), all on device 0.  No reference counterpart (the reference
 * joins one series per process). */
int dtwj_join_batch(const double* const* xs, const int64_t* ns, const int32_t* ms,
                    const int32_t* ws, int32_t count, uint32_t flags, dtwj_result* outs);

/* Reusable context bound to one device: keeps device buffers between calls. */
int dtwj_ctx_create(int device, dtwj_ctx** out);
void dtwj_ctx_destroy(dtwj_ctx* ctx);
int dtwj_ctx_join(dtwj_ctx* ctx, const double* x_host, int64_t n, int32_t m, int32_t w,
                  uint32_t flags, dtwj_result* out);
/* Same, with the series already in device memory (x_dev: n doubles). */
int dtwj_ctx_join_device(dtwj_ctx* ctx, const double* x_dev, int64_t n, int32_t m,
                         int32_t w, uint32_t flags, dtwj_result* out);

/* z-normalised Euclidean matrix profile with exclusion zone m (mpx_v2,
 * CPU_version1/mpx_v2.cpp:13): mp[i] = min over |i-j| >= m, mpi[i] its
 * 0-based argmin (lowest index on ties; -1 and +inf when none).  mp, mpi
 * hold s = n - m + 1 entries.  The FP64 recurrence finds each row's minimum
 * to about 2^-17 relative; every partner within about 2^-16 of it is then
 * measured directly in FP64, and the row takes the smallest (lowest partner
 * on ties).  DTWJ_ERR_OVERFLOW if those near-minimal partners average more
 * than 16 per row (a series of many near-identical windows). */
int dtwj_matrix_profile(const double* x, int64_t n, int32_t m, double* mp, int64_t* mpi);

/* The global CDF mask of the masked diagonal bound (compute_shared_data_global
 * + compute_MASK_global, CPU_version1/compute_shared_data_global.cpp:12,
 * CPU_version1/compute_MASK_global.cpp:10): mask[p] = 1 where the
 * coverage-normalised CDF gap of the windows' envelopes at sample p is at
 * most its mean over the series, else 0 (n floats).  table_len (may be NULL)
 * receives the CDF table length, max(600, 200 floor(max |z|)).  Computed on
 * the device exactly as DTWJ_F_MASKED_CASCADE joins use it. */
int dtwj_global_mask(const double* x, int64_t n, int32_t m, int32_t w, float* mask,
                     int32_t* table_len);

/* Banded DTW distances of explicit pairs of subsequences of x (the exact
 * recurrence MON_dtw computes, CPU_version1/MON_DTW.cpp:20), FP32 on the
 * device (precise=0) or FP64 (precise=1).  dist[k] for (pi[k], pj[k]). */
int dtwj_pair_dtw(const double* x, int64_t n, int32_t m, int32_t w, const int64_t* pi,
                  const int64_t* pj, int64_t count, int32_t precise, double* dist);

/* The two sums LB_Petitjean adds to the endpoint bound (lbPetitjean_new,
 * CPU_version1/LB_PETITJEAN.cpp:10-123, as the join evaluates it at
 * CPU_version1/new_dtw_motifGUI.cpp:517) for window A = pa[k] against window
 * B = pb[k], FP64 on the device: keogh_mid[k] = sum over t in [3, m-4] of
 * (A_t - H_t)^2, H = A projected onto B's envelope; terms[k] = the
 * projection part.  own_env = 1: each window's own clipped envelope of
 * radius w (the reference's subs_U / subs_L); 0: the raw series' envelope
 * normalised per window, as DTWJ_F_PETITJEAN joins read it.  w >= m is taken
 * as m - 1; DTWJ_ERR_ARG where the shared tables (2 (m + 2w) doubles, plus 4m
 * with own_env) exceed 200 KiB. */
int dtwj_pair_lb_petitjean(const double* x, int64_t n, int32_t m, int32_t w, const int64_t* pa,
                           const int64_t* pb, int64_t count, int32_t own_env, double* keogh_mid,
                           double* terms);

/* Allocation-free variant of dtwj_pair_dtw for callers that must not allocate
 * device memory (a host framework that reserves the device at start-up, a
 * latency-bound loop that cannot take cudaMalloc's implicit synchronisation).
 * No counterpart in the reference.  Everything is in device memory and owned
 * by the caller: x_dev (n doubles), pi_dev / pj_dev (count int64 window
 * indices), dist_dev (count doubles, the DTW distances).  Unlike
 * dtwj_pair_dtw, which rejects the whole call with DTWJ_ERR_ARG, an index
 * outside [0, s) is not checked on the host (the indices are device data):
 * that pair's distance is NaN and the other pairs are computed.  w >= m is
 * clamped to m - 1 (the full matrix); m must lie in [8, DTWJ_MAX_M].  Work is
 * enqueued on `stream` (a cudaStream_t; NULL is the legacy default stream)
 * and not waited for.  The only scratch, the window statistics, is a fixed
 * file-scope device array of 6.25 MiB holding at most
 * DTWJ_NOALLOC_MAX_WINDOWS windows; larger series return DTWJ_ERR_SCRATCH.
 * The array's device address is looked up on every call, with the caller's
 * device current, so it stays valid after cudaDeviceReset; the first call on
 * a device also loads the library's device code there, so make that first
 * call before any stream capture.  Every call shares the array, so calls that
 * overlap on the GPU (different streams, devices aside) race; it is rewritten
 * by each call.  Makes no cudaMalloc / cudaFree or other allocating call. */
#define DTWJ_NOALLOC_MAX_WINDOWS 262144
int dtwj_pair_dtw_noalloc(const double* x_dev, int64_t n, int32_t m, int32_t w,
                          const int64_t* pi_dev, const int64_t* pj_dev, int64_t count,
                          int32_t precise, double* dist_dev, void* stream);

/* ---- Learned tile ordering (no counterpart in the reference) ----
 * A small MLP scores each diagonal-sweep tile with a prediction of the
 * smallest DTW distance among its pairs; with DTWJ_F_LEARNED a context sweeps
 * the tiles in ascending order of that score so the best-so-far tightens
 * early.  The score only orders tiles: every pair is still judged by the same
 * bounds and exact DTW, so the result is that of the plain order.
 * Network: 64 -> 128 -> 128 -> 1, ReLU, mean squared error, Adam; BF16
 * weights on the tensor cores with FP32 accumulation and FP32 master weights.
 * Parameters (FP32, DTWJ_MLP_PARAMS values): W1 [128][64], b1 [128],
 * W2 [128][128], b2 [128], w3 [128], b3. */
#define DTWJ_MLP_IN 64
#define DTWJ_MLP_HIDDEN 128
#define DTWJ_MLP_PARAMS 24961
typedef struct dtwj_mlp dtwj_mlp;
/* He-uniform initial weights from `seed`, zero biases. */
int dtwj_mlp_create(int device, uint64_t seed, dtwj_mlp** out);
void dtwj_mlp_destroy(dtwj_mlp* net);
int dtwj_mlp_get(dtwj_mlp* net, float* params);
int dtwj_mlp_set(dtwj_mlp* net, const float* params);  /* also resets Adam */
/* `epochs` passes of Adam over shuffled minibatches of `batch` (<= 8192) rows
 * of x [count][64] against targets y [count]; *last_loss = the last epoch's
 * mean squared error. */
int dtwj_mlp_train(dtwj_mlp* net, const float* x, const float* y, int64_t count,
                   int32_t epochs, int32_t batch, float lr, uint64_t seed, float* last_loss);
int dtwj_mlp_predict(dtwj_mlp* net, const float* x, int64_t count, float* out);
/* Gradient of the mean squared error over one batch (count <= 8192) at the
 * current parameters, in the parameter layout: BF16 tensor-core path
 * (precise = 0, the one training uses) or the FP32 debug path (precise = 1). */
int dtwj_mlp_grad(dtwj_mlp* net, const float* x, const float* y, int64_t count,
                  int32_t precise, float* grad, float* loss);
int dtwj_mlp_save(dtwj_mlp* net, const char* path);
int dtwj_mlp_load(int device, const char* path, dtwj_mlp** out);
/* The network joins with DTWJ_F_LEARNED use on this context (not owned; it
 * must live on the context's device and outlive its use; NULL clears). */
int dtwj_ctx_set_model(dtwj_ctx* ctx, dtwj_mlp* net);
/* The diagonal-sweep tiles of a series, the units the learned order sorts:
 * *count = their number; with non-null arrays of *count entries:
 * desc[4t .. 4t+3] = (first lag, first row, rows, lags of the first row),
 * features[64t ..] = the tile's 64 features, min_dist[t] = the exact smallest
 * DTW distance among the tile's pairs (+inf if none).  min_dist needs a sweep
 * in which every tile prunes only against its own best-so-far: far slower
 * than a join; it produces the training targets of the network. */
int dtwj_ctx_tiles(dtwj_ctx* ctx, const double* x, int64_t n, int32_t m, int32_t w,
                   int64_t* count, int32_t* desc, float* features, double* min_dist);

/* Sharding one join over several GPUs (no counterpart in the reference): a
 * context with shard (rank, world) joins only the diagonal-sweep tiles t with
 * t % world == rank, its ED-profile seeds included.  The tiles are disjoint
 * sets of pairs covering every pair, so the lexicographic minimum of
 * (dist, i, j) over the world's results is the single-context result.  The
 * counters of each result cover its shard.  (0, 1) restores the whole join. */
int dtwj_ctx_set_shard(dtwj_ctx* ctx, int32_t rank, int32_t world);

/* Best-so-far exchange between the shards of one join (no counterpart in the
 * reference).  With an exchange set and world > 1, a sharded join sweeps its
 * tiles in `phases` groups (the same number on every shard, some possibly
 * empty) and calls fn(user, bsf2_dev, count, stream) after each group: bsf2_dev
 * is the context's device best-so-far (count uint32 words, the float bits of
 * a squared DTW distance, which order like the floats) and stream the join's
 * cudaStream_t.  The callback may enqueue on that stream work that lowers
 * the words, e.g. an all-reduce(min) over the shards' contexts, so every
 * shard prunes against the smallest distance any shard has found.  Any value
 * the callback writes must be the squared DTW distance of some pair (or
 * larger): pruning stays exact.  Every shard must pass the same phases.
 * fn = NULL removes the exchange. */
typedef void (*dtwj_exchange_fn)(void* user, uint32_t* bsf2_dev, int32_t count, void* stream);
int dtwj_ctx_set_exchange(dtwj_ctx* ctx, dtwj_exchange_fn fn, void* user, int32_t phases);

/* ---- Autotuning of the DTW band layout (no counterpart in the reference;
 * the reference fixes its layout at compile time with REGISTER_NUM) ----
 * The banded DTW runs a group of G lanes per pair with C band cells per lane
 * (C * G >= 2w + 1).  Every layout computes the same distances, so the choice
 * only changes speed.  dtwj_band_shapes lists the layouts tried for band w
 * (returns how many; writes up to max); dtwj_time_band measures one of them
 * on exact FP32 DTW of `pairs` window pairs of a seeded random walk (band
 * cells per second); dtwj_ctx_set_band makes a context's joins use layout
 * (C, G) for band w (0, 0: back to the default choice).  The default for a
 * join is G = 32 with the smallest C that covers the band (pairs abandon at
 * different rows, and groups sharing a warp would then run one after the
 * other); pair lists (dtwj_pair_dtw) take the layout wasting the fewest
 * cells. */
int dtwj_band_shapes(int32_t w, int32_t* C, int32_t* G, int32_t max);
int dtwj_time_band(int device, int32_t m, int32_t w, int32_t C, int32_t G, int32_t pairs,
                   double* cells_per_s);
int dtwj_ctx_set_band(dtwj_ctx* ctx, int32_t w, int32_t C, int32_t G);
/* Further tunables of a context's joins (no counterpart in the reference):
 * the CTA size of the DTW kernel in warps (1, 2, 4 or 8; each warp is one
 * pair in the default layout) and the tiles per chunk of the diagonal sweep
 * (16 to 4096; a chunk's survivors share the queues).  0 restores a default
 * (4 warps, 1024 tiles).  The result never depends on them. */
int dtwj_ctx_set_tuning(dtwj_ctx* ctx, int32_t dtw_warps, int32_t chunk_tiles);

/* Series files in the formats of the reference's loaders
 * (CPU_version1/loadfile.cpp:14-142, GPU_version1/src/loadfile.cu:13-148):
 *   DTWJ_LOAD_VALUES        every whitespace-separated number (loadfile)
 *   DTWJ_LOAD_EVERY         every param-th of them, from the first (loadfile_apart)
 *   DTWJ_LOAD_FIRST_COLUMN  the first number of every non-empty line of path,
 *                           then of path2 if it is not NULL (loadfile_2)
 *   DTWJ_LOAD_ROWS          the lines as a matrix flattened row by row, each row
 *                           cut to the first row's width (loadfile_); a shorter
 *                           row returns DTWJ_ERR_IO (the reference reads past it)
 *   DTWJ_LOAD_BINARY        raw little-endian float64
 * A token that is not a number ends the read (of the file, or of its line for
 * the line formats), as the reference's stream extraction does.  *n = the
 * series length; up to cap values go to out (out may be NULL with cap 0, to
 * size the buffer).  DTWJ_ERR_IO if a file cannot be read (the reference
 * exits instead). */
#define DTWJ_LOAD_VALUES 0
#define DTWJ_LOAD_EVERY 1
#define DTWJ_LOAD_FIRST_COLUMN 2
#define DTWJ_LOAD_ROWS 3
#define DTWJ_LOAD_BINARY 4
int dtwj_load(const char* path, const char* path2, int32_t format, int32_t param, double* out,
              int64_t cap, int64_t* n);

/* Band from a ratio: ceil(ratio*m) (rounding=0) or the reference's
 * max(round(ratio*m), 1) (rounding=1, GPU_version1/src/AAAA.cu:34). */
int32_t dtwj_band(int32_t m, double ratio, int32_t rounding);

const char* dtwj_strerror(int code);
int dtwj_device_count(void);

#ifdef __cplusplus
}
#endif
#endif
