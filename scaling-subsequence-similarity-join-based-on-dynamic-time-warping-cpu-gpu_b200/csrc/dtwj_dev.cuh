// Internal header: device-side layout of one prepared series and the launch
// entry points of every kernel of the join.  Host orchestration (join.cu)
// only sees the launch functions declared at the bottom.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dtwj {

// Relative slack on squared distances for every pruning and abandoning test.
// FP32 distances and the FP64 diagonal recurrences carry rounding error far
// below this; the slack keeps every pair whose true distance can still be the
// minimum, and the final candidates are re-verified in FP64.
constexpr float kSlack = 1.0f / 512.0f;
// Absolute slack per window sample on squared distances: keeps a pair whose
// distance ties the best-so-far (exact duplicates give 0) above the rounding
// of the FP32 bounds.
constexpr float kAbsSlackPerSample = 1e-6f;

// Pruning / abandoning threshold on squared distances from the best-so-far.
__device__ __forceinline__ float prune_threshold(unsigned int bsf2_bits, int m) {
  return __uint_as_float(bsf2_bits) * (1.0f + kSlack) + kAbsSlackPerSample * (float)m;
}
__device__ __forceinline__ float prune_threshold_now(const unsigned int* bsf2, int m) {
  return prune_threshold(*(volatile const unsigned int*)bsf2, m);
}

// Whether an FP32 lower bound built from block-centered copies (LB_Keogh,
// the block-mean bound) may prune a pair whose windows have error scale r
// (the larger of their DevSeries::rw), against the squared threshold thr.
// Every z-like difference such a bound forms is within dz = 16 * 2^-24 * r of
// its exact value (the centered value, the FP32 reciprocal deviation, the
// block offset and each FMA round once, every term bounded by a few r), so a
// bound sum_k c_k d_k^2 with sum_k c_k <= m is within
// 2 dz sqrt(m * bound) + m dz^2 of the exact one at bound <= thr, plus the
// FP32 summation (at most m / 8 + 8 terms per lane, relative 2^-24 each).
// The pair may be pruned when that error fits in the slack thr keeps above
// the best-so-far: thr - bsf2 = (thr kSlack + kAbsSlackPerSample m) / (1 + kSlack).
__device__ __forceinline__ bool fp32_bound_ok(float r, float thr, int m) {
  const float fm = (float)m;
  const float dz = r * (16.0f / 16777216.0f);
  const float err = 2.0f * dz * sqrtf(fm * thr) + fm * dz * dz +
                    thr * ((fm * 0.125f + 8.0f) * (1.0f / 16777216.0f));
  const float slack = (thr * kSlack + kAbsSlackPerSample * fm) * (1.0f / (1.0f + kSlack));
  return err <= slack;
}

// The largest error scale r for which fp32_bound_ok(r, thr, m) holds (the
// error bound is increasing in r): the positive root of
// a r^2 + b r + c = 0 with a = m k^2, b = 2 k sqrt(m thr), c = summation term
// - slack, k = 16 * 2^-24, in the form -2c / (b + sqrt(b^2 - 4ac)) that does
// not cancel, shrunk by 2^-10 against the rounding of this evaluation; -1 if
// none.
__device__ __forceinline__ float fp32_bound_radius(float thr, int m) {
  const float fm = (float)m, k = 16.0f / 16777216.0f;
  const float slack = (thr * kSlack + kAbsSlackPerSample * fm) * (1.0f / (1.0f + kSlack));
  const float c = thr * ((fm * 0.125f + 8.0f) * (1.0f / 16777216.0f)) - slack;
  if (!(c < 0.0f)) return -1.0f;  // also +inf / NaN thresholds: no FP32 pruning
  const float a = fm * k * k, b = 2.0f * k * sqrtf(fm * thr);
  const float r = -2.0f * c / (b + sqrtf(b * b - 4.0f * a * c));
  return r * (1.0f - 1.0f / 1024.0f);
}

// Endpoint bound width (the reference's BIAS, CPU_version1/diag_mask_global.cpp:8).
constexpr int kBias = 3;
// Seeds taken from the ED matrix profile (CPU_version1/new_dtw_motifGUI.cpp:53).
constexpr int kSeeds = 100;
// The seed profile keys one row in kSeedGrid; each seed pair is widened to
// kSeedSpread pairs on its diagonal (offsets -kSeedGrid/2 .. kSeedGrid/2).
constexpr int kSeedGrid = 7;
constexpr int kSeedSpread = kSeedGrid;
constexpr int kSeedSlots = kSeeds * kSeedSpread;
// Sentinels padding the z-normalised sequences: finite so that no
// inf - inf appears, far enough apart that any cell touching them is
// effectively infinite.
constexpr float kPadQ = 1e18f;
constexpr float kPadT = -1e18f;
constexpr double kPadQd = 1e150;
constexpr double kPadTd = -1e150;

// Lag-block x row-block of the diagonal sweep: pairs (i, i + L) for
// L in [L0, L0 + kLbLags) and i in [i0, i0 + rows), all windows below send.
// Indices are global: in a batch the series sit back to back and a tile
// belongs to one of them.
struct Tile {
  int32_t L0;
  int32_t i0;
  int32_t rows;
  int32_t order;   // position in the queue order (learned or plain)
  int32_t send;    // end of the series' windows (global window index)
  int32_t series;  // series of the batch (0 for a single join)
};
// Diagonal-sweep tiles: 128 threads x kLbPerThread lags x kLbRows rows, one
// survivor bit per pair, kLbWords 32-row words per lag.
constexpr int kLbThreads = 128;
constexpr int kLbPerThread = 7;
constexpr int kLbLags = kLbThreads * kLbPerThread;
constexpr int kLbRows = 18 * kLbPerThread * 32;
constexpr int kLbWords = kLbRows / 32;
// CTAs of the persistent diagonal sweep per SM (launch bounds of k_lb).
constexpr int kLbCtasPerSm = 3;
// Lags per group of the block-mean filter's work items (one lag per lane).
constexpr int kLbGroups = kLbLags / 32;
static_assert(kLbLags % 32 == 0, "lag groups of one warp");
// Longest run of consecutive surviving rows the sweep emits as one item.
constexpr int kRunMax = 256;
// FP32 copies of the series and its envelopes are centered per block of
// 2^kBlkShift samples (value minus the block mean) so that the float rounding
// error stays far below the pruning slack.
constexpr int kBlkShift = 10;
// Blocks of each copy of DevSeries::pq2 (copy 1's block b starts 1024
// samples before copy 0's).
__host__ __device__ inline int64_t kCopyBlocks(int64_t n) { return (n >> 11) + 2; }

// Counters, all uint64 on the device.
enum Counter {
  kPairs = 0,
  kPrunedFast,
  kPrunedKim,
  kPrunedMasked,
  kPrunedKeogh,
  kDtwCalls,
  kDtwAbandoned,
  kDtwCells,
  kCandidates,
  kPrunedPaa,
  kPrunedPetitjean,
  kNumCounters
};

struct Candidate {
  int32_t i, j;
  float d2;
  int32_t series;
};

// All device arrays of one prepared series.
struct DevSeries {
  const double* a;  // n, the series (a batch: all series back to back)
  int64_t n;
  int64_t s;        // n - m + 1
  int m, w;
  const int* sid;   // n, series of each sample (nullptr for a single series)
  const int64_t* sbeg;  // series + 1 sample offsets (nullptr for a single series)
  int nseries;
  double* mu;       // s, window mean
  double* sig;      // s, window population std (1 for flat windows)
  double* isg;      // s, 1/sig (0 for flat windows)
  uint8_t* flat;    // s
  double* U;        // n, upper envelope of the raw series, radius w
  double* L;        // n, lower envelope
  double* E;        // n, U + L
  double* nu;       // s, mean of (U + L) over the window
  double* dfa;      // s, (a[i+m] - a[i]) / 2
  double* dga;      // s, (a[i+m] - mu[i+1]) + (a[i] - mu[i])
  double* dfE;      // s, same for E = U + L
  double* dgE;      // s
  double* A;        // s, 4m + 2N - DUL2   (fast bound row constant)
  double* DUL;      // s, ||nU - nL||
  double* qsig;     // s, sig / 4 (1e300-guarded for flat windows)
  float* mask;      // n, 0/1 mask of the masked bound
  float* MN;        // s, sum_T M (nU^2 + nL^2)
  float* MDUL2;     // s, sum_m M (nU - nL)^2
  float* MDUL;      // s
  double* SM;       // s, sum_T M            (T = [kBias, m-1-kBias])
  double* SME;      // s, sum_T M E
  double* cb;       // (n >> kBlkShift) + 2, block centers
  float* af;        // n, a - cb[block]
  float2* ulf;      // n, (U - cb[block], L - cb[block])
  int paa_b;        // block length of the block-mean bound (8, 16 or 32)
  float4* pq;       // n, means over [p, p + paa_b) of (a, U, L) - cb[block of p], 0
                    //    (windows longer than 1024 samples; else nullptr)
  float* cmax;      // (n >> kBlkShift) + 2, largest |centered FP32 value| per block
  float* rw;        // s, FP32 error scale of window i: isg_i x the largest
                    //    centered magnitude or block offset its FP32 bounds read
  // Windows of at most 1024 samples: the same block means in two copies
  // centered per 2048-sample block, copy 0 on [2048 b, 2048 b + 2048) and
  // copy 1 on [2048 b - 1024, 2048 b + 1024), so every window lies inside one
  // block of one copy and has a single block offset (else all nullptr).
  float4* pq2;      // 2n, copy c at [c n, c n + n)
  float* cmax2;     // 2 kCopyBlocks(n), largest |value| of each copy block
  float4* wrec;     // s, window record: block offset (FP64 in .x/.y), isg as
                    //    FP32 (.z) and the error scale for pq2 (.w)
  int* status;      // device status word (0 ok, else error bits)
};

// Global search state of one join.
struct DevSearch {
  unsigned int* bsf2;           // per series: float bits of the best squared DTW so far
  unsigned long long* counters; // kNumCounters
  Candidate* cand;              // candidate list
  unsigned int* cand_count;
  unsigned int cand_cap;
  int4* runs;                   // runs of fast-bound survivors: (i0, j0, len, 0)
  unsigned int* run_count;
  unsigned int* run_next;
  unsigned int run_cap;
  int2* queue;                  // survivor pairs of the current chunk
  int* qser;                    // their best-so-far slot (nullptr: the series of i)
  unsigned int* queue_count;
  unsigned int* queue_next;
  unsigned int queue_cap;
  int4* kq;                     // LB_Keogh candidates: (i, j, endpoint bound bits, series)
  unsigned int* kq_count;
  unsigned int* kq_next;
  unsigned int kq_cap;
};

// Endpoint bound: minimum cost of any warping path's cells in the first and
// last three layers (LB_KIM, CPU_version1/lb_kim.cpp:10-73).  q = window i,
// t = window j (any indexable sequences); cells are (t index, q index).  The
// reference's fourth option adds the corner cell twice (lb_kim.cpp:55,62);
// here it is added once so that the bound stays admissible.
template <typename V, typename Seq>
__device__ __forceinline__ void kim_bound(const Seq& q, const Seq& t, int m, V* left, V* right) {
  auto D2 = [](V x, V y) { return (x - y) * (x - y); };
  auto mn = [](V x, V y) { return x < y ? x : y; };
  const V o = D2(t[0], q[0]);
  const V lw = mn(D2(t[1], q[0]), D2(t[1], q[1]));
  const V l1 = mn(lw, D2(t[0], q[1]));
  V d = mn(D2(t[1], q[0]) + D2(t[2], q[0]), lw + D2(t[2], q[1]));
  d = mn(d, D2(q[1], t[1]) + D2(q[2], t[2]));
  d = mn(d, l1 + D2(q[2], t[1]));
  d = mn(d, D2(q[1], t[0]) + D2(q[2], t[0]));
  *left = o + d;
  const int e = m - 1;
  const V o2 = D2(t[e], q[e]);
  const V rw = mn(D2(t[e - 1], q[e]), D2(t[e - 1], q[e - 1]));
  const V r1 = mn(rw, D2(t[e], q[e - 1]));
  d = mn(D2(t[e - 1], q[e]) + D2(t[e - 2], q[e]), rw + D2(t[e - 2], q[e - 1]));
  d = mn(d, D2(q[e - 1], t[e - 1]) + D2(q[e - 2], t[e - 2]));
  d = mn(d, r1 + D2(q[e - 2], t[e - 1]));
  d = mn(d, D2(q[e - 1], t[e]) + D2(q[e - 2], t[e]));
  *right = o2 + d;
}

struct BandShape {
  int C;  // cells (diagonals) per lane
  int G;  // lanes per pair
  int warps = 0;  // CTA size of the join's DTW kernel in warps (0: the default, 4)
};
// The join's layout: one pair per warp (G = 32) with the fewest cells per
// lane C in [2, 16] covering 2w+1 diagonals.  Returns false if w > 255.
bool choose_band(int w, BandShape* out);
// Exact DTW lists (no early abandoning): G in {4, 8, 16, 32} and C in
// [2, 16] covering 2w+1 diagonals with the least waste.
bool choose_band_list(int w, BandShape* out);
// (C, G) has a kernel instantiation and covers band w.
bool band_shape_ok(int w, int C, int G);
// The shapes the autotuner tries for band w (per G the two smallest covering
// C); writes up to max, returns how many there are.
int band_shapes(int w, BandShape* out, int max);

// ---- launches (all on `stream`) ----
void launch_check_finite(const double* a, int64_t n, int* status, cudaStream_t st);
// sid[p] = series of sample p for a batch with series offsets sbeg[0..nseries].
void launch_series_ids(const int64_t* sbeg, int nseries, int* sid, int64_t n, cudaStream_t st);
void launch_prep(const DevSeries& S, cudaStream_t st);
void launch_rowterms(const DevSeries& S, bool masked, cudaStream_t st);
// Largest CDF length the mask can need: max |z| <= sqrt(m - 1).
int mask_table_max(int m);
void launch_mask(const DevSeries& S, unsigned int* counts, int lt_max, double* diff,
                 double* mean_acc, float* zmax, cudaStream_t st);
// Row minima over partners j >= i + m on LB tiles (lb.cu layout).
// With tile_best (ntiles entries, 0xffffffff at launch): also each tile's
// smallest key high bits.
void launch_mp(const DevSeries& S, const Tile* tiles, int ntiles, unsigned long long* keys,
               cudaStream_t st, unsigned int* tile_best = nullptr);
// bsf2[t] = an upper bound on tile t's smallest squared DTW (its ED^2 minimum).
void launch_tile_bound(const unsigned int* tile_best, int ntiles, unsigned int* bsf2,
                       cudaStream_t st);
// Full profile: lo = row minima of the reversed series (nullptr: upper only).
void launch_mp_finalize(const DevSeries& S, const unsigned long long* up,
                        const unsigned long long* lo, double* mp, int64_t* mpi,
                        cudaStream_t st);
void launch_reverse(const double* a, int64_t n, double* out, cudaStream_t st);
// Exact profile: want / wrev = the smaller first-pass key of each row (by
// series row / by reversed row); the collect pass lists every pair whose high
// word is near its row's key; the exact pass computes their FP64 distance
// (pick = false: row minima of the bits, true: lowest partner at the minimum;
// reversed: the candidates are rows of the reversed series).
void launch_mp_want(int64_t s, const unsigned long long* up, const unsigned long long* lo,
                    unsigned long long* want, unsigned long long* wrev, cudaStream_t st);
void launch_mp_collect(const DevSeries& S, const Tile* tiles, int ntiles,
                       const unsigned long long* want, int2* cand, unsigned int* count,
                       unsigned int cap, cudaStream_t st);
void launch_mp_exact(const DevSeries& S, const int2* cand, const unsigned int* count,
                     unsigned int cap, bool reversed, bool pick, unsigned long long* rowmin,
                     unsigned long long* rowidx, cudaStream_t st);
void launch_mp_exact_out(int64_t s, const unsigned long long* rowmin,
                         const unsigned long long* rowidx, double* mp, int64_t* mpi,
                         cudaStream_t st);
// kSeeds seeds per series, each with its diagonal neighbours, into
// seeds[series * kSeedSlots ...] (unused slots hold (-1, -1)), their counts
// into nseeds[series].
void launch_seed_select(const DevSeries& S, const unsigned long long* keys, int2* seeds,
                        unsigned int* nseeds, cudaStream_t st);
// Row minima for the join's seeds on the rows of a kSeedGrid grid: FP64
// anchors and stage carries, FP32 increments within a stage (keys only rank
// the seed candidates).
void launch_mp_seed(const DevSeries& S, const Tile* tiles, int ntiles, unsigned long long* keys,
                    cudaStream_t st);
// Series of a sample (0 for a single series).
__device__ __forceinline__ int series_of(const DevSeries& S, int64_t x) {
  return S.sid ? S.sid[x] : 0;
}
// Fast diagonal bound over LB tiles [tile_begin, tile_end); survivors leave
// as bits, [tile][lag][word].  enumerate_all: no pruning (bounds off).
// Persistent: CTAs take tiles from the work counter *next (zero at launch).
void launch_lb(const DevSeries& S, const DevSearch& Q, const Tile* tiles, int tile_begin,
               int tile_end, unsigned int* bits, bool enumerate_all, unsigned int* next,
               int num_sms, cudaStream_t st);
size_t lb_smem_bytes();
// Run filter over the survivor bits of LB tiles [tile_begin, tile_end):
// masked bound, endpoint bound and LB_Keogh for every pair of every run of
// consecutive survivors; pairs that survive go to Q.queue.
void launch_runs(const DevSeries& S, const DevSearch& Q, const Tile* tiles, int tile_begin,
                 int tile_end, const unsigned int* bits, bool masked, bool bounds, int num_sms,
                 cudaStream_t st);
void launch_center(const DevSeries& S, cudaStream_t st);
// 64 features per tile for the learned ordering (features.cu), from the
// profile keys of the series' rows (every row keyed: grid 1; the seed
// profile: grid kSeedGrid); out[64 * t ...] for tile t.
void launch_tile_features(const DevSeries& S, const Tile* tiles, int ntiles,
                          const unsigned long long* keys, int grid, float* out, cudaStream_t st);
// Block-mean lower bound (LB_PAA) over the survivor bits of LB tiles
// [tile_begin, tile_end), then the endpoint bound; survivors go to Q.kq.
void launch_paa(const DevSeries& S, const DevSearch& Q, const Tile* tiles, int tile_begin,
                int tile_end, const unsigned int* bits, int num_sms, cudaStream_t st);
// Block length of the block-mean bound for windows of length m.
int paa_block(int m);
// Sliding block means (pq, or pq2 and wrec for windows of at most 1024
// samples), per-block magnitudes (cmax) and per-window error scales (rw);
// after launch_center.  Returns the number of kernels it launched.
int launch_paa_prep(const DevSeries& S, cudaStream_t st);
// LB_Keogh over the candidates the run filter queued in Q.kq; survivors go to
// Q.queue.
void launch_keogh(const DevSeries& S, const DevSearch& Q, int num_sms, cudaStream_t st);
// LB_Petitjean (csrc/petitjean.cu): the join stage filters the DTW queue of a
// chunk in place (next: a zeroed work counter); it runs when one warp's
// shared tables, 2 (m + 2w) doubles, fit kPjMaxSmemBytes.
constexpr size_t kPjMaxSmemBytes = 200 * 1024;
bool petitjean_fits(int m, int w);
void launch_petitjean(const DevSeries& S, const DevSearch& Q, unsigned int* next, int num_sms,
                      cudaStream_t st);
size_t lbp_list_bytes(int m, int w, bool own_env);
void launch_lbp_list(const DevSeries& S, const int2* pairs, int count, bool own_env,
                     double* keogh_mid, double* terms, int num_sms, cudaStream_t st);
// bounds = false: DTW only (the seeds); true: endpoint bound + LB_Keogh first
void launch_pairs(const DevSeries& S, const DevSearch& Q, const int2* pairs,
                  const unsigned int* npairs, bool bounds, BandShape band, int num_sms,
                  cudaStream_t st);
// FP64 re-verification of the candidates, then per series the lexicographic
// minimum (d2, i, j): best_d2[series] (FP64 squared distance, +inf if none),
// best_ij[series] = i << 32 | j, best_f32[series] = the search's FP32 d2.
void launch_verify(const DevSeries& S, const DevSearch& Q, BandShape band, double* out_d2,
                   unsigned long long* best_d2, unsigned long long* best_ij, float* best_f32,
                   cudaStream_t st);
}  // namespace dtwj
struct dtwj_mlp;
namespace dtwj {
// Tile scores for the learned order (mlp.cu): x_dev [count][64] on the
// device, after the work queued on st; y_dev [count].
int mlp_predict_device(dtwj_mlp* net, const float* x_dev, int64_t count, float* y_dev,
                       cudaStream_t st);
int mlp_device(const dtwj_mlp* net);
void launch_pair_dtw(const DevSeries& S, const int2* pairs, int count, bool precise,
                     BandShape band, double* out_d2, cudaStream_t st);

}  // namespace dtwj
