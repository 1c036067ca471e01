// Host orchestration of the join and the C ABI (include/dtwj.h).
//
// The reference's driver (GPU_version1/src/new_dtw_motifGUI_malloc.cu:30-816)
// prepares everything on the host, allocates one device buffer per
// subsequence and then loops over diagonal blocks with five launches and
// three host synchronisations per block.  Here every phase runs on one
// stream with device-resident state:
//   prep      statistics, envelopes, mask, row constants        (prep.cu)
//   profile   ED matrix profile, row minima                      (mp.cu)
//   seeds     kSeeds smallest profile entries -> exact DTW        (mp.cu, pairs.cu)
//   sweep     per chunk of tiles: diagonal bound -> survivor
//             queue -> endpoint / masked / LB_Keogh / DTW         (lb.cu, pairs.cu)
//   verify    FP64 DTW of every candidate near the final best     (pairs.cu)
// with a single host synchronisation at the end.
#include "../../include/dtwj.h"
#include "dtwj_dev.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

using namespace dtwj;

namespace {

constexpr unsigned int kCandCap = 1u << 20;
constexpr unsigned int kQueueCapMax = 1u << 26;
// Default tiles per chunk of the sweep: kLbChunkRounds tiles for each of the
// diagonal sweep's resident CTAs.  Its tiles take about the same time, so a
// chunk that is not a whole number of rounds leaves CTAs idle in its last
// round (1024 tiles on 444 CTAs: 2.3 rounds, the last one 31 % busy).  On
// the 1M-sample bench series 4 rounds (1776 tiles) measured best: 0.973 s
// per join against 0.998 s at 3 rounds, 0.980 s at 5, 0.985 s at 6 and
// 1.008 s at 1024 tiles.
constexpr int kLbChunkRounds = 4;
// Largest piece an overflowing chunk is swept again in.  Every piece that
// overflows again wastes a full DTW queue of work.  On the 262,144-sample
// ECG-like series at w = 103 nearly every pair reaches LB_Keogh, about 3.5
// million per tile by that join's stage counts, so 32 tiles fit the LB_Keogh
// queue (2^27 entries) and 55 would not.
constexpr int kResweepTiles = 32;
// (m, w) groups of a batch joined at the same time, one context each.
constexpr int kBatchWorkers = 4;

struct Buf {
  void* p = nullptr;
  size_t cap = 0;
};

struct Timer {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double seconds() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

// What one chunk of the sweep left behind: whether one of its queues
// overflowed (pairs were dropped, so the chunk is swept again), and the
// counters after it, so that a chunk swept again can be taken out of them.
struct ChunkNote {
  unsigned long long counters[kNumCounters];
  unsigned int overflow;
  unsigned int pad;
};

// Sort keys of the learned order: ascending score, NaN last; the radix sort
// is stable, so ties keep the plain order.
__global__ void k_order_keys(const float* score, int n, unsigned int* key, int* idx) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float f = score[t];
  const unsigned int u = __float_as_uint(f);
  key[t] = f != f ? 0xffffffffu : ((u & 0x80000000u) ? ~u : (u | 0x80000000u));
  idx[t] = t;
}

// Tiles in the sorted order, each with its position.
__global__ void k_gather_tiles(const Tile* plain, const int* idx, int n, Tile* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  Tile x = plain[idx[t]];
  x.order = t;
  out[t] = x;
}

// Runs after a chunk's last stage on the join's stream: notes the chunk and
// clears the overflow bit for the next one.
__global__ void k_chunk_note(int* status, const unsigned long long* counters, ChunkNote* note) {
  const int t = threadIdx.x;
  if (t < kNumCounters) note->counters[t] = counters[t];
  if (t == 0) {
    const int s = *status;
    note->overflow = (s & 2) ? 1u : 0u;
    *status = s & ~2;
  }
}

}  // namespace

struct dtwj_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  std::vector<Buf> bufs;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<Tile> lbtiles_host;    // kLbLags-lag tiles of the diagonal sweep
  int64_t lbtiles_n = -1, lbtiles_m = -1;  // single-series shape the tiles were built for
  std::vector<unsigned int> host_u32;      // staging of small host -> device copies
  std::vector<Tile> tiles_run;             // the tiles in the order of the current call
  dtwj_mlp* model = nullptr;               // scores tiles for DTWJ_F_LEARNED (not owned)
  std::vector<std::pair<int, BandShape>> band_override;  // band w -> DTW layout (autotuner)
  int dtw_warps = 0;    // CTA size of the join's DTW kernel in warps (0: default)
  int chunk_tiles = 0;  // tiles per chunk of the sweep (0: default)
  int shard_rank = 0, shard_world = 1;  // this context sweeps tiles t with t % world == rank
  dtwj_exchange_fn exchange = nullptr;  // best-so-far exchange between sweep phases
  void* exchange_user = nullptr;
  int exchange_phases = 0;
  std::vector<cudaEvent_t> pool;  // events for per-phase device times
  // the sweep's launches captured as a CUDA graph, replayed while every
  // launch argument is unchanged (same buffers, tiles, band, flags)
  cudaGraphExec_t sweep_exec = nullptr;
  std::vector<unsigned char> sweep_key;
  std::vector<int> sweep_marks;  // phase marks of the capture: (phase, a, b, launches)
  size_t sweep_ev0 = 0, sweep_ev1 = 0;
};

namespace {

enum BufId {
  B_A = 0, B_MU, B_SIG, B_ISG, B_FLAT, B_U, B_L, B_E, B_NU, B_DFA, B_DGA, B_DFE, B_DGE,
  B_AC, B_DUL, B_QSIG, B_MASK, B_MN, B_MDUL2, B_MDUL, B_SM, B_SME, B_STATUS,
  B_COUNTS, B_DIFF, B_MEAN, B_ZMAX, B_KEYS_UP, B_QUEUE, B_QCOUNT,
  B_BSF2, B_COUNTERS, B_CAND, B_CCOUNT, B_SEEDS, B_NSEEDS, B_VERIFY, B_BEST, B_PAIRS, B_OUT,
  B_MP, B_MPI, B_CB, B_AF, B_ULF, B_BITS, B_LBTILES, B_KQ, B_SBEG, B_SID, B_SEEDBSF,
  B_BEST_IJ, B_BEST_F32, B_QSER, B_TILEBEST, B_FEAT, B_SCORE, B_PA, B_CMAX, B_RW,
  B_MPX_WANT, B_MPX_WREV, B_MPX_MIN, B_MPX_IDX, B_MPX_CAND, B_MPX_CNT, B_NOTES, B_NOTES2,
  B_SORT, B_SORT_TEMP, B_LBTILES2, B_CMAX2, B_WREC, B_COUNT_
};

int ensure(dtwj_ctx* c, int id, size_t bytes, void** out) {
  if (c->bufs.size() < (size_t)B_COUNT_) c->bufs.resize(B_COUNT_);
  Buf& b = c->bufs[id];
  if (b.cap < bytes) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    size_t want = bytes < 256 ? 256 : bytes;
    if (cudaMalloc(&b.p, want) != cudaSuccess) {
      cudaGetLastError();
      return DTWJ_ERR_OOM;
    }
    b.cap = want;
  }
  *out = b.p;
  return DTWJ_OK;
}

#define ENSURE(id, bytes, ptr)                                       \
  do {                                                               \
    void* _p = nullptr;                                              \
    int _rc = ensure(ctx, id, (size_t)(bytes), &_p);                 \
    if (_rc) return _rc;                                             \
    ptr = reinterpret_cast<decltype(ptr)>(_p);                       \
  } while (0)

#define CUDA_OK(expr)                                                 \
  do {                                                                \
    cudaError_t _e = (expr);                                          \
    if (_e != cudaSuccess) {                                          \
      if (getenv("DTWJ_DEBUG"))                                       \
        fprintf(stderr, "dtwj: %s failed: %s\n", #expr, cudaGetErrorString(_e)); \
      return DTWJ_ERR_CUDA;                                           \
    }                                                                 \
  } while (0)

// Per-phase device time from CUDA events recorded on the join's stream
// (DTWJ_F_PROFILE); a no-op otherwise.
struct Phases {
  dtwj_ctx* ctx;
  bool on;
  size_t used = 0;
  struct Mark {
    int phase;
    size_t a, b;
    int launches;
  };
  std::vector<Mark> marks;
  size_t open_at = 0;
  Phases(dtwj_ctx* c, bool enabled) : ctx(c), on(enabled) {}
  cudaEvent_t ev(size_t k) {
    while (ctx->pool.size() <= k) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      ctx->pool.push_back(e);
    }
    return ctx->pool[k];
  }
  // While the stream is being captured, records are external: they become
  // event-record nodes of the graph (a plain record would only order the
  // capture, and the external flag is refused outside a capture).
  bool capturing = false;
  void record(cudaEvent_t e) {
    if (capturing) cudaEventRecordWithFlags(e, ctx->stream, cudaEventRecordExternal);
    else cudaEventRecord(e, ctx->stream);
  }
  void begin() {
    if (!on) return;
    open_at = used;
    record(ev(used++));
  }
  void end(int phase, int launches) {
    if (!on) return;
    record(ev(used));
    marks.push_back({phase, open_at, used, launches});
    ++used;
  }
  void collect(dtwj_result* out) {
    for (auto& mk : marks) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ctx->pool[mk.a], ctx->pool[mk.b]) != cudaSuccess) {
        cudaGetLastError();  // a mark without a time must not fail the next call
        ms = 0.f;
      }
      out->phase_seconds[mk.phase] += ms / 1000.0;
      out->phase_launches[mk.phase] += (uint64_t)mk.launches;
    }
  }
};

int check_args(const void* x, int64_t n, int32_t m, int32_t w) {
  if (!x || m < 8 || m > DTWJ_MAX_M || w < 0) return DTWJ_ERR_ARG;
  if (n < 2 * (int64_t)m + 1 || n > (int64_t)INT32_MAX - 4) return DTWJ_ERR_ARG;
  return DTWJ_OK;
}

// Tiles of the profile and the diagonal sweep (kLbLags lags x kLbRows rows)
// for every series; a single series keeps its tiles across calls.
void build_lb_tiles(dtwj_ctx* ctx, int64_t n, int m, const int64_t* sbeg, int nseries) {
  if (!sbeg && ctx->lbtiles_n == n && ctx->lbtiles_m == m) return;
  ctx->lbtiles_host.clear();
  int32_t order = 0;
  for (int r = 0; r < nseries; ++r) {
    const int64_t wb = sbeg ? sbeg[r] : 0;
    const int64_t s = (sbeg ? sbeg[r + 1] - sbeg[r] : n) - m + 1;
    for (int64_t L0 = m; L0 <= s - 1; L0 += kLbLags) {
      const int64_t rows_total = s - L0;
      for (int64_t i0 = 0; i0 < rows_total; i0 += kLbRows) {
        Tile t;
        t.L0 = (int32_t)L0;
        t.i0 = (int32_t)(wb + i0);
        t.rows = (int32_t)(rows_total - i0 < kLbRows ? rows_total - i0 : kLbRows);
        t.order = order++;
        t.send = (int32_t)(wb + s);
        t.series = r;
        ctx->lbtiles_host.push_back(t);
      }
    }
  }
  ctx->lbtiles_n = sbeg ? -1 : n;
  ctx->lbtiles_m = sbeg ? -1 : m;
}

// Allocates and prepares every per-series array; returns the DevSeries.  A
// batch (sbeg != nullptr) holds nseries series back to back in x_dev, series
// r on samples [sbeg[r], sbeg[r + 1]).
int prepare(dtwj_ctx* ctx, const double* x_dev, int64_t n, int m, int w, bool masked,
            const int64_t* sbeg_host, int nseries, DevSeries* out, Phases* ph = nullptr) {
  const int64_t s = n - m + 1;
  DevSeries S;
  memset(&S, 0, sizeof S);
  S.a = x_dev;
  S.n = n;
  S.s = s;
  S.m = m;
  S.w = w;
  S.nseries = nseries;
  if (sbeg_host) {
    int64_t* sbeg;
    int* sid;
    ENSURE(B_SBEG, (size_t)(nseries + 1) * 8, sbeg);
    ENSURE(B_SID, (size_t)n * 4, sid);
    CUDA_OK(cudaMemcpyAsync(sbeg, sbeg_host, (size_t)(nseries + 1) * 8, cudaMemcpyHostToDevice,
                            ctx->stream));
    launch_series_ids(sbeg, nseries, sid, n, ctx->stream);
    S.sbeg = sbeg;
    S.sid = sid;
  }
  ENSURE(B_MU, s * 8, S.mu);
  ENSURE(B_SIG, s * 8, S.sig);
  ENSURE(B_ISG, s * 8, S.isg);
  ENSURE(B_FLAT, s, S.flat);
  ENSURE(B_U, n * 8, S.U);
  ENSURE(B_L, n * 8, S.L);
  ENSURE(B_E, n * 8, S.E);
  ENSURE(B_NU, s * 8, S.nu);
  ENSURE(B_DFA, s * 8, S.dfa);
  ENSURE(B_DGA, s * 8, S.dga);
  ENSURE(B_DFE, s * 8, S.dfE);
  ENSURE(B_DGE, s * 8, S.dgE);
  ENSURE(B_AC, s * 8, S.A);
  ENSURE(B_DUL, s * 8, S.DUL);
  ENSURE(B_QSIG, s * 8, S.qsig);
  ENSURE(B_MASK, n * 4, S.mask);
  ENSURE(B_MN, s * 4, S.MN);
  ENSURE(B_MDUL2, s * 4, S.MDUL2);
  ENSURE(B_MDUL, s * 4, S.MDUL);
  ENSURE(B_SM, s * 8, S.SM);
  ENSURE(B_SME, s * 8, S.SME);
  ENSURE(B_CB, ((n >> kBlkShift) + 4) * 8, S.cb);
  ENSURE(B_AF, n * 4, S.af);
  ENSURE(B_ULF, n * 8, S.ulf);
  if (m <= (1 << kBlkShift)) {
    ENSURE(B_PA, (size_t)n * 32, S.pq2);
    ENSURE(B_CMAX2, (size_t)kCopyBlocks(n) * 8, S.cmax2);
    ENSURE(B_WREC, (size_t)s * 16, S.wrec);
  } else {
    ENSURE(B_PA, (size_t)n * 16, S.pq);
  }
  ENSURE(B_CMAX, ((n >> kBlkShift) + 4) * 4, S.cmax);
  ENSURE(B_RW, s * 4, S.rw);
  S.paa_b = paa_block(m);
  ENSURE(B_STATUS, 4, S.status);
  cudaStream_t st = ctx->stream;
  CUDA_OK(cudaMemsetAsync(S.status, 0, 4, st));
  launch_check_finite(S.a, n, S.status, st);
  int status = 0;
  CUDA_OK(cudaMemcpyAsync(&status, S.status, 4, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  if (status & 1) return DTWJ_ERR_NAN;
  if (ph) ph->begin();
  launch_prep(S, st);
  if (masked) {
    const int lt_max = mask_table_max(m);
    unsigned int* counts;
    double* diff;
    double* mean;
    float* zmax;
    ENSURE(B_COUNTS, (size_t)m * lt_max * 4, counts);
    ENSURE(B_DIFF, n * 8, diff);
    ENSURE(B_MEAN, 8, mean);
    ENSURE(B_ZMAX, 4, zmax);
    if (!sbeg_host) {
      launch_mask(S, counts, lt_max, diff, mean, zmax, st);
    } else {
      // the mask's CDF tables are per series: build it on a view of each one
      for (int r = 0; r < nseries; ++r) {
        const int64_t b = sbeg_host[r], nr = sbeg_host[r + 1] - b;
        DevSeries V = S;
        V.a = S.a + b;
        V.n = nr;
        V.s = nr - m + 1;
        V.mu = S.mu + b;
        V.sig = S.sig + b;
        V.isg = S.isg + b;
        V.flat = S.flat + b;
        V.U = S.U + b;
        V.L = S.L + b;
        V.mask = S.mask + b;
        V.sid = nullptr;
        V.sbeg = nullptr;
        V.nseries = 1;
        launch_mask(V, counts, lt_max, diff, mean, zmax, st);
      }
    }
  } else {
    CUDA_OK(cudaMemsetAsync(S.mask, 0, n * 4, st));
  }
  launch_rowterms(S, masked, st);
  launch_center(S, st);
  const int paa_launches = launch_paa_prep(S, st);
  if (ph) ph->end(DTWJ_PHASE_PREP, (masked ? 11 : 6) + paa_launches);
  CUDA_OK(cudaGetLastError());
  *out = S;
  return DTWJ_OK;
}

int effective_band(int m, int w) { return w > m - 1 ? m - 1 : w; }

// Per-tile outputs of dtwj_ctx_tiles (host arrays, one entry per tile).
struct TileQuery {
  float* features;   // [tiles][64] or nullptr
  double* min_dist;  // exact smallest DTW distance per tile, or nullptr
};

// Joins one series (sbeg == nullptr, nseries == 1) or a batch of nseries
// series of one (m, w) stored back to back (series r on samples
// [sbeg[r], sbeg[r + 1])); outs[r] receives series r's top-1 pair with
// indices relative to its own first sample.  With tq (one series) the call
// reports per-tile values instead of a join: the tile features, and with
// tq->min_dist the exact smallest DTW distance of every tile, found by a sweep
// in which every tile prunes against its own best-so-far only.
int run_join(dtwj_ctx* ctx, const double* x_dev, int64_t n, const int64_t* sbeg, int nseries,
             int32_t m, int32_t w_in, uint32_t flags, dtwj_result* outs, double t_upload,
             const TileQuery* tq = nullptr) {
  Timer wall;
  const int w = effective_band(m, w_in);
  BandShape band;
  if (!choose_band(w, &band)) return DTWJ_ERR_BAND;
  for (const auto& bo : ctx->band_override)
    if (bo.first == w) band = bo.second;
  band.warps = ctx->dtw_warps;
  const bool learned = (flags & DTWJ_F_LEARNED) && !tq;
  if (learned && !ctx->model) return DTWJ_ERR_NOMODEL;
  if (learned && mlp_device(ctx->model) != ctx->device) return DTWJ_ERR_ARG;
  const bool tile_mode = tq && tq->min_dist;
  // the run filter: the block-mean bound (default), or the reference's masked
  // diagonal bound and endpoint bound (DTWJ_F_MASKED_CASCADE)
  const bool cascade = (flags & DTWJ_F_MASKED_CASCADE) != 0;
  const bool masked = cascade && !(flags & DTWJ_F_NO_MASKED) && !(flags & DTWJ_F_NO_DIAG);
  const bool verbose = flags & DTWJ_F_VERBOSE;
  // LB_Petitjean between LB_Keogh and DTW, where its shared tables fit
  const bool petitjean = (flags & DTWJ_F_PETITJEAN) && !(flags & DTWJ_F_NO_DIAG) &&
                         petitjean_fits(m, w);
  cudaStream_t st = ctx->stream;
  Phases ph(ctx, (flags & DTWJ_F_PROFILE) != 0);
  CUDA_OK(cudaEventRecord(ctx->ev0, st));

  DevSeries S;
  int rc = prepare(ctx, x_dev, n, m, w, masked, sbeg, nseries, &S, &ph);
  if (rc) return rc;

  build_lb_tiles(ctx, n, m, sbeg, nseries);
  std::vector<Tile>& th = ctx->tiles_run;
  th = ctx->lbtiles_host;
  if (ctx->shard_world > 1 && !tq) {
    // one shard of the tiles (round robin): the profile, the seeds and the
    // sweep only see these; the shards' results combine by their minimum
    size_t k = 0;
    for (size_t t = 0; t < th.size(); ++t)
      if ((int)(t % (size_t)ctx->shard_world) == ctx->shard_rank) th[k++] = th[t];
    th.resize(k);
  }
  const int nlb = (int)th.size();
  // best-so-far slots: one per series, or one per tile for the tile minima
  const int nslots = tile_mode ? (nlb > 0 ? nlb : 1) : nseries;
  S.nseries = nslots;
  if (tile_mode)
    for (int t = 0; t < nlb; ++t) th[t].series = t;
  Tile* lbtiles;
  ENSURE(B_LBTILES, (size_t)(nlb > 0 ? nlb : 1) * sizeof(Tile), lbtiles);
  if (nlb > 0)
    CUDA_OK(cudaMemcpyAsync(lbtiles, th.data(), (size_t)nlb * sizeof(Tile),
                            cudaMemcpyHostToDevice, st));

  // search state
  DevSearch Q;
  memset(&Q, 0, sizeof Q);
  unsigned int qcap = kQueueCapMax;
  if (const char* env = getenv("DTWJ_QUEUE_CAP")) {  // smaller queue (profiling, tests)
    const long v = atol(env);
    if (v >= 1024 && v < (long)kQueueCapMax) qcap = (unsigned int)v;
  }
  ENSURE(B_QUEUE, (size_t)qcap * sizeof(int2), Q.queue);
  // LB_Keogh candidates of one chunk: twice the DTW queue (most are pruned)
  ENSURE(B_KQ, (size_t)qcap * 2 * sizeof(int4), Q.kq);
  unsigned int* qc;
  ENSURE(B_QCOUNT, 32, qc);
  Q.queue_count = qc;
  Q.queue_next = qc + 1;
  Q.run_count = qc + 2;
  Q.run_next = qc + 3;
  Q.kq_count = qc + 4;
  Q.kq_next = qc + 5;
  unsigned int* lb_next = qc + 6;
  Q.queue_cap = qcap;
  Q.kq_cap = qcap * 2;
  Q.runs = nullptr;
  Q.run_cap = 0;
  ENSURE(B_BSF2, (size_t)nslots * 4, Q.bsf2);
  ENSURE(B_COUNTERS, kNumCounters * 8, Q.counters);
  // the tile minima keep a few candidates per tile
  const unsigned int cand_cap =
      tile_mode && 16u * (unsigned int)nlb > kCandCap ? 16u * (unsigned int)nlb : kCandCap;
  ENSURE(B_CAND, (size_t)cand_cap * sizeof(Candidate), Q.cand);
  ENSURE(B_CCOUNT, 4, Q.cand_count);
  Q.cand_cap = cand_cap;
  if (tile_mode) ENSURE(B_QSER, (size_t)qcap * sizeof(int), Q.qser);
  CUDA_OK(cudaMemsetAsync(Q.counters, 0, kNumCounters * 8, st));
  CUDA_OK(cudaMemsetAsync(Q.cand_count, 0, 4, st));
  ctx->host_u32.assign((size_t)nslots + 1, 0x7f800000u);  // +inf per slot
  CUDA_OK(cudaMemcpyAsync(Q.bsf2, ctx->host_u32.data(), (size_t)nslots * 4,
                          cudaMemcpyHostToDevice, st));
  unsigned int* seed_bsf;
  ENSURE(B_SEEDBSF, (size_t)nslots * 4, seed_bsf);

  // ---- ED matrix profile (row minima; per tile for the tile minima) ----
  const bool want_features = learned || (tq && tq->features);
  unsigned long long* keys = nullptr;
  if (nlb > 0 && (tile_mode || want_features || !(flags & DTWJ_F_NO_SEED))) {
    ENSURE(B_KEYS_UP, S.s * 8, keys);
    unsigned int* tbest = nullptr;
    if (tile_mode) {
      ENSURE(B_TILEBEST, (size_t)nlb * 4, tbest);
      CUDA_OK(cudaMemsetAsync(tbest, 0xff, (size_t)nlb * 4, st));
    }
    ph.begin();
    // a join only ranks seed candidates by these keys (mixed precision, one
    // row in kSeedGrid); the per-tile minima and the exported features take
    // the exact FP64 profile of every row
    if (tq) launch_mp(S, lbtiles, nlb, keys, st, tbest);
    else launch_mp_seed(S, lbtiles, nlb, keys, st);
    if (tile_mode) launch_tile_bound(tbest, nlb, Q.bsf2, st);
    ph.end(DTWJ_PHASE_PROFILE, 2);
  }
  // ---- tile features; the learned order sorts the tiles by their score ----
  if (want_features && nlb > 0) {
    float* feat;
    ENSURE(B_FEAT, (size_t)nlb * DTWJ_MLP_IN * 4, feat);
    launch_tile_features(S, lbtiles, nlb, keys, tq ? 1 : kSeedGrid, feat, st);
    if (tq && tq->features)
      CUDA_OK(cudaMemcpyAsync(tq->features, feat, (size_t)nlb * DTWJ_MLP_IN * 4,
                              cudaMemcpyDeviceToHost, st));
    if (learned) {
      float* score;
      ENSURE(B_SCORE, (size_t)nlb * 4, score);
      rc = mlp_predict_device(ctx->model, feat, nlb, score, st);
      if (rc) return rc;
      // ascending predicted minimum; ties (and NaN scores, last) keep the
      // plain order: a stable radix sort of (score key, tile) on the device,
      // then the tiles gathered in that order
      unsigned int* sk;
      ENSURE(B_SORT, (size_t)nlb * 16, sk);
      unsigned int* sk_out = sk + nlb;
      int* si = reinterpret_cast<int*>(sk + 2 * (size_t)nlb);
      int* si_out = si + nlb;
      const unsigned int nb = (unsigned int)((nlb + 255) / 256);
      k_order_keys<<<nb, 256, 0, st>>>(score, nlb, sk, si);
      size_t temp_bytes = 0;
      CUDA_OK(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, sk, sk_out, si, si_out, nlb,
                                              0, 32, st));
      void* temp;
      ENSURE(B_SORT_TEMP, temp_bytes > 0 ? temp_bytes : 16, temp);
      CUDA_OK(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, sk, sk_out, si, si_out, nlb, 0,
                                              32, st));
      Tile* sorted;
      ENSURE(B_LBTILES2, (size_t)nlb * sizeof(Tile), sorted);
      k_gather_tiles<<<nb, 256, 0, st>>>(lbtiles, si_out, nlb, sorted);
      CUDA_OK(cudaMemcpyAsync(lbtiles, sorted, (size_t)nlb * sizeof(Tile),
                              cudaMemcpyDeviceToDevice, st));
    }
  }
  if (tq && !tile_mode) {
    CUDA_OK(cudaStreamSynchronize(st));
    return DTWJ_OK;
  }

  // ---- ED profile seeds ----
  if (!tile_mode && !(flags & DTWJ_F_NO_SEED) && nlb > 0) {
    int2* seeds;
    unsigned int* nseeds;  // [nseries] counts, total slots, work counter
    ENSURE(B_SEEDS, (size_t)nseries * kSeedSlots * sizeof(int2), seeds);
    ENSURE(B_NSEEDS, ((size_t)nseries + 2) * 4, nseeds);
    ctx->host_u32[0] = (unsigned int)(nseries * kSeedSlots);
    CUDA_OK(cudaMemcpyAsync(nseeds + nseries, ctx->host_u32.data(), 4, cudaMemcpyHostToDevice,
                            st));
    CUDA_OK(cudaMemsetAsync(nseeds + nseries + 1, 0, 4, st));
    ph.begin();
    launch_seed_select(S, keys, seeds, nseeds, st);
    DevSearch Qs = Q;
    Qs.qser = nullptr;
    Qs.queue_next = nseeds + nseries + 1;
    Qs.queue_cap = (unsigned int)(nseries * kSeedSlots);
    launch_pairs(S, Qs, seeds, nseeds + nseries, false, band, ctx->num_sms, st);
    ph.end(DTWJ_PHASE_SEEDS, 2);
  }
  CUDA_OK(cudaMemcpyAsync(seed_bsf, Q.bsf2, (size_t)nslots * 4, cudaMemcpyDeviceToDevice, st));

  // ---- diagonal sweep in chunks of LB tiles ----
  const bool enumerate_all = flags & DTWJ_F_NO_DIAG;
  const double tile_pairs = (double)kLbLags * kLbRows;
  int chunk = ctx->chunk_tiles > 0 ? ctx->chunk_tiles
                                   : kLbChunkRounds * kLbCtasPerSm * ctx->num_sms;
  if (enumerate_all) chunk = (int)((double)qcap / tile_pairs) > 0 ? (int)((double)qcap / tile_pairs) : 1;
  unsigned int* bits;
  ENSURE(B_BITS, (size_t)(chunk < nlb ? chunk : (nlb > 0 ? nlb : 1)) * kLbLags * kLbWords * 4, bits);
  // the stages after the diagonal bound of one chunk: run filter, LB_Keogh, DTW
  auto filter_chunk = [&](int t0, int t1) {
    ph.begin();
    if (enumerate_all || cascade)
      launch_runs(S, Q, lbtiles, t0, t1, bits, masked, !enumerate_all, ctx->num_sms, st);
    else
      launch_paa(S, Q, lbtiles, t0, t1, bits, ctx->num_sms, st);
    ph.end(DTWJ_PHASE_RUNS, 1);
    if (!enumerate_all) {
      ph.begin();
      launch_keogh(S, Q, ctx->num_sms, st);
      if (petitjean) launch_petitjean(S, Q, qc + 7, ctx->num_sms, st);
      ph.end(DTWJ_PHASE_KEOGH, petitjean ? 2 : 1);
    }
    ph.begin();
    launch_pairs(S, Q, Q.queue, Q.queue_count, true, band, ctx->num_sms, st);
    ph.end(DTWJ_PHASE_PAIRS, 1);
  };
  // one pass over tile ranges: bound sweep, run filter, LB_Keogh, DTW, and a
  // note of each range (queue overflow, counters after it); notes[0] holds
  // the counters before the pass, notes[c + 1] those after range c
  using Range = std::pair<int, int>;
  auto sweep_range = [&](const Range& r, ChunkNote* note) {
    CUDA_OK(cudaMemsetAsync(qc, 0, 32, st));
    ph.begin();
    launch_lb(S, Q, lbtiles, r.first, r.second, bits, enumerate_all, lb_next, ctx->num_sms, st);
    ph.end(DTWJ_PHASE_DIAG, 1);
    filter_chunk(r.first, r.second);
    k_chunk_note<<<1, 32, 0, st>>>(S.status, Q.counters, note);
    return DTWJ_OK;
  };
  auto sweep = [&](const std::vector<Range>& rg, ChunkNote* notes) -> int {
    k_chunk_note<<<1, 32, 0, st>>>(S.status, Q.counters, notes);
    for (size_t c = 0; c < rg.size(); ++c) sweep_range(rg[c], notes + c + 1);
    CUDA_OK(cudaGetLastError());
    return DTWJ_OK;
  };
  std::vector<Range> ranges;
  for (int t0 = 0; t0 < nlb; t0 += chunk) ranges.push_back({t0, t0 + chunk < nlb ? t0 + chunk : nlb});
  ChunkNote* notes;
  ENSURE(B_NOTES, (ranges.size() + 1) * sizeof(ChunkNote), notes);
  // a sharded join with an exchange sweeps its tiles in phases and lets the
  // caller lower the best-so-far between them (direct launches)
  const bool exchanging = ctx->exchange && ctx->shard_world > 1 && !tq;
  auto sweep_phased = [&]() -> int {
    const int P = ctx->exchange_phases;
    k_chunk_note<<<1, 32, 0, st>>>(S.status, Q.counters, notes);
    size_t c = 0;
    for (int ph_i = 0; ph_i < P; ++ph_i) {
      const int b = (int)((int64_t)nlb * (ph_i + 1) / P);
      for (; c < ranges.size() && ranges[c].second <= b; ++c)
        sweep_range(ranges[c], notes + c + 1);
      ctx->exchange(ctx->exchange_user, Q.bsf2, nslots, (void*)st);
    }
    for (; c < ranges.size(); ++c) sweep_range(ranges[c], notes + c + 1);
    CUDA_OK(cudaGetLastError());
    return DTWJ_OK;
  };
  // A batch sweeps chunk by chunk and checks each one: its short series put
  // many tiles' survivors into one chunk, and when a chunk's queues
  // overflow, the counters go back to before it, it is swept again in
  // chunks an eighth its size, and the size grows back after chunks that
  // fit, up to half the size that overflowed (a pass that is checked only at
  // its end would sweep every overflowing chunk twice).
  const bool adaptive = sbeg != nullptr && !exchanging && nlb > 0;
  if (adaptive) {
    ChunkNote* an;
    ENSURE(B_NOTES2, 2 * sizeof(ChunkNote), an);
    k_chunk_note<<<1, 32, 0, st>>>(S.status, Q.counters, an);
    int ch = chunk, ch_max = chunk;
    size_t resweeps = 0;
    for (int t0 = 0; t0 < nlb;) {
      const int t1 = t0 + ch < nlb ? t0 + ch : nlb;
      sweep_range({t0, t1}, an + 1);
      ChunkNote h[2];
      CUDA_OK(cudaMemcpyAsync(h, an, sizeof h, cudaMemcpyDeviceToHost, st));
      CUDA_OK(cudaStreamSynchronize(st));
      if (!h[1].overflow) {
        CUDA_OK(cudaMemcpyAsync(an, an + 1, sizeof(ChunkNote), cudaMemcpyDeviceToDevice, st));
        t0 = t1;
        ch = 2 * ch < ch_max ? 2 * ch : ch_max;
        continue;
      }
      if (t1 - t0 == 1) return DTWJ_ERR_OVERFLOW;
      ++resweeps;
      CUDA_OK(cudaMemcpyAsync(Q.counters, h[0].counters, sizeof h[0].counters,
                              cudaMemcpyHostToDevice, st));
      CUDA_OK(cudaStreamSynchronize(st));  // h is read before it goes out of scope
      ch_max = (t1 - t0) / 2 > 0 ? (t1 - t0) / 2 : 1;
      ch = (t1 - t0) / 8 > 0 ? (t1 - t0) / 8 : 1;
    }
    CUDA_OK(cudaGetLastError());
    if (verbose && resweeps)
      fprintf(stderr, "dtwj: %zu chunks swept again in smaller chunks\n", resweeps);
    ranges.clear();
  }
  for (int attempt = 0; !adaptive; ++attempt) {
    bool swept = false;
    ChunkNote* pass_notes = notes;
    // only the first pass exchanges: a shard whose queues overflowed sweeps
    // those chunks again alone, and every shard must make the same exchange
    // calls
    if (exchanging && attempt == 0) {
      const int src = sweep_phased();
      if (src) return src;
      swept = true;
    }
    if (!swept && attempt == 0 && !(flags & DTWJ_F_NO_GRAPH) && nlb > 0) {
      // the first pass runs as a CUDA graph: replayed if this context captured
      // the same launches before, captured (then launched) otherwise
      std::vector<unsigned char> key;
      auto put = [&key](const void* p, size_t bytes) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        key.insert(key.end(), b, b + bytes);
      };
      const int band_cg[3] = {band.C, band.G, band.warps};
      const int64_t misc[12] = {nlb, chunk, enumerate_all, masked, cascade, petitjean,
                                ctx->num_sms, ph.on,
                                (int64_t)ph.used, (int64_t)(uintptr_t)lbtiles,
                                (int64_t)(uintptr_t)bits, (int64_t)(uintptr_t)notes};
      put(&S, sizeof S);
      put(&Q, sizeof Q);
      put(band_cg, sizeof band_cg);
      put(misc, sizeof misc);
      if (ctx->sweep_exec && key == ctx->sweep_key) {
        CUDA_OK(cudaGraphLaunch(ctx->sweep_exec, st));
        for (size_t k = 0; k + 3 < ctx->sweep_marks.size(); k += 4)
          ph.marks.push_back({ctx->sweep_marks[k], (size_t)ctx->sweep_marks[k + 1],
                              (size_t)ctx->sweep_marks[k + 2], ctx->sweep_marks[k + 3]});
        ph.used = ctx->sweep_ev1;
        swept = true;
      } else {
        if (ctx->sweep_exec) cudaGraphExecDestroy(ctx->sweep_exec);
        ctx->sweep_exec = nullptr;
        ctx->sweep_key.clear();
        const size_t u0 = ph.used, m0 = ph.marks.size();
        // events the capture records must exist before it starts
        if (ph.on) ph.ev(u0 + 8 * ranges.size() + 8);
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        bool ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
          ph.capturing = true;
          const int src = sweep(ranges, notes);
          ph.capturing = false;
          ok = cudaStreamEndCapture(st, &graph) == cudaSuccess && src == DTWJ_OK && graph;
        }
        if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
        if (graph) cudaGraphDestroy(graph);
        if (ok && cudaGraphLaunch(exec, st) == cudaSuccess) {
          ctx->sweep_exec = exec;
          ctx->sweep_key = key;
          ctx->sweep_marks.clear();
          for (size_t k = m0; k < ph.marks.size(); ++k) {
            const auto& mk = ph.marks[k];
            ctx->sweep_marks.insert(ctx->sweep_marks.end(),
                                    {mk.phase, (int)mk.a, (int)mk.b, mk.launches});
          }
          ctx->sweep_ev0 = u0;
          ctx->sweep_ev1 = ph.used;
          swept = true;
        } else {
          // not capturable here: fall back to direct launches
          if (exec) cudaGraphExecDestroy(exec);
          cudaGetLastError();
          ph.used = u0;
          ph.marks.resize(m0);
        }
      }
    }
    if (!swept) {
      if (attempt > 0) {
        // the chunks swept again get notes of their own (the first pass's
        // buffer stays as the captured graph knows it)
        ENSURE(B_NOTES2, (ranges.size() + 1) * sizeof(ChunkNote), pass_notes);
      }
      const int src = sweep(ranges, pass_notes);
      if (src) return src;
    }
    // a chunk whose queue overflowed lost pairs: take its counts out and
    // sweep it again in smaller chunks (the other chunks stand)
    if (ranges.empty()) break;
    std::vector<ChunkNote> nh(ranges.size() + 1);
    CUDA_OK(cudaMemcpyAsync(nh.data(), pass_notes, nh.size() * sizeof(ChunkNote),
                            cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    std::vector<Range> again;
    unsigned long long drop[kNumCounters] = {0};
    size_t nbad = 0;
    for (size_t c = 0; c < ranges.size(); ++c) {
      if (!nh[c + 1].overflow) continue;
      ++nbad;
      for (int k = 0; k < kNumCounters; ++k)
        drop[k] += nh[c + 1].counters[k] - nh[c].counters[k];
      const int t0 = ranges[c].first, t1 = ranges[c].second;
      if (t1 - t0 == 1 || attempt >= 4) return DTWJ_ERR_OVERFLOW;
      int sub = (t1 - t0) / 32;
      if (sub > kResweepTiles) sub = kResweepTiles;
      if (sub < 1) sub = 1;
      for (int u = t0; u < t1; u += sub) again.push_back({u, u + sub < t1 ? u + sub : t1});
    }
    if (again.empty()) break;
    if (verbose)
      fprintf(stderr, "dtwj: queue overflow in %zu of %zu chunks, sweeping them again in %zu\n",
              nbad, ranges.size(), again.size());
    unsigned long long kept[kNumCounters];
    for (int k = 0; k < kNumCounters; ++k) kept[k] = nh.back().counters[k] - drop[k];
    CUDA_OK(cudaMemcpyAsync(Q.counters, kept, sizeof kept, cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaStreamSynchronize(st));  // kept is read before it goes out of scope
    ranges.swap(again);
  }

  // ---- FP64 verification of the candidates, per-series minimum ----
  double* vd2;
  ENSURE(B_VERIFY, (size_t)kCandCap * 8, vd2);
  unsigned long long *best_d2, *best_ij;
  float* best_f32;
  ENSURE(B_BEST, (size_t)nslots * 8, best_d2);
  ENSURE(B_BEST_IJ, (size_t)nslots * 8, best_ij);
  ENSURE(B_BEST_F32, (size_t)nslots * 4, best_f32);
  ph.begin();
  launch_verify(S, Q, band, vd2, best_d2, best_ij, best_f32, st);
  ph.end(DTWJ_PHASE_VERIFY, 4);
  CUDA_OK(cudaEventRecord(ctx->ev1, st));

  std::vector<unsigned long long> d2_h(nslots), ij_h(nslots);
  std::vector<unsigned int> f32_h(nslots), seed_h(nslots);
  unsigned long long cnt_h[kNumCounters];
  unsigned int cand_h = 0;
  int status_h = 0;
  CUDA_OK(cudaMemcpyAsync(d2_h.data(), best_d2, (size_t)nslots * 8, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaMemcpyAsync(ij_h.data(), best_ij, (size_t)nslots * 8, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaMemcpyAsync(f32_h.data(), best_f32, (size_t)nslots * 4, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaMemcpyAsync(seed_h.data(), seed_bsf, (size_t)nslots * 4, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaMemcpyAsync(cnt_h, Q.counters, sizeof cnt_h, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaMemcpyAsync(&cand_h, Q.cand_count, 4, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaMemcpyAsync(&status_h, S.status, 4, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  if (status_h & 2) return DTWJ_ERR_OVERFLOW;
  if (cand_h > cand_cap) return DTWJ_ERR_OVERFLOW;
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  if (tile_mode) {
    for (int t = 0; t < nlb; ++t) {
      double d2;
      memcpy(&d2, &d2_h[t], 8);
      tq->min_dist[t] = d2_h[t] != ~0ull ? std::sqrt(d2) : INFINITY;
    }
    return DTWJ_OK;
  }

  for (int r = 0; r < nseries; ++r) {
    dtwj_result* out = &outs[r];
    memset(out, 0, sizeof *out);
    const int64_t base = sbeg ? sbeg[r] : 0;
    out->n = sbeg ? sbeg[r + 1] - sbeg[r] : n;
    out->m = m;
    out->w = w_in;
    if (d2_h[r] != ~0ull) {
      double d2;
      memcpy(&d2, &d2_h[r], 8);
      float f2;
      memcpy(&f2, &f32_h[r], 4);
      out->i = (int64_t)(ij_h[r] >> 32) - base;
      out->j = (int64_t)(ij_h[r] & 0xffffffffull) - base;
      out->dist = std::sqrt(d2);
      out->dist_fp32 = std::sqrt((double)f2);
    } else {
      out->i = out->j = -1;
      out->dist = out->dist_fp32 = INFINITY;
    }
    float sb;
    memcpy(&sb, &seed_h[r], 4);
    out->seed_bsf = std::sqrt((double)sb);
    out->seconds_join = ms / 1000.0;
    out->seconds_total = wall.seconds() + t_upload;
    if (!sbeg) {  // the counters are the whole call's: per series only for a single join
      out->pairs = cnt_h[kPairs];
      out->pruned_fast = cnt_h[kPrunedFast];
      out->pruned_kim = cnt_h[kPrunedKim];
      out->pruned_masked = cnt_h[kPrunedMasked];
      out->pruned_keogh = cnt_h[kPrunedKeogh];
      out->pruned_paa = cnt_h[kPrunedPaa];
      out->pruned_petitjean = cnt_h[kPrunedPetitjean];
      out->dtw_calls = cnt_h[kDtwCalls];
      out->dtw_abandoned = cnt_h[kDtwAbandoned];
      out->dtw_cells = cnt_h[kDtwCells];
      out->candidates = cand_h;
      ph.collect(out);
    }
  }
  if (verbose)
    fprintf(stderr, "dtwj: %d series, %.3fs device, %u candidates\n", nseries, ms / 1000.0, cand_h);
  return DTWJ_OK;
}

int join_device(dtwj_ctx* ctx, const double* x_dev, int64_t n, int32_t m, int32_t w_in,
                uint32_t flags, dtwj_result* out, double t_upload) {
  return run_join(ctx, x_dev, n, nullptr, 1, m, w_in, flags, out, t_upload);
}

int upload(dtwj_ctx* ctx, const double* x, int64_t n, double** dev) {
  ENSURE(B_A, n * 8, *dev);
  CUDA_OK(cudaMemcpyAsync(*dev, x, n * 8, cudaMemcpyHostToDevice, ctx->stream));
  return DTWJ_OK;
}

}  // namespace

extern "C" {

int dtwj_device_count(void) {
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return c;
}

int dtwj_ctx_create(int device, dtwj_ctx** out) {
  if (!out) return DTWJ_ERR_ARG;
  *out = nullptr;
  if (dtwj_device_count() <= device || device < 0) return DTWJ_ERR_NODEVICE;
  dtwj_ctx* c = new (std::nothrow) dtwj_ctx();
  if (!c) return DTWJ_ERR_OOM;
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete c;
    return DTWJ_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
    delete c;
    return DTWJ_ERR_CUDA;
  }
  c->bufs.resize(B_COUNT_);
  *out = c;
  return DTWJ_OK;
}

void dtwj_ctx_destroy(dtwj_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (auto& b : c->bufs)
    if (b.p) cudaFree(b.p);
  if (c->sweep_exec) cudaGraphExecDestroy(c->sweep_exec);
  for (auto e : c->pool) cudaEventDestroy(e);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int dtwj_ctx_join_device(dtwj_ctx* ctx, const double* x_dev, int64_t n, int32_t m, int32_t w,
                         uint32_t flags, dtwj_result* out) {
  if (!ctx || !out) return DTWJ_ERR_ARG;
  int rc = check_args(x_dev, n, m, w);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  return join_device(ctx, x_dev, n, m, w, flags, out, 0.0);
}

int dtwj_band_shapes(int32_t w, int32_t* C, int32_t* G, int32_t max) {
  if (w < 0 || max < 0 || (max > 0 && (!C || !G))) return DTWJ_ERR_ARG;
  BandShape b[16];
  const int k = band_shapes(w, b, 16);
  for (int q = 0; q < k && q < max && q < 16; ++q) {
    C[q] = b[q].C;
    G[q] = b[q].G;
  }
  return k;
}

int dtwj_ctx_set_band(dtwj_ctx* ctx, int32_t w, int32_t C, int32_t G) {
  if (!ctx || w < 0) return DTWJ_ERR_ARG;
  auto& v = ctx->band_override;
  for (size_t q = 0; q < v.size(); ++q)
    if (v[q].first == w) {
      v.erase(v.begin() + q);
      break;
    }
  if (C == 0 && G == 0) return DTWJ_OK;
  if (!band_shape_ok(w, C, G)) return DTWJ_ERR_BAND;
  v.push_back({w, BandShape{C, G}});
  return DTWJ_OK;
}

int dtwj_ctx_set_tuning(dtwj_ctx* ctx, int32_t dtw_warps, int32_t chunk_tiles) {
  if (!ctx) return DTWJ_ERR_ARG;
  if (dtw_warps != 0 && dtw_warps != 1 && dtw_warps != 2 && dtw_warps != 4 && dtw_warps != 8)
    return DTWJ_ERR_ARG;
  if (chunk_tiles != 0 && (chunk_tiles < 16 || chunk_tiles > 4096)) return DTWJ_ERR_ARG;
  ctx->dtw_warps = dtw_warps;
  ctx->chunk_tiles = chunk_tiles;
  return DTWJ_OK;
}

int dtwj_time_band(int device, int32_t m, int32_t w, int32_t C, int32_t G, int32_t pairs,
                   double* cells_per_s) {
  if (!cells_per_s || m < 8 || m > DTWJ_MAX_M || w < 0 || pairs < 1) return DTWJ_ERR_ARG;
  const int we = effective_band(m, w);
  if (!band_shape_ok(we, C, G)) return DTWJ_ERR_BAND;
  dtwj_ctx* ctx = nullptr;
  int rc = dtwj_ctx_create(device, &ctx);
  if (rc) return rc;
  do {
    // a seeded random walk of 8m samples, pairs of windows drawn from it
    const int64_t n = 8 * (int64_t)m;
    std::vector<double> x((size_t)n);
    uint64_t st = 0x9e3779b97f4a7c15ull;
    double v = 0.0;
    for (int64_t p = 0; p < n; ++p) {
      st = st * 6364136223846793005ull + 1442695040888963407ull;
      v += ((double)(st >> 11) * (1.0 / 9007199254740992.0)) - 0.5;
      x[(size_t)p] = v;
    }
    double* dev = nullptr;
    if ((rc = upload(ctx, x.data(), n, &dev))) break;
    DevSeries S;
    if ((rc = prepare(ctx, dev, n, m, we, false, nullptr, 1, &S))) break;
    std::vector<int2> pr((size_t)pairs);
    const int64_t s = n - m + 1;
    for (int q = 0; q < pairs; ++q) {
      st = st * 6364136223846793005ull + 1442695040888963407ull;
      const int a = (int)((st >> 33) % (uint64_t)(s - m));
      st = st * 6364136223846793005ull + 1442695040888963407ull;
      const int b = a + m + (int)((st >> 33) % (uint64_t)(s - m - a));
      pr[(size_t)q] = make_int2(a, b);
    }
    int2* dp;
    double* out;
    if ((rc = ensure(ctx, B_PAIRS, (size_t)pairs * sizeof(int2), (void**)&dp))) break;
    if ((rc = ensure(ctx, B_OUT, (size_t)pairs * 8, (void**)&out))) break;
    if (cudaMemcpyAsync(dp, pr.data(), (size_t)pairs * sizeof(int2), cudaMemcpyHostToDevice,
                        ctx->stream) != cudaSuccess) {
      rc = DTWJ_ERR_CUDA;
      break;
    }
    const BandShape b = {C, G};
    launch_pair_dtw(S, dp, pairs, false, b, out, ctx->stream);  // warm-up
    cudaEventRecord(ctx->ev0, ctx->stream);
    for (int r = 0; r < 3; ++r) launch_pair_dtw(S, dp, pairs, false, b, out, ctx->stream);
    cudaEventRecord(ctx->ev1, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
      rc = DTWJ_ERR_CUDA;
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    const double cells = 3.0 * pairs * ((double)m * (2 * we + 1) - (double)we * (we + 1));
    *cells_per_s = ms > 0 ? cells / (ms * 1e-3) : 0.0;
  } while (0);
  dtwj_ctx_destroy(ctx);
  return rc;
}

int dtwj_ctx_set_shard(dtwj_ctx* ctx, int32_t rank, int32_t world) {
  if (!ctx || world < 1 || rank < 0 || rank >= world) return DTWJ_ERR_ARG;
  ctx->shard_rank = rank;
  ctx->shard_world = world;
  return DTWJ_OK;
}

int dtwj_ctx_set_exchange(dtwj_ctx* ctx, dtwj_exchange_fn fn, void* user, int32_t phases) {
  if (!ctx || (fn && phases < 1)) return DTWJ_ERR_ARG;
  ctx->exchange = fn;
  ctx->exchange_user = fn ? user : nullptr;
  ctx->exchange_phases = fn ? phases : 0;
  return DTWJ_OK;
}

int dtwj_ctx_set_model(dtwj_ctx* ctx, dtwj_mlp* net) {
  if (!ctx) return DTWJ_ERR_ARG;
  if (net && mlp_device(net) != ctx->device) return DTWJ_ERR_ARG;
  ctx->model = net;
  return DTWJ_OK;
}

int dtwj_ctx_tiles(dtwj_ctx* ctx, const double* x, int64_t n, int32_t m, int32_t w,
                   int64_t* count, int32_t* desc, float* features, double* min_dist) {
  if (!ctx || !count) return DTWJ_ERR_ARG;
  int rc = check_args(x, n, m, w);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  build_lb_tiles(ctx, n, m, nullptr, 1);
  const int64_t nt = (int64_t)ctx->lbtiles_host.size();
  *count = nt;
  if (desc) {
    const int64_t s = n - m + 1;
    for (int64_t t = 0; t < nt; ++t) {
      const Tile& T = ctx->lbtiles_host[t];
      const int64_t lags = s - T.i0 - T.L0 < kLbLags ? s - T.i0 - T.L0 : kLbLags;
      desc[4 * t] = T.L0;
      desc[4 * t + 1] = T.i0;
      desc[4 * t + 2] = T.rows;
      desc[4 * t + 3] = (int32_t)lags;
    }
  }
  if (!features && !min_dist) return DTWJ_OK;
  double* dev = nullptr;
  rc = upload(ctx, x, n, &dev);
  if (rc) return rc;
  TileQuery tq;
  tq.features = features;
  tq.min_dist = min_dist;
  if (min_dist && features) {
    // features first (a plain pass), then the minima sweep
    TileQuery f1 = {features, nullptr};
    rc = run_join(ctx, dev, n, nullptr, 1, m, w, 0, nullptr, 0.0, &f1);
    if (rc) return rc;
    tq.features = nullptr;
  }
  return run_join(ctx, dev, n, nullptr, 1, m, w, DTWJ_F_NO_GRAPH, nullptr, 0.0, &tq);
}

int dtwj_ctx_join(dtwj_ctx* ctx, const double* x, int64_t n, int32_t m, int32_t w,
                  uint32_t flags, dtwj_result* out) {
  if (!ctx || !out) return DTWJ_ERR_ARG;
  int rc = check_args(x, n, m, w);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  Timer t;
  double* dev = nullptr;
  rc = upload(ctx, x, n, &dev);
  if (rc) return rc;
  rc = join_device(ctx, dev, n, m, w, flags, out, 0.0);
  if (rc == DTWJ_OK) out->seconds_total = t.seconds();
  return rc;
}

int dtwj_join(const double* x, int64_t n, int32_t m, int32_t w, uint32_t flags,
              dtwj_result* out) {
  if (!out) return DTWJ_ERR_ARG;
  int rc = check_args(x, n, m, w);
  if (rc) return rc;
  dtwj_ctx* ctx = nullptr;
  rc = dtwj_ctx_create(0, &ctx);
  if (rc) return rc;
  rc = dtwj_ctx_join(ctx, x, n, m, w, flags, out);
  dtwj_ctx_destroy(ctx);
  return rc;
}

int dtwj_join_batch(const double* const* xs, const int64_t* ns, const int32_t* ms,
                    const int32_t* ws, int32_t count, uint32_t flags, dtwj_result* outs) {
  if (!xs || !ns || !ms || !ws || !outs || count < 0) return DTWJ_ERR_ARG;
  int rc = DTWJ_OK;
  for (int32_t k = 0; k < count && rc == DTWJ_OK; ++k) rc = check_args(xs[k], ns[k], ms[k], ws[k]);
  if (rc || count == 0) return rc;
  // series of one (m, effective band) are joined together, back to back
  std::vector<int32_t> order(count);
  for (int32_t k = 0; k < count; ++k) order[k] = k;
  auto key = [&](int32_t k) {
    return ((int64_t)ms[k] << 32) | (uint32_t)effective_band(ms[k], ws[k]);
  };
  std::stable_sort(order.begin(), order.end(),
                   [&](int32_t a, int32_t b) { return key(a) < key(b); });
  std::vector<std::pair<int32_t, int32_t>> groups;  // [g0, g1) of order
  for (int32_t g0 = 0; g0 < count;) {
    int32_t g1 = g0;
    while (g1 < count && key(order[g1]) == key(order[g0])) ++g1;
    groups.push_back({g0, g1});
    g0 = g1;
  }
  // One group's pass on a context: its series stored back to back, joined
  // together, each result written to its own slot of outs.
  auto run_group = [&](dtwj_ctx* ctx, int32_t g0, int32_t g1, std::vector<double>& cat,
                       std::vector<int64_t>& sbeg, std::vector<dtwj_result>& res) -> int {
    const int nser = g1 - g0;
    sbeg.assign(1, 0);
    for (int32_t q = g0; q < g1; ++q) sbeg.push_back(sbeg.back() + ns[order[q]]);
    const int64_t total = sbeg.back();
    if (total > (int64_t)INT32_MAX - 4) return DTWJ_ERR_ARG;
    cat.resize((size_t)total);
    for (int32_t q = g0; q < g1; ++q)
      memcpy(cat.data() + sbeg[q - g0], xs[order[q]], (size_t)ns[order[q]] * 8);
    double* dev = nullptr;
    Timer t;
    int grc = upload(ctx, cat.data(), total, &dev);
    if (grc) return grc;
    res.resize((size_t)nser);
    grc = run_join(ctx, dev, total, sbeg.data(), nser, ms[order[g0]], ws[order[g0]], flags,
                   res.data(), 0.0);
    for (int q = 0; q < nser && grc == DTWJ_OK; ++q) {
      res[q].w = ws[order[g0 + q]];
      res[q].seconds_total = t.seconds();
      outs[order[g0 + q]] = res[q];
    }
    return grc;
  };
  // Groups run concurrently, up to kBatchWorkers at a time: each worker
  // thread owns a context (its own stream and buffers) and takes the next
  // group until none is left, so one group's host checks and small launches
  // overlap another's kernels.
  const int workers = (int)groups.size() < kBatchWorkers ? (int)groups.size() : kBatchWorkers;
  std::atomic<int> next_group{0};
  std::atomic<int> first_error{DTWJ_OK};
  auto worker = [&]() {
    dtwj_ctx* ctx = nullptr;
    int wrc = dtwj_ctx_create(0, &ctx);
    std::vector<double> cat;
    std::vector<int64_t> sbeg;
    std::vector<dtwj_result> res;
    while (wrc == DTWJ_OK && first_error.load() == DTWJ_OK) {
      const int gi = next_group.fetch_add(1);
      if (gi >= (int)groups.size()) break;
      wrc = run_group(ctx, groups[gi].first, groups[gi].second, cat, sbeg, res);
    }
    if (wrc != DTWJ_OK) {
      int expected = DTWJ_OK;
      first_error.compare_exchange_strong(expected, wrc);
    }
    dtwj_ctx_destroy(ctx);
  };
  std::vector<std::thread> pool;
  if (workers > 1) {
    try {
      for (int k = 0; k < workers; ++k) pool.emplace_back(worker);
    } catch (...) {
      // no more threads: the workers already started take every group
    }
  }
  if (pool.empty()) worker();
  for (auto& th : pool) th.join();
  return first_error.load();
}

int dtwj_matrix_profile(const double* x, int64_t n, int32_t m, double* mp, int64_t* mpi) {
  if (!mp || !mpi) return DTWJ_ERR_ARG;
  int rc = check_args(x, n, m, 0);
  if (rc) return rc;
  // Row minima over partners j >= i + m come from the series, those over
  // j <= i - m from the reversed series: reversing both windows keeps their
  // z-normalised distance, and window i becomes window s-1-i.
  dtwj_ctx* ctx = nullptr;
  dtwj_ctx* rev = nullptr;
  rc = dtwj_ctx_create(0, &ctx);
  if (rc) return rc;
  rc = dtwj_ctx_create(0, &rev);
  if (rc) {
    dtwj_ctx_destroy(ctx);
    return rc;
  }
  do {
    double* dev = nullptr;
    if ((rc = upload(ctx, x, n, &dev))) break;
    void* p;
    if ((rc = ensure(rev, B_A, n * 8, &p))) break;
    double* rdev = (double*)p;
    launch_reverse(dev, n, rdev, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
      rc = DTWJ_ERR_CUDA;
      break;
    }
    DevSeries S, R;
    if ((rc = prepare(ctx, dev, n, m, 0, false, nullptr, 1, &S))) break;
    if ((rc = prepare(rev, rdev, n, m, 0, false, nullptr, 1, &R))) break;
    build_lb_tiles(ctx, n, m, nullptr, 1);
    const int nlb = (int)ctx->lbtiles_host.size();
    if ((rc = ensure(ctx, B_LBTILES, (size_t)nlb * sizeof(Tile), &p))) break;
    Tile* tiles = (Tile*)p;
    cudaMemcpy(tiles, ctx->lbtiles_host.data(), (size_t)nlb * sizeof(Tile), cudaMemcpyHostToDevice);
    const int64_t s = n - m + 1;
    if ((rc = ensure(ctx, B_KEYS_UP, s * 8, &p))) break;
    unsigned long long* up = (unsigned long long*)p;
    if ((rc = ensure(rev, B_KEYS_UP, s * 8, &p))) break;
    unsigned long long* lo = (unsigned long long*)p;
    launch_mp(S, tiles, nlb, up, ctx->stream);
    launch_mp(R, tiles, nlb, lo, rev->stream);
    if (cudaStreamSynchronize(rev->stream) != cudaSuccess) {
      rc = DTWJ_ERR_CUDA;
      break;
    }
    if ((rc = ensure(ctx, B_MP, s * 8, &p))) break;
    double* dmp = (double*)p;
    if ((rc = ensure(ctx, B_MPI, s * 8, &p))) break;
    int64_t* dmpi = (int64_t*)p;
    // Exact pass.  The first pass keeps about 17 mantissa bits of ED^2 per
    // row; every pair whose key lies within ten 20-bit units of its row's
    // smallest key (either direction) is a candidate, its FP64 distance is
    // computed directly, and the row takes the smallest, lowest partner on
    // ties.
    unsigned long long *want, *wrev, *rowmin, *rowidx;
    if ((rc = ensure(ctx, B_MPX_WANT, s * 8, &p))) break;
    want = (unsigned long long*)p;
    if ((rc = ensure(ctx, B_MPX_WREV, s * 8, &p))) break;
    wrev = (unsigned long long*)p;
    if ((rc = ensure(ctx, B_MPX_MIN, s * 8, &p))) break;
    rowmin = (unsigned long long*)p;
    if ((rc = ensure(ctx, B_MPX_IDX, s * 8, &p))) break;
    rowidx = (unsigned long long*)p;
    const unsigned int cap =
        (unsigned int)(s * 16 + 4096 < (1ll << 31) ? s * 16 + 4096 : (1ll << 31));
    if ((rc = ensure(ctx, B_MPX_CAND, (size_t)cap * sizeof(int2), &p))) break;
    int2* cand_up = (int2*)p;
    if ((rc = ensure(rev, B_MPX_CAND, (size_t)cap * sizeof(int2), &p))) break;
    int2* cand_lo = (int2*)p;
    if ((rc = ensure(ctx, B_MPX_CNT, 8, &p))) break;
    unsigned int* cnt = (unsigned int*)p;
    cudaStream_t st = ctx->stream;
    launch_mp_want(s, up, lo, want, wrev, st);
    cudaMemsetAsync(cnt, 0, 8, st);
    cudaMemsetAsync(rowmin, 0xff, s * 8, st);
    cudaMemsetAsync(rowidx, 0xff, s * 8, st);
    launch_mp_collect(S, tiles, nlb, want, cand_up, cnt, cap, st);
    launch_mp_collect(R, tiles, nlb, wrev, cand_lo, cnt + 1, cap, st);
    for (int pick = 0; pick < 2; ++pick) {
      launch_mp_exact(S, cand_up, cnt, cap, false, pick != 0, rowmin, rowidx, st);
      launch_mp_exact(S, cand_lo, cnt + 1, cap, true, pick != 0, rowmin, rowidx, st);
    }
    launch_mp_exact_out(s, rowmin, rowidx, dmp, dmpi, st);
    unsigned int cnt_h[2] = {0, 0};
    if (cudaMemcpyAsync(cnt_h, cnt, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      rc = DTWJ_ERR_CUDA;
      break;
    }
    if (cnt_h[0] > cap || cnt_h[1] > cap) {
      rc = DTWJ_ERR_OVERFLOW;
      break;
    }
    if (cudaMemcpyAsync(mp, dmp, s * 8, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
        cudaMemcpyAsync(mpi, dmpi, s * 8, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
      rc = DTWJ_ERR_CUDA;
      break;
    }
  } while (0);
  dtwj_ctx_destroy(rev);
  dtwj_ctx_destroy(ctx);
  return rc;
}

int dtwj_global_mask(const double* x, int64_t n, int32_t m, int32_t w, float* mask,
                     int32_t* table_len) {
  if (!mask) return DTWJ_ERR_ARG;
  int rc = check_args(x, n, m, w);
  if (rc) return rc;
  const int we = effective_band(m, w);
  dtwj_ctx* ctx = nullptr;
  rc = dtwj_ctx_create(0, &ctx);
  if (rc) return rc;
  do {
    double* dev = nullptr;
    if ((rc = upload(ctx, x, n, &dev))) break;
    DevSeries S;
    if ((rc = prepare(ctx, dev, n, m, we, true, nullptr, 1, &S))) break;
    if (cudaMemcpyAsync(mask, S.mask, (size_t)n * 4, cudaMemcpyDeviceToHost, ctx->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
      rc = DTWJ_ERR_CUDA;
      break;
    }
    if (table_len) {
      // the table length the mask used: 200 floor(max |z|), at least 600
      float zmax = 0.0f;
      void* p = nullptr;
      if ((rc = ensure(ctx, B_ZMAX, 4, &p))) break;
      if (cudaMemcpy(&zmax, p, 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
        rc = DTWJ_ERR_CUDA;
        break;
      }
      const int lt = (int)(std::floor((double)zmax) * 200.0);
      *table_len = lt > 600 ? lt : 600;
    }
  } while (0);
  dtwj_ctx_destroy(ctx);
  return rc;
}

int dtwj_pair_dtw(const double* x, int64_t n, int32_t m, int32_t w, const int64_t* pi,
                  const int64_t* pj, int64_t count, int32_t precise, double* dist) {
  if (!pi || !pj || !dist || count < 0) return DTWJ_ERR_ARG;
  int rc = check_args(x, n, m, w);
  if (rc) return rc;
  const int64_t s = n - m + 1;
  std::vector<int2> pairs((size_t)count);
  for (int64_t k = 0; k < count; ++k) {
    if (pi[k] < 0 || pj[k] < 0 || pi[k] >= s || pj[k] >= s) return DTWJ_ERR_ARG;
    pairs[k] = make_int2((int)pi[k], (int)pj[k]);
  }
  if (count == 0) return DTWJ_OK;
  const int we = effective_band(m, w);
  BandShape band;
  if (!choose_band_list(we, &band)) return DTWJ_ERR_BAND;
  dtwj_ctx* ctx = nullptr;
  rc = dtwj_ctx_create(0, &ctx);
  if (rc) return rc;
  do {
    double* dev = nullptr;
    if ((rc = upload(ctx, x, n, &dev))) break;
    DevSeries S;
    if ((rc = prepare(ctx, dev, n, m, we, false, nullptr, 1, &S))) break;
    void* p;
    if ((rc = ensure(ctx, B_PAIRS, (size_t)count * sizeof(int2), &p))) break;
    int2* dp = (int2*)p;
    if ((rc = ensure(ctx, B_OUT, (size_t)count * 8, &p))) break;
    double* dout = (double*)p;
    cudaMemcpyAsync(dp, pairs.data(), (size_t)count * sizeof(int2), cudaMemcpyHostToDevice,
                    ctx->stream);
    launch_pair_dtw(S, dp, (int)count, precise != 0, band, dout, ctx->stream);
    if (cudaMemcpyAsync(dist, dout, (size_t)count * 8, cudaMemcpyDeviceToHost, ctx->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
      rc = DTWJ_ERR_CUDA;
      break;
    }
    for (int64_t k = 0; k < count; ++k) dist[k] = std::sqrt(dist[k]);
  } while (0);
  dtwj_ctx_destroy(ctx);
  return rc;
}

int dtwj_pair_lb_petitjean(const double* x, int64_t n, int32_t m, int32_t w, const int64_t* pa,
                           const int64_t* pb, int64_t count, int32_t own_env, double* keogh_mid,
                           double* terms) {
  if (!pa || !pb || !keogh_mid || !terms || count < 0 || count > INT32_MAX) return DTWJ_ERR_ARG;
  int rc = check_args(x, n, m, w);
  if (rc) return rc;
  const int we = effective_band(m, w);
  if (lbp_list_bytes(m, we, own_env != 0) > kPjMaxSmemBytes) return DTWJ_ERR_ARG;
  const int64_t s = n - m + 1;
  std::vector<int2> pairs((size_t)count);
  for (int64_t k = 0; k < count; ++k) {
    if (pa[k] < 0 || pb[k] < 0 || pa[k] >= s || pb[k] >= s) return DTWJ_ERR_ARG;
    pairs[k] = make_int2((int)pa[k], (int)pb[k]);
  }
  if (count == 0) return DTWJ_OK;
  dtwj_ctx* ctx = nullptr;
  rc = dtwj_ctx_create(0, &ctx);
  if (rc) return rc;
  do {
    double* dev = nullptr;
    if ((rc = upload(ctx, x, n, &dev))) break;
    DevSeries S;
    if ((rc = prepare(ctx, dev, n, m, we, false, nullptr, 1, &S))) break;
    void* p;
    if ((rc = ensure(ctx, B_PAIRS, (size_t)count * sizeof(int2), &p))) break;
    int2* dp = (int2*)p;
    if ((rc = ensure(ctx, B_OUT, (size_t)count * 16, &p))) break;
    double* dout = (double*)p;
    cudaMemcpyAsync(dp, pairs.data(), (size_t)count * sizeof(int2), cudaMemcpyHostToDevice,
                    ctx->stream);
    launch_lbp_list(S, dp, (int)count, own_env != 0, dout, dout + count, ctx->num_sms,
                    ctx->stream);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(keogh_mid, dout, (size_t)count * 8, cudaMemcpyDeviceToHost,
                        ctx->stream) != cudaSuccess ||
        cudaMemcpyAsync(terms, dout + count, (size_t)count * 8, cudaMemcpyDeviceToHost,
                        ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
      rc = DTWJ_ERR_CUDA;
      break;
    }
  } while (0);
  dtwj_ctx_destroy(ctx);
  return rc;
}

int32_t dtwj_band(int32_t m, double ratio, int32_t rounding) {
  double v = ratio * (double)m;
  int32_t w;
  if (rounding == 1) w = (int32_t)std::floor(v + 0.5);
  else w = (int32_t)std::ceil(v - 1e-9);
  return w < 1 ? 1 : w;
}

const char* dtwj_strerror(int code) {
  switch (code) {
    case DTWJ_OK: return "ok";
    case DTWJ_ERR_ARG: return "invalid argument";
    case DTWJ_ERR_NAN: return "input contains NaN or infinity";
    case DTWJ_ERR_CUDA: return "CUDA error";
    case DTWJ_ERR_OOM: return "device out of memory";
    case DTWJ_ERR_BAND: return "band too wide (w must be <= 255)";
    case DTWJ_ERR_OVERFLOW: return "candidate or survivor list overflow";
    case DTWJ_ERR_TIMEOUT: return "device-side wait ran out";
    case DTWJ_ERR_NODEVICE: return "no CUDA device";
    case DTWJ_ERR_IO: return "file could not be read or written";
    case DTWJ_ERR_NOMODEL: return "learned ordering requested but no model is loaded";
    case DTWJ_ERR_SCRATCH: return "series exceeds the fixed scratch of the allocation-free entry point";
    default: return "unknown error";
  }
}

}  // extern "C"
