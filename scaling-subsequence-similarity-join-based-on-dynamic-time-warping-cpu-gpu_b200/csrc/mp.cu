// z-normalised Euclidean matrix profile (the reference's mpx_v2) and the
// ED-seeded best-so-far.
//
// mpx_v2 (CPU_version1/mpx_v2.cpp:79-113, GPU_version1/src/mpx_v2.cu:80-115)
// walks every diagonal with the covariance recurrence
//   cov -= dr_bwd * dc_bwd;  cov += dr_fwd * dc_fwd
// on one host thread.  Here one thread owns one lag L and walks a block of
// rows with the equivalent centered FP64 update
//   C(i, j) = C(i-1, j-1) + df[i-1] dg[j-1] + df[j-1] dg[i-1],
// re-anchored exactly at the first row of every tile, and the row minimum of
// ED^2 = 2m - 2 C / (sig_i sig_j) is reduced across the warp in one REDUX.
// A key packs the high 32 bits of ED^2 (sign, exponent, 20 mantissa bits:
// monotone for non-negative doubles; the lowest 3 bits give way to the lag
// inside a thread's minimum) above the partner index, so a 64-bit atomicMin
// keeps the nearest neighbour at that resolution.  That is all the seeds
// need; the matrix profile (dtwj_matrix_profile) then decides every row at
// FP64 among the partners whose key is near the row's (launch_mp_collect).
//
// The seeds are the kSeeds smallest row minima, as in
// CPU_version1/new_dtw_motifGUI.cpp:53-74 (min_v_k + exact DTW per seed).
#include "dtwj_dev.cuh"

#include <cfloat>
#include <climits>

namespace dtwj {
namespace {

// Row minima of ED^2 over the upper triangle (partners j >= i + m).  Tile and
// staging as in the diagonal sweep (lb.cu): 128 threads x kLbPerThread lags
// x kLbRows rows, column operands (df[j-1], dg[j-1], 1/sig_j and the flat
// guard 2m | 1e300) staged per kStage rows in shared memory and slid through
// registers.  Per row a thread keeps its best of kLbPerThread lags, the warp
// reduces the high words with one REDUX, and the winner lane folds its key
// into the tile's row minima with a shared 64-bit atomicMin.
constexpr int kStage = kLbPerThread * 32;
constexpr int kCols = kLbLags + kStage;

// High words of ED^2 keys at or above this (ED^2 >= 2^513) come from the
// 1e300 offset of a column past the series or of a flat window, not a pair.
constexpr unsigned int kKeyReal = 0x60000000u;
static_assert(kLbPerThread <= 8, "the lag fits the key's 3 low bits");

struct MpShared {
  double p1[kCols], p2[kCols], is[kCols], c2[kCols];
  double r1[kStage], r2[kStage], ci[kStage];
  unsigned int lim[kStage];
  unsigned long long rowbest[kStage];  // row minima of the current stage
};

// Candidate list of the exact profile (COLLECT): every pair whose high word
// is within ten units of its row's smallest key.
struct MpCollect {
  const unsigned long long* want;  // per row: the smallest key of the first pass
  int2* cand;
  unsigned int* count;
  unsigned int cap;
};

template <bool COLLECT>
__global__ void __launch_bounds__(kLbThreads, 4) k_mp(DevSeries S, const Tile* tiles,
                                                      unsigned long long* keys,
                                                      unsigned int* tile_best, int tile_base,
                                                      MpCollect col) {
  extern __shared__ __align__(16) unsigned char smraw[];
  MpShared& sh = *reinterpret_cast<MpShared*>(smraw);
  const Tile T = tiles[blockIdx.x];
  const int64_t s = T.send;  // windows of the tile's series end here
  const int m = S.m;
  const int t = threadIdx.x, lane = t & 31;
  const int64_t L0 = T.L0, i0 = T.i0;
  const int64_t Lt = L0 + (int64_t)t * kLbPerThread;

  // exact anchors C(i0, i0 + L) for the thread's lags
  double C[kLbPerThread];
  {
    double mj[kLbPerThread], wa[kLbPerThread];
    const int64_t jb = i0 + Lt;
#pragma unroll
    for (int l = 0; l < kLbPerThread; ++l) {
      C[l] = 0.0;
      mj[l] = S.mu[jb + l < s ? jb + l : s - 1];
      wa[l] = S.a[jb + l < S.n ? jb + l : S.n - 1];
    }
    const double mi = S.mu[i0];
    for (int k = 0; k < m; ++k) {
      const double ai = S.a[i0 + k] - mi;
#pragma unroll
      for (int l = 0; l < kLbPerThread; ++l) C[l] = fma(ai, wa[l] - mj[l], C[l]);
#pragma unroll
      for (int l = 0; l < kLbPerThread - 1; ++l) wa[l] = wa[l + 1];
      const int64_t x = jb + kLbPerThread + k < S.n ? jb + kLbPerThread + k : S.n - 1;
      wa[kLbPerThread - 1] = S.a[x];
    }
  }
  double w1[kLbPerThread], w2[kLbPerThread], wi[kLbPerThread], wc[kLbPerThread];
  const double two_m = 2.0 * m;
  unsigned int tmin = 0xffffffffu;  // the tile's smallest key (high bits of ED^2)
  for (int st = 0; st < T.rows; st += kStage) {
    const int64_t r0 = i0 + st, c0 = r0 + L0;
    __syncthreads();
    if (!COLLECT)
      for (int x = t; x < kStage; x += kLbThreads) sh.rowbest[x] = ULLONG_MAX;
    for (int x = t; x < kCols; x += kLbThreads) {
      const int64_t j = c0 + x;
      const bool in = j >= 0 && j < s, up = j >= 1 && j < s;  // update terms exist for j >= 1
      sh.p1[x] = up ? S.dfa[j - 1] : 0.0;
      sh.p2[x] = up ? S.dga[j - 1] : 0.0;
      sh.is[x] = in ? S.isg[j] : 0.0;
      sh.c2[x] = (in && !S.flat[j]) ? two_m : 1e300;
    }
    for (int x = t; x < kStage; x += kLbThreads) {
      const int64_t i = r0 + x;
      const bool in = i >= 0 && i < s, up = i >= 1 && i < s;
      sh.r1[x] = up ? S.dfa[i - 1] : 0.0;
      sh.r2[x] = up ? S.dga[i - 1] : 0.0;
      sh.ci[x] = (in && !S.flat[i]) ? -2.0 * S.isg[i] : 0.0;
      if (COLLECT) {
        // the first pass's key is the row's smallest high word with its 3
        // low bits cleared: its partners lie within 8 units, plus 2 of margin
        const unsigned long long k = in ? col.want[i] : ULLONG_MAX;
        sh.lim[x] = k == ULLONG_MAX ? 0u : (unsigned int)(k >> 32) + 10u;
      }
    }
    __syncthreads();
    const int cb = t * kLbPerThread;
#pragma unroll
    for (int l = 0; l < kLbPerThread; ++l) {
      w1[l] = sh.p1[cb + l];
      w2[l] = sh.p2[cb + l];
      wi[l] = sh.is[cb + l];
      wc[l] = sh.c2[cb + l];
    }
    for (int qq = 0; qq < kStage / kLbPerThread; ++qq) {
#pragma unroll
      for (int u = 0; u < kLbPerThread; ++u) {
        const int r = qq * kLbPerThread + u;
        const int64_t i = r0 + r;
        const bool first = (st == 0 && r == 0);
        const double q1 = sh.r1[r], q2 = sh.r2[r], qc = sh.ci[r];
        const unsigned int lim = COLLECT ? sh.lim[r] : 0u;
        // rows of the tile with a non-flat window (warp-uniform); a column past
        // the series or flat has weight 0 and offset 1e300, so its key is far
        // above any real one and it never needs a test of its own
        const bool row_ok = (st + r < T.rows) && qc != 0.0;
        unsigned int best = UINT_MAX;
#pragma unroll
        for (int l = 0; l < kLbPerThread; ++l) {
          const int sl = (u + l) % kLbPerThread;
          if (!first) {
            C[l] = fma(q1, w2[sl], C[l]);
            C[l] = fma(w1[sl], q2, C[l]);
          }
          const double e2 = fmax(fma(C[l] * qc, wi[sl], wc[sl]), 0.0);
          const unsigned int hi = (unsigned int)__double2hiint(e2);
          if (COLLECT) {
            if (row_ok && hi <= lim) {
              const unsigned int slot = atomicAdd(col.count, 1u);
              if (slot < col.cap) col.cand[slot] = make_int2((int)i, (int)(i + Lt + l));
            }
          } else {
            // the high word with its lowest 3 bits replaced by the lag: one
            // minimum keeps the nearest lag (17 mantissa bits of ED^2)
            best = min(best, (hi & ~7u) | (unsigned int)l);
          }
        }
        const int nx = cb + r + kLbPerThread;
        w1[u] = sh.p1[nx];
        w2[u] = sh.p2[nx];
        wi[u] = sh.is[nx];
        wc[u] = sh.c2[nx];
        if (!COLLECT && row_ok) {  // flat rows have no neighbour
          const unsigned int wbest = __reduce_min_sync(0xffffffffu, best);
          if (wbest < kKeyReal) {
            const unsigned int ballot = __ballot_sync(0xffffffffu, best == wbest);
            if (lane == __ffs(ballot) - 1) {
              const unsigned long long key =
                  ((unsigned long long)(wbest & ~7u) << 32) |
                  (unsigned long long)(unsigned int)(i + Lt + (wbest & 7u));
              atomicMin(&sh.rowbest[r], key);
            }
          }
        }
      }
    }
    if (!COLLECT) {
      // the stage's row minima into the series' keys (each row once per tile)
      __syncthreads();
      const int nrow = T.rows - st < kStage ? T.rows - st : kStage;
      for (int x = t; x < nrow; x += kLbThreads) {
        const unsigned long long v = sh.rowbest[x];
        if (v != ULLONG_MAX) {
          atomicMin(&keys[r0 + x], v);
          tmin = min(tmin, (unsigned int)(v >> 32));
        }
      }
    }
  }
  if (COLLECT) return;
  if (tile_best) {
    for (int o = 16; o > 0; o >>= 1) tmin = min(tmin, __shfl_xor_sync(0xffffffffu, tmin, o));
    if (lane == 0 && tmin != 0xffffffffu) atomicMin(&tile_best[tile_base + blockIdx.x], tmin);
  }
}

// Row minima for the join's seeds only.  The seeds choose which pairs get an
// exact DTW first; nothing else depends on these keys (the join's starting
// best-so-far comes from those exact DTWs, and the result never depends on
// it), so this pass samples and approximates:
//  - only the rows on a grid of kSeedGrid rows (i - i0 a multiple of
//    kSeedGrid; every tile starts on the grid of its series) get a key.  The
//    covariance recurrence still steps every row, but the ED^2, the minimum
//    and the row reduction run on one row in kSeedGrid.  A seed (i, j) is
//    later widened to its diagonal neighbours (i + d, j + d), |d| <=
//    kSeedGrid / 2, which covers every row of the grid cell;
//  - the pass keeps the tile's exact FP64 anchor and carries the covariance
//    in FP64 from stage to stage, but accumulates the per-row increments of a
//    stage (224 rows) in FP32 on FP32 copies of the update terms.  On random
//    walks that leaves ED^2 within about 1e-4 of the FP64 recurrence; the keys
//    keep 20 mantissa bits.
static_assert(kSeedGrid == kLbPerThread, "grid rows are the first of each unrolled group");
static_assert(kLbRows % kSeedGrid == 0 && kStage % kSeedGrid == 0, "tiles and stages on the grid");

struct MpSeedShared {
  float2 p[kCols];   // (dfa, dga) of column j - 1: one 8-byte read per row and thread
  float is[kCols], c2[kCols];
  float4 r[kStage];  // (dfa, dga of row i - 1, -2 isg of row i, 0): one broadcast read per row
  unsigned long long rowbest[kStage / kSeedGrid];
};

__global__ void __launch_bounds__(kLbThreads, 6) k_mp_seed(DevSeries S, const Tile* tiles,
                                                           unsigned long long* keys) {
  extern __shared__ __align__(16) unsigned char smraw[];
  MpSeedShared& sh = *reinterpret_cast<MpSeedShared*>(smraw);
  const Tile T = tiles[blockIdx.x];
  const int64_t s = T.send;
  const int m = S.m;
  const int t = threadIdx.x, lane = t & 31;
  const int64_t L0 = T.L0, i0 = T.i0;
  const int64_t Lt = L0 + (int64_t)t * kLbPerThread;
  // exact anchors C(i0, i0 + L) for the thread's lags (FP64)
  double C[kLbPerThread];
  {
    double mj[kLbPerThread], wa[kLbPerThread];
    const int64_t jb = i0 + Lt;
#pragma unroll
    for (int l = 0; l < kLbPerThread; ++l) {
      C[l] = 0.0;
      mj[l] = S.mu[jb + l < s ? jb + l : s - 1];
      wa[l] = S.a[jb + l < S.n ? jb + l : S.n - 1];
    }
    const double mi = S.mu[i0];
    for (int k = 0; k < m; ++k) {
      const double ai = S.a[i0 + k] - mi;
#pragma unroll
      for (int l = 0; l < kLbPerThread; ++l) C[l] = fma(ai, wa[l] - mj[l], C[l]);
#pragma unroll
      for (int l = 0; l < kLbPerThread - 1; ++l) wa[l] = wa[l + 1];
      const int64_t x = jb + kLbPerThread + k < S.n ? jb + kLbPerThread + k : S.n - 1;
      wa[kLbPerThread - 1] = S.a[x];
    }
  }
  float w1[kLbPerThread], w2[kLbPerThread];
  const float two_m = 2.0f * (float)m;
  const unsigned int kReal = __float_as_uint(1e20f);  // above: a guard column, not a pair
  for (int st = 0; st < T.rows; st += kStage) {
    const int64_t r0 = i0 + st, c0 = r0 + L0;
    __syncthreads();
    for (int x = t; x < kStage / kSeedGrid; x += kLbThreads) sh.rowbest[x] = ULLONG_MAX;
    for (int x = t; x < kCols; x += kLbThreads) {
      const int64_t j = c0 + x;
      const bool in = j >= 0 && j < s, up = j >= 1 && j < s;
      sh.p[x] = make_float2(up ? (float)S.dfa[j - 1] : 0.0f, up ? (float)S.dga[j - 1] : 0.0f);
      sh.is[x] = in ? (float)S.isg[j] : 0.0f;
      sh.c2[x] = (in && !S.flat[j]) ? two_m : 1e30f;
    }
    for (int x = t; x < kStage; x += kLbThreads) {
      const int64_t i = r0 + x;
      const bool in = i >= 0 && i < s, up = i >= 1 && i < s;
      sh.r[x] = make_float4(up ? (float)S.dfa[i - 1] : 0.0f, up ? (float)S.dga[i - 1] : 0.0f,
                            (in && !S.flat[i]) ? (float)(-2.0 * S.isg[i]) : 0.0f, 0.0f);
    }
    __syncthreads();
    const int cb = t * kLbPerThread;
    float Cb[kLbPerThread], D[kLbPerThread];
#pragma unroll
    for (int l = 0; l < kLbPerThread; ++l) {
      const float2 pc = sh.p[cb + l];
      w1[l] = pc.x;
      w2[l] = pc.y;
      Cb[l] = (float)C[l];
      D[l] = 0.0f;
    }
    for (int qq = 0; qq < kStage / kLbPerThread; ++qq) {
#pragma unroll
      for (int u = 0; u < kLbPerThread; ++u) {
        const int r = qq * kLbPerThread + u;
        const bool first = (st == 0 && r == 0);
        const float4 rq = sh.r[r];
        const float q1 = rq.x, q2 = rq.y;
        if (!first) {
#pragma unroll
          for (int l = 0; l < kLbPerThread; ++l) {
            const int sl = (u + l) % kLbPerThread;  // ring slot of lag l at this row
            D[l] = fmaf(q1, w2[sl], D[l]);
            D[l] = fmaf(w1[sl], q2, D[l]);
          }
        }
        // a grid row (u == 0: lag l's column sits in ring slot l and at
        // stage column cb + r + l)
        const float qc = rq.z;
        if (u == 0 && st + r < T.rows && qc != 0.0f) {
          unsigned int best = UINT_MAX;
#pragma unroll
          for (int l = 0; l < kLbPerThread; ++l) {
            const float e2 =
                fmaxf(fmaf((Cb[l] + D[l]) * qc, sh.is[cb + r + l], sh.c2[cb + r + l]), 0.0f);
            best = min(best, (__float_as_uint(e2) & ~7u) | (unsigned int)l);
          }
          const unsigned int wbest = __reduce_min_sync(0xffffffffu, best);
          if (wbest < kReal) {
            const unsigned int ballot = __ballot_sync(0xffffffffu, best == wbest);
            if (lane == __ffs(ballot) - 1) {
              // the float (20 mantissa bits kept) in the FP64 key format
              const unsigned int hi =
                  (unsigned int)__double2hiint((double)__uint_as_float(wbest & ~7u));
              const unsigned long long key =
                  ((unsigned long long)(hi & ~7u) << 32) |
                  (unsigned long long)(unsigned int)(r0 + r + Lt + (wbest & 7u));
              atomicMin(&sh.rowbest[r / kSeedGrid], key);
            }
          }
        }
        const int nx = cb + r + kLbPerThread;
        const float2 pn = sh.p[nx];
        w1[u] = pn.x;
        w2[u] = pn.y;
      }
    }
#pragma unroll
    for (int l = 0; l < kLbPerThread; ++l) C[l] += (double)D[l];
    __syncthreads();
    const int nrow = T.rows - st < kStage ? T.rows - st : kStage;
    for (int x = t; x * kSeedGrid < nrow; x += kLbThreads) {
      const unsigned long long v = sh.rowbest[x];
      if (v != ULLONG_MAX) atomicMin(&keys[r0 + (int64_t)x * kSeedGrid], v);
    }
  }
}

// Per tile, an upper bound on its smallest squared DTW distance: the ED^2 of
// its closest pair (ED >= DTW), from the truncated key rounded up.
__global__ void k_tile_bound(const unsigned int* tile_best, int ntiles, unsigned int* bsf2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  const unsigned int hi = tile_best[t];
  if (hi == 0xffffffffu) {
    bsf2[t] = 0x7f800000u;
    return;
  }
  // the key's high word has its 3 low bits cleared: the pair's ED^2 is below
  // the next multiple of 8 units
  const unsigned long long bits = ((unsigned long long)(hi & ~7u) + 8ull) << 32;
  bsf2[t] = __float_as_uint(__double2float_ru(__longlong_as_double((long long)bits)));
}

__global__ void k_fill_u64(unsigned long long* p, int64_t n, unsigned long long v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

// Exact FP64 distance of each row's nearest neighbour.
__global__ void k_mp_finalize(DevSeries S, const unsigned long long* up,
                              const unsigned long long* lo, double* mp, int64_t* mpi) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= S.s) return;
  unsigned long long k = up[i];
  if (lo) {
    // lo holds the row minima of the reversed series: row s-1-i, partner s-1-j
    unsigned long long k2 = lo[S.s - 1 - i];
    if (k2 != ULLONG_MAX)
      k2 = (k2 & 0xffffffff00000000ull) |
           (unsigned long long)(unsigned int)(S.s - 1 - (int64_t)(k2 & 0xffffffffu));
    // tie on the distance key: lowest partner index
    if ((k2 >> 32) < (k >> 32) || ((k2 >> 32) == (k >> 32) && (k2 & 0xffffffffu) < (k & 0xffffffffu)))
      k = k2;
  }
  if (k == ULLONG_MAX) {
    mp[i] = __longlong_as_double(0x7ff0000000000000LL);
    mpi[i] = -1;
    return;
  }
  const int64_t j = (int64_t)(k & 0xffffffffu);
  const double mi = S.mu[i], mj = S.mu[j], si = S.isg[i], sj = S.isg[j];
  double d2 = 0.0;
  for (int q = 0; q < S.m; ++q) {
    const double d = (S.a[i + q] - mi) * si - (S.a[j + q] - mj) * sj;
    d2 = fma(d, d, d2);
  }
  mp[i] = sqrt(d2);
  mpi[i] = j;
}

// Exact squared distance of candidate pairs, one warp per pair (the same
// arithmetic as k_mp_finalize).  A candidate (i, j) of the reversed series is
// the pair (s-1-i, s-1-j) of the series.  pick == false: rowmin[i] = the
// smallest FP64 bits over the row's candidates (non-negative doubles order as
// their bits); pick == true: rowidx[i] = the lowest partner reaching it.
__global__ void k_mp_exact(DevSeries S, const int2* cand, const unsigned int* count,
                           unsigned int cap, bool reversed, bool pick,
                           unsigned long long* rowmin, unsigned long long* rowidx) {
  const int lane = threadIdx.x & 31;
  const unsigned int total = *count < cap ? *count : cap;
  for (unsigned int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < total;
       c += (gridDim.x * blockDim.x) >> 5) {
    const int2 p = cand[c];
    const int64_t i = reversed ? S.s - 1 - p.x : p.x, j = reversed ? S.s - 1 - p.y : p.y;
    const double mi = S.mu[i], mj = S.mu[j], si = S.isg[i], sj = S.isg[j];
    double d2 = 0.0;
    for (int q = lane; q < S.m; q += 32) {
      const double d = (S.a[i + q] - mi) * si - (S.a[j + q] - mj) * sj;
      d2 = fma(d, d, d2);
    }
    for (int o = 16; o > 0; o >>= 1) d2 += __shfl_xor_sync(0xffffffffu, d2, o);
    if (lane == 0) {
      const unsigned long long b = (unsigned long long)__double_as_longlong(d2);
      if (!pick) atomicMin(&rowmin[i], b);
      else if (b == rowmin[i]) atomicMin(&rowidx[i], (unsigned long long)j);
    }
  }
}

// mp[i] = sqrt of the row's exact minimum, mpi[i] its lowest partner.
__global__ void k_mp_exact_out(int64_t s, const unsigned long long* rowmin,
                               const unsigned long long* rowidx, double* mp, int64_t* mpi) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= s) return;
  if (rowidx[i] == ULLONG_MAX) {
    mp[i] = __longlong_as_double(0x7ff0000000000000LL);
    mpi[i] = -1;
    return;
  }
  mp[i] = sqrt(__longlong_as_double((long long)rowmin[i]));
  mpi[i] = (int64_t)rowidx[i];
}

// want[i] = the smaller of row i's keys over j > i (up) and over j < i (lo,
// rows of the reversed series); wrev is the same indexed by reversed rows.
__global__ void k_mp_want(int64_t s, const unsigned long long* up, const unsigned long long* lo,
                          unsigned long long* want, unsigned long long* wrev) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= s) return;
  const unsigned long long a = up[i], b = lo[s - 1 - i];
  const unsigned long long ha = a == ULLONG_MAX ? ULLONG_MAX : (a >> 32);
  const unsigned long long hb = b == ULLONG_MAX ? ULLONG_MAX : (b >> 32);
  const unsigned long long h = ha < hb ? ha : hb;
  const unsigned long long k = h == ULLONG_MAX ? ULLONG_MAX : (h << 32);
  want[i] = k;
  wrev[s - 1 - i] = k;
}

constexpr int kSelThreads = 1024;
constexpr int kLocal = 8;

// kSeeds smallest row minima (by ED^2 key, then row index).  Each thread
// keeps the kLocal best of a strided slice; kSeeds rounds of block minimum
// then pop the global order.  Writes each seed pair with its diagonal
// neighbours (kSeedSpread slots per seed, (-1, -1) where a neighbour leaves
// the series) and the seed count.
__global__ void __launch_bounds__(kSelThreads) k_seed_select(DevSeries S,
                                                              const unsigned long long* keys,
                                                              int2* seeds, unsigned int* nseeds) {
  // block b selects the seeds of series b (windows [wb, we))
  const int b = blockIdx.x;
  const int64_t wb = S.sbeg ? S.sbeg[b] : 0;
  const int64_t we = S.sbeg ? S.sbeg[b + 1] - S.m + 1 : S.s;
  seeds += (size_t)b * kSeedSlots;
  for (int x = threadIdx.x; x < kSeedSlots; x += blockDim.x) seeds[x] = make_int2(-1, -1);
  unsigned long long loc[kLocal];
  int part[kLocal];
#pragma unroll
  for (int q = 0; q < kLocal; ++q) { loc[q] = ULLONG_MAX; part[q] = -1; }
  for (int64_t i = wb + threadIdx.x; i < we; i += blockDim.x) {
    const unsigned long long k = keys[i];
    if (k == ULLONG_MAX) continue;
    const unsigned long long sk = (k & 0xffffffff00000000ull) | (unsigned long long)(unsigned int)i;
    if (sk >= loc[kLocal - 1]) continue;
    const int pj = (int)(k & 0xffffffffu);
    // insertion into the ascending local list
    bool done = false;
#pragma unroll
    for (int q = kLocal - 1; q > 0; --q) {
      if (!done) {
        if (loc[q - 1] > sk) {
          loc[q] = loc[q - 1];
          part[q] = part[q - 1];
        } else {
          loc[q] = sk;
          part[q] = pj;
          done = true;
        }
      }
    }
    if (!done) {
      loc[0] = sk;
      part[0] = pj;
    }
  }
  __shared__ unsigned long long red[kSelThreads / 32];
  __shared__ unsigned long long winner;
  int head = 0;
  unsigned int count = 0;
  for (int round = 0; round < kSeeds; ++round) {
    // head of the local list (select through the unrolled registers)
    unsigned long long v = ULLONG_MAX;
#pragma unroll
    for (int q = 0; q < kLocal; ++q) if (q == head) v = loc[q];
    unsigned long long wv = v;
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long t = __shfl_xor_sync(0xffffffffu, wv, o);
      wv = t < wv ? t : wv;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = wv;
    __syncthreads();
    if (threadIdx.x < 32) {
      unsigned long long t = red[threadIdx.x];
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long u = __shfl_xor_sync(0xffffffffu, t, o);
        t = u < t ? u : t;
      }
      if (threadIdx.x == 0) winner = t;
    }
    __syncthreads();
    const unsigned long long wn = winner;
    if (wn == ULLONG_MAX) break;
    if (v == wn) {
      int pj = -1;
#pragma unroll
      for (int q = 0; q < kLocal; ++q) if (q == head) pj = part[q];
      const int i = (int)(wn & 0xffffffffu);
      const int lo = i < pj ? i : pj, hi = i < pj ? pj : i;
      // the pair and its diagonal neighbours that lie in the series
      for (int d = 0; d < kSeedSpread; ++d) {
        const int off = d - kSeedSpread / 2;
        const bool ok = lo + off >= wb && hi + off < we;
        seeds[round * kSeedSpread + d] = ok ? make_int2(lo + off, hi + off) : make_int2(-1, -1);
      }
      ++head;
    }
    ++count;
    __syncthreads();
  }
  if (threadIdx.x == 0) nseeds[b] = count;
}

__global__ void k_reverse(const double* a, int64_t n, double* out) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x)
    out[p] = a[n - 1 - p];
}

}  // namespace

void launch_reverse(const double* a, int64_t n, double* out, cudaStream_t st) {
  k_reverse<<<1024, 256, 0, st>>>(a, n, out);
}

void launch_tile_bound(const unsigned int* tile_best, int ntiles, unsigned int* bsf2,
                       cudaStream_t st) {
  if (ntiles > 0) k_tile_bound<<<(ntiles + 255) / 256, 256, 0, st>>>(tile_best, ntiles, bsf2);
}

void launch_mp(const DevSeries& S, const Tile* tiles, int ntiles, unsigned long long* keys,
               cudaStream_t st, unsigned int* tile_best) {
  k_fill_u64<<<1024, 256, 0, st>>>(keys, S.s, ULLONG_MAX);
  if (ntiles <= 0) return;
  cudaFuncSetAttribute(k_mp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(MpShared));
  const int slab = 1 << 20;
  for (int b = 0; b < ntiles; b += slab) {
    const int cnt = ntiles - b < slab ? ntiles - b : slab;
    k_mp<false><<<cnt, kLbThreads, sizeof(MpShared), st>>>(S, tiles + b, keys, tile_best, b,
                                                           MpCollect{});
  }
}

void launch_mp_seed(const DevSeries& S, const Tile* tiles, int ntiles, unsigned long long* keys,
                    cudaStream_t st) {
  k_fill_u64<<<1024, 256, 0, st>>>(keys, S.s, ULLONG_MAX);
  if (ntiles <= 0) return;
  cudaFuncSetAttribute(k_mp_seed, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(MpSeedShared));
  const int slab = 1 << 20;
  for (int b = 0; b < ntiles; b += slab) {
    const int cnt = ntiles - b < slab ? ntiles - b : slab;
    k_mp_seed<<<cnt, kLbThreads, sizeof(MpSeedShared), st>>>(S, tiles + b, keys);
  }
}

void launch_mp_collect(const DevSeries& S, const Tile* tiles, int ntiles,
                       const unsigned long long* want, int2* cand, unsigned int* count,
                       unsigned int cap, cudaStream_t st) {
  if (ntiles <= 0) return;
  cudaFuncSetAttribute(k_mp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(MpShared));
  const int slab = 1 << 20;
  for (int b = 0; b < ntiles; b += slab) {
    const int cnt = ntiles - b < slab ? ntiles - b : slab;
    k_mp<true><<<cnt, kLbThreads, sizeof(MpShared), st>>>(S, tiles + b, nullptr, nullptr, b,
                                                          MpCollect{want, cand, count, cap});
  }
}

void launch_mp_want(int64_t s, const unsigned long long* up, const unsigned long long* lo,
                    unsigned long long* want, unsigned long long* wrev, cudaStream_t st) {
  k_mp_want<<<(unsigned)((s + 255) / 256), 256, 0, st>>>(s, up, lo, want, wrev);
}

void launch_mp_exact(const DevSeries& S, const int2* cand, const unsigned int* count,
                     unsigned int cap, bool reversed, bool pick, unsigned long long* rowmin,
                     unsigned long long* rowidx, cudaStream_t st) {
  k_mp_exact<<<148 * 8, 256, 0, st>>>(S, cand, count, cap, reversed, pick, rowmin, rowidx);
}

void launch_mp_exact_out(int64_t s, const unsigned long long* rowmin,
                         const unsigned long long* rowidx, double* mp, int64_t* mpi,
                         cudaStream_t st) {
  k_mp_exact_out<<<(unsigned)((s + 255) / 256), 256, 0, st>>>(s, rowmin, rowidx, mp, mpi);
}

void launch_mp_finalize(const DevSeries& S, const unsigned long long* up,
                        const unsigned long long* lo, double* mp, int64_t* mpi,
                        cudaStream_t st) {
  k_mp_finalize<<<(unsigned)((S.s + 255) / 256), 256, 0, st>>>(S, up, lo, mp, mpi);
}

void launch_seed_select(const DevSeries& S, const unsigned long long* keys, int2* seeds,
                        unsigned int* nseeds, cudaStream_t st) {
  k_seed_select<<<S.nseries, kSelThreads, 0, st>>>(S, keys, seeds, nseeds);
}

}  // namespace dtwj
