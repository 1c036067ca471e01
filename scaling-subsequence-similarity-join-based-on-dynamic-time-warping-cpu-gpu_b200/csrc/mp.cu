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
// monotone for non-negative doubles) above the partner index, so a 64-bit
// atomicMin keeps the nearest neighbour with the lowest index on ties at that
// resolution; the finalize pass recomputes the exact FP64 distance.
//
// The seeds are the kSeeds smallest row minima, as in
// CPU_version1/new_dtw_motifGUI.cpp:53-74 (min_v_k + exact DTW per seed).
#include "dtwj_dev.cuh"

#include <cfloat>
#include <climits>

namespace dtwj {
namespace {

constexpr int kMpRowsMax = 4096;

// LOWER = false: pairs (r, r + L), reduction to row r  (j > i neighbours)
// LOWER = true:  pairs (r, r - L), reduction to row r  (j < i neighbours)
template <bool LOWER>
__global__ void __launch_bounds__(kTileLags) k_mp(DevSeries S, const Tile* tiles,
                                                  unsigned long long* keys) {
  __shared__ unsigned long long rowbest[kMpRowsMax];
  const Tile T = tiles[blockIdx.x];
  const int64_t L = (int64_t)T.L0 + threadIdx.x;
  const int64_t s = S.s;
  const int m = S.m;
  // rows of this tile (upper: i; lower: r = i + L0)
  const int64_t rbase = LOWER ? (int64_t)T.L0 + T.i0 : (int64_t)T.i0;
  const int rows = T.rows;
  for (int x = threadIdx.x; x < rows; x += blockDim.x) rowbest[x] = ULLONG_MAX;
  __syncthreads();

  int64_t r_start, r_end;  // this thread's rows [r_start, r_end)
  if (LOWER) {
    r_start = rbase > L ? rbase : L;
    r_end = rbase + rows < s ? rbase + rows : s;
  } else {
    r_start = rbase;
    r_end = rbase + rows < s - L ? rbase + rows : s - L;
  }
  const bool any = L < s && r_start < r_end;

  double C = 0.0;
  if (any) {
    const int64_t c0 = LOWER ? r_start - L : r_start + L;
    const double mr = S.mu[r_start], mc = S.mu[c0];
    for (int k = 0; k < m; ++k) C = fma(S.a[r_start + k] - mr, S.a[c0 + k] - mc, C);
  }
  const int lane = threadIdx.x & 31;
  for (int x = 0; x < rows; ++x) {
    const int64_t r = rbase + x;
    unsigned int hi = UINT_MAX;
    int64_t c = 0;
    if (any && r >= r_start && r < r_end) {
      c = LOWER ? r - L : r + L;
      if (r > r_start) {
        C = fma(S.dfa[r - 1], S.dga[c - 1], C);
        C = fma(S.dfa[c - 1], S.dga[r - 1], C);
      }
      if (!S.flat[r] && !S.flat[c]) {
        double e2 = fma(-2.0 * C * S.isg[r], S.isg[c], 2.0 * m);
        e2 = fmax(e2, 0.0);
        hi = (unsigned int)__double2hiint(e2);
      }
    }
    const unsigned int best = __reduce_min_sync(0xffffffffu, hi);
    if (best != UINT_MAX) {
      const unsigned int ballot = __ballot_sync(0xffffffffu, hi == best);
      // lowest partner index: lowest lane (upper) or highest lane (lower)
      const int win = LOWER ? 31 - __clz(ballot) : __ffs(ballot) - 1;
      if (lane == win) {
        const unsigned long long key =
            ((unsigned long long)best << 32) | (unsigned long long)(unsigned int)c;
        atomicMin(&rowbest[x], key);
      }
    }
  }
  __syncthreads();
  for (int x = threadIdx.x; x < rows; x += blockDim.x) {
    const unsigned long long v = rowbest[x];
    if (v != ULLONG_MAX) atomicMin(&keys[rbase + x], v);
  }
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
    const unsigned long long k2 = lo[i];
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

constexpr int kSelThreads = 1024;
constexpr int kLocal = 8;

// kSeeds smallest row minima (by ED^2 key, then row index).  Each thread
// keeps the kLocal best of a strided slice; kSeeds rounds of block minimum
// then pop the global order.  Writes the seed pairs, their count and the
// initial best-so-far (the smallest ED^2, rounded up: ED >= DTW).
__global__ void __launch_bounds__(kSelThreads) k_seed_select(DevSeries S,
                                                              const unsigned long long* keys,
                                                              int2* seeds, unsigned int* nseeds,
                                                              unsigned int* bsf2) {
  unsigned long long loc[kLocal];
  int part[kLocal];
#pragma unroll
  for (int q = 0; q < kLocal; ++q) { loc[q] = ULLONG_MAX; part[q] = -1; }
  for (int64_t i = threadIdx.x; i < S.s; i += blockDim.x) {
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
      seeds[round] = make_int2(i < pj ? i : pj, i < pj ? pj : i);
      if (round == 0) {
        const unsigned long long bits = ((wn >> 32) + 1ull) << 32;
        const float e2 = __double2float_ru(__longlong_as_double((long long)bits));
        *bsf2 = __float_as_uint(e2);
      }
      ++head;
    }
    ++count;
    __syncthreads();
  }
  if (threadIdx.x == 0) *nseeds = count;
}

}  // namespace

void launch_mp(const DevSeries& S, const Tile* tiles, int ntiles, unsigned long long* keys,
               bool lower, cudaStream_t st) {
  k_fill_u64<<<1024, 256, 0, st>>>(keys, S.s, ULLONG_MAX);
  if (ntiles <= 0) return;
  // grid limit is 2^31-1 blocks; tiles are launched in slabs to stay far below
  const int slab = 1 << 20;
  for (int b = 0; b < ntiles; b += slab) {
    const int cnt = ntiles - b < slab ? ntiles - b : slab;
    if (lower)
      k_mp<true><<<cnt, kTileLags, 0, st>>>(S, tiles + b, keys);
    else
      k_mp<false><<<cnt, kTileLags, 0, st>>>(S, tiles + b, keys);
  }
}

void launch_mp_finalize(const DevSeries& S, const unsigned long long* up,
                        const unsigned long long* lo, double* mp, int64_t* mpi,
                        cudaStream_t st) {
  k_mp_finalize<<<(unsigned)((S.s + 255) / 256), 256, 0, st>>>(S, up, lo, mp, mpi);
}

void launch_seed_select(const DevSeries& S, const unsigned long long* keys, int2* seeds,
                        unsigned int* nseeds, unsigned int* bsf2, cudaStream_t st) {
  k_seed_select<<<1, kSelThreads, 0, st>>>(S, keys, seeds, nseeds, bsf2);
}

}  // namespace dtwj
