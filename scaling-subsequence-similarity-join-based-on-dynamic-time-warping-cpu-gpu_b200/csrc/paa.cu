// Block-mean lower bound (LB_PAA) on the survivors of the diagonal sweep.
//
// LB_Keogh (CPU_version1/lb_keogh.cpp:9-72, GPU_version1/src/LB_keogh_warp.cu:
// 74-96) sums, over the samples k of the query window, the squared distance
// of q_k to the envelope [L_k, U_k] of the other window.  Over a block of B
// consecutive samples, Cauchy-Schwarz gives
//   sum_{k in block} max(q_k - U_k, 0)^2 >= B max(qbar - Ubar, 0)^2
// (and the same for L), with qbar, Ubar, Lbar the block means, so
//   LB_PAA = B sum_blocks max(qbar - Ubar, Lbar - qbar, 0)^2  <=  LB_Keogh
// is a lower bound of the DTW distance as well (Keogh's PAA bound).  With
// the sliding means of the series and of its raw envelope precomputed, one
// pair costs m / B block terms per direction instead of m samples, and on
// random walks it prunes nearly every pair the O(1) diagonal bound lets
// through (99.5 % at m = 1024, B = 32, w = 52), where the reference's masked
// diagonal bound and endpoint bound prune about 86 %.
//
// Work items are (tile, 32-row word, group of 32 lags) of the diagonal
// sweep's survivor bits, stored [tile][word][lag].  Windows of at most 1024
// samples go to k_paa_lags (lanes on lags, described there).  For longer
// ones (k_paa), a warp loads the 32 words of its lag group in one coalesced
// read; for every lag L with survivors, lane p takes row i = i0 + p of the
// word (survivors cluster: a nonzero word
// holds about 28 of 32 rows).  The blocks are aligned to absolute sample
// positions: block [x, x + B) of window i, x a multiple of B, meets block
// [x + L, x + L + B) of window j, so every lane of the batch reads the same
// two block means (broadcast loads) and only the per-window normalisation
// differs between lanes.  The aligned blocks inside every lane's window are
// shared; each lane adds the window-relative blocks that fit in its own
// window before and after them (the rows are consecutive, so those reads are
// coalesced).  A window's block offset changes where a block crosses a
// 1024-sample boundary; for aligned blocks that happens at the same block in
// every lane, so the shared blocks run in warp-wide segments with constant
// offsets: two loads and ten FP32 operations per block.  The lanes vote every
// four blocks; the batch stops as soon as every live lane is pruned.  The
// endpoint bound (LB_Kim, CPU_version1/lb_kim.cpp:10-73) then runs in FP64 on
// the survivors, which go to the LB_Keogh queue.
//
// Precision: the sliding means are FP32, centered per block, and normalised
// per window by an FP64 block offset.  For windows longer than 1024 samples
// the blocks are the 1024-sample blocks of the LB_Keogh copies; for shorter
// ones, 2048-sample blocks in two copies shifted by 1024 samples, so that a
// window lies in one block (one offset per window).  A pair is pruned only
// when the FP32 error bound of its windows (rw, or the window record's scale)
// fits in the slack the threshold keeps above the best-so-far
// (fp32_bound_ok).
#include "../../include/dtwj.h"
#include "dtwj_dev.cuh"

namespace dtwj {
namespace {

constexpr int kPaaWarps = 8;

__device__ __forceinline__ float max3f(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}

// Centers of the two copies of the block means for windows of at most 1024
// samples: block b of copy 0 is [2048 b, 2048 b + 2048), block b of copy 1 is
// [2048 b - 1024, 2048 b + 1024); each is centered on the mean of the two
// 1024-sample blocks it spans (cb, padded past the end).
__device__ __forceinline__ int64_t copy_block(int copy, int64_t p) { return (p + copy * 1024) >> 11; }
__device__ __forceinline__ double copy_center(const DevSeries& S, int copy, int64_t b) {
  const int64_t k = 2 * b - copy;
  return k < 0 ? S.cb[0] : 0.5 * (S.cb[k] + S.cb[k + 1]);
}
// The copy whose blocks hold window [i, i + m), m <= 1024: copy 0 when the
// window ends inside its 2048-sample block, else copy 1 (then i mod 2048 >
// 1024 and the window lies in [2048 b + 1024, 2048 b + 3072)).
__device__ __forceinline__ int win_copy(int64_t i, int m) { return (int)(i & 2047) + m > 2048 ? 1 : 0; }

// Sliding block means over [p, p + B) of a, U and L, centered: on the
// 1024-sample block of p (pq, windows longer than 1024 samples), or on the
// block of p in each of the two copies (pq2).  Entries whose block runs past
// the series are zero (never read: a window's blocks end inside it).
__global__ void k_slide_means(DevSeries S, int B) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= S.n) return;
  if (p + B > S.n) {
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (S.pq2) {
      S.pq2[p] = z;
      S.pq2[S.n + p] = z;
    } else {
      S.pq[p] = z;
    }
    return;
  }
  double sa = 0.0, su = 0.0, sl = 0.0;
  for (int k = 0; k < B; ++k) {
    sa += S.a[p + k];
    su += S.U[p + k];
    sl += S.L[p + k];
  }
  const double ib = 1.0 / (double)B;
  const double ma = sa * ib, mu = su * ib, ml = sl * ib;
  if (S.pq2) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const double x = copy_center(S, c, copy_block(c, p));
      S.pq2[c * S.n + p] = make_float4((float)(ma - x), (float)(mu - x), (float)(ml - x), 0.0f);
    }
  } else {
    const double x = S.cb[p >> kBlkShift];
    S.pq[p] = make_float4((float)(ma - x), (float)(mu - x), (float)(ml - x), 0.0f);
  }
}

__device__ __forceinline__ float block_max_reduce(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  __shared__ float red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  float t = 0.0f;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmaxf(t, red[w]);
  return t;
}

// cmax[b] = the largest magnitude of any centered FP32 value of block b
// (af, ulf and, when built, pq), read by LB_Keogh and the block-mean bound.
__global__ void k_block_max(DevSeries S, int nb) {
  const int b = blockIdx.x;
  if (b >= nb) return;
  const int64_t lo = (int64_t)b << kBlkShift;
  int64_t hi = lo + (1 << kBlkShift);
  if (hi > S.n) hi = S.n;
  float v = 0.0f;
  for (int64_t p = lo + threadIdx.x; p < hi; p += blockDim.x) {
    const float2 u = S.ulf[p];
    v = fmaxf(v, fmaxf(fabsf(S.af[p]), fmaxf(fabsf(u.x), fabsf(u.y))));
    if (S.pq) {
      const float4 q = S.pq[p];
      v = fmaxf(v, fmaxf(fabsf(q.x), fmaxf(fabsf(q.y), fabsf(q.z))));
    }
  }
  const float t = block_max_reduce(v);
  if (threadIdx.x == 0) S.cmax[b] = t;
}

// cmax2[c * kCopyBlocks + b] = the largest magnitude of pq2 over block b of
// copy c (grid: 2 kCopyBlocks(n) blocks).
__global__ void k_block_max2(DevSeries S) {
  const int64_t nbc = kCopyBlocks(S.n);
  const int c = (int)(blockIdx.x / nbc);
  const int64_t b = blockIdx.x - c * nbc;
  int64_t lo = b * 2048 - c * 1024, hi = lo + 2048;
  if (lo < 0) lo = 0;
  if (hi > S.n) hi = S.n;
  const float4* q = S.pq2 + c * S.n;
  float v = 0.0f;
  for (int64_t p = lo + threadIdx.x; p < hi; p += blockDim.x) {
    const float4 x = q[p];
    v = fmaxf(v, fmaxf(fabsf(x.x), fmaxf(fabsf(x.y), fabsf(x.z))));
  }
  const float t = block_max_reduce(v);
  if (threadIdx.x == 0) S.cmax2[blockIdx.x] = t;
}

// rw[i] = isg_i * max over the blocks window i covers of (cmax[b] +
// |cb[b] - mu_i|): bounds every z-like value the FP32 bounds form for it.
__global__ void k_window_scale(DevSeries S) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= S.s) return;
  const double mu = S.mu[i];
  const int64_t b0 = i >> kBlkShift, b1 = (i + S.m - 1) >> kBlkShift;
  double r = 0.0;
  for (int64_t b = b0; b <= b1; ++b) r = fmax(r, (double)S.cmax[b] + fabs(S.cb[b] - mu));
  S.rw[i] = (float)(r * S.isg[i] * (1.0 + 1e-6));
}

// Window records for pq2: the block offset (x_c - mu_i) isg_i of the copy
// block holding window i (center x_c), FP64; isg_i as FP32; and the error
// scale isg_i (cmax2 + |x_c - mu_i|) of the values the block-mean bound forms
// for it (the rw of pq2).
__global__ void k_window_rec(DevSeries S) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= S.s) return;
  const int c = win_copy(i, S.m);
  const int64_t b = copy_block(c, i);
  const double x = copy_center(S, c, b), mu = S.mu[i], is = S.isg[i];
  const double off = (x - mu) * is;
  const double r = ((double)S.cmax2[c * kCopyBlocks(S.n) + b] + fabs(x - mu)) * is * (1.0 + 1e-6);
  S.wrec[i] = make_float4(__int_as_float(__double2loint(off)), __int_as_float(__double2hiint(off)),
                          (float)is, (float)r);
}

// Scaled block offset of window x at 1024-sample block b, FP64.
__device__ __forceinline__ double win_offset(const DevSeries& S, int64_t b, double mu, double is) {
  return (S.cb[b] - mu) * is;
}

// The six end samples of a window as a sequence of length 6 for kim_bound:
// indices 0..2 and e-2..e (e = 5) are its first and last three samples.
struct Ends6 {
  const double* v;
  __device__ double operator[](int k) const { return v[k]; }
};

// One block term of both directions: query i (block mean qi) against the
// envelope of j (uj, lj) and query j against the envelope of i, with
// q - U = P - U s and L - q = L s - P, P = q s + (offset of q - offset of U).
__device__ __forceinline__ void block_terms(const float4 bi, const float4 bj, float si, float sj,
                                            float oij, float& acc1, float& acc2) {
  const float p1 = fmaf(bi.x, si, oij);
  const float d1 = max3f(fmaf(-bj.y, sj, p1), fmaf(bj.z, sj, -p1), 0.0f);
  acc1 = fmaf(d1, d1, acc1);
  const float p2 = fmaf(bj.x, sj, -oij);
  const float d2 = max3f(fmaf(-bi.y, si, p2), fmaf(bi.z, si, -p2), 0.0f);
  acc2 = fmaf(d2, d2, acc2);
}

template <int B>
__global__ void __launch_bounds__(kPaaWarps * 32, 3) k_paa(DevSeries S, DevSearch Q,
                                                           const Tile* tiles,
                                                           const unsigned int* bits,
                                                           unsigned int total_items) {
  __shared__ unsigned long long cnt_paa, cnt_kim;
  if (threadIdx.x == 0) cnt_paa = cnt_kim = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int m = S.m;
  constexpr int kSpan = 1 << kBlkShift;
  unsigned int npaa = 0, nkim = 0;
  for (;;) {
    unsigned int item = 0;
    if (lane == 0) item = atomicAdd(Q.run_next, 1u);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= total_items) break;
    const unsigned int tk = item / (kLbWords * kLbGroups);
    const unsigned int rem = item - tk * (kLbWords * kLbGroups);
    const int wi = (int)(rem / kLbGroups), g = (int)(rem % kLbGroups);
    const unsigned int word = bits[((size_t)tk * kLbWords + wi) * kLbLags + g * 32 + lane];
    unsigned int nz = __ballot_sync(0xffffffffu, word != 0u);
    if (!nz) continue;
    const Tile T = tiles[tk];
    const unsigned int* bsf2 = Q.bsf2 + T.series;
    // positions fit 32 bits (n <= INT32_MAX - 4)
    const int ib = T.i0 + wi * 32;  // the batch's first row
    const int i_row = ib + lane;    // this lane's row
    // aligned blocks inside every row's window [ib + p, ib + p + m), p < 32
    // (none when m is short: each lane then covers its window by itself)
    int x_lo = (ib + 31 + B - 1) / B * B, x_hi = (ib + m) / B * B;
    const bool shared = x_lo < x_hi;
    if (!shared) x_lo = x_hi = 0;
    // the threshold, once per item (a later, lower best-so-far only prunes
    // more: the one read here stays valid), and the largest error scale
    // whose FP32 bound may prune against it
    const float thr = prune_threshold_now(bsf2, m);
    const float r_ok = fp32_bound_radius(thr, m);
    // the row side, the same for every lag of the item: window statistics and
    // the offsets of the (at most two) 1024-blocks of the shared range
    const int i_own = i_row < T.send ? i_row : T.send - 1;  // a valid row for the loads
    const double mi_own = S.mu[i_own], si_own = S.isg[i_own];
    // the error scale a partner may have and still prune with this row (-1: none)
    const float r_lane = S.rw[i_own] <= r_ok ? r_ok : -1.0f;
    const int b_lo = x_lo >> kBlkShift;
    const double oi0_own = win_offset(S, b_lo, mi_own, si_own);
    const double oi1_own = win_offset(S, b_lo + 1, mi_own, si_own);
    while (nz) {
      const int l = __ffs(nz) - 1;
      nz &= nz - 1u;
      const unsigned int wb = __shfl_sync(0xffffffffu, word, l);
      const bool live = (wb >> lane) & 1u;  // the sweep set only bits of valid pairs
      const int L = T.L0 + g * 32 + l;
      // a lane without a pair computes the first live lane's pair (valid
      // addresses, result ignored), so the block loops need no predicate
      const int src = __ffs(wb) - 1;
      const int i = ib + (live ? lane : src), j = i + L;
      const double mi = mi_own, si = si_own;  // a borrowed pair's are only approximate: ignored
      const double mj = S.mu[j], sj = S.isg[j];
      const float thr_lane = live && S.rw[j] <= r_lane ? thr : __int_as_float(0x7f800000);
      const float fsi = (float)si, fsj = (float)sj;
      float acc1 = 0.0f, acc2 = 0.0f;
      // ---- this lane's own blocks before and after the shared ones ----
      {
        // head [i, x_lo) and tail [x_hi, i + m) are each at most 30 + B
        // samples long; without shared blocks the head is the whole window
        // (m < 31 + 2B, so at most 2 (30 + B) / B blocks as well)
        const int nh = shared ? (x_lo - i) / B : m / B;
        const int nt = shared ? (i + m - x_hi) / B : 0;
        constexpr int kEdgeMax = 2 * ((30 + B) / B);
#pragma unroll 1
        for (int e = 0; e < kEdgeMax; ++e) {
          const bool head = e < nh, tail = e >= nh && e < nh + nt;
          if (head || tail) {
            const int xi = head ? i + e * B : x_hi + (e - nh) * B;
            const int xj = xi + L;
            const float o = (float)(win_offset(S, xi >> kBlkShift, mi, si) -
                                    win_offset(S, xj >> kBlkShift, mj, sj));
            block_terms(S.pq[xi], S.pq[xj], fsi, fsj, o, acc1, acc2);
          }
        }
      }
      // ---- the shared aligned blocks, in segments of constant offsets ----
      bool pruned = !live || (float)B * fmaxf(acc1, acc2) > thr_lane;
      int x = x_lo;
      while (x < x_hi && !__all_sync(0xffffffffu, pruned)) {
        // the next block whose i or j side starts in another 1024-sample block
        const int ci = ((x >> kBlkShift) + 1) << kBlkShift;
        const int cj = (((((x + L) >> kBlkShift) + 1) << kBlkShift) - L + B - 1) / B * B;
        int seg = ci < cj ? ci : cj;
        if (seg > x_hi) seg = x_hi;
        const int bx = x >> kBlkShift;
        const double oi = bx == b_lo ? oi0_own
                        : (bx == b_lo + 1 ? oi1_own : win_offset(S, bx, mi, si));
        const float oij = (float)(oi - win_offset(S, (x + L) >> kBlkShift, mj, sj));
        const float4* qi = S.pq + x;
        const float4* qj = S.pq + x + L;
        const int nblk = (seg - x) / B;
        int k = 0;
        for (; k + 4 <= nblk; k += 4, qi += 4 * B, qj += 4 * B) {
#pragma unroll
          for (int u = 0; u < 4; ++u) block_terms(qi[u * B], qj[u * B], fsi, fsj, oij, acc1, acc2);
          pruned = pruned || (float)B * fmaxf(acc1, acc2) > thr_lane;
          if (__all_sync(0xffffffffu, pruned)) break;
        }
        if (k + 4 <= nblk) break;  // every lane pruned
        for (; k < nblk; ++k, qi += B, qj += B) block_terms(qi[0], qj[0], fsi, fsj, oij, acc1, acc2);
        pruned = pruned || (float)B * fmaxf(acc1, acc2) > thr_lane;
        x = seg;
      }
      bool alive = live && !pruned;
      npaa += (live && pruned) ? 1u : 0u;
      float kim = 0.0f;
      if (alive) {
        // endpoint bound on the survivors (FP64, the end samples normalised)
        double qv[6], tv[6];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          qv[k] = (S.a[i + k] - mi) * si;
          qv[3 + k] = (S.a[i + m - 3 + k] - mi) * si;
          tv[k] = (S.a[j + k] - mj) * sj;
          tv[3 + k] = (S.a[j + m - 3 + k] - mj) * sj;
        }
        double dl, dr;
        kim_bound<double>(Ends6{qv}, Ends6{tv}, 6, &dl, &dr);
        kim = (float)(dl + dr);
        if (dl + dr > (double)thr) {
          alive = false;
          ++nkim;
        }
      }
      const unsigned int sv = __ballot_sync(0xffffffffu, alive);
      if (sv) {
        unsigned int base = 0;
        if (lane == 0) base = atomicAdd(Q.kq_count, (unsigned int)__popc(sv));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (alive) {
          const unsigned int slot = base + __popc(sv & ((1u << lane) - 1u));
          if (slot < Q.kq_cap) {
            Q.kq[slot] = make_int4(i, j, __float_as_int(kim), T.series);
          } else {
            atomicOr(S.status, 2);
          }
        }
      }
    }
  }
  unsigned long long a = npaa, b = nkim;
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if (lane == 0) {
    if (a) atomicAdd(&cnt_paa, a);
    if (b) atomicAdd(&cnt_kim, b);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (cnt_paa) atomicAdd(&Q.counters[kPrunedPaa], cnt_paa);
    if (cnt_kim) atomicAdd(&Q.counters[kPrunedKim], cnt_kim);
  }
}

// The block-mean filter for windows of at most 1024 samples, with the lanes
// of a batch on 32 consecutive lags of one row instead of 32 rows of one lag.
// A row's window [i, i + m) is cut into nb = m / B blocks relative to the
// window (block k: [i + kB, i + kB + B)); its block means are the same for
// every lane (broadcast loads) and the partner's [j + kB, j + kB + B), j =
// i + L, sit at consecutive lags (coalesced loads), so no lane needs blocks
// of its own at the window ends.  The means come from pq2, where every window
// lies inside one block of one copy: a pair's block offset is one FP32 value,
// the difference of its windows' FP64 offsets (wrec), and a block term is
// two loads and ten FP32 operations.  The blocks run in a stride-4 order
// (k = 0, 4, 8, ..., then 1, 5, 9, ...), which spreads the first terms over
// the whole window: on the bench series a batch is settled after 7.6 blocks
// on average against 9.2 in position order (CPU measurement over sampled lag
// groups); the lanes vote every four blocks.
template <int B>
__global__ void __launch_bounds__(kPaaWarps * 32, 3) k_paa_lags(DevSeries S, DevSearch Q,
                                                                const Tile* tiles,
                                                                const unsigned int* bits,
                                                                unsigned int total_items) {
  __shared__ unsigned long long cnt_paa, cnt_kim;
  if (threadIdx.x == 0) cnt_paa = cnt_kim = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int m = S.m;
  const int nb = m / B;  // blocks per window (a short tail past nb B is left out)
  const float INF = __int_as_float(0x7f800000);
  unsigned int npaa = 0, nkim = 0;
  for (;;) {
    unsigned int item = 0;
    if (lane == 0) item = atomicAdd(Q.run_next, 1u);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= total_items) break;
    const unsigned int tk = item / (kLbWords * kLbGroups);
    const unsigned int rem = item - tk * (kLbWords * kLbGroups);
    const int wi = (int)(rem / kLbGroups), g = (int)(rem % kLbGroups);
    // lane l holds lag L0 + 32 g + l: bit r is row i0 + 32 wi + r
    const unsigned int word = bits[((size_t)tk * kLbWords + wi) * kLbLags + g * 32 + lane];
    unsigned int rows = __reduce_or_sync(0xffffffffu, word);
    if (!rows) continue;
    const Tile T = tiles[tk];
    const unsigned int* bsf2 = Q.bsf2 + T.series;
    // positions fit 32 bits (n <= INT32_MAX - 4)
    const int ib = T.i0 + wi * 32;
    const int L = T.L0 + g * 32 + lane;
    // the threshold, once per item (a later, lower best-so-far only prunes
    // more: the one read here stays valid), and the largest error scale
    // whose FP32 bound may prune against it
    const float thr = prune_threshold_now(bsf2, m);
    const float r_ok = fp32_bound_radius(thr, m);
    while (rows) {
      const int r = __ffs(rows) - 1;
      rows &= rows - 1u;
      const bool live = (word >> r) & 1u;  // the sweep set only bits of valid pairs
      const unsigned int lm = __ballot_sync(0xffffffffu, live);
      const int i = ib + r;
      // a lane without a pair computes the first live lane's pair (valid
      // addresses, result ignored), so the block loop needs no predicate
      const int j = i + (live ? L : L - lane + __ffs(lm) - 1);
      const float4 wri = S.wrec[i];  // broadcast
      const float4 wrj = S.wrec[j];  // consecutive lags: coalesced
      const float thr_lane = live && wri.w <= r_ok && wrj.w <= r_ok ? thr : INF;
      const float o = (float)(__hiloint2double(__float_as_int(wri.y), __float_as_int(wri.x)) -
                              __hiloint2double(__float_as_int(wrj.y), __float_as_int(wrj.x)));
      const float fsi = wri.z, fsj = wrj.z;
      const float4* pi = S.pq2 + (win_copy(i, m) ? S.n : 0) + i;
      const float4* pj = S.pq2 + (win_copy(j, m) ? S.n : 0) + j;
      float acc1 = 0.0f, acc2 = 0.0f;
      bool pruned = !live;
      // stride-4 order, a vote after every four blocks
#pragma unroll 1
      for (int r4 = 0; r4 < 4; ++r4) {
        int k = r4;
        // block k's means at qi[0], qj[0]; the group's four at immediate offsets
        const float4* qi = pi + r4 * B;
        const float4* qj = pj + r4 * B;
        for (; k + 12 < nb; k += 16, qi += 16 * B, qj += 16 * B) {
#pragma unroll
          for (int u = 0; u < 4; ++u) block_terms(qi[4 * u * B], qj[4 * u * B], fsi, fsj, o, acc1, acc2);
          pruned = pruned || (float)B * fmaxf(acc1, acc2) > thr_lane;
          if (__all_sync(0xffffffffu, pruned)) break;
        }
        if (k + 12 < nb) break;  // every lane pruned
        if (k < nb) {
          for (; k < nb; k += 4, qi += 4 * B, qj += 4 * B) block_terms(qi[0], qj[0], fsi, fsj, o, acc1, acc2);
          pruned = pruned || (float)B * fmaxf(acc1, acc2) > thr_lane;
          if (__all_sync(0xffffffffu, pruned)) break;
        }
      }
      bool alive = live && !pruned;
      npaa += (live && pruned) ? 1u : 0u;
      float kim = 0.0f;
      if (alive) {
        // endpoint bound on the survivors (FP64, the end samples normalised)
        const double mi = S.mu[i], si = S.isg[i], mj = S.mu[j], sj = S.isg[j];
        double qv[6], tv[6];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          qv[k] = (S.a[i + k] - mi) * si;
          qv[3 + k] = (S.a[i + m - 3 + k] - mi) * si;
          tv[k] = (S.a[j + k] - mj) * sj;
          tv[3 + k] = (S.a[j + m - 3 + k] - mj) * sj;
        }
        double dl, dr;
        kim_bound<double>(Ends6{qv}, Ends6{tv}, 6, &dl, &dr);
        kim = (float)(dl + dr);
        if (dl + dr > (double)thr) {
          alive = false;
          ++nkim;
        }
      }
      const unsigned int sv = __ballot_sync(0xffffffffu, alive);
      if (sv) {
        unsigned int base = 0;
        if (lane == 0) base = atomicAdd(Q.kq_count, (unsigned int)__popc(sv));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (alive) {
          const unsigned int slot = base + __popc(sv & ((1u << lane) - 1u));
          if (slot < Q.kq_cap) {
            Q.kq[slot] = make_int4(i, j, __float_as_int(kim), T.series);
          } else {
            atomicOr(S.status, 2);
          }
        }
      }
    }
  }
  unsigned long long a = npaa, b = nkim;
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if (lane == 0) {
    if (a) atomicAdd(&cnt_paa, a);
    if (b) atomicAdd(&cnt_kim, b);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (cnt_paa) atomicAdd(&Q.counters[kPrunedPaa], cnt_paa);
    if (cnt_kim) atomicAdd(&Q.counters[kPrunedKim], cnt_kim);
  }
}

}  // namespace

int paa_block(int m) {
  if (m >= 1024) return 32;
  if (m >= 512) return 16;
  return 8;
}

int launch_paa_prep(const DevSeries& S, cudaStream_t st) {
  const int nb = (int)((S.n + (1 << kBlkShift) - 1) >> kBlkShift);
  k_slide_means<<<(unsigned)((S.n + 255) / 256), 256, 0, st>>>(S, S.paa_b);
  k_block_max<<<nb, 256, 0, st>>>(S, nb);
  k_window_scale<<<(unsigned)((S.s + 255) / 256), 256, 0, st>>>(S);
  if (!S.pq2) return 3;
  k_block_max2<<<(unsigned)(2 * kCopyBlocks(S.n)), 256, 0, st>>>(S);
  k_window_rec<<<(unsigned)((S.s + 255) / 256), 256, 0, st>>>(S);
  return 5;
}

void launch_paa(const DevSeries& S, const DevSearch& Q, const Tile* tiles, int tile_begin,
                int tile_end, const unsigned int* bits, int num_sms, cudaStream_t st) {
  if (tile_end <= tile_begin) return;
  const unsigned int items = (unsigned int)(tile_end - tile_begin) * kLbWords * kLbGroups;
  auto go = [&](auto kern) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPaaWarps * 32, 0);
    if (per_sm < 1) per_sm = 1;
    kern<<<num_sms * per_sm, kPaaWarps * 32, 0, st>>>(S, Q, tiles + tile_begin, bits, items);
  };
  // windows of at most 1024 samples: lanes on lags (window-relative blocks,
  // no per-lane window ends); longer windows: lanes on rows
  if (S.m <= (1 << kBlkShift)) {
    if (S.paa_b == 32) go(k_paa_lags<32>);
    else if (S.paa_b == 16) go(k_paa_lags<16>);
    else go(k_paa_lags<8>);
  } else {
    if (S.paa_b == 32) go(k_paa<32>);
    else if (S.paa_b == 16) go(k_paa<16>);
    else go(k_paa<8>);
  }
}

}  // namespace dtwj
