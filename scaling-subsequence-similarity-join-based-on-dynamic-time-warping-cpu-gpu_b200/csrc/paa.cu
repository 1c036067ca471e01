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
// sweep's survivor bits, stored [tile][word][lag].  A warp loads the 32 words
// of its lag group in one coalesced read; for every lag with survivors, lane p
// takes row p of the word, so the 32 pairs are consecutive on one diagonal and
// every block read (pa, pul at i + B k and j + B k) is one contiguous line per
// warp.  Survivors on a lag cluster: a nonzero word holds about 28 of 32 rows.
// The lanes run the block terms of both directions together and vote every
// four blocks; the batch stops as soon as every live lane is pruned.  The
// blocks run in warp-wide segments between the points where some lane's
// window crosses into the next 1024-sample block (its offset changes there),
// so the loop body is loads at immediate offsets and the block terms only.  The
// endpoint bound (LB_Kim, CPU_version1/lb_kim.cpp:10-73) then runs in FP64 on
// the survivors, which go to the LB_Keogh queue.
//
// Precision: the sliding means are FP32, centered per 1024-sample block like
// the LB_Keogh copies, and normalised per window by an FP64 block offset.  A
// pair is pruned only when the FP32 error bound of its windows (rw) fits in
// the slack the threshold keeps above the best-so-far (fp32_bound_ok).
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

// Sliding block means, centered on the 1024-sample block of their first
// sample: pa[p] = mean a[p, p + B) - cb[p >> kBlkShift], pul likewise for
// (U, L).  Entries whose block runs past the series are zero (never read:
// a window's blocks end inside it).
__global__ void k_slide_means(DevSeries S, int B) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= S.n) return;
  if (p + B > S.n) {
    S.pa[p] = 0.0f;
    S.pul[p] = make_float2(0.0f, 0.0f);
    return;
  }
  double sa = 0.0, su = 0.0, sl = 0.0;
  for (int k = 0; k < B; ++k) {
    sa += S.a[p + k];
    su += S.U[p + k];
    sl += S.L[p + k];
  }
  const double c = S.cb[p >> kBlkShift], ib = 1.0 / (double)B;
  S.pa[p] = (float)(sa * ib - c);
  S.pul[p] = make_float2((float)(su * ib - c), (float)(sl * ib - c));
}

// cmax[b] = the largest magnitude of any centered FP32 value of block b
// (af, ulf, pa, pul), read by LB_Keogh and the block-mean bound.
__global__ void k_block_max(DevSeries S, int nb) {
  const int b = blockIdx.x;
  if (b >= nb) return;
  const int64_t lo = (int64_t)b << kBlkShift;
  int64_t hi = lo + (1 << kBlkShift);
  if (hi > S.n) hi = S.n;
  float v = 0.0f;
  for (int64_t p = lo + threadIdx.x; p < hi; p += blockDim.x) {
    const float2 u = S.ulf[p], pu = S.pul[p];
    v = fmaxf(v, fmaxf(fabsf(S.af[p]), fmaxf(fabsf(u.x), fabsf(u.y))));
    v = fmaxf(v, fmaxf(fabsf(S.pa[p]), fmaxf(fabsf(pu.x), fabsf(pu.y))));
  }
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  __shared__ float red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmaxf(t, red[w]);
    S.cmax[b] = t;
  }
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

template <int B>
__global__ void __launch_bounds__(kPaaWarps * 32, 4) k_paa(DevSeries S, DevSearch Q,
                                                           const Tile* tiles,
                                                           const unsigned int* bits,
                                                           unsigned int total_items) {
  __shared__ unsigned long long cnt_paa, cnt_kim;
  if (threadIdx.x == 0) cnt_paa = cnt_kim = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int m = S.m;
  const int nb = m / B;  // whole blocks; a partial tail block is left out (terms >= 0)
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
    const int64_t i_row = (int64_t)T.i0 + wi * 32 + lane;  // this lane's row
    while (nz) {
      const int l = __ffs(nz) - 1;
      nz &= nz - 1u;
      const unsigned int wb = __shfl_sync(0xffffffffu, word, l);
      const bool live = (wb >> lane) & 1u;  // the sweep set only bits of valid pairs
      // a lane without a pair computes the first live lane's pair (valid
      // addresses, result ignored), so the block loop needs no predicate
      const int64_t i_src = __shfl_sync(0xffffffffu, i_row, __ffs(wb) - 1);
      const int64_t i = live ? i_row : i_src;
      const int64_t j = i + (int64_t)T.L0 + g * 32 + l;
      const float thr = prune_threshold_now(bsf2, m);
      const double mi = S.mu[i], si = S.isg[i], mj = S.mu[j], sj = S.isg[j];
      // a pair whose FP32 error bound does not fit the slack is never pruned here
      const float thr_lane =
          live && fp32_bound_ok(fmaxf(S.rw[i], S.rw[j]), thr, m) ? thr : __int_as_float(0x7f800000);
      const float fsi = (float)si, fsj = (float)sj;
      const float* pai = S.pa + i;
      const float* paj = S.pa + j;
      const float2* pui = S.pul + i;
      const float2* puj = S.pul + j;
      // the block offsets change where a window's block start crosses a
      // 1024-sample boundary: block ci (i) and cj (j), then every 1024 / B
      int ci = (int)((((i >> kBlkShift) + 1) << kBlkShift) - i + B - 1) / B;
      int cj = (int)((((j >> kBlkShift) + 1) << kBlkShift) - j + B - 1) / B;
      float oij = (float)(win_offset(S, i >> kBlkShift, mi, si) - win_offset(S, j >> kBlkShift, mj, sj));
      float acc1 = 0.0f, acc2 = 0.0f;
      bool pruned = !live;
      int k = 0;
      while (k < nb) {
        // a segment of blocks in which no lane's offsets change
        int seg = min(ci, cj);
        seg = __reduce_min_sync(0xffffffffu, (unsigned int)min(seg, nb));
        for (; k + 4 <= seg; k += 4) {
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int x = (k + u) * B;
            const float ai = pai[x], aj = paj[x];
            const float2 ui = pui[x], uj = puj[x];
            // query i against the envelope of j: q - U = P - Uj sj, L - q = Lj sj - P
            const float p1 = fmaf(ai, fsi, oij);
            const float d1 = max3f(fmaf(-uj.x, fsj, p1), fmaf(uj.y, fsj, -p1), 0.0f);
            acc1 = fmaf(d1, d1, acc1);
            // query j against the envelope of i
            const float p2 = fmaf(aj, fsj, -oij);
            const float d2 = max3f(fmaf(-ui.x, fsi, p2), fmaf(ui.y, fsi, -p2), 0.0f);
            acc2 = fmaf(d2, d2, acc2);
          }
          pruned = pruned || (float)B * fmaxf(acc1, acc2) > thr_lane;
          if (__all_sync(0xffffffffu, pruned)) break;
        }
        if (__all_sync(0xffffffffu, pruned)) break;
        for (; k < seg; ++k) {
          const int x = k * B;
          const float ai = pai[x], aj = paj[x];
          const float2 ui = pui[x], uj = puj[x];
          const float p1 = fmaf(ai, fsi, oij);
          const float d1 = max3f(fmaf(-uj.x, fsj, p1), fmaf(uj.y, fsj, -p1), 0.0f);
          acc1 = fmaf(d1, d1, acc1);
          const float p2 = fmaf(aj, fsj, -oij);
          const float d2 = max3f(fmaf(-ui.x, fsi, p2), fmaf(ui.y, fsi, -p2), 0.0f);
          acc2 = fmaf(d2, d2, acc2);
        }
        if (k >= nb) break;
        // at block k some lanes cross into the next 1024-sample block
        if (k == ci || k == cj) {
          if (k == ci) ci += (1 << kBlkShift) / B;
          if (k == cj) cj += (1 << kBlkShift) / B;
          const int64_t xi = i + (int64_t)k * B, xj = j + (int64_t)k * B;
          oij = (float)(win_offset(S, xi >> kBlkShift, mi, si) -
                        win_offset(S, xj >> kBlkShift, mj, sj));
        }
      }
      pruned = pruned || (float)B * fmaxf(acc1, acc2) > thr_lane;
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
            Q.kq[slot] = make_int4((int)i, (int)j, __float_as_int(kim), T.series);
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

void launch_paa_prep(const DevSeries& S, cudaStream_t st) {
  const int nb = (int)((S.n + (1 << kBlkShift) - 1) >> kBlkShift);
  k_slide_means<<<(unsigned)((S.n + 255) / 256), 256, 0, st>>>(S, S.paa_b);
  k_block_max<<<nb, 256, 0, st>>>(S, nb);
  k_window_scale<<<(unsigned)((S.s + 255) / 256), 256, 0, st>>>(S);
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
  if (S.paa_b == 32) go(k_paa<32>);
  else if (S.paa_b == 16) go(k_paa<16>);
  else go(k_paa<8>);
}

}  // namespace dtwj
