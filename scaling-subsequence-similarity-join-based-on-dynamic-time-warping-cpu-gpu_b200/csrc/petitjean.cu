// LB_Petitjean on the device (lbPetitjean_new, CPU_version1/LB_PETITJEAN.cpp:10-123;
// the reference evaluates it between LB_Keogh and MON_dtw,
// CPU_version1/new_dtw_motifGUI.cpp:517-519).
//
// For windows A (rows) and B (columns) with envelopes (LA, UA) and (LB, UB):
//   H_k = A_k projected onto [LB_k, UB_k] for k in [3, m-4], H_k = A_k on the
//         three end samples of each side (the reference's copy of q, :24-39);
//   (LH, UH) = the clipped envelope of H, radius w (:41-88);
//   bound = endpoint bound + sum_{k=3}^{m-4} (A_k - H_k)^2
//         + sum_{k=3}^{m-4} g(B_k), g the distance of B_k to [LH_k, UH_k],
//           refined against A's envelope where UH_k > UA_k or LH_k < LA_k
//           (:89-110).
// Every cell (r, c) of a warping path costs at least (A_r - H_r)^2 + g(B_c)
// when H_r is the projection of A_r onto an interval that holds B_c and
// UA_c / LA_c bound A_r: the first sum charges one cell in each row, the
// second one cell in each column, and the endpoint bound the corner cells,
// which lie in neither those rows nor those columns.  So any envelopes that
// contain the windows keep the bound admissible: the join reads the raw
// series' envelope normalised per window; dtwj_pair_lb_petitjean can also
// build each window's own clipped envelope, as the reference does.
//
// One warp per pair, FP64 throughout (the projection term's difference of
// squares cancels, which an FP32 evaluation could not bound within the
// pruning slack).  The clipped envelopes come from doubling passes over a
// shared-memory table of m + 2w entries padded with -inf / +inf.
#include "../../include/dtwj.h"
#include "dtwj_dev.cuh"

#include <cmath>

namespace dtwj {
namespace {

constexpr int kPjWarps = 4;  // most warps per CTA of the join stage

__device__ __forceinline__ double pos_inf() { return __longlong_as_double(0x7ff0000000000000ll); }

// A z-normalised window read from the series.
struct ZWin {
  const double* a;
  int64_t o;
  double mu, is;
  __device__ __forceinline__ double operator[](int k) const { return (a[o + k] - mu) * is; }
};

// Sliding extrema by doubling.  tx / tn hold L = m + 2w entries; entry x is
// the value at sample x - w (-inf in tx, +inf in tn outside [0, m)).  Pass r
// replaces entry x by the extremum of entries x and x + r; after the passes
// r = 1, 2, ..., p / 2 (p the largest power of two <= 2w + 1) entry x covers
// [x, x + p), so the clipped envelope of radius w at sample k is the
// extremum of entries k and k + 2w + 1 - p.  A warp updates the table in
// place 32 entries at a time, in ascending order: an update reads only
// entries at or above its own, none of which the pass has written yet.
__device__ void extrema_passes(double* tx, double* tn, int L, int w, int lane) {
  for (int r = 1; 2 * r <= 2 * w + 1; r <<= 1) {
    for (int x0 = 0; x0 < L; x0 += 32) {
      const int x = x0 + lane;
      double vx = 0.0, vn = 0.0;
      if (x < L) {
        vx = tx[x];
        vn = tn[x];
        if (x + r < L) {
          vx = fmax(vx, tx[x + r]);
          vn = fmin(vn, tn[x + r]);
        }
      }
      __syncwarp();
      if (x < L) {
        tx[x] = vx;
        tn[x] = vn;
      }
      __syncwarp();
    }
  }
}

__device__ __forceinline__ int env_shift(int w) {
  int p = 1;
  while (2 * p <= 2 * w + 1) p <<= 1;
  return 2 * w + 1 - p;
}

// Fills the table with a window's z-normalised values and runs the passes.
__device__ void window_tables(const ZWin& z, int m, int w, double* tx, double* tn, int lane) {
  const int L = m + 2 * w;
  for (int x = lane; x < L; x += 32) {
    const int k = x - w;
    const bool in = k >= 0 && k < m;
    const double v = in ? z[k] : 0.0;
    tx[x] = in ? v : -pos_inf();
    tn[x] = in ? v : pos_inf();
  }
  __syncwarp();
  extrema_passes(tx, tn, L, w, lane);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// The two sums of the bound for windows ia (A) and ib (B), on every lane.
// OWN_ENV: each window's own clipped envelope, built here (ev holds 4m
// doubles: LA, UA, LB, UB); otherwise the raw envelope S.L / S.U normalised
// with the window's statistics.  tx / tn: m + 2w doubles each.
template <bool OWN_ENV>
__device__ void lbp_pair(const DevSeries& S, int64_t ia, int64_t ib, double* tx, double* tn,
                         double* ev, int lane, double* keogh_mid, double* terms) {
  const int m = S.m, w = S.w, L = m + 2 * w, sh = env_shift(w);
  const ZWin A{S.a, ia, S.mu[ia], S.isg[ia]};
  const ZWin B{S.a, ib, S.mu[ib], S.isg[ib]};
  if (OWN_ENV) {
    for (int side = 0; side < 2; ++side) {
      window_tables(side ? B : A, m, w, tx, tn, lane);
      double* lo = ev + 2 * side * m;
      double* up = lo + m;
      for (int k = lane; k < m; k += 32) {
        lo[k] = fmin(tn[k], tn[k + sh]);
        up[k] = fmax(tx[k], tx[k + sh]);
      }
      __syncwarp();
    }
  }
  // H and the first sum
  double km = 0.0;
  for (int x = lane; x < L; x += 32) {
    const int k = x - w;
    double hx = -pos_inf(), hn = pos_inf();
    if (k >= 0 && k < m) {
      const double za = A[k];
      double h = za;
      if (k >= kBias && k < m - kBias) {
        double lo, up;
        if (OWN_ENV) {
          lo = ev[2 * m + k];
          up = ev[3 * m + k];
        } else {
          lo = (S.L[ib + k] - B.mu) * B.is;
          up = (S.U[ib + k] - B.mu) * B.is;
        }
        h = fmin(fmax(za, lo), up);
        const double d = za - h;
        km = fma(d, d, km);
      }
      hx = h;
      hn = h;
    }
    tx[x] = hx;
    tn[x] = hn;
  }
  __syncwarp();
  extrema_passes(tx, tn, L, w, lane);
  // the second sum
  double t = 0.0;
  for (int k = kBias + lane; k < m - kBias; k += 32) {
    const double x = B[k];
    const double uh = fmax(tx[k], tx[k + sh]), lh = fmin(tn[k], tn[k + sh]);
    double ua, la;
    if (OWN_ENV) {
      la = ev[k];
      ua = ev[m + k];
    } else {
      la = (S.L[ia + k] - A.mu) * A.is;
      ua = (S.U[ia + k] - A.mu) * A.is;
    }
    double d = 0.0;
    if (x > uh && uh > ua) d = (x - ua) * (x - ua) - (uh - ua) * (uh - ua);
    else if (x < lh && lh < la) d = (x - la) * (x - la) - (lh - la) * (lh - la);
    else if (x > uh) d = (x - uh) * (x - uh);
    else if (x < lh) d = (x - lh) * (x - lh);
    t += d;
  }
  *keogh_mid = warp_sum(km);
  *terms = warp_sum(t);
  __syncwarp();  // the tables are rewritten by the next pair
}

// Join stage: filters the DTW queue of one chunk in place.  A pair whose
// bound exceeds its series' threshold gets i = -1, which the DTW stage skips.
__global__ void __launch_bounds__(kPjWarps * 32) k_petitjean(DevSeries S, DevSearch Q,
                                                              unsigned int* next, int warp_doubles) {
  extern __shared__ __align__(16) double smd[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double* tx = smd + (size_t)wid * warp_doubles;
  double* tn = tx + (S.m + 2 * S.w);
  const unsigned int total = *Q.queue_count < Q.queue_cap ? *Q.queue_count : Q.queue_cap;
  unsigned long long pruned = 0;
  for (;;) {
    unsigned int idx = 0;
    if (lane == 0) idx = atomicAdd(next, 1u);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    if (idx >= total) break;
    const int2 pr = Q.queue[idx];
    if (pr.x < 0) continue;
    const int sr = Q.qser ? Q.qser[idx] : series_of(S, pr.x);
    // one threshold for the whole warp (no kernel changes it during this one)
    float thr = 0.0f;
    if (lane == 0) thr = prune_threshold_now(Q.bsf2 + sr, S.m);
    thr = __shfl_sync(0xffffffffu, thr, 0);
    if (!(thr < __int_as_float(0x7f800000))) continue;  // nothing to prune against yet
    double kl = 0.0, kr = 0.0;
    if (lane == 0) {
      const ZWin A{S.a, pr.x, S.mu[pr.x], S.isg[pr.x]};
      const ZWin B{S.a, pr.y, S.mu[pr.y], S.isg[pr.y]};
      kim_bound<double>(A, B, S.m, &kl, &kr);
    }
    double km, t;
    lbp_pair<false>(S, pr.x, pr.y, tx, tn, nullptr, lane, &km, &t);
    if (lane == 0 && kl + kr + km + t > (double)thr) {
      Q.queue[idx] = make_int2(-1, pr.y);
      ++pruned;
    }
  }
  if (lane == 0 && pruned) atomicAdd(&Q.counters[kPrunedPetitjean], pruned);
}

// The two sums for explicit pairs (dtwj_pair_lb_petitjean): one warp per CTA.
template <bool OWN_ENV>
__global__ void __launch_bounds__(32) k_lbp_list(DevSeries S, const int2* pairs, int count,
                                                  double* keogh_mid, double* terms) {
  extern __shared__ __align__(16) double smd[];
  const int L = S.m + 2 * S.w;
  double* tx = smd;
  double* tn = smd + L;
  double* ev = smd + 2 * L;
  for (int p = blockIdx.x; p < count; p += gridDim.x) {
    const int2 pr = pairs[p];
    double km, t;
    lbp_pair<OWN_ENV>(S, pr.x, pr.y, tx, tn, ev, threadIdx.x, &km, &t);
    if (threadIdx.x == 0) {
      keogh_mid[p] = km;
      terms[p] = t;
    }
  }
}

}  // namespace

size_t petitjean_warp_bytes(int m, int w) { return (size_t)2 * (m + 2 * w) * sizeof(double); }

bool petitjean_fits(int m, int w) { return petitjean_warp_bytes(m, w) <= kPjMaxSmemBytes; }

void launch_petitjean(const DevSeries& S, const DevSearch& Q, unsigned int* next, int num_sms,
                      cudaStream_t st) {
  const size_t per_warp = petitjean_warp_bytes(S.m, S.w);
  if (per_warp > kPjMaxSmemBytes) return;  // callers check petitjean_fits first
  int warps = (int)(kPjMaxSmemBytes / per_warp);
  if (warps > kPjWarps) warps = kPjWarps;
  const size_t smem = per_warp * warps;
  cudaFuncSetAttribute(k_petitjean, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_petitjean, warps * 32, smem);
  if (per_sm < 1) per_sm = 1;
  k_petitjean<<<num_sms * per_sm, warps * 32, smem, st>>>(S, Q, next,
                                                          (int)(per_warp / sizeof(double)));
}

size_t lbp_list_bytes(int m, int w, bool own_env) {
  return ((size_t)2 * (m + 2 * w) + (own_env ? (size_t)4 * m : 0)) * sizeof(double);
}

void launch_lbp_list(const DevSeries& S, const int2* pairs, int count, bool own_env,
                     double* keogh_mid, double* terms, int num_sms, cudaStream_t st) {
  if (count <= 0) return;
  const size_t smem = lbp_list_bytes(S.m, S.w, own_env);
  const int grid = count < num_sms * 8 ? count : num_sms * 8;
  if (own_env) {
    cudaFuncSetAttribute(k_lbp_list<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_lbp_list<true><<<grid, 32, smem, st>>>(S, pairs, count, keogh_mid, terms);
  } else {
    cudaFuncSetAttribute(k_lbp_list<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    k_lbp_list<false><<<grid, 32, smem, st>>>(S, pairs, count, keogh_mid, terms);
  }
}

}  // namespace dtwj
