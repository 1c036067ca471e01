// Run filter: the stages the reference applies to every pair that passes
// diag_fast, applied here to runs of consecutive pairs on one diagonal.
//
//   masked bound    diag_mask_global      CPU_version1/diag_mask_global.cpp:11-245,
//                                         GPU_version1/lib/diag_mask_global.cu:12-164
//   endpoint bound  its LB_KIM tail       CPU_version1/diag_mask_global.cpp:247-311
//   LB_Keogh        lb_keogh_stride_with_nomalise (raw-series envelope
//                   normalised per window) GPU_version1/src/LB_keogh_warp.cu:74-96
//
// Work items are (tile, lag) pairs of the diagonal sweep: a warp reads the
// lag's survivor bits, cuts them into runs of consecutive rows (at most
// kRunMax long) and owns each run (i0 + p, j0 + p), p < len.  Lane p of a batch of 32
// holds pair p.  The masked bound needs six running sums along the diagonal;
// their per-row increments are independent, so the warp computes all of a
// batch's increments at once and turns them into the sums with one inclusive
// scan, anchored by an exact O(m) evaluation at the run's first pair (FP64
// throughout, as in the reference's recurrence).  The endpoint bound is one
// lane's work per pair.  LB_Keogh then runs pair by pair with the lanes
// spread over positions, in rounds of 256 positions that stop as soon as
// either direction exceeds the best-so-far; the run's windows overlap, so
// consecutive pairs re-read the same lines from L1.  It reads FP32 copies of
// the series and envelope centered per 1024-sample block, normalised per
// window.  Survivors go to the DTW queue.
#include "dtwj_dev.cuh"

namespace dtwj {
namespace {

constexpr int kRunWarps = 4;
constexpr int kMaxWinBlocks = 64;  // windows up to 62 * 1024 samples

// Masked bound for env = r, query = c from the raw FP64 sums
// F1 = sum_T M_r a_c, F2 = sum_T M_r a_c^2, F3 = sum_T M_r E_r a_c.
__device__ inline double masked_lb(const DevSeries& S, int64_t r, int64_t c, double F1,
                                   double F2, double F3) {
  const double mr = S.mu[r], mc = S.mu[c], ir = S.isg[r], ic = S.isg[c];
  const double SM = S.SM[r];
  const double mnorm = (F2 - 2.0 * mc * F1 + mc * mc * SM) * ic * ic;
  const double t = (F3 - 2.0 * mr * F1 - mc * S.SME[r] + 2.0 * mr * mc * SM) * ir * ic;
  const double dist = 2.0 * mnorm - 2.0 * t + (double)S.MN[r];
  const double d2 = (double)S.MDUL2[r];
  if (dist < d2) return 0.0;
  return 0.5 * (sqrt(2.0 * dist - d2) - (double)S.MDUL[r]);
}

struct ZEnds {
  double v[6];
  int m;
  __device__ double operator[](int k) const { return k < 3 ? v[k] : v[k - (m - 3) + 3]; }
};

__device__ inline ZEnds z_ends(const DevSeries& S, int64_t w0) {
  ZEnds z;
  z.m = S.m;
  const double mu = S.mu[w0], is = S.isg[w0];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    z.v[k] = (S.a[w0 + k] - mu) * is;
    z.v[3 + k] = (S.a[w0 + S.m - 3 + k] - mu) * is;
  }
  return z;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_iscan(double v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

__device__ __forceinline__ float keogh_term(float x, float U, float L) {
  const float du = x - U, dl = x - L;
  return x > U ? du * du : (x < L ? dl * dl : 0.0f);
}

// Cuts the survivor bits of one lag into runs; returns how many runs were
// written to `list` (at most `cap`) and advances *pos past them.
__device__ int cut_runs(const unsigned int* w, int* pos, int2* list, int cap) {
  int cnt = 0;
  int p = *pos;
  while (p < kLbRows && cnt < cap) {
    const int wi = p >> 5, b = p & 31;
    const unsigned int v = w[wi] >> b;
    if (v == 0u) {
      p = (wi + 1) << 5;
      continue;
    }
    const int start = p + __ffs(v) - 1;
    int e = start;
    for (;;) {
      const int wj = e >> 5, bj = e & 31;
      const int ones = __ffs(~(w[wj] >> bj)) - 1;  // consecutive ones from bit bj
      const int avail = 32 - bj;
      if (ones < 0 || ones >= avail) {
        e += avail;
        if (e >= kLbRows) break;
      } else {
        e += ones;
        break;
      }
    }
    for (int r = start; r < e && cnt < cap; r += kRunMax) {
      const int len = e - r < kRunMax ? e - r : kRunMax;
      list[cnt++] = make_int2(r, len);
      p = r + len;
    }
    if (p < e) break;  // list full in the middle of a run
  }
  *pos = p;
  return cnt;
}

constexpr int kRunList = 32;

__global__ void __launch_bounds__(kRunWarps * 32) k_runs(DevSeries S, DevSearch Q,
                                                         const Tile* tiles,
                                                         const unsigned int* bits,
                                                         unsigned int total_items, bool masked,
                                                         bool bounds) {
  __shared__ float offs[kRunWarps][2][kMaxWinBlocks];
  __shared__ unsigned int wbits[kRunWarps][kLbWords];
  __shared__ int2 rlist[kRunWarps][kRunList];
  __shared__ unsigned long long cnt[kNumCounters];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m = S.m, lo = kBias, hi = S.m - 1 - kBias;
  const int nblk = ((m - 1) >> kBlkShift) + 2;
  for (int x = threadIdx.x; x < kNumCounters; x += blockDim.x) cnt[x] = 0;
  __syncthreads();
  float* oi = offs[warp][0];
  float* oj = offs[warp][1];
  unsigned int* wb = wbits[warp];
  int2* rl = rlist[warp];
  for (;;) {
    unsigned int item = 0;
    if (lane == 0) item = atomicAdd(Q.run_next, 1u);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= total_items) break;
    const unsigned int* src = bits + (size_t)item * kLbWords;
    const Tile T = tiles[item / kLbLags];
    const int64_t L = (int64_t)T.L0 + (int64_t)(item % kLbLags);
    // rows this lag really has in the tile: r < rows and i0 + r + L < s
    int64_t nrow = S.s - L - T.i0;
    if (nrow > T.rows) nrow = T.rows;
    bool nz = false;
    for (int x = lane; x < kLbWords; x += 32) {
      unsigned int v = src[x];
      const int64_t lo_row = (int64_t)x * 32;
      if (lo_row >= nrow) v = 0u;
      else if (lo_row + 32 > nrow) v &= (1u << (nrow - lo_row)) - 1u;
      wb[x] = v;
      nz |= v != 0u;
    }
    if (!__any_sync(0xffffffffu, nz)) continue;
    __syncwarp();
    int pos = 0;
    for (;;) {
      int nr = 0;
      if (lane == 0) nr = cut_runs(wb, &pos, rl, kRunList);
      nr = __shfl_sync(0xffffffffu, nr, 0);
      __syncwarp();
      if (nr == 0) break;
      for (int ri = 0; ri < nr; ++ri) {
    const int64_t i0 = (int64_t)T.i0 + rl[ri].x, j0 = i0 + L;
    const int len = rl[ri].y;
    if (!bounds) {
      // no bounds: every pair of the run goes to the DTW stage
      for (int p = lane; p < len; p += 32) {
        const unsigned int slot = atomicAdd(Q.queue_count, 1u);
        if (slot < Q.queue_cap) Q.queue[slot] = make_int2((int)(i0 + p), (int)(j0 + p));
        else atomicOr(S.status, 2);
      }
      continue;
    }
    float thr = prune_threshold_now(Q.bsf2, S.m);
    // ---- masked sums at the run's first pair (exact, FP64) ----
    double F1 = 0, F2 = 0, F3 = 0, R1 = 0, R2 = 0, R3 = 0;
    if (masked) {
      for (int k = lo + lane; k <= hi; k += 32) {
        const double ai = S.a[i0 + k], aj = S.a[j0 + k];
        const double Mi = S.mask[i0 + k], Mj = S.mask[j0 + k];
        F1 = fma(Mi, aj, F1);
        F2 = fma(Mi * aj, aj, F2);
        F3 = fma(Mi * S.E[i0 + k], aj, F3);
        R1 = fma(Mj, ai, R1);
        R2 = fma(Mj * ai, ai, R2);
        R3 = fma(Mj * S.E[j0 + k], ai, R3);
      }
      F1 = warp_sum(F1);
      F2 = warp_sum(F2);
      F3 = warp_sum(F3);
      R1 = warp_sum(R1);
      R2 = warp_sum(R2);
      R3 = warp_sum(R3);
    }
    for (int b = 0; b < len; b += 32) {
      const int p = b + lane;
      const bool valid = p < len;
      const int64_t i = i0 + p, j = j0 + p;
      double lbm = 0.0;
      if (masked) {
        // per-row increments: the window start (k = lo) of the previous row
        // leaves, the window end (k = hi) of this row enters
        double d1 = 0, d2 = 0, d3 = 0, e1 = 0, e2 = 0, e3 = 0;
        if (valid && p > 0) {
          const int64_t io = i - 1 + lo, in = i + hi, jo = j - 1 + lo, jn = j + hi;
          const double Mio = S.mask[io], Min = S.mask[in], Mjo = S.mask[jo], Mjn = S.mask[jn];
          const double ajo = S.a[jo], ajn = S.a[jn], aio = S.a[io], ain = S.a[in];
          d1 = Min * ajn - Mio * ajo;
          d2 = Min * ajn * ajn - Mio * ajo * ajo;
          d3 = Min * S.E[in] * ajn - Mio * S.E[io] * ajo;
          e1 = Mjn * ain - Mjo * aio;
          e2 = Mjn * ain * ain - Mjo * aio * aio;
          e3 = Mjn * S.E[jn] * ain - Mjo * S.E[jo] * aio;
        }
        const double f1 = F1 + warp_iscan(d1, lane), f2 = F2 + warp_iscan(d2, lane);
        const double f3 = F3 + warp_iscan(d3, lane), r1 = R1 + warp_iscan(e1, lane);
        const double r2 = R2 + warp_iscan(e2, lane), r3 = R3 + warp_iscan(e3, lane);
        if (valid) lbm = fmax(masked_lb(S, i, j, f1, f2, f3), masked_lb(S, j, i, r1, r2, r3));
        F1 = __shfl_sync(0xffffffffu, f1, 31);
        F2 = __shfl_sync(0xffffffffu, f2, 31);
        F3 = __shfl_sync(0xffffffffu, f3, 31);
        R1 = __shfl_sync(0xffffffffu, r1, 31);
        R2 = __shfl_sync(0xffffffffu, r2, 31);
        R3 = __shfl_sync(0xffffffffu, r3, 31);
      }
      bool alive = valid;
      if (alive && masked && lbm * lbm > (double)thr) {
        alive = false;
        atomicAdd(&cnt[kPrunedMasked], 1ull);
      }
      float kl = 0.0f, kr = 0.0f;
      if (alive) {
        const ZEnds zi = z_ends(S, i), zj = z_ends(S, j);
        double dl, dr;
        kim_bound<double>(zi, zj, m, &dl, &dr);
        kl = (float)dl;
        kr = (float)dr;
        if (dl + dr + lbm * lbm > (double)thr) {
          alive = false;
          atomicAdd(&cnt[kPrunedKim], 1ull);
        }
      }
      // ---- LB_Keogh, one pair at a time ----
      unsigned int bits = __ballot_sync(0xffffffffu, alive);
      while (bits) {
        const int qd = __ffs(bits) - 1;
        bits &= bits - 1;
        const int64_t pi = __shfl_sync(0xffffffffu, i, qd);
        const int64_t pj = __shfl_sync(0xffffffffu, j, qd);
        const float ends = __shfl_sync(0xffffffffu, kl + kr, qd);
        const double mui = S.mu[pi], muj = S.mu[pj];
        const float si = (float)S.isg[pi], sj = (float)S.isg[pj];
        const int64_t bi = pi >> kBlkShift, bj = pj >> kBlkShift;
        if (lane < nblk) {
          oi[lane] = (float)(S.cb[bi + lane] - mui);
          oj[lane] = (float)(S.cb[bj + lane] - muj);
        }
        __syncwarp();
        float s_e1 = 0, s_m1 = 0, s_e2 = 0, s_m2 = 0;
        bool dead = false;
        for (int base = 0; base < m && !dead; base += 256) {
          const int lim = base + 256 < m ? base + 256 : m;
          for (int k = base + lane; k < lim; k += 32) {
            const int64_t xi = pi + k, xj = pj + k;
            const float ofi = oi[(xi >> kBlkShift) - bi], ofj = oj[(xj >> kBlkShift) - bj];
            const float qi = (S.af[xi] + ofi) * si, tj = (S.af[xj] + ofj) * sj;
            const float t1 = keogh_term(qi, (S.Uf[xj] + ofj) * sj, (S.Lf[xj] + ofj) * sj);
            const float t2 = keogh_term(tj, (S.Uf[xi] + ofi) * si, (S.Lf[xi] + ofi) * si);
            if (k < kBias || k >= m - kBias) {
              s_e1 += t1;
              s_e2 += t2;
            } else {
              s_m1 += t1;
              s_m2 += t2;
            }
          }
          const float lb1 = fmaxf(warp_sumf(s_e1), ends) + warp_sumf(s_m1);
          const float lb2 = fmaxf(warp_sumf(s_e2), ends) + warp_sumf(s_m2);
          if (lb1 > thr || lb2 > thr) dead = true;
        }
        if (lane == 0) {
          if (dead) {
            atomicAdd(&cnt[kPrunedKeogh], 1ull);
          } else {
            const unsigned int slot = atomicAdd(Q.queue_count, 1u);
            if (slot < Q.queue_cap) Q.queue[slot] = make_int2((int)pi, (int)pj);
            else atomicOr(S.status, 2);
          }
        }
        __syncwarp();
      }
      // a fresh best-so-far tightens the rest of the run
      thr = fminf(thr, prune_threshold_now(Q.bsf2, S.m));
    }
      }
      __syncwarp();
    }
  }
  __syncthreads();
  for (int x = threadIdx.x; x < kNumCounters; x += blockDim.x)
    if (cnt[x]) atomicAdd(&Q.counters[x], cnt[x]);
}

// Block means of the series (centers of the FP32 copies).
__global__ void k_block_mean(DevSeries S, int nb) {
  const int b = blockIdx.x;
  if (b >= nb) return;
  const int64_t lo = (int64_t)b << kBlkShift;
  int64_t hi = lo + (1 << kBlkShift);
  if (hi > S.n) hi = S.n;
  double acc = 0.0;
  for (int64_t p = lo + threadIdx.x; p < hi; p += blockDim.x) acc += S.a[p];
  __shared__ double red[8];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    S.cb[b] = hi > lo ? t / (double)(hi - lo) : (b > 0 ? S.cb[b - 1] : 0.0);
  }
}

__global__ void k_center(DevSeries S, int nb) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p < S.n) {
    const double c = S.cb[p >> kBlkShift];
    S.af[p] = (float)(S.a[p] - c);
    S.Uf[p] = (float)(S.U[p] - c);
    S.Lf[p] = (float)(S.L[p] - c);
  }
  // two padding blocks past the end repeat the last center
  if (p < 2) S.cb[nb + p] = S.cb[nb - 1];
}

}  // namespace

void launch_center(const DevSeries& S, cudaStream_t st) {
  const int nb = (int)((S.n + (1 << kBlkShift) - 1) >> kBlkShift);
  k_block_mean<<<nb, 256, 0, st>>>(S, nb);
  k_center<<<(unsigned)((S.n + 255) / 256), 256, 0, st>>>(S, nb);
}

void launch_runs(const DevSeries& S, const DevSearch& Q, const Tile* tiles, int tile_begin,
                 int tile_end, const unsigned int* bits, bool masked, bool bounds, int num_sms,
                 cudaStream_t st) {
  if (tile_end <= tile_begin) return;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_runs, kRunWarps * 32, 0);
  if (per_sm < 1) per_sm = 1;
  const unsigned int items = (unsigned int)(tile_end - tile_begin) * kLbLags;
  k_runs<<<num_sms * per_sm, kRunWarps * 32, 0, st>>>(S, Q, tiles + tile_begin, bits, items,
                                                       masked, bounds);
}

}  // namespace dtwj
