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
// spread over positions, one direction at a time (the second only when the
// first stays within the best-so-far), checking the warp's running sum every
// kKeoghCheck samples; most pairs that reach it are pruned within the first
// few hundred samples of the first direction.  The run's windows overlap, so
// consecutive pairs re-read the same lines from L1.  It reads FP32 copies of
// the series and of the envelope (U, L pairs), centered per 1024-sample
// block and normalised per window.  Survivors go to the DTW queue.
#include "../../include/dtwj.h"
#include "dtwj_dev.cuh"

namespace dtwj {
namespace {

constexpr int kRunWarps = 4;
constexpr int kKeoghCheck = 128;  // samples between two best-so-far checks of LB_Keogh
constexpr int kKeoghWarps = 8;    // warps per block of the LB_Keogh kernel
constexpr int kKeoghBatch = 8;    // consecutive queue entries a warp takes at once

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

// max(a, b, c) in one instruction (three-input max.f32, sm_100).
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}

// Adds one LB_Keogh term: query sample a (block-centered, scale sq, offset o
// = query block offset - envelope block offset, both already scaled) against
// the block-centered envelope ul = (U, L) (scale se).  With q = a sq + o,
// max(q - U, 0)^2 + min(q - L, 0)^2 = max(q - U, L - q, 0)^2 since L <= U.
__device__ __forceinline__ float keogh_acc(float a, float2 ul, float sq, float se, float o,
                                           float acc) {
  const float q = fmaf(a, sq, o);
  const float d = max3f(fmaf(ul.x, -se, q), fmaf(ul.y, se, -q), 0.0f);
  return fmaf(d, d, acc);
}

__device__ __forceinline__ float block_offset(const DevSeries& S, unsigned int b, double mu,
                                              double is) {
  return (float)((S.cb[b] - mu) * is);
}

// One window of a queued LB_Keogh candidate, prefetched into shared memory.
struct KeoghSide {
  double mu, is;     // window mean and 1 / deviation
  float o0, o1;      // (cb - mu) * is of the window's first block and of the next
  unsigned int x;    // window start (below 2^31: n <= INT32_MAX - 4)
  unsigned int pad;
};

// Scaled offset of block b for window side w: the prefetched ones for its
// first two blocks, FP64 otherwise (windows longer than a block).
__device__ __forceinline__ float side_offset(const DevSeries& S, const KeoghSide& w,
                                             unsigned int b) {
  const unsigned int b0 = w.x >> kBlkShift;
  return b == b0 ? w.o0 : (b == b0 + 1 ? w.o1 : block_offset(S, b, w.mu, w.is));
}

// One direction of LB_Keogh for one pair: query window q against the
// envelope of window e, over the middle samples [kBias, m - kBias); `ends` is
// the end samples' share (max of their terms and the endpoint bound).  The
// samples run in segments over which both windows stay in one block (constant
// offset), each in stretches of kKeoghCheck after which the warp compares the
// running sum with thr; a segment's remainder joins the sum unchecked.
// Returns true when the whole bound stays within thr, false as soon as it
// exceeds it.  Every branch is warp-uniform.
__device__ bool keogh_within(const DevSeries& S, const KeoghSide& q, const KeoghSide& e,
                             float ends, float thr, int lane) {
  const int kend = S.m - kBias;
  const unsigned int qx = q.x, ex = e.x;
  const float sq = (float)q.is, se = (float)e.is;
  const float* A = S.af + qx + lane;
  const float2* UL = S.ulf + ex + lane;
  unsigned int bq = (qx + kBias) >> kBlkShift, be = (ex + kBias) >> kBlkShift;
  float oq = side_offset(S, q, bq), oe = side_offset(S, e, be);
  float acc = 0.0f;
  int k = kBias;
  for (;;) {
    // first samples of the next blocks, relative to the window starts
    const int nq = (int)(((bq + 1) << kBlkShift) - qx), ne = (int)(((be + 1) << kBlkShift) - ex);
    const int seg = min(kend, min(nq, ne));
    const float o = oq - oe;
    for (; k + kKeoghCheck <= seg; k += kKeoghCheck) {
#pragma unroll
      for (int u = 0; u < kKeoghCheck / 32; ++u)
        acc = keogh_acc(A[k + 32 * u], UL[k + 32 * u], sq, se, o, acc);
      if (ends + warp_sumf(acc) > thr) return false;
    }
#pragma unroll
    for (int u = 0; u < kKeoghCheck / 32; ++u)
      if (k + 32 * u + lane < seg) acc = keogh_acc(A[k + 32 * u], UL[k + 32 * u], sq, se, o, acc);
    k = seg;
    if (k >= kend) break;
    if (nq == seg) oq = side_offset(S, q, ++bq);
    if (ne == seg) oe = side_offset(S, e, ++be);
  }
  return ends + warp_sumf(acc) <= thr;
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

__global__ void __launch_bounds__(kRunWarps * 32, 8) k_runs(DevSeries S, DevSearch Q,
                                                         const Tile* tiles,
                                                         const unsigned int* bits,
                                                         unsigned int total_items, bool masked,
                                                         bool bounds) {
  __shared__ unsigned int wbits[kRunWarps][kLbWords];
  __shared__ int2 rlist[kRunWarps][kRunList];
  __shared__ unsigned long long cnt[kNumCounters];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m = S.m, lo = kBias, hi = S.m - 1 - kBias;
  for (int x = threadIdx.x; x < kNumCounters; x += blockDim.x) cnt[x] = 0;
  __syncthreads();
  unsigned int* wb = wbits[warp];
  int2* rl = rlist[warp];
  for (;;) {
    unsigned int item = 0;
    if (lane == 0) item = atomicAdd(Q.run_next, 1u);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= total_items) break;
    // the lag's words, [tile][word][lag]
    const unsigned int* src = bits + (size_t)(item / kLbLags) * kLbLags * kLbWords + item % kLbLags;
    const Tile T = tiles[item / kLbLags];
    const int64_t L = (int64_t)T.L0 + (int64_t)(item % kLbLags);
    // rows this lag really has in the tile: r < rows and i0 + r + L < s
    int64_t nrow = (int64_t)T.send - L - T.i0;
    if (nrow > T.rows) nrow = T.rows;
    bool nz = false;
    for (int x = lane; x < kLbWords; x += 32) {
      unsigned int v = src[(size_t)x * kLbLags];
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
            if (slot < Q.queue_cap) {
              Q.queue[slot] = make_int2((int)(i0 + p), (int)(j0 + p));
              if (Q.qser) Q.qser[slot] = T.series;
            } else {
              atomicOr(S.status, 2);
            }
          }
          continue;
        }
        const unsigned int* bsf2 = Q.bsf2 + T.series;
        float thr = prune_threshold_now(bsf2, S.m);
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
          float kim = 0.0f;
          if (alive) {
            const ZEnds zi = z_ends(S, i), zj = z_ends(S, j);
            double dl, dr;
            kim_bound<double>(zi, zj, m, &dl, &dr);
            kim = (float)(dl + dr);
            if (dl + dr + lbm * lbm > (double)thr) {
              alive = false;
              atomicAdd(&cnt[kPrunedKim], 1ull);
            }
          }
          // ---- survivors go to the LB_Keogh queue, in run order ----
          const unsigned int bits = __ballot_sync(0xffffffffu, alive);
          if (bits) {
            unsigned int base = 0;
            if (lane == 0) base = atomicAdd(Q.kq_count, (unsigned int)__popc(bits));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (alive) {
              const unsigned int slot = base + __popc(bits & ((1u << lane) - 1u));
              if (slot < Q.kq_cap) {
                Q.kq[slot] = make_int4((int)i, (int)j, __float_as_int(kim), T.series);
              } else {
                atomicOr(S.status, 2);
              }
            }
          }
          // a fresh best-so-far tightens the rest of the run
          thr = fminf(thr, prune_threshold_now(bsf2, S.m));
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();
  for (int x = threadIdx.x; x < kNumCounters; x += blockDim.x)
    if (cnt[x]) atomicAdd(&Q.counters[x], cnt[x]);
}

// LB_Keogh over the queued candidates.  Entries sit in the order the run
// filter found them, so the kKeoghBatch consecutive pairs a warp takes are
// mostly neighbours on one diagonal and share L1 lines.  Lane e prefetches
// entry e of the batch (indices, endpoint bound, window statistics, block
// offsets) into shared memory, so the dependent loads are paid once per
// batch; then the lanes run over the samples of one pair at a time.  The
// first direction (query i against the envelope of j) decides most pairs,
// the second runs only when the first stays within the best-so-far.
__global__ void __launch_bounds__(kKeoghWarps * 32, 5) k_keogh(DevSeries S, DevSearch Q) {
  __shared__ KeoghSide side[kKeoghWarps][kKeoghBatch][2];
  __shared__ float endsv[kKeoghWarps][kKeoghBatch][2];
  __shared__ int serv[kKeoghWarps][kKeoghBatch];
  __shared__ float errv[kKeoghWarps][kKeoghBatch];  // FP32 error scale of the pair
  __shared__ unsigned long long pruned_block;
  if (threadIdx.x == 0) pruned_block = 0;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned int total = *Q.kq_count < Q.kq_cap ? *Q.kq_count : Q.kq_cap;
  unsigned long long pruned = 0;
  for (;;) {
    unsigned int idx = 0;
    if (lane == 0) idx = atomicAdd(Q.kq_next, (unsigned int)kKeoghBatch);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    if (idx >= total) break;
    const int cnt = total - idx < (unsigned int)kKeoghBatch ? (int)(total - idx) : kKeoghBatch;
    __syncwarp();  // the previous batch is no longer read
    if (lane < 2 * cnt) {
      // lane (e, d): window d of entry e, and the end samples of direction d
      // (query = window d, envelope = the other window) in FP64
      const int e = lane >> 1, d = lane & 1;
      const int4 r = Q.kq[idx + e];
      const unsigned int xe = (unsigned int)(d ? r.x : r.y);
      KeoghSide w;
      w.x = (unsigned int)(d ? r.y : r.x);
      w.mu = S.mu[w.x];
      w.is = S.isg[w.x];
      const unsigned int b0 = w.x >> kBlkShift;
      w.o0 = block_offset(S, b0, w.mu, w.is);
      w.o1 = block_offset(S, b0 + 1, w.mu, w.is);
      w.pad = 0;
      side[warp][e][d] = w;
      const double me = S.mu[xe], ie = S.isg[xe];
      double t = 0.0;
#pragma unroll
      for (int c = 0; c < 2 * kBias; ++c) {
        const int k = c < kBias ? c : S.m - 2 * kBias + c;
        const double z = (S.a[w.x + k] - w.mu) * w.is;
        const double u = (S.U[xe + k] - me) * ie, l = (S.L[xe + k] - me) * ie;
        const double dd = fmax(fmax(z - u, l - z), 0.0);
        t = fma(dd, dd, t);
      }
      endsv[warp][e][d] = (float)fmax((double)__int_as_float(r.z), t);
      if (d == 0) {
        serv[warp][e] = r.w;
        errv[warp][e] = fmaxf(S.rw[r.x], S.rw[r.y]);
      }
    }
    __syncwarp();
    for (int e = 0; e < cnt; ++e) {
      float thr = prune_threshold_now(Q.bsf2 + serv[warp][e], S.m);
      // a pair whose FP32 error bound does not fit the slack is never pruned here
      if (!fp32_bound_ok(errv[warp][e], thr, S.m)) thr = __int_as_float(0x7f800000);
      const KeoghSide& wi = side[warp][e][0];
      const KeoghSide& wj = side[warp][e][1];
      bool live = keogh_within(S, wi, wj, endsv[warp][e][0], thr, lane);
      if (live) live = keogh_within(S, wj, wi, endsv[warp][e][1], thr, lane);
      if (lane == 0) {
        if (!live) {
          ++pruned;
        } else {
          const unsigned int slot = atomicAdd(Q.queue_count, 1u);
          if (slot < Q.queue_cap) {
            Q.queue[slot] = make_int2((int)wi.x, (int)wj.x);
            if (Q.qser) Q.qser[slot] = serv[warp][e];
          } else {
            atomicOr(S.status, 2);
          }
        }
      }
    }
  }
  if (lane == 0 && pruned) atomicAdd(&pruned_block, pruned);
  __syncthreads();
  if (threadIdx.x == 0 && pruned_block) atomicAdd(&Q.counters[kPrunedKeogh], pruned_block);
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
    S.ulf[p] = make_float2((float)(S.U[p] - c), (float)(S.L[p] - c));
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

void launch_keogh(const DevSeries& S, const DevSearch& Q, int num_sms, cudaStream_t st) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_keogh, kKeoghWarps * 32, 0);
  if (per_sm < 1) per_sm = 1;
  k_keogh<<<num_sms * per_sm, kKeoghWarps * 32, 0, st>>>(S, Q);
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
