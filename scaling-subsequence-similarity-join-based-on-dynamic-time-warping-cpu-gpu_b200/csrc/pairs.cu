// Per-pair stages for the survivors of the diagonal sweep: endpoint bound,
// LB_Keogh in both directions with its cumulative bound, and the banded DTW.
//
// Reference counterparts:
//   endpoint bound  LB_KIM / the tail of diag_mask_global
//                   CPU_version1/lb_kim.cpp:10-73, GPU_version1/lib/diag_mask_global.cu:165-228
//   LB_Keogh        LB_KK             CPU_version1/lb_keogh.cpp:9-72,
//                   lb_keogh_stride_with_nomalise  GPU_version1/src/LB_keogh_warp.cu:74-96
//   DTW             MON_dtw           CPU_version1/MON_DTW.cpp:20-108,
//                   DTW_stairs_*      GPU_version1/src/DTW_stairs*.cu
//   bsf update      atomicMinFloat + syn_bsfs  GPU_version1/lib/GLOBAL_DIAG.cu:18-27
//
// Band layout (the register "stairs" of the reference, with the band width a
// runtime template choice instead of the REGISTER_NUM recompile): a group of
// G lanes computes one pair; lane g owns the C consecutive diagonals
// d = -w + gC .. -w + gC + C - 1 (cell (r, r + d)).  Lane g handles row
// r = tau - g at step tau: cell (r, d) needs (r, d-1) from the left lane's
// previous step (a shuffle of its last cell) and (r-1, d+1) from the right
// lane's first cell of this step (a shuffle right after it is computed), so
// every lane computes a full row of its C cells per step with two shuffles.
// The join runs one pair per warp (G = 32); pair lists pack several.  q and t
// are z-normalised in shared memory with finite sentinels outside [0, m) so
// out-of-range cells are effectively infinite without branches; a lane keeps
// the q and t values of C consecutive steps in registers.
#include "dtwj_dev.cuh"

#include <cfloat>
#include <climits>

namespace dtwj {
namespace {

template <typename T> struct Pad;
template <> struct Pad<float> {
  static __device__ __forceinline__ float q() { return kPadQ; }
  static __device__ __forceinline__ float t() { return kPadT; }
  static __device__ __forceinline__ float inf() { return __int_as_float(0x7f800000); }
};
template <> struct Pad<double> {
  static __device__ __forceinline__ double q() { return kPadQd; }
  static __device__ __forceinline__ double t() { return kPadTd; }
  static __device__ __forceinline__ double inf() { return __longlong_as_double(0x7ff0000000000000LL); }
};

__device__ __forceinline__ float fmin_(float a, float b) { return fminf(a, b); }
// min(a, b, c) in one instruction for FP32 (three-input min.f32, sm_100).
__device__ __forceinline__ float fmin3_(float a, float b, float c) {
  float d;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}
__device__ __forceinline__ double fmin3_(double a, double b, double c) { return fmin(fmin(a, b), c); }
__device__ __forceinline__ double fmin_(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ float fmax_(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double fmax_(double a, double b) { return fmax(a, b); }

template <int G>
__device__ __forceinline__ unsigned int group_mask() {
  if (G == 32) return 0xffffffffu;
  const unsigned int lane = threadIdx.x & 31;
  constexpr unsigned int bits = G < 32 ? (1u << (G % 32)) - 1u : 0xffffffffu;
  return bits << (lane & ~(unsigned)(G - 1));
}

template <int G, typename V>
__device__ __forceinline__ V group_sum(V v, unsigned int gm) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gm, v, o, G);
  return v;
}

// Shared-memory footprint of one group (in elements of T).
struct GroupLayout {
  int pq, pt;     // padding of q and t on each side
  int nc;         // cumulative-bound chunks
  int q_off, t_off, cb_off, total;
};

__host__ __device__ inline GroupLayout group_layout(int m, int w, int C, int G, bool bounds) {
  GroupLayout l;
  l.pq = G + 1;
  l.pt = G * C + G + 2;  // t is read at offsets [-(G + w), m + G + GC)
  l.nc = (m + 7) / 8;
  l.q_off = l.pq;
  l.t_off = l.pq + m + l.pq + l.pt;
  l.cb_off = l.t_off + m + l.pt;
  l.total = l.cb_off + l.nc + 2;
  // groups of a warp read their own q and t at a stride of C - 1 floats per
  // lane: an odd group stride (17 mod 32) keeps two groups off each other's
  // shared-memory banks
  l.total = l.total + ((17 - l.total % 32) + 32) % 32;
  return l;
}

// One row step of a lane, in place: A holds row r - 1 of its C diagonals
// (r = tau - g) and receives row r.  Cell (r, d) takes the minimum of
// (r, d-1) (the cell to its left: A[c-1] already updated, or the left lane's
// last cell of the previous step), (r-1, d) (A[c], not yet updated) and
// (r-1, d+1) (A[c+1], or the right lane's first cell of this step), plus
// (q[r] - t[r + d])^2; pen[c] is +inf for diagonals past the band.  qr is
// q[r] and tw(c) returns t[r + d_lo + c].  With LIVE false the lane keeps its
// row (a lane that has not reached row 0 yet), and its neighbours read its
// unchanged cells: for row 0 those are the virtual row -1 (0 on d = 0, +inf
// elsewhere), exactly what row 0 needs.  HI selects the cells that take the
// band mask: every cell (HI = -2), none (HI = -1) or cell HI alone (the
// layouts of dtw_band that keep the lanes past the band huge by their q).
template <typename T, int C, int G, int HI, typename TW>
__device__ __forceinline__ void band_step(T qr, const TW& tw, bool live, int g, unsigned int gm,
                                          const T (&pen)[C], T (&A)[C]) {
  // Lane 0's left neighbour and lane G-1's right neighbour wrap around the
  // group, so no lane needs a select: C G is even and 2w + 1 odd, so C G >
  // 2w + 1 and lane G-1's last cell lies past the band; its +inf penalty
  // (or its huge cost) keeps it huge, which is what lane 0's first cell
  // (d = -w) needs on its left, and makes whatever comes from the right
  // irrelevant to it.
  const T left = __shfl_sync(gm, A[C - 1], (g + G - 1) & (G - 1), G);
  {
    const T d = qr - tw(0);
    const T v = fmin3_(A[1], A[0], left);
    T x = fma(d, d, v);
    if (HI == -2 || HI == 0) x = fmax_(x, pen[0]);
    A[0] = live ? x : A[0];
  }
  const T right = __shfl_sync(gm, A[0], (g + 1) & (G - 1), G);
#pragma unroll
  for (int c = 1; c < C; ++c) {
    const T up = (c + 1 < C) ? A[c + 1 < C ? c + 1 : 0] : right;
    const T d = qr - tw(c);
    const T v = fmin3_(up, A[c], A[c - 1]);
    T x = fma(d, d, v);
    if (HI == -2 || HI == c) x = fmax_(x, pen[c]);
    A[c] = live ? x : A[c];
  }
}

// Banded DTW of q (rows) against t (columns), squared cost.  A group of G
// lanes computes one pair; lane g owns the C consecutive diagonals
// d = -w + gC .. -w + gC + C - 1 and handles row tau - g at step tau.  The
// first G steps (the lanes starting one after another) and the last few read
// q and t from shared memory cell by cell.  In between the steps run in
// blocks of C: a lane needs q[tau - g + k] and t[tau + k + x], k < C,
// x < 2C - 1, over a block (its cells of consecutive steps overlap in t), so
// it loads C values of q and C new values of t per block into registers and
// keeps the C - 1 values of t the next block shares: two shared-memory loads
// and two shuffles per step for C cells.  The blocks run two per loop
// iteration over a ring of 2C registers of t, so no value is copied between
// registers and the loop's pointer and counter updates come once per 2C
// steps.  With ABANDON the group checks about
// every 16 steps whether every lane's latest row, plus the cumulative bound
// of the rows still ahead, exceeds the threshold; it then returns +inf and
// reports the cells it swept.
//
// Band mask: HI = -2 masks every cell past the band.  Otherwise HI is the
// cell, (2w + 1) mod C, at which diagonal w + 1 (the first past the band)
// sits in its lane (-1 when that is the lane's first cell), and only that
// cell is masked: it walls the band off from the diagonals beyond, and the
// lanes whose cells all lie past the band (after that lane, or from it when
// HI = -1) read the q sentinel instead of q, so every cell they compute is at
// least 1e36 with no mask.  Lane 0's left neighbour is then such a cell, the
// cells between the wall and those lanes only see huge values, and every cell
// of the band, the abandoning test and the result are the same as with the
// full mask.
template <typename T, int C, int G, bool ABANDON, int HI = -2>
__device__ T dtw_band(const T* __restrict__ q, const T* __restrict__ t, int m, int w,
                      const float* __restrict__ cbc, int nc, float thr,
                      const unsigned int* bsf2, unsigned int gm, int g,
                      unsigned long long* cells, bool* abandoned) {
  static_assert(C >= 2, "a lane's first cell must not need its right neighbour's");
  const T INF = Pad<T>::inf();
  const int d_lo = -w + g * C;
  T pen[C], A[C];
#pragma unroll
  for (int c = 0; c < C; ++c) {
    pen[c] = (d_lo + c <= w) ? T(0) : INF;
    A[c] = (d_lo + c == 0) ? T(0) : INF;  // virtual row -1: D(-1, 0) = 0
  }
  const T* qg = q - g;         // qg[tau] = q[row]
  const T* tg = t - g + d_lo;  // tg[tau + c] = t[row + d_lo + c]
  const int g_past = (2 * w + 1) / C + (HI == -1 ? 0 : 1);
  const bool past = HI != -2 && g >= g_past;  // reads the sentinel q[-1 - x]
  const T PQ = Pad<T>::q();
  const int g0 = w / C, c0 = w % C;
  const int tau_end = m - 1 + g0;  // lane g0 (cell c0 on d = 0) reaches row m - 1
  *abandoned = false;
  // warm-up: a lane that has not reached row 0 keeps its initial row
  const int warm = G < tau_end + 1 ? G : tau_end + 1;
  int tau = 0;
  for (; tau < warm; ++tau) {
    const T* tp = tg + tau;
    band_step<T, C, G, HI>(past ? PQ : qg[tau], [tp](int c) { return tp[c]; }, tau - g >= 0, g,
                           gm, pen, A);
  }
  // blocks of C steps with q and t in registers, two per iteration: W is a
  // ring of 2C values of t (offset x from the iteration's first step at
  // W[x mod 2C]), so no value moves between registers
  constexpr int kAbEvery = (16 + 2 * C - 1) / (2 * C);  // iterations between abandon checks
  int ab_count = kAbEvery;
  T W[2 * C];
  if (tau + C - 1 <= tau_end) {
#pragma unroll
    for (int x = 0; x < C - 1; ++x) W[x] = tg[tau + x];
  }
  const T* tb = tg + tau + C - 1;  // the blocks' new values of t, and of q,
  const T* qb = past ? q - 2 * C : qg + tau;  // at immediate offsets from two pointers
  const int qstep = past ? 0 : 2 * C;
  while (tau + 2 * C - 1 <= tau_end) {
    T Qv[2 * C];
#pragma unroll
    for (int x = 0; x < C; ++x) W[C - 1 + x] = tb[x];
#pragma unroll
    for (int x = 0; x < 2 * C; ++x) Qv[x] = qb[x];
#pragma unroll
    for (int k = 0; k < C; ++k)
      band_step<T, C, G, HI>(Qv[k], [&W, k](int c) { return W[k + c]; }, true, g, gm, pen, A);
#pragma unroll
    for (int x = 0; x < C; ++x) W[(2 * C - 1 + x) % (2 * C)] = tb[C + x];
#pragma unroll
    for (int k = 0; k < C; ++k)
      band_step<T, C, G, HI>(Qv[C + k], [&W, k](int c) { return W[(C + k + c) % (2 * C)]; }, true,
                             g, gm, pen, A);
    tb += 2 * C;
    qb += qstep;
    tau += 2 * C;
    if (ABANDON && --ab_count == 0 && tau <= tau_end) {
      ab_count = kAbEvery;
      const int r = tau - 1 - g;  // this lane's latest row
      T fm = A[0];
#pragma unroll
      for (int c = 1; c < C; ++c) fm = fmin_(fm, A[c]);
      int idx = r + w + 1;
      idx = idx < 0 ? 0 : (idx + 7) >> 3;
      const float cbv = cbc[idx < nc ? idx : nc];
      thr = fminf(thr, prune_threshold_now(bsf2, m));
      const bool over = (float)fm + cbv > thr;
      if ((__ballot_sync(gm, over) & gm) == gm) {
        // cells swept so far: rows [0, rows_done) of each owned diagonal
        const int rows_done = r + 1 < 0 ? 0 : (r + 1 > m ? m : r + 1);
        unsigned long long cnt = 0;
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const int d = d_lo + c;
          if (d > w) continue;
          const int lo = d < 0 ? -d : 0;
          const int hi = rows_done < m - d ? rows_done : m - d;
          if (hi > lo) cnt += (unsigned long long)(hi - lo);
        }
        *cells = group_sum<G>(cnt, gm);
        *abandoned = true;
        return INF;
      }
    }
  }
  // one more block when it fits (W holds offsets 0 .. C - 2 of tau)
  if (tau + C - 1 <= tau_end) {
    T Qv[C];
#pragma unroll
    for (int x = 0; x < C; ++x) {
      W[C - 1 + x] = tb[x];
      Qv[x] = qb[x];
    }
#pragma unroll
    for (int k = 0; k < C; ++k)
      band_step<T, C, G, HI>(Qv[k], [&W, k](int c) { return W[k + c]; }, true, g, gm, pen, A);
    tau += C;
  }
  // the last steps (fewer than C)
  for (; tau <= tau_end; ++tau) {
    const T* tp = tg + tau;
    band_step<T, C, G, HI>(past ? PQ : qg[tau], [tp](int c) { return tp[c]; }, true, g, gm, pen,
                           A);
  }
  T result = INF;
#pragma unroll
  for (int c = 0; c < C; ++c)
    if (c == c0) result = A[c];
  result = __shfl_sync(gm, result, g0, G);
  *cells = (unsigned long long)m * (2 * w + 1) - (unsigned long long)w * (w + 1);
  return result;
}

// The pair consumer: every group takes pairs from the queue until it is
// drained.  flags bit 0: run the bounds (otherwise DTW only, for seeds).
template <int C, int G, int HI>
__global__ void __launch_bounds__(256) k_pairs(DevSeries S, DevSearch Q, const int2* pairs,
                                                const unsigned int* npairs, int flags,
                                                int group_floats) {
  extern __shared__ __align__(16) unsigned char smraw[];
  float* sm = reinterpret_cast<float*>(smraw);
  __shared__ unsigned long long cnt[kNumCounters];
  const bool bounds = flags & 1;
  const int m = S.m, w = S.w;
  const int gib = threadIdx.x / G, g = threadIdx.x % G;
  const unsigned int gm = group_mask<G>();
  const GroupLayout lay = group_layout(m, w, C, G, bounds);
  float* base = sm + (size_t)gib * group_floats;
  float* q = base + lay.q_off;
  float* t = base + lay.t_off;
  float* cbc = base + lay.cb_off;
  for (int x = threadIdx.x; x < kNumCounters; x += blockDim.x) cnt[x] = 0;
  // sentinels (written once; the interior is rewritten per pair)
  for (int x = g; x < lay.pq; x += G) {
    q[-1 - x] = kPadQ;
    q[m + x] = kPadQ;
  }
  for (int x = g; x < lay.pt; x += G) {
    t[-1 - x] = kPadT;
    t[m + x] = kPadT;
  }
  __syncthreads();
  const unsigned int total = *npairs < Q.queue_cap ? *npairs : Q.queue_cap;
  for (;;) {
    unsigned int idx = 0;
    if (g == 0) idx = atomicAdd(Q.queue_next, 1u);
    idx = __shfl_sync(gm, idx, 0, G);
    if (idx >= total) break;
    const int2 pr = pairs[idx];
    if (pr.x < 0) continue;  // an unused seed slot
    const int64_t i = pr.x, j = pr.y;
    const int sr = Q.qser ? Q.qser[idx] : series_of(S, i);
    unsigned int* bsf2 = Q.bsf2 + sr;
    const double mi = S.mu[i], si = S.isg[i], mj = S.mu[j], sj = S.isg[j];
    float thr = prune_threshold_now(bsf2, S.m);
    for (int x = g; x <= lay.nc + 1; x += G) cbc[x] = 0.0f;
    if (!bounds) {
      for (int k = g; k < m; k += G) {
        q[k] = (float)((S.a[i + k] - mi) * si);
        t[k] = (float)((S.a[j + k] - mj) * sj);
      }
      __syncwarp(gm);
    } else {
      // ---- z-normalised windows and the endpoint bound's two parts ----
      for (int k = g; k < m; k += G) {
        q[k] = (float)((S.a[i + k] - mi) * si);
        t[k] = (float)((S.a[j + k] - mj) * sj);
      }
      __syncwarp(gm);
      float kl = 0.0f, kr = 0.0f;
      if (g == 0) kim_bound<float>(q, t, m, &kl, &kr);
      kl = __shfl_sync(gm, kl, 0, G);
      kr = __shfl_sync(gm, kr, 0, G);
      // ---- cumulative bound for abandoning: LB_Keogh terms of the rows (q)
      // against the envelope of window j, summed over 8-row chunks, then
      // suffix-summed over the chunks.  The group takes G consecutive rows
      // at a time (coalesced envelope loads, conflict-free reads of q); the
      // rows of a chunk sit in min(G, 8) consecutive lanes and are added by
      // shuffles (two passes of four lanes when G = 4). ----
      constexpr int kSeg = G < 8 ? G : 8;
      float hold = 0.0f;
      for (int k0 = 0; k0 < m; k0 += G) {
        const int k = k0 + g;
        float term = 0.0f;
        if (k < m) {
          if (k < kBias || k >= m - kBias) {
            term = k == 0 ? kl : (k == m - kBias ? kr : 0.0f);
          } else {
            const float U = (float)((S.U[j + k] - mj) * sj), L = (float)((S.L[j + k] - mj) * sj);
            const float d = fmaxf(fmaxf(q[k] - U, L - q[k]), 0.0f);
            term = d * d;
          }
        }
#pragma unroll
        for (int o = 1; o < kSeg; o <<= 1) term += __shfl_xor_sync(gm, term, o, G);
        if (kSeg == 8) {
          if ((g & 7) == 0 && k < m) cbc[k >> 3] = term;
        } else if (g == 0) {
          if ((k0 & 4) == 0) {
            hold = term;
            if (k0 + 4 >= m) cbc[k0 >> 3] = hold;
          } else {
            cbc[k0 >> 3] = hold + term;
          }
        }
      }
      __syncwarp(gm);
      // lane g owns chunks [g per, g per + per): it suffix-sums its own from
      // the end, then adds the totals of the lanes above it
      const int per = (lay.nc + G - 1) / G;
      float run = 0.0f;
      for (int u = per - 1; u >= 0; --u) {
        const int x = g * per + u;
        if (x >= lay.nc) continue;
        run += cbc[x];
        cbc[x] = run;
      }
      float above = run;  // inclusive suffix scan of the lane totals
#pragma unroll
      for (int o = 1; o < G; o <<= 1) {
        const float v = __shfl_down_sync(gm, above, o, G);
        if (g + o < G) above += v;
      }
      above -= run;
      for (int u = 0; u < per; ++u) {
        const int x = g * per + u;
        if (x < lay.nc) cbc[x] += above;
      }
      if (g == 0) {
        cbc[lay.nc] = 0.0f;
        cbc[lay.nc + 1] = 0.0f;
      }
      __syncwarp(gm);
      // the whole bound (LB_Keogh of q against j's envelope with the endpoint
      // parts) already exceeds the best-so-far: no DTW
      if (cbc[0] > thr) {
        if (g == 0) atomicAdd(&cnt[kPrunedKeogh], 1ull);
        __syncwarp(gm);
        continue;
      }
    }
    // ---- banded DTW (FP32, early abandoning) ----
    unsigned long long cells = 0;
    bool ab = false;
    const float d2 =
        dtw_band<float, C, G, true, HI>(q, t, m, w, cbc, lay.nc, thr, bsf2, gm, g, &cells, &ab);
    if (g == 0) {
      atomicAdd(&cnt[kDtwCalls], 1ull);
      atomicAdd(&cnt[kDtwCells], cells);
      if (ab) {
        atomicAdd(&cnt[kDtwAbandoned], 1ull);
      } else {
        const float now = prune_threshold_now(bsf2, S.m);
        if (d2 <= now) {
          atomicMin(bsf2, __float_as_uint(d2));
          const unsigned int slot = atomicAdd(Q.cand_count, 1u);
          if (slot < Q.cand_cap) {
            Candidate cd;
            cd.i = (int)i;
            cd.j = (int)j;
            cd.d2 = d2;
            cd.series = sr;
            Q.cand[slot] = cd;
          }
        }
      }
    }
    __syncwarp(gm);
  }
  __syncthreads();
  for (int x = threadIdx.x; x < kNumCounters; x += blockDim.x)
    if (cnt[x]) atomicAdd(&Q.counters[x], cnt[x]);
}

// Exact DTW of a list of pairs (no bounds, no abandoning), FP32 or FP64.
// With `cands`, pairs come from the candidate list and any candidate above
// the final best-so-far (plus slack) is skipped with +inf.
template <typename T, int C, int G>
__global__ void __launch_bounds__(128) k_dtw_list(DevSeries S, const int2* pairs,
                                                   const Candidate* cands,
                                                   const unsigned int* count_ptr, int count,
                                                   const unsigned int* bsf2, double* out,
                                                   int group_elems) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sm = reinterpret_cast<T*>(smraw);
  const int m = S.m, w = S.w;
  const int gib = threadIdx.x / G, g = threadIdx.x % G;
  const unsigned int gm = group_mask<G>();
  const int groups = blockDim.x / G;
  const int pq = G + 1, pt = G * C + G + 2;
  T* q = sm + (size_t)gib * group_elems + pq;
  T* t = q + m + pq + pt;
  for (int x = g; x < pq; x += G) {
    q[-1 - x] = Pad<T>::q();
    q[m + x] = Pad<T>::q();
  }
  for (int x = g; x < pt; x += G) {
    t[-1 - x] = Pad<T>::t();
    t[m + x] = Pad<T>::t();
  }
  __syncwarp(gm);
  int n = count;
  if (count_ptr) {
    const unsigned int c = *count_ptr;
    n = (int)(c < (unsigned)count ? c : (unsigned)count);
  }
  for (int k = blockIdx.x * groups + gib; k < n; k += gridDim.x * groups) {
    int64_t i, j;
    if (cands) {
      const Candidate cd = cands[k];
      i = cd.i;
      j = cd.j;
      if (bsf2 && cd.d2 > prune_threshold(bsf2[cd.series], S.m)) {
        if (g == 0) out[k] = __longlong_as_double(0x7ff0000000000000LL);
        continue;
      }
    } else {
      i = pairs[k].x;
      j = pairs[k].y;
    }
    const double mi = S.mu[i], si = S.isg[i], mj = S.mu[j], sj = S.isg[j];
    for (int x = g; x < m; x += G) {
      q[x] = (T)((S.a[i + x] - mi) * si);
      t[x] = (T)((S.a[j + x] - mj) * sj);
    }
    __syncwarp(gm);
    unsigned long long cells;
    bool ab;
    const T d2 = dtw_band<T, C, G, false>(q, t, m, w, nullptr, 0, 0.0f, nullptr, gm, g, &cells,
                                         &ab);
    if (g == 0) out[k] = (double)d2;
    __syncwarp(gm);
  }
}

// Per series lexicographic minimum (d2, i, j) over the verified candidates,
// in three passes of atomicMin on 64-bit keys (non-negative doubles order
// like their bit patterns): the distance, then i << 32 | j among the
// candidates at that distance, then the FP32 search distance of that pair.
__global__ void k_best_d2(const Candidate* cands, const unsigned int* count_ptr, int cap,
                          const double* d2, unsigned long long* best_d2) {
  const unsigned int c = *count_ptr;
  const int n = (int)(c < (unsigned)cap ? c : (unsigned)cap);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const double v = d2[k];
    if (v < __longlong_as_double(0x7ff0000000000000LL))
      atomicMin(best_d2 + cands[k].series, (unsigned long long)__double_as_longlong(v));
  }
}

__global__ void k_best_ij(const Candidate* cands, const unsigned int* count_ptr, int cap,
                          const double* d2, const unsigned long long* best_d2,
                          unsigned long long* best_ij) {
  const unsigned int c = *count_ptr;
  const int n = (int)(c < (unsigned)cap ? c : (unsigned)cap);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const Candidate cd = cands[k];
    if ((unsigned long long)__double_as_longlong(d2[k]) == best_d2[cd.series])
      atomicMin(best_ij + cd.series,
                ((unsigned long long)(unsigned int)cd.i << 32) | (unsigned int)cd.j);
  }
}

__global__ void k_best_f32(const Candidate* cands, const unsigned int* count_ptr, int cap,
                           const double* d2, const unsigned long long* best_d2,
                           const unsigned long long* best_ij, unsigned int* best_f32) {
  const unsigned int c = *count_ptr;
  const int n = (int)(c < (unsigned)cap ? c : (unsigned)cap);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const Candidate cd = cands[k];
    const unsigned long long ij = ((unsigned long long)(unsigned int)cd.i << 32) | (unsigned int)cd.j;
    if ((unsigned long long)__double_as_longlong(d2[k]) == best_d2[cd.series] &&
        ij == best_ij[cd.series])
      atomicMin(best_f32 + cd.series, __float_as_uint(cd.d2));
  }
}

// ---- dispatch ----

template <int C, int G, int HI>
void run_pairs(const DevSeries& S, const DevSearch& Q, const int2* pairs,
               const unsigned int* npairs, int flags, int num_sms, cudaStream_t st,
               int warps) {
  const bool bounds = flags & 1;
  const GroupLayout lay = group_layout(S.m, S.w, C, G, bounds);
  int threads = warps > 0 ? 32 * warps : 128;
  if (threads < G) threads = G;
  size_t bytes = (size_t)(threads / G) * lay.total * sizeof(float);
  // keep at least two blocks per SM when the series is long
  while (bytes > 100 * 1024 && threads > G && threads > 32) {
    threads /= 2;
    bytes /= 2;
  }
  const int gpb = threads / G;
  bytes = (size_t)gpb * lay.total * sizeof(float);
  cudaFuncSetAttribute(k_pairs<C, G, HI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       200 * 1024);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pairs<C, G, HI>, threads, bytes);
  if (per_sm < 1) per_sm = 1;
  k_pairs<C, G, HI><<<num_sms * per_sm, threads, bytes, st>>>(S, Q, pairs, npairs, flags,
                                                              lay.total);
}

// The one-pair-per-warp layouts with at most 8 cells per lane run with the
// single-cell band mask (HI = (2w + 1) mod C, -1 for 0; an even C only sees
// odd values); the others mask every cell.
template <int C, int G, int K>
bool run_pairs_hi(int hi, const DevSeries& S, const DevSearch& Q, const int2* pairs,
                  const unsigned int* npairs, int flags, int num_sms, cudaStream_t st,
                  int warps) {
  if constexpr (K < C) {
    if constexpr (C % 2 == 1 || K % 2 == 1) {
      if (hi == K) {
        run_pairs<C, G, K == 0 ? -1 : K>(S, Q, pairs, npairs, flags, num_sms, st, warps);
        return true;
      }
    }
    return run_pairs_hi<C, G, K + 1>(hi, S, Q, pairs, npairs, flags, num_sms, st, warps);
  } else {
    return false;
  }
}

template <int C, int G>
void run_pairs_band(const DevSeries& S, const DevSearch& Q, const int2* pairs,
                    const unsigned int* npairs, int flags, int num_sms, cudaStream_t st,
                    int warps) {
  if constexpr (G == 32 && C <= 8) {
    if (run_pairs_hi<C, G, 0>((2 * S.w + 1) % C, S, Q, pairs, npairs, flags, num_sms, st, warps))
      return;
  }
  run_pairs<C, G, -2>(S, Q, pairs, npairs, flags, num_sms, st, warps);
}

template <typename T, int C, int G>
void run_list(const DevSeries& S, const int2* pairs, const Candidate* cands,
              const unsigned int* count_ptr, int count, const unsigned int* bsf2, double* out,
              cudaStream_t st) {
  const int pq = G + 1, pt = G * C + G + 2;
  int elems = 2 * pq + 2 * pt + 2 * S.m;
  elems += sizeof(T) == 4 ? ((17 - elems % 32) + 32) % 32 : ((9 - elems % 16) + 16) % 16;
  int threads = 128;
  size_t bytes = (size_t)(threads / G) * elems * sizeof(T);
  while (bytes > 100 * 1024 && threads > G && threads > 32) {
    threads /= 2;
    bytes /= 2;
  }
  bytes = (size_t)(threads / G) * elems * sizeof(T);
  cudaFuncSetAttribute(k_dtw_list<T, C, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       200 * 1024);
  const int groups = threads / G;
  int blocks = (count + groups - 1) / groups;
  if (blocks < 1) blocks = 1;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_dtw_list<T, C, G><<<blocks, threads, bytes, st>>>(S, pairs, cands, count_ptr, count, bsf2,
                                                      out, elems);
}

#define DTWJ_BAND_CASES(X) \
  X(2, 4) X(3, 4) X(4, 4) X(5, 4) X(6, 4) X(7, 4) X(8, 4) \
  X(2, 8) X(3, 8) X(4, 8) X(5, 8) X(6, 8) X(7, 8) X(8, 8) \
  X(2, 16) X(3, 16) X(4, 16) X(5, 16) X(6, 16) X(7, 16) X(8, 16) \
  X(2, 32) X(3, 32) X(4, 32) X(5, 32) X(6, 32) X(7, 32) X(8, 32) \
  X(10, 32) X(12, 32) X(16, 32)

bool band_supported(int C, int G) {
#define X(c, g) if (C == c && G == g) return true;
  DTWJ_BAND_CASES(X)
#undef X
  return false;
}

}  // namespace

bool band_shape_ok(int w, int C, int G) {
  return w >= 0 && band_supported(C, G) && C * G >= 2 * w + 1;
}

int band_shapes(int w, BandShape* out, int max) {
  // per G, the smallest supported C covering the band and the next one up
  int k = 0;
  const int Gs[4] = {4, 8, 16, 32};
  for (int gi = 0; gi < 4; ++gi) {
    const int G = Gs[gi];
    int found = 0;
    for (int C = 2; C <= 16 && found < 2; ++C) {
      if (!band_shape_ok(w, C, G)) continue;
      if (k < max) out[k] = {C, G};
      ++k;
      ++found;
    }
  }
  return k;
}

bool choose_band(int w, BandShape* out) {
  // One pair per warp (G = 32), with the fewest cells per lane that cover
  // the band.  The groups of a warp that hold different pairs leave the band
  // loop at different steps (early abandoning) and the warp then runs their
  // loops one after the other, which costs more than the lanes' cells
  // outside the band: measured in joins of ECG-like series at w = 3, 13, 52
  // and 103, G = 32 was fastest at every w, up to 4.9x ahead of the layout
  // with the fewest wasted cells (w = 13: (7, 4) 58.9 s against (2, 32)
  // 12.0 s of DTW).
  int C = (2 * w + 1 + 31) / 32;
  if (C < 2) C = 2;
  while (C <= 16 && !band_supported(C, 32)) ++C;
  if (C > 16) return false;
  out->C = C;
  out->G = 32;
  return true;
}

bool choose_band_list(int w, BandShape* out) {
  // Lists of exact DTWs run every pair to the end, so the groups of a warp
  // stay in step: the layout that wastes the fewest cells.
  const int cells = 2 * w + 1;
  const int Gs[4] = {32, 16, 8, 4};
  double best = 2.0;
  BandShape pick = {0, 0};
  for (int gi = 0; gi < 4; ++gi) {
    const int G = Gs[gi];
    int C = (cells + G - 1) / G;
    if (C < 2) C = 2;
    while (C <= 16 && !band_supported(C, G)) ++C;
    if (C > 16) continue;
    const double waste = (double)(G * C - cells) / (double)(G * C);
    if (waste < best - 1e-9) {
      best = waste;
      pick.C = C;
      pick.G = G;
    }
  }
  if (pick.G == 0) return false;
  *out = pick;
  return true;
}

void launch_pairs(const DevSeries& S, const DevSearch& Q, const int2* pairs,
                  const unsigned int* npairs, bool bounds, BandShape band, int num_sms,
                  cudaStream_t st) {
  const int flags = bounds ? 1 : 0;
#define X(c, g) \
  if (band.C == c && band.G == g) {                                               \
    run_pairs_band<c, g>(S, Q, pairs, npairs, flags, num_sms, st, band.warps);     \
    return;                                                                        \
  }
  DTWJ_BAND_CASES(X)
#undef X
}

void launch_verify(const DevSeries& S, const DevSearch& Q, BandShape band, double* out_d2,
                   unsigned long long* best_d2, unsigned long long* best_ij, float* best_f32,
                   cudaStream_t st) {
#define X(c, g)                                                                          \
  if (band.C == c && band.G == g) {                                                      \
    run_list<double, c, g>(S, nullptr, Q.cand, Q.cand_count, (int)Q.cand_cap, Q.bsf2,   \
                           out_d2, st);                                                  \
  }
  DTWJ_BAND_CASES(X)
#undef X
  const int ns = S.nseries;
  cudaMemsetAsync(best_d2, 0xff, (size_t)ns * 8, st);
  cudaMemsetAsync(best_ij, 0xff, (size_t)ns * 8, st);
  cudaMemsetAsync(best_f32, 0xff, (size_t)ns * 4, st);
  const int cap = (int)Q.cand_cap;
  k_best_d2<<<256, 256, 0, st>>>(Q.cand, Q.cand_count, cap, out_d2, best_d2);
  k_best_ij<<<256, 256, 0, st>>>(Q.cand, Q.cand_count, cap, out_d2, best_d2, best_ij);
  k_best_f32<<<256, 256, 0, st>>>(Q.cand, Q.cand_count, cap, out_d2, best_d2, best_ij,
                                  reinterpret_cast<unsigned int*>(best_f32));
}

void launch_pair_dtw(const DevSeries& S, const int2* pairs, int count, bool precise,
                     BandShape band, double* out_d2, cudaStream_t st) {
#define X(c, g)                                                                       \
  if (band.C == c && band.G == g) {                                                   \
    if (precise)                                                                      \
      run_list<double, c, g>(S, pairs, nullptr, nullptr, count, nullptr, out_d2, st); \
    else                                                                              \
      run_list<float, c, g>(S, pairs, nullptr, nullptr, count, nullptr, out_d2, st);  \
  }
  DTWJ_BAND_CASES(X)
#undef X
}

}  // namespace dtwj

// ---- device-resident pair lists (allocation-free entry point) ----

namespace dtwj {
namespace {

// Exact banded DTW distances (sqrt applied) of int64 pair lists that live in
// device memory; a pair with an index outside [0, s) yields NaN.
template <typename T, int C, int G>
__global__ void __launch_bounds__(128) k_dtw_pairs64(DevSeries S, const int64_t* pi,
                                                      const int64_t* pj, int64_t count,
                                                      double* out, int group_elems) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sm = reinterpret_cast<T*>(smraw);
  const int m = S.m, w = S.w;
  const int gib = threadIdx.x / G, g = threadIdx.x % G;
  const unsigned int gm = group_mask<G>();
  const int groups = blockDim.x / G;
  const int pq = G + 1, pt = G * C + G + 2;
  T* q = sm + (size_t)gib * group_elems + pq;
  T* t = q + m + pq + pt;
  for (int x = g; x < pq; x += G) {
    q[-1 - x] = Pad<T>::q();
    q[m + x] = Pad<T>::q();
  }
  for (int x = g; x < pt; x += G) {
    t[-1 - x] = Pad<T>::t();
    t[m + x] = Pad<T>::t();
  }
  __syncwarp(gm);
  for (int64_t k = (int64_t)blockIdx.x * groups + gib; k < count;
       k += (int64_t)gridDim.x * groups) {
    const int64_t i = pi[k], j = pj[k];
    if (i < 0 || j < 0 || i >= S.s || j >= S.s) {
      if (g == 0) out[k] = __longlong_as_double(0x7ff8000000000000LL);
      continue;
    }
    const double mi = S.mu[i], si = S.isg[i], mj = S.mu[j], sj = S.isg[j];
    for (int x = g; x < m; x += G) {
      q[x] = (T)((S.a[i + x] - mi) * si);
      t[x] = (T)((S.a[j + x] - mj) * sj);
    }
    __syncwarp(gm);
    unsigned long long cells;
    bool ab;
    const T d2 = dtw_band<T, C, G, false>(q, t, m, w, nullptr, 0, 0.0f, nullptr, gm, g, &cells,
                                         &ab);
    if (g == 0) out[k] = sqrt((double)d2);
    __syncwarp(gm);
  }
}

template <typename T, int C, int G>
void run_pairs64(const DevSeries& S, const int64_t* pi, const int64_t* pj, int64_t count,
                 double* out, cudaStream_t st) {
  const int pq = G + 1, pt = G * C + G + 2;
  int elems = 2 * pq + 2 * pt + 2 * S.m;
  elems += sizeof(T) == 4 ? ((17 - elems % 32) + 32) % 32 : ((9 - elems % 16) + 16) % 16;
  int threads = 128;
  size_t bytes = (size_t)(threads / G) * elems * sizeof(T);
  while (bytes > 100 * 1024 && threads > G && threads > 32) {
    threads /= 2;
    bytes /= 2;
  }
  bytes = (size_t)(threads / G) * elems * sizeof(T);
  cudaFuncSetAttribute(k_dtw_pairs64<T, C, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       200 * 1024);
  const int groups = threads / G;
  int64_t blocks = (count + groups - 1) / groups;
  if (blocks < 1) blocks = 1;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_dtw_pairs64<T, C, G><<<(unsigned)blocks, threads, bytes, st>>>(S, pi, pj, count, out, elems);
}

}  // namespace

void launch_pair_dtw64(const DevSeries& S, const int64_t* pi, const int64_t* pj, int64_t count,
                       bool precise, BandShape band, double* out, cudaStream_t st) {
#define X(c, g)                                                 \
  if (band.C == c && band.G == g) {                             \
    if (precise)                                                \
      run_pairs64<double, c, g>(S, pi, pj, count, out, st);     \
    else                                                        \
      run_pairs64<float, c, g>(S, pi, pj, count, out, st);      \
  }
  DTWJ_BAND_CASES(X)
#undef X
}

}  // namespace dtwj
