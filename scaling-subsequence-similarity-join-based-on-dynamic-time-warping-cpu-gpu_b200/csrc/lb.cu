// Diagonal lower-bound sweep: the first stage of the reference's GLOBAL_DIAG
// kernel (GPU_version1/lib/GLOBAL_DIAG.cu:29-73), diag_fast
// (GPU_version1/lib/diag_fast.cu:13-90, CPU_version1/diag_fast.cpp:12-88).
//
// For pair (i, j), j = i + L, and the raw-series envelope U, L (radius w)
// normalised by window r, the reference bounds the z-normalised DTW by
//   lb = (sqrt(2 S - DUL2_r) - DUL_r) / 2,   S = 2m + N_r - 2 X,
//   X  = sum_k z_q[k] (nU_r[k] + nL_r[k])
// in both directions (env = i, query = j and env = j, query = i), updating X
// along the diagonal in O(1).  lb > bsf  <=>  X < (A_r - (2 bsf + DUL_r)^2)/4
// with A_r = 4m + 2N_r - DUL2_r, and X = C / (sig_q sig_r) with the centered
// FP64 cross covariance C(r, q) = sum_k (a[q+k] - mu_q) (E[r+k] - nu_r),
// E = U + L, which moves along a diagonal as
//   C(r, q) = C(r-1, q-1) + df_a[q-1] dg_E[r-1] + df_E[r-1] dg_a[q-1].
// A direction therefore prunes iff  G_r sig_q - C > 0  with
// G_r = sig_r (A_r - (2 bsf + DUL_r)^2) / 4: two FP64 recurrences (4 DFMA)
// and two DFMA tests per pair, no division and no square root.
//
// Tile: 128 threads x kLbPerThread consecutive lags x kLbRows rows.  Rows are
// processed in stages of kStage rows: the block stages the column operands
// (df_a, dg_a, df_E, dg_E of index j-1, sig and G of j) for the stage's
// kLbLags + kStage columns and the row operands for its rows in shared
// memory, with G computed from the current best-so-far while staging.  Each
// thread keeps a sliding window of its kLbPerThread columns in registers, so
// every shared load feeds kLbPerThread pairs (kLbPerThread is odd, so the
// strided FP64 reads are bank-conflict free).  Survivors are written as one
// bit per pair, 32 rows per word, [tile][word][lag]: the kLbLags words of one
// row word are contiguous, so a warp's seven stores of a word index fill the
// same seven lines.  The block-mean filter (paa.cu) reads a word of 32
// consecutive lags per warp; the run filter (runs.cu) reads one lag's words.
#include "dtwj_dev.cuh"

namespace dtwj {
namespace {

constexpr int kStage = kLbPerThread * 32;          // rows per shared-memory stage
constexpr int kCols = kLbLags + kStage;            // staged columns per stage
static_assert(kLbRows % kStage == 0, "tile rows must be whole stages");

struct LbShared {
  double p1[kCols], p2[kCols], p3[kCols], p4[kCols], sg[kCols], g[kCols];
  double r1[kStage], r2[kStage], r3[kStage], r4[kStage], rs[kStage], rg[kStage];
};

// G of window x; flat windows (A = 1e300) get +1e300 whatever the
// best-so-far, so every pair with a flat window is pruned, also while the
// best-so-far is still +inf or with the bounds off.
__device__ __forceinline__ double g_of(const DevSeries& S, int64_t x, double twoB) {
  const double A = S.A[x];
  if (A >= 1e299) return 1e300;
  const double t = twoB + S.DUL[x];
  return S.qsig[x] * fma(-t, t, A);
}

// One tile of the sweep (the body of the persistent k_lb below).
__device__ __forceinline__ void lb_tile(const DevSeries& S, const DevSearch& Q, const Tile& T,
                                        unsigned int* out, bool enumerate_all, LbShared& sh,
                                        unsigned int& npairs, unsigned int& nfast) {
  const int64_t s = T.send;  // windows of the tile's series end here
  const int m = S.m;
  const int t = threadIdx.x;
  const int64_t L0 = T.L0, i0 = T.i0;
  const int64_t Lt = L0 + (int64_t)t * kLbPerThread;  // this thread's first lag

  const float b2 =
      enumerate_all ? __int_as_float(0x7f800000) : prune_threshold_now(Q.bsf2 + T.series, m);
  const double twoB = 2.0 * sqrt((double)b2);

  // ---- exact anchors at the tile's first row ----
  double Cf[kLbPerThread], Cr[kLbPerThread];
#pragma unroll
  for (int l = 0; l < kLbPerThread; ++l) Cf[l] = Cr[l] = 0.0;
  {
    double mj[kLbPerThread], nj[kLbPerThread];
#pragma unroll
    for (int l = 0; l < kLbPerThread; ++l) {
      const int64_t j = i0 + Lt + l < s ? i0 + Lt + l : s - 1;
      mj[l] = S.mu[j];
      nj[l] = S.nu[j];
    }
    const double mi = S.mu[i0], ni = S.nu[i0];
    const int64_t jb = i0 + Lt;
    // sliding windows of a and E over the thread's columns
    double wa[kLbPerThread], we[kLbPerThread];
#pragma unroll
    for (int l = 0; l < kLbPerThread; ++l) {
      const int64_t x = jb + l < S.n ? jb + l : S.n - 1;
      wa[l] = S.a[x];
      we[l] = S.E[x];
    }
    for (int k = 0; k < m; ++k) {
      const double ei = S.E[i0 + k] - ni, ai = S.a[i0 + k] - mi;
#pragma unroll
      for (int l = 0; l < kLbPerThread; ++l) {
        Cf[l] = fma(wa[l] - mj[l], ei, Cf[l]);
        Cr[l] = fma(ai, we[l] - nj[l], Cr[l]);
      }
#pragma unroll
      for (int l = 0; l < kLbPerThread - 1; ++l) {
        wa[l] = wa[l + 1];
        we[l] = we[l + 1];
      }
      const int64_t x = jb + kLbPerThread + k < S.n ? jb + kLbPerThread + k : S.n - 1;
      wa[kLbPerThread - 1] = S.a[x];
      we[kLbPerThread - 1] = S.E[x];
    }
  }

  double w1[kLbPerThread], w2[kLbPerThread], w3[kLbPerThread], w4[kLbPerThread];
  double ws[kLbPerThread], wg[kLbPerThread];
  for (int st = 0; st < T.rows; st += kStage) {
    const int64_t r0 = i0 + st;         // first row of the stage
    const int64_t c0 = r0 + L0;         // first staged column
    __syncthreads();
    for (int x = t; x < kCols; x += kLbThreads) {
      const int64_t j = c0 + x;
      const bool in = j >= 0 && j < s, up = j >= 1 && j < s;  // update terms exist for j >= 1
      sh.p1[x] = up ? S.dfa[j - 1] : 0.0;
      sh.p2[x] = up ? S.dga[j - 1] : 0.0;
      sh.p3[x] = up ? S.dfE[j - 1] : 0.0;
      sh.p4[x] = up ? S.dgE[j - 1] : 0.0;
      sh.sg[x] = in ? S.sig[j] : 1.0;
      sh.g[x] = in ? g_of(S, j, twoB) : 1e300;
    }
    for (int x = t; x < kStage; x += kLbThreads) {
      const int64_t i = r0 + x;
      const bool in = i >= 0 && i < s, up = i >= 1 && i < s;
      sh.r1[x] = up ? S.dfa[i - 1] : 0.0;
      sh.r2[x] = up ? S.dga[i - 1] : 0.0;
      sh.r3[x] = up ? S.dfE[i - 1] : 0.0;
      sh.r4[x] = up ? S.dgE[i - 1] : 0.0;
      sh.rs[x] = in ? S.sig[i] : 1.0;
      sh.rg[x] = in ? g_of(S, i, twoB) : 1e300;
    }
    __syncthreads();
    // windows: column of lag l at stage row 0 is stage column t*K + l
    const int cb = t * kLbPerThread;
#pragma unroll
    for (int l = 0; l < kLbPerThread; ++l) {
      w1[l] = sh.p1[cb + l];
      w2[l] = sh.p2[cb + l];
      w3[l] = sh.p3[cb + l];
      w4[l] = sh.p4[cb + l];
      ws[l] = sh.sg[cb + l];
      wg[l] = sh.g[cb + l];
    }
    // survivor bits enter at the bottom of each lag's word (word = 2 word +
    // bit), so after 32 rows row r of the word sits at bit 31 - r; the word is
    // reversed and masked to the pairs that exist when it is stored
    unsigned int word[kLbPerThread];
#pragma unroll
    for (int l = 0; l < kLbPerThread; ++l) word[l] = 0u;
    for (int qq = 0; qq < kStage / kLbPerThread; ++qq) {
#pragma unroll
      for (int u = 0; u < kLbPerThread; ++u) {
        const int r = qq * kLbPerThread + u;   // stage row; r % K == u
        const bool first = (st == 0 && r == 0);
        const double q1 = sh.r1[r], q2 = sh.r2[r], q3 = sh.r3[r], q4 = sh.r4[r];
        const double qs = sh.rs[r], qg = sh.rg[r];
#pragma unroll
        for (int l = 0; l < kLbPerThread; ++l) {
          const int sl = (u + l) % kLbPerThread;  // ring slot of lag l at this row
          if (!first) {
            Cf[l] = fma(w1[sl], q4, Cf[l]);
            Cf[l] = fma(q3, w2[sl], Cf[l]);
            Cr[l] = fma(q1, w4[sl], Cr[l]);
            Cr[l] = fma(w3[sl], q2, Cr[l]);
          }
          // a direction prunes when G sigma - C > 0; the sign of the high word
          // decides (hi > 0: positive; zero, denormals and negatives survive,
          // which only keeps more pairs).  With the bounds off (best-so-far
          // +inf) only flat windows prune.
          const int hf = __double2hiint(fma(qg, ws[sl], -Cf[l]));
          const int hr = __double2hiint(fma(wg[sl], qs, -Cr[l]));
          word[l] = word[l] * 2u + (max(hf, hr) <= 0 ? 1u : 0u);
        }
        // the column lag K-1 needs at the next row replaces the one lag 0 used
        const int nx = cb + r + kLbPerThread;
        w1[u] = sh.p1[nx];
        w2[u] = sh.p2[nx];
        w3[u] = sh.p3[nx];
        w4[u] = sh.p4[nx];
        ws[u] = sh.sg[nx];
        wg[u] = sh.g[nx];
        if ((r & 31) == 31) {
          const int wi = (st + r) >> 5;
          // pairs that exist: tile row x < rows and i0 + x + Lt + l < s
          const int64_t room = s - i0 - Lt - (int64_t)wi * 32;
          const int64_t rows_left = (int64_t)T.rows - (int64_t)wi * 32;
#pragma unroll
          for (int l = 0; l < kLbPerThread; ++l) {
            const int64_t lim = room - l < rows_left ? room - l : rows_left;
            const unsigned int vm =
                lim >= 32 ? 0xffffffffu : (lim <= 0 ? 0u : (1u << (int)lim) - 1u);
            const unsigned int wv = __brev(word[l]) & vm;
            npairs += __popc(vm);
            nfast += __popc(vm & ~wv);
            out[(size_t)wi * kLbLags + t * kLbPerThread + l] = wv;
            word[l] = 0u;
          }
        }
      }
    }
  }
  // words past the tile's last stage (short tiles) are zero, never stale
  for (int wi = ((T.rows + kStage - 1) / kStage) * (kStage / 32); wi < kLbWords; ++wi) {
#pragma unroll
    for (int l = 0; l < kLbPerThread; ++l) out[(size_t)wi * kLbLags + t * kLbPerThread + l] = 0u;
  }
}

// Persistent sweep: each CTA takes tiles from the work counter *next until
// the chunk is exhausted; tile k of the chunk writes its bits to slot k.
__global__ void __launch_bounds__(kLbThreads, kLbCtasPerSm) k_lb(DevSeries S, DevSearch Q,
                                                      const Tile* tiles, int ntiles,
                                                      unsigned int* bits, bool enumerate_all,
                                                      unsigned int* next) {
  extern __shared__ __align__(16) unsigned char smraw[];
  LbShared& sh = *reinterpret_cast<LbShared*>(smraw);
  __shared__ unsigned int tile_idx;
  const int lane = threadIdx.x & 31;
  unsigned int npairs = 0, nfast = 0;
  for (;;) {
    __syncthreads();  // every thread has read tile_idx and left the previous tile's staging
    if (threadIdx.x == 0) tile_idx = atomicAdd(next, 1u);
    __syncthreads();
    const unsigned int k = tile_idx;
    if (k >= (unsigned int)ntiles) break;
    const Tile T = tiles[k];
    lb_tile(S, Q, T, bits + (size_t)k * kLbLags * kLbWords, enumerate_all, sh, npairs, nfast);
  }
  unsigned long long np = npairs, nf = nfast;
  for (int o = 16; o > 0; o >>= 1) {
    np += __shfl_xor_sync(0xffffffffu, np, o);
    nf += __shfl_xor_sync(0xffffffffu, nf, o);
  }
  if (lane == 0 && np) {
    atomicAdd(&Q.counters[kPairs], np);
    atomicAdd(&Q.counters[kPrunedFast], nf);
  }
}

}  // namespace

size_t lb_smem_bytes() { return sizeof(LbShared); }

void launch_lb(const DevSeries& S, const DevSearch& Q, const Tile* tiles, int tile_begin,
               int tile_end, unsigned int* bits, bool enumerate_all, unsigned int* next,
               int num_sms, cudaStream_t st) {
  if (tile_end <= tile_begin) return;
  cudaFuncSetAttribute(k_lb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(LbShared));
  const int ntiles = tile_end - tile_begin;
  const int resident = kLbCtasPerSm * num_sms;  // launch bounds, 64.5 KB shared each
  k_lb<<<ntiles < resident ? ntiles : resident, kLbThreads, sizeof(LbShared), st>>>(
      S, Q, tiles + tile_begin, ntiles, bits, enumerate_all, next);
}

}  // namespace dtwj
