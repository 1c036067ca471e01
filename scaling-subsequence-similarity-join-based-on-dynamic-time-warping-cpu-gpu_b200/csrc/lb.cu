// Diagonal lower-bound sweep: the reference's GLOBAL_DIAG kernel
// (GPU_version1/lib/GLOBAL_DIAG.cu:29-73), i.e. diag_fast
// (GPU_version1/lib/diag_fast.cu:13-90, CPU_version1/diag_fast.cpp:12-88)
// followed by diag_mask_global and its endpoint bound
// (GPU_version1/lib/diag_mask_global.cu:12-230,
// CPU_version1/diag_mask_global.cpp:11-313), for a tile of 128 lags x up to
// 4096 rows.
//
// Fast bound.  For pair (i, j), j = i + L, and the raw-series envelope U, L
// (radius w) normalised by window r, the reference bounds the z-normalised
// DTW by
//   lb = (sqrt(2 S - DUL2_r) - DUL_r) / 2,   S = 2m + N_r - 2 X,
//   X  = sum_k z_q[k] (nU_r[k] + nL_r[k])
// in both directions (env = i, query = j and env = j, query = i).
// lb > bsf  <=>  X < (A_r - (2 bsf + DUL_r)^2)/4  with A_r = 4m + 2N_r - DUL2_r,
// and X = C / (sig_q sig_r) with the centered FP64 cross covariance
// C(r, q) = sum_k (a[q+k] - mu_q) (E[r+k] - nu_r), E = U + L.  A direction
// therefore prunes iff  G_r sig_q - C > 0,  G_r = sig_r (A_r - (2 bsf + DUL_r)^2)/4:
// two FP64 recurrences (4 DFMA) and two DFMA tests per pair, no division and
// no square root.
//
// Masked bound (MASKED).  The same construction restricted to the positions
// T = [3, m-4] where the global mask M is 1, with the raw FP64 running sums
//   F1 = sum_T M_i a_j,  F2 = sum_T M_i a_j^2,  F3 = sum_T M_i E_i a_j
// (and R1..R3 with i and j swapped), updated by one leaving and one entering
// term per row as in diag_mask_global.cpp:187-195.  It is evaluated only for
// pairs the fast bound keeps.
//
// Endpoint bound.  Pairs still alive get the LB_KIM-style bound of their
// first and last three path layers, plus the masked bound squared.
//
// One thread owns one lag and walks the tile's rows; the block's 128 lags
// share each row, so row operands are broadcast and column operands are
// consecutive.  Survivors go to the chunk's queue with one atomic per warp
// and row.
#include "dtwj_dev.cuh"

namespace dtwj {
namespace {

// The six endpoint values of a z-normalised window.
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

// Masked bound for env = r, query = c from the raw sums F1..F3.
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

template <bool MASKED>
__global__ void __launch_bounds__(kTileLags) k_lb(DevSeries S, DevSearch Q, const Tile* tiles,
                                                  bool enumerate_all) {
  const Tile T = tiles[blockIdx.x];
  const int64_t L = (int64_t)T.L0 + threadIdx.x;
  const int64_t s = S.s;
  const int m = S.m;
  const int lo = kBias, hi = m - 1 - kBias;
  const int64_t i_begin = T.i0;
  const int64_t i_end = (int64_t)T.i0 + T.rows < s - L ? (int64_t)T.i0 + T.rows : s - L;
  const bool any = L < s && i_begin < i_end;
  const int lane = threadIdx.x & 31;

  const float b2 = __uint_as_float(*(volatile unsigned int*)Q.bsf2) * (1.0f + kSlack);
  const double B = sqrt((double)b2);
  const double twoB = 2.0 * B;

  double Cf = 0.0, Cr = 0.0;
  double F1 = 0, F2 = 0, F3 = 0, R1 = 0, R2 = 0, R3 = 0;
  if (any) {
    const int64_t i = i_begin, j = i_begin + L;
    const double mi = S.mu[i], mj = S.mu[j], ni = S.nu[i], nj = S.nu[j];
    for (int k = 0; k < m; ++k) {
      const double ai = S.a[i + k], aj = S.a[j + k], Ei = S.E[i + k], Ej = S.E[j + k];
      Cf = fma(aj - mj, Ei - ni, Cf);
      Cr = fma(ai - mi, Ej - nj, Cr);
      if (MASKED && k >= lo && k <= hi) {
        const double Mi = S.mask[i + k], Mj = S.mask[j + k];
        F1 = fma(Mi, aj, F1);
        F2 = fma(Mi * aj, aj, F2);
        F3 = fma(Mi * Ei, aj, F3);
        R1 = fma(Mj, ai, R1);
        R2 = fma(Mj * ai, ai, R2);
        R3 = fma(Mj * Ej, ai, R3);
      }
    }
  }
  unsigned long long npairs = 0, nfast = 0, nmasked = 0, nkim = 0;
  for (int x = 0; x < T.rows; ++x) {
    const int64_t i = i_begin + x;
    bool survive = false;
    int64_t j = 0;
    if (any && i < i_end) {
      j = i + L;
      if (x > 0) {
        Cf = fma(S.dfa[j - 1], S.dgE[i - 1], Cf);
        Cf = fma(S.dfE[i - 1], S.dga[j - 1], Cf);
        Cr = fma(S.dfa[i - 1], S.dgE[j - 1], Cr);
        Cr = fma(S.dfE[j - 1], S.dga[i - 1], Cr);
        if (MASKED) {
          // window start leaves (k = lo of the previous row), end enters
          const int64_t io = i - 1 + lo, jo = j - 1 + lo, in = i + hi, jn = j + hi;
          const double Mio = S.mask[io], Min = S.mask[in];
          const double Mjo = S.mask[jo], Mjn = S.mask[jn];
          const double ajo = S.a[jo], ajn = S.a[jn], aio = S.a[io], ain = S.a[in];
          F1 += Min * ajn - Mio * ajo;
          F2 += Min * ajn * ajn - Mio * ajo * ajo;
          F3 += Min * S.E[in] * ajn - Mio * S.E[io] * ajo;
          R1 += Mjn * ain - Mjo * aio;
          R2 += Mjn * ain * ain - Mjo * aio * aio;
          R3 += Mjn * S.E[jn] * ain - Mjo * S.E[jo] * aio;
        }
      }
      const double ti = twoB + S.DUL[i];
      const double Gi = S.qsig[i] * fma(-ti, ti, S.A[i]);
      const double tj = twoB + S.DUL[j];
      const double Gj = S.qsig[j] * fma(-tj, tj, S.A[j]);
      const bool prune = !enumerate_all &&
                         (fma(Gi, S.sig[j], -Cf) > 0.0 || fma(Gj, S.sig[i], -Cr) > 0.0);
      ++npairs;
      if (prune) {
        ++nfast;
      } else if (enumerate_all) {
        survive = true;
      } else {
        // rare path: masked bound, then the endpoint bound
        double lbm = 0.0;
        bool dead = false;
        if (MASKED) {
          lbm = fmax(masked_lb(S, i, j, F1, F2, F3), masked_lb(S, j, i, R1, R2, R3));
          if (lbm > B) {
            ++nmasked;
            dead = true;
          }
        }
        if (!dead) {
          const ZEnds zi = z_ends(S, i), zj = z_ends(S, j);
          double kl, kr;
          kim_bound<double>(zi, zj, m, &kl, &kr);
          if (kl + kr + lbm * lbm > (double)b2) ++nkim;
          else survive = true;
        }
      }
    }
    const unsigned int ballot = __ballot_sync(0xffffffffu, survive);
    if (ballot) {
      const int leader = __ffs(ballot) - 1;
      unsigned int base = 0;
      if (lane == leader) base = atomicAdd(Q.queue_count, (unsigned int)__popc(ballot));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (survive) {
        const unsigned int slot = base + __popc(ballot & ((1u << lane) - 1u));
        if (slot < Q.queue_cap) Q.queue[slot] = make_int2((int)i, (int)j);
        else atomicOr(S.status, 2);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    npairs += __shfl_xor_sync(0xffffffffu, npairs, o);
    nfast += __shfl_xor_sync(0xffffffffu, nfast, o);
    nmasked += __shfl_xor_sync(0xffffffffu, nmasked, o);
    nkim += __shfl_xor_sync(0xffffffffu, nkim, o);
  }
  if (lane == 0 && npairs) {
    atomicAdd(&Q.counters[kPairs], npairs);
    atomicAdd(&Q.counters[kPrunedFast], nfast);
    if (nmasked) atomicAdd(&Q.counters[kPrunedMasked], nmasked);
    if (nkim) atomicAdd(&Q.counters[kPrunedKim], nkim);
  }
}

}  // namespace

void launch_lb(const DevSeries& S, const DevSearch& Q, const Tile* tiles, int tile_begin,
               int tile_end, bool masked, bool enumerate_all, cudaStream_t st) {
  if (tile_end <= tile_begin) return;
  if (masked && !enumerate_all)
    k_lb<true><<<tile_end - tile_begin, kTileLags, 0, st>>>(S, Q, tiles + tile_begin, false);
  else
    k_lb<false><<<tile_end - tile_begin, kTileLags, 0, st>>>(S, Q, tiles + tile_begin,
                                                             enumerate_all);
}

}  // namespace dtwj
