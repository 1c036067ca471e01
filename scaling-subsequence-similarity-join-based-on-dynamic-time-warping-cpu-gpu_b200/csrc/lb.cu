// Diagonal lower-bound sweep: the first stage of the reference's GLOBAL_DIAG
// kernel (GPU_version1/lib/GLOBAL_DIAG.cu:29-73), diag_fast
// (GPU_version1/lib/diag_fast.cu:13-90, CPU_version1/diag_fast.cpp:12-88),
// for a tile of 128 lags x up to 4096 rows.
//
// For pair (i, j), j = i + L, and the raw-series envelope U, L (radius w)
// normalised by window r, the reference bounds the z-normalised DTW by
//   lb = (sqrt(2 S - DUL2_r) - DUL_r) / 2,   S = 2m + N_r - 2 X,
//   X  = sum_k z_q[k] (nU_r[k] + nL_r[k])
// in both directions (env = i, query = j and env = j, query = i), updating X
// along the diagonal in O(1).  lb > bsf  <=>  X < (A_r - (2 bsf + DUL_r)^2)/4
// with A_r = 4m + 2N_r - DUL2_r, and X = C / (sig_q sig_r) with the centered
// FP64 cross covariance C(r, q) = sum_k (a[q+k] - mu_q) (E[r+k] - nu_r),
// E = U + L.  A direction therefore prunes iff  G_r sig_q - C > 0  with
// G_r = sig_r (A_r - (2 bsf + DUL_r)^2) / 4: two FP64 recurrences (4 DFMA)
// and two DFMA tests per pair, no division and no square root.
//
// One thread owns one lag and walks the tile's rows; the block's 128 lags
// share each row, so row operands are broadcast and column operands are
// consecutive.  Survivors of one lag come in long runs of consecutive rows
// (the bound moves slowly along a diagonal), so a thread emits
// (i0, j0, length) per run, capped at kRunMax rows, with one atomic per warp
// and row; the run filter (runs.cu) then reuses each run's data across its
// pairs.
#include "dtwj_dev.cuh"

namespace dtwj {
namespace {

__global__ void __launch_bounds__(kTileLags) k_lb(DevSeries S, DevSearch Q, const Tile* tiles,
                                                  bool enumerate_all) {
  const Tile T = tiles[blockIdx.x];
  const int64_t L = (int64_t)T.L0 + threadIdx.x;
  const int64_t s = S.s;
  const int m = S.m;
  const int64_t i_begin = T.i0;
  const int64_t i_end = (int64_t)T.i0 + T.rows < s - L ? (int64_t)T.i0 + T.rows : s - L;
  const bool any = L < s && i_begin < i_end;
  const int lane = threadIdx.x & 31;

  const float b2 = prune_threshold_now(Q.bsf2, S.m);
  const double twoB = 2.0 * sqrt((double)b2);

  double Cf = 0.0, Cr = 0.0;
  if (any) {
    const int64_t i = i_begin, j = i_begin + L;
    const double mi = S.mu[i], mj = S.mu[j], ni = S.nu[i], nj = S.nu[j];
    for (int k = 0; k < m; ++k) {
      Cf = fma(S.a[j + k] - mj, S.E[i + k] - ni, Cf);
      Cr = fma(S.a[i + k] - mi, S.E[j + k] - nj, Cr);
    }
  }
  unsigned long long npairs = 0, nfast = 0;
  int64_t run_start = -1;
  int run_len = 0;
  for (int x = 0; x <= T.rows; ++x) {
    const int64_t i = i_begin + x;
    bool survive = false;
    if (x < T.rows && any && i < i_end) {
      const int64_t j = i + L;
      if (x > 0) {
        Cf = fma(S.dfa[j - 1], S.dgE[i - 1], Cf);
        Cf = fma(S.dfE[i - 1], S.dga[j - 1], Cf);
        Cr = fma(S.dfa[i - 1], S.dgE[j - 1], Cr);
        Cr = fma(S.dfE[j - 1], S.dga[i - 1], Cr);
      }
      const double ti = twoB + S.DUL[i];
      const double Gi = S.qsig[i] * fma(-ti, ti, S.A[i]);
      const double tj = twoB + S.DUL[j];
      const double Gj = S.qsig[j] * fma(-tj, tj, S.A[j]);
      const bool prune = !enumerate_all &&
                         (fma(Gi, S.sig[j], -Cf) > 0.0 || fma(Gj, S.sig[i], -Cr) > 0.0);
      ++npairs;
      if (prune) ++nfast;
      else survive = true;
    }
    // run bookkeeping: close a run when it breaks, hits kRunMax or the tile ends
    bool emit = false;
    int64_t e_start = 0;
    int e_len = 0;
    if (survive) {
      if (run_start < 0) {
        run_start = i;
        run_len = 0;
      }
      ++run_len;
      if (run_len == kRunMax) {
        emit = true;
        e_start = run_start;
        e_len = run_len;
        run_start = -1;
      }
    } else if (run_start >= 0) {
      emit = true;
      e_start = run_start;
      e_len = run_len;
      run_start = -1;
    }
    const unsigned int ballot = __ballot_sync(0xffffffffu, emit);
    if (ballot) {
      const int leader = __ffs(ballot) - 1;
      unsigned int base = 0;
      if (lane == leader) base = atomicAdd(Q.run_count, (unsigned int)__popc(ballot));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (emit) {
        const unsigned int slot = base + __popc(ballot & ((1u << lane) - 1u));
        if (slot < Q.run_cap) Q.runs[slot] = make_int4((int)e_start, (int)(e_start + L), e_len, 0);
        else atomicOr(S.status, 2);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    npairs += __shfl_xor_sync(0xffffffffu, npairs, o);
    nfast += __shfl_xor_sync(0xffffffffu, nfast, o);
  }
  if (lane == 0 && npairs) {
    atomicAdd(&Q.counters[kPairs], npairs);
    atomicAdd(&Q.counters[kPrunedFast], nfast);
  }
}

}  // namespace

void launch_lb(const DevSeries& S, const DevSearch& Q, const Tile* tiles, int tile_begin,
               int tile_end, bool enumerate_all, cudaStream_t st) {
  if (tile_end <= tile_begin) return;
  k_lb<<<tile_end - tile_begin, kTileLags, 0, st>>>(S, Q, tiles + tile_begin, enumerate_all);
}

}  // namespace dtwj
