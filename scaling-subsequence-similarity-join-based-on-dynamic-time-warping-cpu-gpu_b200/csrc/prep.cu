// Per-series preparation kernels: window statistics, envelopes, the row
// constants of the diagonal bounds, the centered update terms of the FP64
// diagonal recurrences, and the global CDF mask.
//
// Reference counterparts (all host loops there):
//   stats       mvmean                    CPU_version1/allmatrixop/movmean.cpp:9-33
//               (GPU_version1/allmatrixop/movmean.cu:9-33 runs it in FP32)
//   envelope    lower_upper_lemire(a, ...) GPU_version1/src/new_dtw_motifGUI_malloc.cu:122-124
//   row terms   DUL2_fast / DUL_fast / norm_U_plus_norm_L_trans
//                                         GPU_version1/src/new_dtw_motifGUI_malloc.cu:150-176
//   mask        compute_shared_data_global + compute_MASK_global
//                                         GPU_version1/src/compute_shared_data_global.cu:48-80,
//                                         GPU_version1/src/compute_MASK_global.cu:92-170
#include "dtwj_dev.cuh"

#include <cfloat>
#include <cmath>

namespace dtwj {
namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(int64_t n, int threads = kThreads) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > (int64_t)1 << 30) b = (int64_t)1 << 30;
  return (unsigned)b;
}

__global__ void k_check_finite(const double* a, int64_t n, int* status) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    if (!isfinite(a[p])) atomicOr(status, 1);
  }
}

// Series of every sample of a batch: the r with sbeg[r] <= p < sbeg[r + 1].
__global__ void k_series_ids(const int64_t* sbeg, int nseries, int* sid, int64_t n) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = nseries - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (sbeg[mid] <= p) lo = mid;
      else hi = mid - 1;
    }
    sid[p] = lo;
  }
}

// Exact two-pass mean and population deviation of each window, FP64.
__global__ void k_stats(DevSeries S) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= S.s) return;
  const double* x = S.a + i;
  double sum = 0.0;
  for (int k = 0; k < S.m; ++k) sum += x[k];
  const double mean = sum / S.m;
  double ss = 0.0;
  for (int k = 0; k < S.m; ++k) {
    double d = x[k] - mean;
    ss = fma(d, d, ss);
  }
  const double sd = sqrt(ss / S.m);
  const double rms = sqrt(mean * mean + sd * sd);
  const bool flat = !(sd > 1e-12 * rms) || sd == 0.0;
  S.mu[i] = mean;
  S.sig[i] = flat ? 1.0 : sd;
  S.isg[i] = flat ? 0.0 : 1.0 / sd;
  S.flat[i] = flat ? 1 : 0;
}

// Clipped Sakoe-Chiba envelope of the raw series: U[p] = max a[p-w .. p+w],
// clipped to the sample's own series in a batch.
__global__ void k_envelope(DevSeries S) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= S.n) return;
  int64_t b = 0, e = S.n;
  if (S.sid) {
    const int r = S.sid[p];
    b = S.sbeg[r];
    e = S.sbeg[r + 1];
  }
  const int64_t lo = p - S.w > b ? p - S.w : b;
  const int64_t hi = p + S.w < e - 1 ? p + S.w : e - 1;
  double u = S.a[lo], l = S.a[lo];
  for (int64_t q = lo + 1; q <= hi; ++q) {
    double v = S.a[q];
    u = fmax(u, v);
    l = fmin(l, v);
  }
  S.U[p] = u;
  S.L[p] = l;
  S.E[p] = u + l;
}

// Row constants.  With nU = (U - mu)/sig and nL likewise over the window:
//   N    = sum nU^2 + nL^2
//   DUL2 = sum (nU - nL)^2,   A = 4m + 2N - DUL2
// so that the diagonal bound lb = (sqrt(2S - DUL2) - DUL)/2 with
// S = 2m + N - 2X (diag_fast.cpp:35) prunes iff X < (A - (2 bsf + DUL)^2)/4.
// Masked terms over T = [kBias, m-1-kBias] (diag_mask_global.cpp:117-128):
//   MN = sum_T M (nU^2 + nL^2), MDUL2 = sum_m M (nU - nL)^2.
__global__ void k_rowterms(DevSeries S, bool masked) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= S.s) return;
  const double mu = S.mu[i], isg = S.isg[i];
  double N = 0, D2 = 0, sE = 0, MN = 0, MD2 = 0, SM = 0, SME = 0;
  const int m = S.m;
  for (int k = 0; k < m; ++k) {
    const double U = S.U[i + k], L = S.L[i + k];
    sE += U + L;
    const double u = (U - mu) * isg, l = (L - mu) * isg;
    N = fma(u, u, fma(l, l, N));
    D2 = fma(u - l, u - l, D2);
    if (masked) {
      const double M = S.mask[i + k];
      if (k >= kBias && k <= m - 1 - kBias) {
        MN += M * (u * u + l * l);
        SM += M;
        SME += M * (U + L);
      }
      MD2 += M * (u - l) * (u - l);
    }
  }
  S.nu[i] = sE / m;
  if (S.flat[i]) {
    S.A[i] = 1e300;  // every pair touching a flat window is pruned
    S.DUL[i] = 0.0;
    S.qsig[i] = 0.25;
  } else {
    S.A[i] = 4.0 * m + 2.0 * N - D2;
    S.DUL[i] = sqrt(fmax(D2, 0.0));
    S.qsig[i] = 0.25 * S.sig[i];
  }
  if (masked) {
    S.MN[i] = (float)MN;
    S.MDUL2[i] = (float)MD2;
    S.MDUL[i] = (float)sqrt(fmax(MD2, 0.0));
    S.SM[i] = SM;
    S.SME[i] = SME;
  }
}

// Centered update terms of the diagonal covariance recurrence
//   C(i+1, j+1) = C(i, j) + df_x[i] dg_y[j] + df_y[j] dg_x[i]
// for C(i, j) = sum_k (x[i+k] - mean_x(i)) (y[j+k] - mean_y(j)).
__global__ void k_diffs(DevSeries S) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= S.s) return;
  if (i == S.s - 1) {
    S.dfa[i] = S.dga[i] = S.dfE[i] = S.dgE[i] = 0.0;
    return;
  }
  const int m = S.m;
  const double a0 = S.a[i], a1 = S.a[i + m];
  const double e0 = S.E[i], e1 = S.E[i + m];
  S.dfa[i] = 0.5 * (a1 - a0);
  S.dga[i] = (a1 - S.mu[i + 1]) + (a0 - S.mu[i]);
  S.dfE[i] = 0.5 * (e1 - e0);
  S.dgE[i] = (e1 - S.nu[i + 1]) + (e0 - S.nu[i]);
}

// ---- global CDF mask ----

// Largest |z| over every non-flat window and offset (real_max/real_min of
// new_dtw_motifGUI_malloc.cu:185-199).
__global__ void k_zmax(DevSeries S, float* zmax) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  float v = 0.0f;
  if (i < S.s && !S.flat[i]) {
    double mx = -DBL_MAX, mn = DBL_MAX;
    for (int k = 0; k < S.m; ++k) {
      double x = S.a[i + k];
      mx = fmax(mx, x);
      mn = fmin(mn, x);
    }
    double z = fmax(fabs((mx - S.mu[i]) * S.isg[i]), fabs((mn - S.mu[i]) * S.isg[i]));
    // rounded down: the table length takes floor(max |z|), which a value just
    // below an integer must not reach by rounding up
    v = __double2float_rd(z);
  }
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomicMax((unsigned int*)zmax, __float_as_uint(v));
}

__device__ inline int table_len_from(const float* zmax) {
  // len_of_table_global = max(600, floor(max|z|) * 200)  (new_dtw_motifGUI.cpp:195-197)
  double lt = floor((double)*zmax) * 200.0;
  return lt > 600.0 ? (int)lt : 600;
}

__device__ inline int bucket(double z, int lt) {
  // FIND_POS_GLOBAL clamped to [1, lt] (compute_shared_data_global.cpp:25-31)
  double pp = floor(z * 100.0 + lt * 0.5);
  if (pp <= 0) pp = 1;
  if (pp > lt) pp = lt;
  return (int)pp - 1;
}

// Histogram of z values per offset k: counts[k][bucket].
__global__ void k_hist(DevSeries S, unsigned int* counts, const float* zmax, int lt_max) {
  const int lt = table_len_from(zmax);
  const int64_t total = S.s * (int64_t)S.m;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / S.m;
    const int k = (int)(e - i * S.m);
    if (S.flat[i]) continue;
    const double z = (S.a[i + k] - S.mu[i]) * S.isg[i];
    atomicAdd(&counts[(int64_t)k * lt_max + bucket(z, lt)], 1u);
  }
}

// In-place cumulative sum per offset (the CDF).
__global__ void k_cdf(int m, unsigned int* counts, const float* zmax, int lt_max) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const int lt = table_len_from(zmax);
  unsigned int acc = 0;
  unsigned int* row = counts + (int64_t)k * lt_max;
  for (int b = 0; b < lt; ++b) {
    acc += row[b];
    row[b] = acc;
  }
}

// Contribution of window i to DIFF[p] given the clipped envelope extremes
// (raw values) of window i at offset k = p - i.
__device__ inline double cdf_gap(const DevSeries& S, const unsigned int* cdf, int lt,
                                 int lt_max, int64_t i, int k, double U, double L) {
  const double zu = (U - S.mu[i]) * S.isg[i], zl = (L - S.mu[i]) * S.isg[i];
  const unsigned int* row = cdf + (int64_t)k * lt_max;
  return (double)row[bucket(zu, lt)] - (double)row[bucket(zl, lt)];
}

// DIFF[p] = (1/coverage) sum over windows i covering p of
//   (CDF_k(U_i[k]) - CDF_k(L_i[k])) / s,  k = p - i,
// with U_i / L_i the clipped envelopes of z-normalised window i
// (compute_MASK_global.cpp:28-62).  Window i's envelope at p spans
// [max(i, p-w), min(i+m-1, p+w)]: the raw envelope U[p], L[p] in the interior
// and a window that grows monotonically over the two edge ranges of i, which
// are walked with running extremes.
__global__ void k_diff(DevSeries S, const unsigned int* cdf, const float* zmax, int lt_max,
                       double* diff, double* mean_acc) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double local = 0.0;
  if (p < S.n) {
    const int lt = table_len_from(zmax);
    const int m = S.m, w = S.w;
    const int64_t ilo = p - m + 1 > 0 ? p - m + 1 : 0;
    const int64_t ihi = p < S.s - 1 ? p : S.s - 1;
    double acc = 0.0;
    if (m >= 2 * w + 2) {
      // phase A: i < p + w - m + 1 -> window [p - w, i + m - 1], growing in i
      const int64_t a_end = p + w - m + 1;  // exclusive
      int64_t i = ilo;
      if (i < a_end && i <= ihi) {
        double U = S.a[p - w], L = U;
        for (int64_t q = p - w + 1; q <= i + m - 1; ++q) {
          U = fmax(U, S.a[q]);
          L = fmin(L, S.a[q]);
        }
        for (; i < a_end && i <= ihi; ++i) {
          const double v = S.a[i + m - 1];
          U = fmax(U, v);
          L = fmin(L, v);
          if (!S.flat[i]) acc += cdf_gap(S, cdf, lt, lt_max, i, (int)(p - i), U, L);
        }
      }
      // phase B: interior -> raw envelope
      const int64_t c_begin = p - w + 1;  // phase C: i >= p - w + 1
      const double Up = S.U[p], Lp = S.L[p];
      for (; i <= ihi && i < c_begin; ++i)
        if (!S.flat[i]) acc += cdf_gap(S, cdf, lt, lt_max, i, (int)(p - i), Up, Lp);
      // phase C: i > p - w -> window [i, p + w], growing as i decreases
      if (i <= ihi) {
        const int64_t first = i;
        double U = S.a[p + w], L = U;
        for (int64_t q = ihi; q < p + w; ++q) {
          U = fmax(U, S.a[q]);
          L = fmin(L, S.a[q]);
        }
        double accC = 0.0;
        for (int64_t k2 = ihi; k2 >= first; --k2) {
          const double v = S.a[k2];
          U = fmax(U, v);
          L = fmin(L, v);
          if (!S.flat[k2]) accC += cdf_gap(S, cdf, lt, lt_max, k2, (int)(p - k2), U, L);
        }
        acc += accC;
      }
    } else {
      for (int64_t i = ilo; i <= ihi; ++i) {
        if (S.flat[i]) continue;
        const int64_t lo = (p - w > i) ? p - w : i;
        const int64_t hi = (p + w < i + m - 1) ? p + w : i + m - 1;
        double U = S.a[lo], L = U;
        for (int64_t q = lo + 1; q <= hi; ++q) {
          U = fmax(U, S.a[q]);
          L = fmin(L, S.a[q]);
        }
        acc += cdf_gap(S, cdf, lt, lt_max, i, (int)(p - i), U, L);
      }
    }
    acc /= (double)S.s;
    // coverage 1..m, m, ..., m..1 (compute_MASK_global.cpp:15-23)
    double cov = (double)m;
    if (p < m) cov = (double)(p + 1);
    if (p >= S.n - m) cov = (double)(S.n - p);
    acc /= cov;
    diff[p] = acc;
    local = acc;
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(mean_acc, local);
}

__global__ void k_mask(DevSeries S, const double* diff, const double* mean_acc) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= S.n) return;
  const double mean = *mean_acc / (double)S.n;
  S.mask[p] = diff[p] <= mean ? 1.0f : 0.0f;
}

}  // namespace

void launch_series_ids(const int64_t* sbeg, int nseries, int* sid, int64_t n, cudaStream_t st) {
  k_series_ids<<<1024, 256, 0, st>>>(sbeg, nseries, sid, n);
}

void launch_check_finite(const double* a, int64_t n, int* status, cudaStream_t st) {
  unsigned g = grid_for(n);
  if (g > 4096) g = 4096;
  k_check_finite<<<g, kThreads, 0, st>>>(a, n, status);
}

void launch_prep(const DevSeries& S, cudaStream_t st) {
  k_stats<<<grid_for(S.s), kThreads, 0, st>>>(S);
  k_envelope<<<grid_for(S.n), kThreads, 0, st>>>(S);
}

void launch_stats(const DevSeries& S, cudaStream_t st) {
  k_stats<<<grid_for(S.s), kThreads, 0, st>>>(S);
}

int mask_table_max(int m) {
  int z = (int)floor(sqrt((double)(m > 1 ? m - 1 : 1))) + 1;
  int lt = z * 200;
  return lt > 600 ? lt : 600;
}

void launch_rowterms(const DevSeries& S, bool masked, cudaStream_t st) {
  k_rowterms<<<grid_for(S.s), kThreads, 0, st>>>(S, masked);
  k_diffs<<<grid_for(S.s), kThreads, 0, st>>>(S);
}

void launch_mask(const DevSeries& S, unsigned int* counts, int lt_max, double* diff,
                 double* mean_acc, float* zmax, cudaStream_t st) {
  cudaMemsetAsync(zmax, 0, sizeof(float), st);
  cudaMemsetAsync(mean_acc, 0, sizeof(double), st);
  cudaMemsetAsync(counts, 0, sizeof(unsigned int) * (size_t)S.m * lt_max, st);
  k_zmax<<<grid_for(S.s), kThreads, 0, st>>>(S, zmax);
  unsigned g = grid_for(S.s * (int64_t)S.m);
  if (g > 148 * 64) g = 148 * 64;
  k_hist<<<g, kThreads, 0, st>>>(S, counts, zmax, lt_max);
  k_cdf<<<grid_for(S.m, 128), 128, 0, st>>>(S.m, counts, zmax, lt_max);
  k_diff<<<grid_for(S.n), kThreads, 0, st>>>(S, counts, zmax, lt_max, diff, mean_acc);
  k_mask<<<grid_for(S.n), kThreads, 0, st>>>(S, diff, mean_acc);
}

}  // namespace dtwj
