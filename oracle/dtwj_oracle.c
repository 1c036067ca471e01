/* TEST INFRASTRUCTURE ONLY — the oracle.  See dtwj_oracle.h.
 *
 * FP64 restatement of the reference's CPU join, function by function:
 *   orc_stats      mvmean                  CPU_version1/allmatrixop/movmean.cpp:9-33
 *                  (restated as an exact two-pass mean / population std)
 *   orc_envelope   lower_upper_lemire      CPU_version1/allmatrixop/lower_upper_lemire.cpp:7-43
 *   orc_dtw2       banded DTW recurrence   CPU_version1/MON_DTW.cpp:20-108 (no pruning)
 *   orc_dtw2_ea    MON_dtw early abandon   CPU_version1/MON_DTW.cpp:30,48 (UB = bsf - cb[i+w+1])
 *   orc_mp         mpx_v2                  CPU_version1/mpx_v2.cpp:13-150
 *   orc_mask       compute_shared_data_global + compute_MASK_global
 *                                          CPU_version1/compute_shared_data_global.cpp:12-46,
 *                                          CPU_version1/compute_MASK_global.cpp:10-92
 *   orc_lb_keogh2  LB_KK / LB_KK_FIRST      CPU_version1/lb_keogh.cpp:9-146
 *   orc_kim2       LB_KIM endpoint bound   CPU_version1/lb_kim.cpp:10-73
 *   orc_join       new_dtw_motifGUI        CPU_version1/new_dtw_motifGUI.cpp:21-586
 *                  seeds :53-74, diag_fast :376 (diag_fast.cpp:12-88),
 *                  diag_mask_global :389 (diag_mask_global.cpp:11-226),
 *                  LB_KK x2 + cb + MON_dtw :503-547
 *
 * Deliberate differences from the reference, each an exactness fix:
 *  - the endpoint bound's fourth option adds the corner cell once, not twice
 *    (lb_kim.cpp:55,62 and diag_mask_global.cpp:205,212 add it twice, which
 *    can overestimate);
 *  - diag_mask_global's first pair uses the high index's norm term like every
 *    other pair (diag_mask_global.cpp:77 indexes the low one);
 *  - pruning tests are strict with a 1e-9 relative slack, so a pair whose DTW
 *    equals the best-so-far is always evaluated, and ties resolve to the lowest
 *    (dist, i, j) instead of the last pair in visit order;
 *  - flat windows (sigma == 0) are excluded instead of producing inf/NaN;
 *  - the CPU-only extra stages (local CDF masks with alpha search,
 *    LB_Petitjean) are not restated: the join is exact without them.
 */
#include "dtwj_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_INF 1e300
#define REL_SLACK 1e-9
#define KIM_BIAS 3

static double sq(double x) { return x * x; }
/* a window with (numerically) zero deviation has no z-normalisation */
static int is_flat(double mu, double sig) {
  double rms = sqrt(mu * mu + sig * sig);
  return !(sig > 1e-12 * rms) || sig == 0.0;
}
static double now_seconds(void) {
#ifdef _OPENMP
  return omp_get_wtime();
#else
  return 0.0;
#endif
}

void orc_stats(const double* a, int64_t n, int m, double* mu, double* sig) {
  int64_t s = n - m + 1;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < s; ++i) {
    double sum = 0.0;
    for (int k = 0; k < m; ++k) sum += a[i + k];
    double mean = sum / m, ss = 0.0;
    for (int k = 0; k < m; ++k) ss += sq(a[i + k] - mean);
    mu[i] = mean;
    sig[i] = sqrt(ss / m);
  }
}

/* lower[p] = min a[max(0,p-r) .. min(n-1,p+r)], upper likewise (clipped
 * Sakoe-Chiba envelope), with monotone deques. */
void orc_envelope(const double* a, int64_t n, int r, double* lower, double* upper) {
  int64_t* qu = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
  int64_t* ql = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
  int64_t hu = 0, tu = 0, hl = 0, tl = 0; /* [head, tail) */
  int64_t next = 0;
  for (int64_t p = 0; p < n; ++p) {
    int64_t hi = p + r < n - 1 ? p + r : n - 1;
    while (next <= hi) {
      while (tu > hu && a[qu[tu - 1]] <= a[next]) --tu;
      qu[tu++] = next;
      while (tl > hl && a[ql[tl - 1]] >= a[next]) --tl;
      ql[tl++] = next;
      ++next;
    }
    while (qu[hu] < p - r) ++hu;
    while (ql[hl] < p - r) ++hl;
    upper[p] = a[qu[hu]];
    lower[p] = a[ql[hl]];
  }
  free(qu);
  free(ql);
}

/* Squared banded DTW, exact (no pruning).  Cells (r, c) with |r - c| <= w.
 * Row buffers hold cell (r, c) at index c + 1; only the band is touched per
 * row (index c0 is reset to +inf as the left border, indices right of the
 * band have never been written and stay +inf). */
static double dtw2_rows(const double* q, const double* t, const double* cb, int m, int w,
                        double bsf2, double* prev, double* cur) {
  if (w > m) w = m;
  for (int c = 0; c <= m + 1; ++c) { prev[c] = ORC_INF; cur[c] = ORC_INF; }
  int r;
  for (r = 0; r < m; ++r) {
    int c0 = r - w > 0 ? r - w : 0, c1 = r + w < m - 1 ? r + w : m - 1;
    cur[c0] = ORC_INF;
    double rowmin = ORC_INF;
    for (int c = c0; c <= c1; ++c) {
      double best;
      if (r == 0 && c == 0) best = 0.0;
      else {
        double up = prev[c + 1], left = cur[c], diag = prev[c];
        best = up < left ? up : left;
        best = best < diag ? best : diag;
      }
      double v = best + sq(q[r] - t[c]);
      cur[c + 1] = v;
      if (v < rowmin) rowmin = v;
    }
    if (cb) {
      double rest = (r + w + 1 < m) ? cb[r + w + 1] : 0.0;
      if (rowmin + rest > bsf2) return ORC_INF;
    }
    double* tmp = prev; prev = cur; cur = tmp;
  }
  return prev[m];
}

double orc_dtw2(const double* q, const double* t, int m, int w) {
  double* buf = (double*)malloc(sizeof(double) * (size_t)(2 * m + 4));
  double d = dtw2_rows(q, t, NULL, m, w, ORC_INF, buf, buf + m + 2);
  free(buf);
  return d;
}

/* Early-abandoning squared DTW (the semantics of MON_dtw): returns the exact
 * squared DTW when it is <= bsf2, otherwise ORC_INF.  After row r every path
 * still has to cross rows/columns >= r + w + 1, whose cost is bounded below
 * by cb[r + w + 1] (cb is a suffix sum, zero past m; MON_DTW.cpp:48). */
double orc_dtw2_ea(const double* q, const double* t, const double* cb, int m, int w,
                   double bsf2) {
  double* buf = (double*)malloc(sizeof(double) * (size_t)(2 * m + 4));
  double d = dtw2_rows(q, t, cb, m, w, bsf2, buf, buf + m + 2);
  free(buf);
  return d;
}

/* ED matrix profile with exclusion zone m (mpx_v2, minlag = m): diagonal
 * covariance recurrence in FP64, mp[i] = min_j z-ED(i, j) over |i-j| >= m,
 * mpi[i] the 0-based argmin (lowest index on ties), -1 / inf when none. */
void orc_mp(const double* a, int64_t n, int m, double* mp, int64_t* mpi) {
  int64_t s = n - m + 1;
  double* mu = (double*)malloc(sizeof(double) * (size_t)s);
  double* sig = (double*)malloc(sizeof(double) * (size_t)s);
  orc_stats(a, n, m, mu, sig);
  double* corr_best = (double*)malloc(sizeof(double) * (size_t)s);
  unsigned char* flat = (unsigned char*)malloc((size_t)s);
  for (int64_t i = 0; i < s; ++i) {
    corr_best[i] = -ORC_INF;
    mpi[i] = -1;
    flat[i] = (unsigned char)is_flat(mu[i], sig[i]);
  }
#pragma omp parallel
  {
    double* cb = (double*)malloc(sizeof(double) * (size_t)s);
    int64_t* ci = (int64_t*)malloc(sizeof(int64_t) * (size_t)s);
    for (int64_t i = 0; i < s; ++i) { cb[i] = -ORC_INF; ci[i] = -1; }
#pragma omp for schedule(dynamic, 16)
    for (int64_t L = m; L < s; ++L) {
      double cov = 0.0;
      for (int64_t i = 0; i + L < s; ++i) {
        int64_t j = i + L;
        if ((i & 1023) == 0) { /* exact re-anchor */
          cov = 0.0;
          for (int k = 0; k < m; ++k) cov += (a[i + k] - mu[i]) * (a[j + k] - mu[j]);
        } else {
          /* centered update: C(i,j) = C(i-1,j-1) + df(i-1)dg(j-1) + df(j-1)dg(i-1) */
          double dfi = 0.5 * (a[i - 1 + m] - a[i - 1]);
          double dfj = 0.5 * (a[j - 1 + m] - a[j - 1]);
          double dgi = (a[i - 1 + m] - mu[i]) + (a[i - 1] - mu[i - 1]);
          double dgj = (a[j - 1 + m] - mu[j]) + (a[j - 1] - mu[j - 1]);
          cov += dfi * dgj + dfj * dgi;
        }
        if (flat[i] || flat[j]) continue;
        double corr = cov / (m * sig[i] * sig[j]);
        if (corr > cb[i] || (corr == cb[i] && j < ci[i])) { cb[i] = corr; ci[i] = j; }
        if (corr > cb[j] || (corr == cb[j] && i < ci[j])) { cb[j] = corr; ci[j] = i; }
      }
    }
#pragma omp critical
    for (int64_t i = 0; i < s; ++i) {
      if (ci[i] < 0) continue;
      if (cb[i] > corr_best[i] || (cb[i] == corr_best[i] && ci[i] < mpi[i])) {
        corr_best[i] = cb[i];
        mpi[i] = ci[i];
      }
    }
    free(cb);
    free(ci);
  }
  for (int64_t i = 0; i < s; ++i) {
    if (mpi[i] < 0) { mp[i] = INFINITY; continue; }
    double d2 = 2.0 * m * (1.0 - corr_best[i]);
    mp[i] = sqrt(d2 > 0 ? d2 : 0.0);
  }
  free(corr_best);
  free(flat);
  free(mu);
  free(sig);
}

/* Global CDF table over z-normalised values per offset and the binary mask
 * derived from it (compute_shared_data_global + compute_MASK_global).
 * Returns 0, or -1 if n < 2m.  *table_len receives the CDF length. */
int orc_mask(const double* a, int64_t n, int m, int w, double* mask, int* table_len) {
  int64_t s = n - m + 1;
  if (n < 2 * (int64_t)m) return -1;
  double* mu = (double*)malloc(sizeof(double) * (size_t)s);
  double* sig = (double*)malloc(sizeof(double) * (size_t)s);
  orc_stats(a, n, m, mu, sig);
  double vmax = -ORC_INF, vmin = ORC_INF;
  for (int64_t i = 0; i < s; ++i)
    for (int k = 0; k < m && !is_flat(mu[i], sig[i]); ++k) {
      double v = (a[i + k] - mu[i]) / sig[i];
      if (v > vmax) vmax = v;
      if (v < vmin) vmin = v;
    }
  double amax = fabs(vmax) > fabs(vmin) ? fabs(vmax) : fabs(vmin);
  double lt_d = floor(amax) * 2 * 100;
  int lt = lt_d > 600 ? (int)lt_d : 600;
  *table_len = lt;
  double* cdf = (double*)calloc((size_t)m * lt, sizeof(double));
  double* z = (double*)malloc(sizeof(double) * m);
  double* zl = (double*)malloc(sizeof(double) * m);
  double* zu = (double*)malloc(sizeof(double) * m);
  for (int64_t i = 0; i < s; ++i)
    for (int k = 0; k < m && !is_flat(mu[i], sig[i]); ++k) {
      double v = (a[i + k] - mu[i]) / sig[i];
      double pp = floor(v * 100 + lt * 0.5);
      if (pp <= 0) pp = 1;
      if (pp > lt) pp = lt;
      cdf[(size_t)k * lt + (size_t)pp - 1] += 1.0;
    }
  for (int k = 0; k < m; ++k) {
    double acc = 0;
    for (int b = 0; b < lt; ++b) { acc += cdf[(size_t)k * lt + b]; cdf[(size_t)k * lt + b] = acc; }
  }
  double* diff = (double*)calloc((size_t)n, sizeof(double));
  for (int64_t i = 0; i < s; ++i) {
    if (is_flat(mu[i], sig[i])) continue;
    for (int k = 0; k < m; ++k) z[k] = (a[i + k] - mu[i]) / sig[i];
    orc_envelope(z, m, w, zl, zu);
    for (int k = 0; k < m; ++k) {
      double pl = floor(zl[k] * 100 + lt * 0.5), pu = floor(zu[k] * 100 + lt * 0.5);
      if (pl <= 0) pl = 1;
      if (pl > lt) pl = lt;
      if (pu <= 0) pu = 1;
      if (pu > lt) pu = lt;
      double d = cdf[(size_t)k * lt + (size_t)pu - 1] - cdf[(size_t)k * lt + (size_t)pl - 1];
      diff[i + k] += d / (double)s;
    }
  }
  double mean = 0;
  for (int64_t p = 0; p < n; ++p) {
    /* coverage: 1..m, then m, then m..1 (compute_MASK_global.cpp:15-23) */
    double cov = (double)m;
    if (p < m) cov = (double)(p + 1);
    if (p >= n - m) cov = (double)(n - p);
    diff[p] /= cov;
    mean += diff[p];
  }
  mean /= (double)n;
  for (int64_t p = 0; p < n; ++p) mask[p] = diff[p] <= mean ? 1.0 : 0.0;
  free(diff); free(cdf); free(z); free(zl); free(zu); free(mu); free(sig);
  return 0;
}

double orc_lb_keogh2(const double* q, const double* lower, const double* upper, int m) {
  double d = 0.0;
  for (int k = 0; k < m; ++k) {
    if (q[k] > upper[k]) d += sq(q[k] - upper[k]);
    else if (q[k] < lower[k]) d += sq(q[k] - lower[k]);
  }
  return d;
}

/* Endpoint bound (LB_KIM, lb_kim.cpp:10-73): minimum cost of the path cells
 * in the first (left) and last (right) three layers.  q = subsequence i,
 * t = subsequence j; cells are (t index, q index).  Fourth option fixed to
 * count the corner once. */
void orc_kim2(const double* q, const double* t, int m, double* left, double* right) {
#define D(x, y) sq((x) - (y))
  double o = D(t[0], q[0]);
  double lw = fmin(D(t[1], q[0]), D(t[1], q[1]));
  double l1 = fmin(lw, D(t[0], q[1]));
  double d = fmin(D(t[1], q[0]) + D(t[2], q[0]), lw + D(t[2], q[1]));
  d = fmin(d, D(q[1], t[1]) + D(q[2], t[2]));
  d = fmin(d, l1 + D(q[2], t[1]));
  d = fmin(d, D(q[1], t[0]) + D(q[2], t[0]));
  *left = o + d;
  const int e = m - 1;
  double o2 = D(t[e], q[e]);
  double rw = fmin(D(t[e - 1], q[e]), D(t[e - 1], q[e - 1]));
  double r1 = fmin(rw, D(t[e], q[e - 1]));
  d = fmin(D(t[e - 1], q[e]) + D(t[e - 2], q[e]), rw + D(t[e - 2], q[e - 1]));
  d = fmin(d, D(q[e - 1], t[e - 1]) + D(q[e - 2], t[e - 2]));
  d = fmin(d, r1 + D(q[e - 2], t[e - 1]));
  d = fmin(d, D(q[e - 1], t[e]) + D(q[e - 2], t[e]));
  *right = o2 + d;
#undef D
}

/* ---------------------------------------------------------------- join --- */

typedef struct {
  const double* a;
  int64_t n, s;
  int m, w;
  double *mu, *sig, *isg;
  unsigned char* flat;
  double *U, *L, *E;
  double *N, *DUL2, *DUL;          /* fast bound row terms              */
  double *mask;                    /* masked bound                        */
  double *MN, *MDUL2, *MDUL;       /* masked row terms: sum M(nU^2+nL^2)  */
  double *sumE;                    /* sum_k E[i+k]                        */
  double *SM, *SME;                /* sum_T M, sum_T M*E  (T = [3, m-4])  */
} orc_ctx;

static void znorm(const orc_ctx* c, int64_t i, double* z) {
  for (int k = 0; k < c->m; ++k) z[k] = (c->a[i + k] - c->mu[i]) / c->sig[i];
}

/* fast bound (diag_fast): env = row r, query = column q, cross term X */
static double fast_lb(const orc_ctx* c, int64_t r, double X) {
  double S = 2.0 * c->m + c->N[r] - 2.0 * X;
  double v = 2.0 * S - c->DUL2[r];
  if (!(v >= 0)) return -ORC_INF; /* reference: sqrt of negative -> NaN -> not pruned */
  return 0.5 * (sqrt(v) - c->DUL[r]);
}



/* masked bound (diag_mask_global) for env = row r, query = column q, from the
 * raw masked sums over T = [3, m-4]: F1 = sum M_r a_q, F2 = sum M_r a_q^2,
 * F3 = sum M_r E_r a_q. */
static double masked_lb(const orc_ctx* c, int64_t r, int64_t q, double F1, double F2,
                        double F3) {
  double mq = c->mu[q], mr = c->mu[r];
  double mnorm = (F2 - 2.0 * mq * F1 + mq * mq * c->SM[r]) * sq(c->isg[q]);
  double t = (F3 - 2.0 * mr * F1 - mq * c->SME[r] + 2.0 * mr * mq * c->SM[r]) * c->isg[q] *
             c->isg[r];
  double dist = 2.0 * mnorm - 2.0 * t + c->MN[r];
  if (dist < c->MDUL2[r]) return 0.0;
  return 0.5 * (sqrt(2.0 * dist - c->MDUL2[r]) - c->MDUL[r]);
}

static double atomic_read(const double* p) {
  double v;
#pragma omp atomic read
  v = *p;
  return v;
}

typedef struct {
  double d2;
  int64_t i, j;
} best_t;

static int better(double d2, int64_t i, int64_t j, const best_t* b) {
  if (d2 < b->d2) return 1;
  if (d2 > b->d2) return 0;
  return (i < b->i) || (i == b->i && j < b->j);
}

/* Clipped envelope of z-normalised window j, the reference's subs_U/subs_L
 * (lower_upper_lemire on each subsequence, new_dtw_motifGUI.cpp:37-46):
 * lo[k] = min z_j[max(0, k-w) .. min(m-1, k+w)].  Because z = (a - mu) * isg
 * is monotone in a, the minimum of z is z of the minimum of a: positions
 * w <= k <= m-1-w read the raw-series envelope of radius w, the first and
 * last w positions take running extremes over the window.  Scaled by the
 * reciprocal deviation (LB_Keogh is a bound; the 1e-9 slack covers the last
 * bits). */
static void window_envelope(const orc_ctx* c, int64_t j, double* lo, double* up) {
  const int m = c->m, w = c->w;
  const double mu = c->mu[j], is = c->isg[j];
  const double* x = c->a + j;
  if (2 * w >= m - 1) { /* band covers most of the window: direct */
    for (int k = 0; k < m; ++k) {
      int k0 = k - w > 0 ? k - w : 0, k1 = k + w < m - 1 ? k + w : m - 1;
      double mn = x[k0], mx = x[k0];
      for (int t = k0 + 1; t <= k1; ++t) { mn = fmin(mn, x[t]); mx = fmax(mx, x[t]); }
      lo[k] = (mn - mu) * is;
      up[k] = (mx - mu) * is;
    }
    return;
  }
  for (int k = w; k <= m - 1 - w; ++k) {
    lo[k] = (c->L[j + k] - mu) * is;
    up[k] = (c->U[j + k] - mu) * is;
  }
  double mn = x[0], mx = x[0];
  for (int t = 1; t < w; ++t) { mn = fmin(mn, x[t]); mx = fmax(mx, x[t]); }
  for (int k = 0; k < w; ++k) {
    mn = fmin(mn, x[k + w]); mx = fmax(mx, x[k + w]);
    lo[k] = (mn - mu) * is;
    up[k] = (mx - mu) * is;
  }
  mn = x[m - 1]; mx = x[m - 1];
  for (int t = m - w; t < m - 1; ++t) { mn = fmin(mn, x[t]); mx = fmax(mx, x[t]); }
  for (int k = m - 1; k >= m - w; --k) {
    mn = fmin(mn, x[k - w]); mx = fmax(mx, x[k - w]);
    lo[k] = (mn - mu) * is;
    up[k] = (mx - mu) * is;
  }
}

/* One candidate pair through Kim -> Keogh x2 -> DTW.  Returns squared DTW or
 * ORC_INF.  stage: 0 pruned by kim, 1 by keogh, 2 dtw evaluated.
 * LB_KK (lb_keogh.cpp:9-72): the three end terms of each side against the
 * endpoint bound, then the middle terms with an early exit once the sum
 * passes the threshold; the surviving direction with the larger bound gives
 * the per-position terms whose suffix sums abandon the DTW
 * (new_dtw_motifGUI.cpp:508-547). */
static double eval_pair(const orc_ctx* c, int64_t i, int64_t j, double lbm, double bsf2,
                        double* buf, int* stage) {
  const int m = c->m, w = c->w;
  double *zi = buf, *zj = buf + m, *lo = buf + 2 * m, *up = buf + 3 * m;
  double *cb1 = buf + 4 * m, *cb2 = buf + 5 * m, *cb = buf + 6 * m; /* m + w + 2 */
  double *prev = buf + 7 * m + w + 4, *cur = prev + m + 2;
  double thr = bsf2 * (1.0 + REL_SLACK);
  /* endpoint bound from the three samples at each end, normalised as znorm */
  double qi[6], tj[6];
  for (int k = 0; k < 3; ++k) {
    qi[k] = (c->a[i + k] - c->mu[i]) / c->sig[i];
    tj[k] = (c->a[j + k] - c->mu[j]) / c->sig[j];
    qi[5 - k] = (c->a[i + m - 1 - k] - c->mu[i]) / c->sig[i];
    tj[5 - k] = (c->a[j + m - 1 - k] - c->mu[j]) / c->sig[j];
  }
  double kl, kr;
  orc_kim2(qi, tj, 6, &kl, &kr);
  if (kl + kr + lbm * lbm > thr) { *stage = 0; return ORC_INF; }
  double lbk[2];
  for (int dir = 0; dir < 2; ++dir) {
    const int64_t qw = dir == 0 ? i : j, ew = dir == 0 ? j : i;
    double* cbx = dir == 0 ? cb1 : cb2;
    window_envelope(c, ew, lo, up);
    const double mq = c->mu[qw], iq = c->isg[qw];
    const double* xq = c->a + qw;
    double ends = 0.0;
    for (int h = 0; h < 2 * KIM_BIAS; ++h) {
      int k = h < KIM_BIAS ? h : m - 2 * KIM_BIAS + h;
      double v = (xq[k] - mq) * iq, d = 0.0;
      if (v > up[k]) d = sq(v - up[k]);
      else if (v < lo[k]) d = sq(v - lo[k]);
      ends += d;
      cbx[k] = 0.0;
    }
    double dist = ends > kl + kr ? ends : kl + kr;
    int k;
    for (k = KIM_BIAS; k < m - KIM_BIAS; ++k) {
      double v = (xq[k] - mq) * iq, d = 0.0;
      if (v > up[k]) d = sq(v - up[k]);
      else if (v < lo[k]) d = sq(v - lo[k]);
      cbx[k] = d;
      dist += d;
      if (dist > thr) break;
    }
    if (k < m - KIM_BIAS) { *stage = 1; return ORC_INF; }
    cbx[0] = kl;
    cbx[m - KIM_BIAS] = kr;
    lbk[dir] = dist;
  }
  const double* src = lbk[0] > lbk[1] ? cb1 : cb2;
  for (int k = m; k < m + w + 2; ++k) cb[k] = 0.0;
  cb[m - 1] = src[m - 1];
  for (int k = m - 2; k >= 0; --k) cb[k] = cb[k + 1] + src[k];
  znorm(c, i, zi);
  znorm(c, j, zj);
  *stage = 2;
  return dtw2_rows(zi, zj, cb, m, w, thr, prev, cur);
}

double orc_pair_dist(const double* a, int64_t n, int m, int w, int64_t i, int64_t j) {
  double* zi = (double*)malloc(sizeof(double) * m);
  double* zj = (double*)malloc(sizeof(double) * m);
  double mi, si, mj, sj;
  {
    double sum = 0, ss = 0;
    for (int k = 0; k < m; ++k) sum += a[i + k];
    mi = sum / m;
    for (int k = 0; k < m; ++k) ss += sq(a[i + k] - mi);
    si = sqrt(ss / m);
    sum = 0; ss = 0;
    for (int k = 0; k < m; ++k) sum += a[j + k];
    mj = sum / m;
    for (int k = 0; k < m; ++k) ss += sq(a[j + k] - mj);
    sj = sqrt(ss / m);
  }
  (void)n;
  for (int k = 0; k < m; ++k) { zi[k] = (a[i + k] - mi) / si; zj[k] = (a[j + k] - mj) / sj; }
  double d = sqrt(orc_dtw2(zi, zj, m, w));
  free(zi);
  free(zj);
  return d;
}

int orc_join(const double* a, int64_t n, int m, int w, unsigned flags, int threads,
             orc_result* out) {
  memset(out, 0, sizeof *out);
  if (m < 8 || w < 0 || n < 2 * (int64_t)m + 1) return -1;
  for (int64_t p = 0; p < n; ++p)
    if (!isfinite(a[p])) return -2;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
  out->threads = omp_get_max_threads();
#else
  out->threads = 1;
#endif
  double t0 = now_seconds();
  orc_ctx c;
  memset(&c, 0, sizeof c);
  c.a = a; c.n = n; c.m = m; c.w = w;
  int64_t s = n - m + 1;
  c.s = s;
  c.mu = (double*)malloc(sizeof(double) * s);
  c.sig = (double*)malloc(sizeof(double) * s);
  c.isg = (double*)malloc(sizeof(double) * s);
  c.flat = (unsigned char*)calloc((size_t)s, 1);
  orc_stats(a, n, m, c.mu, c.sig);
  for (int64_t i = 0; i < s; ++i) {
    c.flat[i] = is_flat(c.mu[i], c.sig[i]);
    c.isg[i] = c.flat[i] ? 0.0 : 1.0 / c.sig[i];
  }
  c.U = (double*)malloc(sizeof(double) * n);
  c.L = (double*)malloc(sizeof(double) * n);
  c.E = (double*)malloc(sizeof(double) * n);
  orc_envelope(a, n, w, c.L, c.U);
  for (int64_t p = 0; p < n; ++p) c.E[p] = c.U[p] + c.L[p];
  c.N = (double*)malloc(sizeof(double) * s);
  c.DUL2 = (double*)malloc(sizeof(double) * s);
  c.DUL = (double*)malloc(sizeof(double) * s);
  const int use_diag = !(flags & ORC_NO_DIAG);
  const int use_masked = use_diag && !(flags & ORC_NO_MASKED);
  for (int64_t i = 0; i < s; ++i) {
    double nn = 0, dd = 0;
    for (int k = 0; k < m; ++k) {
      double u = (c.U[i + k] - c.mu[i]) * c.isg[i], l = (c.L[i + k] - c.mu[i]) * c.isg[i];
      nn += u * u + l * l;
      dd += sq(u - l);
    }
    c.N[i] = nn; c.DUL2[i] = dd; c.DUL[i] = sqrt(dd);
  }
  c.sumE = (double*)malloc(sizeof(double) * s);
  for (int64_t i = 0; i < s; ++i) {
    double acc = 0;
    for (int k = 0; k < m; ++k) acc += c.E[i + k];
    c.sumE[i] = acc;
  }
  if (use_masked) {
    int lt;
    c.mask = (double*)malloc(sizeof(double) * n);
    orc_mask(a, n, m, w, c.mask, &lt);
    c.MN = (double*)malloc(sizeof(double) * s);
    c.MDUL2 = (double*)malloc(sizeof(double) * s);
    c.MDUL = (double*)malloc(sizeof(double) * s);
    for (int64_t i = 0; i < s; ++i) {
      double nn = 0, dd = 0;
      for (int k = 0; k < m; ++k) {
        double M = c.mask[i + k];
        double u = (c.U[i + k] - c.mu[i]) * c.isg[i], l = (c.L[i + k] - c.mu[i]) * c.isg[i];
        if (k >= KIM_BIAS && k <= m - 1 - KIM_BIAS) nn += M * (u * u + l * l);
        dd += M * sq(u - l); /* over all m, as diag_mask_global's DUL2_global */
      }
      c.MN[i] = nn; c.MDUL2[i] = dd; c.MDUL[i] = sqrt(dd);
    }
    c.SM = (double*)malloc(sizeof(double) * s);
    c.SME = (double*)malloc(sizeof(double) * s);
    for (int64_t i = 0; i < s; ++i) {
      double sm = 0, sme = 0;
      for (int k = KIM_BIAS; k <= m - 1 - KIM_BIAS; ++k) {
        sm += c.mask[i + k];
        sme += c.mask[i + k] * c.E[i + k];
      }
      c.SM[i] = sm; c.SME[i] = sme;
    }
  }

  /* ---- seeds: k = 100 smallest ED-profile entries -> exact DTW ---- */
  best_t best = {ORC_INF, -1, -1};
  double bsf = ORC_INF;
  if (!(flags & ORC_NO_SEED)) {
    double* mp = (double*)malloc(sizeof(double) * s);
    int64_t* mpi = (int64_t*)malloc(sizeof(int64_t) * s);
    orc_mp(a, n, m, mp, mpi);
    const int K = 100;
    int64_t sel[100];
    int ns = 0;
    unsigned char* taken = (unsigned char*)calloc((size_t)s, 1);
    for (int r = 0; r < K; ++r) {
      int64_t bi = -1;
      for (int64_t i = 0; i < s; ++i) {
        if (taken[i] || mpi[i] < 0 || c.flat[i] || c.flat[mpi[i]]) continue;
        if (bi < 0 || mp[i] < mp[bi]) bi = i;
      }
      if (bi < 0) break;
      taken[bi] = 1;
      sel[ns++] = bi;
    }
    if (ns > 0) bsf = mp[sel[0]];
    double* zi = (double*)malloc(sizeof(double) * m);
    double* zj = (double*)malloc(sizeof(double) * m);
    for (int r = 0; r < ns; ++r) {
      int64_t i = sel[r], j = mpi[sel[r]];
      if (i > j) { int64_t t = i; i = j; j = t; }
      znorm(&c, i, zi);
      znorm(&c, j, zj);
      double d2 = orc_dtw2(zi, zj, m, w);
      if (better(d2, i, j, &best)) { best.d2 = d2; best.i = i; best.j = j; }
    }
    if (best.i >= 0 && sqrt(best.d2) < bsf) bsf = sqrt(best.d2);
    free(zi); free(zj); free(taken); free(mp); free(mpi);
  }
  out->seed_bsf = bsf;

  /* ---- sweep every diagonal (lag L = j - i >= m) ---- */
  uint64_t n_pairs = 0, n_fast = 0, n_masked = 0, n_kim = 0, n_keogh = 0, n_dtw = 0, n_ab = 0;
#pragma omp parallel reduction(+ : n_pairs, n_fast, n_masked, n_kim, n_keogh, n_dtw, n_ab)
  {
    double* buf = (double*)malloc(sizeof(double) * (size_t)(9 * m + w + 12));
#pragma omp for schedule(dynamic, 8)
    for (int64_t L = m; L < s; ++L) {
      /* raw cross sums along the diagonal, re-anchored every 512 rows:
       * fast (diag_fast.cpp:24-27,59-63)  cf = sum a_j E_i, cr = sum a_i E_j
       * masked (diag_mask_global.cpp:117-128,187-195) F* env i, R* env j */
      double cf = 0, cr = 0, F1 = 0, F2 = 0, F3 = 0, R1 = 0, R2 = 0, R3 = 0;
      const int lo = KIM_BIAS, hi = m - 1 - KIM_BIAS;
      for (int64_t i = 0; i + L < s; ++i) {
        int64_t j = i + L;
        if (use_diag) {
          if ((i & 511) == 0) {
            cf = cr = F1 = F2 = F3 = R1 = R2 = R3 = 0.0;
            for (int k = 0; k < m; ++k) { cf += a[j + k] * c.E[i + k]; cr += a[i + k] * c.E[j + k]; }
            if (use_masked)
              for (int k = lo; k <= hi; ++k) {
                double Mi = c.mask[i + k], Mj = c.mask[j + k];
                F1 += Mi * a[j + k]; F2 += Mi * a[j + k] * a[j + k]; F3 += Mi * c.E[i + k] * a[j + k];
                R1 += Mj * a[i + k]; R2 += Mj * a[i + k] * a[i + k]; R3 += Mj * c.E[j + k] * a[i + k];
              }
          } else {
            cf += a[j + m - 1] * c.E[i + m - 1] - a[j - 1] * c.E[i - 1];
            cr += a[i + m - 1] * c.E[j + m - 1] - a[i - 1] * c.E[j - 1];
            if (use_masked) {
              int64_t oi = i - 1 + lo, oj = j - 1 + lo, ni = i + hi, nj = j + hi;
              double Mo = c.mask[oi], Mn = c.mask[ni];
              F1 += Mn * a[nj] - Mo * a[oj];
              F2 += Mn * a[nj] * a[nj] - Mo * a[oj] * a[oj];
              F3 += Mn * c.E[ni] * a[nj] - Mo * c.E[oi] * a[oj];
              Mo = c.mask[oj]; Mn = c.mask[nj];
              R1 += Mn * a[ni] - Mo * a[oi];
              R2 += Mn * a[ni] * a[ni] - Mo * a[oi] * a[oi];
              R3 += Mn * c.E[nj] * a[ni] - Mo * c.E[oj] * a[oi];
            }
          }
        }
        if (c.flat[i] || c.flat[j]) continue;
        ++n_pairs;
        double cur_bsf = atomic_read(&bsf);
        double lbm = 0.0;
        if (use_diag) {
          /* X = (sum a_q E_r - mu_q sum E_r) / (sig_q sig_r) */
          double Xf = (cf - c.mu[j] * c.sumE[i]) * c.isg[j] * c.isg[i];
          double Xr = (cr - c.mu[i] * c.sumE[j]) * c.isg[i] * c.isg[j];
          double lbf = fast_lb(&c, i, Xf), lbr = fast_lb(&c, j, Xr);
          double lb = lbf > lbr ? lbf : lbr;
          if (lb > cur_bsf * (1.0 + REL_SLACK) + 1e-12) { ++n_fast; continue; }
          if (use_masked) {
            double m1 = masked_lb(&c, i, j, F1, F2, F3), m2 = masked_lb(&c, j, i, R1, R2, R3);
            lbm = m1 > m2 ? m1 : m2;
            if (lbm > cur_bsf * (1.0 + REL_SLACK) + 1e-12) { ++n_masked; continue; }
          }
        }
        int stage;
        double d2 = eval_pair(&c, i, j, lbm, cur_bsf * cur_bsf, buf, &stage);
        if (stage == 0) { ++n_kim; continue; }
        if (stage == 1) { ++n_keogh; continue; }
        ++n_dtw;
        if (d2 >= ORC_INF) { ++n_ab; continue; }
#pragma omp critical(orc_best)
        {
          if (better(d2, i, j, &best)) {
            best.d2 = d2; best.i = i; best.j = j;
            double d = sqrt(d2);
            if (d < bsf) {
#pragma omp atomic write
              bsf = d;
            }
          }
        }
      }
    }
    free(buf);
  }
  out->i = best.i;
  out->j = best.j;
  out->dist = best.i >= 0 ? sqrt(best.d2) : INFINITY;
  out->pairs = n_pairs;
  out->pruned_fast = n_fast;
  out->pruned_masked = n_masked;
  out->pruned_kim = n_kim;
  out->pruned_keogh = n_keogh;
  out->dtw_calls = n_dtw;
  out->dtw_abandoned = n_ab;
  out->seconds = now_seconds() - t0;
  free(c.mu); free(c.sig); free(c.isg); free(c.flat); free(c.U); free(c.L); free(c.E);
  free(c.N); free(c.DUL2); free(c.DUL);
  free(c.mask); free(c.MN); free(c.MDUL2); free(c.MDUL); free(c.sumE); free(c.SM); free(c.SME);
  return 0;
}

/* ---- LB_Petitjean (CPU_version1/LB_PETITJEAN.cpp:10-123) ----
 * The bound adds to LB_Keogh of A against B's envelope a second term for B:
 * H is A projected onto B's envelope (LB_PETITJEAN.cpp:27-39; the three end
 * samples of each side keep A's own values, as the reference's copy of q
 * does at :24), (UH, LH) is H's clipped envelope (:41-88), and each B_k on
 * k in [3, m-4] adds its distance to [LH_k, UH_k], refined against A's own
 * envelope where that envelope lies inside (:89-110). */
static void pj_window(const double* a, int64_t n, int m, int w, int64_t p, int env_mode,
                      double* z, double* lo, double* up) {
  double sum = 0.0, ss = 0.0;
  for (int k = 0; k < m; ++k) sum += a[p + k];
  const double mu = sum / m;
  for (int k = 0; k < m; ++k) ss += sq(a[p + k] - mu);
  const double sg = sqrt(ss / m);
  for (int k = 0; k < m; ++k) z[k] = (a[p + k] - mu) / sg;
  if (env_mode) {
    orc_envelope(z, m, w, lo, up);
    return;
  }
  /* raw envelope of radius w over the series, taken on the slice that holds
   * every sample the window's envelope reads (clipping at the series ends) */
  const int64_t b0 = p - w > 0 ? p - w : 0;
  const int64_t b1 = p + m + w < n ? p + m + w : n;
  double* sl = (double*)malloc(sizeof(double) * (size_t)(b1 - b0));
  double* su = (double*)malloc(sizeof(double) * (size_t)(b1 - b0));
  orc_envelope(a + b0, b1 - b0, w, sl, su);
  for (int k = 0; k < m; ++k) {
    lo[k] = (sl[p + k - b0] - mu) / sg;
    up[k] = (su[p + k - b0] - mu) / sg;
  }
  free(sl);
  free(su);
}

void orc_lb_petitjean(const double* a, int64_t n, int m, int w, int64_t ia, int64_t ib,
                      int env_mode, double* keogh_full, double* keogh_mid, double* terms) {
  if (w > m - 1) w = m - 1;
  double* buf = (double*)malloc(sizeof(double) * (size_t)m * 9);
  double *za = buf, *la = buf + m, *ua = buf + 2 * m;
  double *zb = buf + 3 * m, *lb = buf + 4 * m, *ub = buf + 5 * m;
  double *h = buf + 6 * m, *lh = buf + 7 * m, *uh = buf + 8 * m;
  pj_window(a, n, m, w, ia, env_mode, za, la, ua);
  pj_window(a, n, m, w, ib, env_mode, zb, lb, ub);
  double km = 0.0;
  if (keogh_full) *keogh_full = orc_lb_keogh2(za, lb, ub, m);
  for (int k = 0; k < m; ++k) {
    h[k] = za[k];
    if (k >= KIM_BIAS && k < m - KIM_BIAS) {
      if (za[k] > ub[k]) h[k] = ub[k];
      else if (za[k] < lb[k]) h[k] = lb[k];
      km += sq(za[k] - h[k]);
    }
  }
  orc_envelope(h, m, w, lh, uh);
  double t = 0.0;
  for (int k = KIM_BIAS; k < m - KIM_BIAS; ++k) {
    const double x = zb[k];
    if (x > uh[k] && uh[k] > ua[k]) t += sq(x - ua[k]) - sq(uh[k] - ua[k]);
    else if (x < lh[k] && lh[k] < la[k]) t += sq(x - la[k]) - sq(lh[k] - la[k]);
    else if (x > uh[k]) t += sq(x - uh[k]);
    else if (x < lh[k]) t += sq(x - lh[k]);
  }
  *keogh_mid = km;
  *terms = t;
  free(buf);
}
