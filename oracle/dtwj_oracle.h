/* TEST INFRASTRUCTURE ONLY — the oracle.
 *
 * A plain-C FP64 restatement of the reference's top-1 z-normalised DTW
 * subsequence self-join (CPU_version1/new_dtw_motifGUI.cpp:21-586 and the
 * functions it calls).  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load it, and only as the checker; the product library
 * never links it.  Build: oracle/Makefile -> oracle/_build/liboracle.so.
 *
 * Conventions (shared with the product):
 *   n  series length, m subsequence length, w Sakoe-Chiba band,
 *   s = n - m + 1 subsequences, pair (i, j) with j - i >= m (exclusion zone
 *   of the reference: minlag = m, new_dtw_motifGUI.cpp:182), 0-based.
 *   Distances are z-normalised DTW (not squared) unless a name ends in 2.
 */
#ifndef DTWJ_ORACLE_H
#define DTWJ_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int64_t i, j;            /* top-1 pair, 0-based, i < j, lowest (dist, i, j) */
  double dist;             /* DTW distance (sqrt of the squared cost)         */
  double seed_bsf;         /* best-so-far after the ED-seeded DTW seeds        */
  uint64_t pairs;          /* candidate pairs (j - i >= m, no flat window)    */
  uint64_t pruned_fast;    /* pruned by diag_fast                              */
  uint64_t pruned_masked;  /* pruned by diag_mask_global's masked bound        */
  uint64_t pruned_kim;     /* pruned by the endpoint (LB_Kim-style) bound      */
  uint64_t pruned_keogh;   /* pruned by LB_Keogh (either direction)            */
  uint64_t dtw_calls;      /* early-abandoning DTW evaluations                 */
  uint64_t dtw_abandoned;  /* of which abandoned                               */
  double seconds;          /* wall time of the join                            */
  int threads;             /* OpenMP threads used                              */
} orc_result;

/* flags for orc_join */
#define ORC_NO_DIAG    1u   /* skip the diagonal bounds (LB_Keogh + DTW only) */
#define ORC_NO_MASKED  2u   /* skip diag_mask_global's masked bound          */
#define ORC_NO_SEED    4u   /* start from an infinite best-so-far            */

void orc_stats(const double* a, int64_t n, int m, double* mu, double* sig);
void orc_envelope(const double* a, int64_t n, int r, double* lower, double* upper);
double orc_dtw2(const double* q, const double* t, int m, int w);
double orc_dtw2_ea(const double* q, const double* t, const double* cb, int m, int w,
                   double bsf2);
void orc_mp(const double* a, int64_t n, int m, double* mp, int64_t* mpi);
int orc_mask(const double* a, int64_t n, int m, int w, double* mask, int* table_len);
double orc_lb_keogh2(const double* q, const double* lower, const double* upper, int m);
void orc_kim2(const double* q, const double* t, int m, double* left, double* right);
int orc_join(const double* a, int64_t n, int m, int w, unsigned flags, int threads,
             orc_result* out);
double orc_pair_dist(const double* a, int64_t n, int m, int w, int64_t i, int64_t j);
/* LB_Petitjean of window A = a[ia, ia + m) against window B = a[ib, ib + m)
 * (lbPetitjean_new, CPU_version1/LB_PETITJEAN.cpp:10-123).  env_mode 1: the
 * clipped per-window envelopes of the z-normalised windows, as the reference
 * builds them (subs_U / subs_L, new_dtw_motifGUI.cpp:45); env_mode 0: the
 * raw series' envelope of radius w, normalised with each window's own
 * statistics (what the GPU join reads).  w >= m is taken as m - 1.
 * keogh_full = squared LB_Keogh of A against B's envelope over all m samples
 * (may be NULL); keogh_mid = the same over k in [3, m-4], i.e. the sum of
 * (A_k - H_k)^2 with H = A projected onto B's envelope; terms = the
 * projection part summed over the same k. */
void orc_lb_petitjean(const double* a, int64_t n, int m, int w, int64_t ia, int64_t ib,
                      int env_mode, double* keogh_full, double* keogh_mid, double* terms);

#ifdef __cplusplus
}
#endif
#endif
