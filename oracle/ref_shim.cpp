// Test infrastructure only (the oracle): a C ABI around the reference's own
// FP64 CPU implementation (CPU_version1), linked from objects that
// oracle/build_ref.sh compiles out of the reference tree.  Tests, smoke() and
// bench.py's CPU-baseline leg call it through ctypes as the checker; the
// product never links it.
//
// Every function here forwards to the reference function it names:
//   ref_join      -> DTWMotifDiscoveryGUI   CPU_version1/DTWMotifDiscoveryGUI.cpp:12
//                    (mpx_v2 + new_dtw_motifGUI, CPU_version1/new_dtw_motifGUI.cpp:21)
//   ref_mon_dtw   -> MON_dtw                CPU_version1/MON_DTW.cpp:20
//   ref_mvmean    -> mvmean                 CPU_version1/allmatrixop/movmean.cpp:9
//   ref_lemire    -> lower_upper_lemire     CPU_version1/allmatrixop/lower_upper_lemire.cpp:7
//   ref_mpx       -> mpx_v2                 CPU_version1/mpx_v2.cpp:13
//   ref_load      -> loadfile / loadfile_apart / loadfile_2 / loadfile_
//                                           CPU_version1/loadfile.cpp:14,35,63,114
//   ref_mask      -> compute_shared_data_global + compute_MASK_global
//                                           CPU_version1/compute_shared_data_global.cpp:12,
//                                           CPU_version1/compute_MASK_global.cpp:10
//                    with the set-up of new_dtw_motifGUI.cpp:29-45,155-207
//   ref_lb_petitjean -> LB_KK + lbPetitjean_new
//                                           CPU_version1/lb_keogh.cpp:9,
//                                           CPU_version1/LB_PETITJEAN.cpp:10
//                    on windows set up as new_dtw_motifGUI.cpp:28-46 does
#include "alldef/matrix.h"
#include "alldef/allstruct.h"
#include "allunder/underdtw.h"
#include <unistd.h>
#include <fcntl.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <chrono>

RETURN_MPX mpx_v2(const vector<DOUBLE>& timeSeries, int minlag, int subseqlen);
void compute_shared_data_global(const vector<DOUBLE>& ts, int subseqLen,
                                const vector<vector<DOUBLE>>& my_subs, int len_of_table_global,
                                vector<vector<DOUBLE>>& count_table_global);
void compute_MASK_global(const vector<DOUBLE>& a, int subseqLen,
                         const vector<vector<DOUBLE>>& my_subs, int len_of_table_global,
                         vector<vector<DOUBLE>>& count_table_global,
                         const vector<vector<DOUBLE>>& subs_U, const vector<vector<DOUBLE>>& subs_L,
                         vector<DOUBLE>& MASK_global);
vector<DOUBLE> loadfile(string filename);
vector<DOUBLE> loadfile_apart(string filename, int apart);
vector<DOUBLE> loadfile_2(string filename1, string filename2);
vector<DOUBLE> loadfile_(string filename);
void DTWMotifDiscoveryGUI(const vector<DOUBLE>& TS, int subseqlen, int maxwarp,
                          const char* output_time_file_path);

namespace {

// Runs fn() with file descriptor 1 pointed at a temporary file and returns
// everything the reference printed.
template <class F>
std::string capture_stdout(F fn) {
  fflush(stdout);
  std::cout.flush();
  char path[] = "/tmp/dtwj_ref_XXXXXX";
  int fd = mkstemp(path);
  if (fd < 0) { fn(); return std::string(); }
  int saved = dup(1);
  dup2(fd, 1);
  fn();
  fflush(stdout);
  std::cout.flush();
  dup2(saved, 1);
  close(saved);
  std::string out;
  lseek(fd, 0, SEEK_SET);
  char buf[65536];
  ssize_t k;
  while ((k = read(fd, buf, sizeof buf)) > 0) out.append(buf, (size_t)k);
  close(fd);
  unlink(path);
  return out;
}

bool find_double_after(const std::string& s, const char* key, double* v) {
  size_t p = s.rfind(key);
  if (p == std::string::npos) return false;
  return sscanf(s.c_str() + p + strlen(key), "%lf", v) == 1;
}

}  // namespace

extern "C" {

// Squared banded DTW of two equal-length sequences with no early abandoning
// (cumulative bound all zeros, best-so-far effectively infinite).
double ref_mon_dtw(const double* q, const double* t, int m, int w) {
  std::vector<double> a(q, q + m), b(t, t + m), cb((size_t)m + w + 2, 0.0);
  return MON_dtw(a, b, cb, m, w, 1e300);
}

void ref_mvmean(const double* a, long n, int m, double* mu, double* sig) {
  std::vector<double> v(a, a + n);
  long s = n - m + 1;
  std::vector<double> mv(s), sv(s);
  mvmean(v, m, mv, sv);
  for (long i = 0; i < s; ++i) { mu[i] = mv[i]; sig[i] = sv[i]; }
}

// LB_Petitjean of window A = a[ia..) against window B = a[ib..) as the
// reference's join evaluates it (new_dtw_motifGUI.cpp:508-519, with A the
// window i + diag - 2 and B the window i - 1): the windows z-normalised with
// mvmean's statistics and each given its clipped envelope by
// lower_upper_lemire.  keogh = LB_KK of A against B's envelope with no
// endpoint part and no threshold (the squared LB_Keogh over all m samples);
// terms = what lbPetitjean_new adds to a zero lbk2 with no threshold.
void ref_lb_petitjean(const double* a, long n, int m, int w, long ia, long ib,
                      double* keogh, double* terms) {
  std::vector<double> v(a, a + n);
  const long s = n - m + 1;
  std::vector<double> mu(s), sig(s);
  mvmean(v, m, mu, sig);
  std::vector<double> A(m), B(m), la(m), ua(m), lb(m), ub(m);
  for (int k = 0; k < m; ++k) {
    A[k] = (a[ia + k] - mu[ia]) / sig[ia];
    B[k] = (a[ib + k] - mu[ib]) / sig[ib];
  }
  lower_upper_lemire(A, m, w, la, ua);
  lower_upper_lemire(B, m, w, lb, ub);
  std::vector<double> cb(m, 0.0), proj(m), up(m), lp(m);
  double sv[2] = {0.0, 0.0};
  double lbk = 0.0;
  LB_KK(A, ub.data(), lb.data(), m, 1e300, cb, sv, lbk);
  *keogh = lbk;
  double t = 0.0;
  std::fill(cb.begin(), cb.end(), 0.0);
  lbPetitjean_new(proj, A, up, lp, ua.data(), la.data(), B, ub.data(), lb.data(), w, m, 1e300,
                  t, cb, mu[ia], sig[ia]);
  *terms = t;
}

void ref_lemire(const double* a, int n, int r, double* lower, double* upper) {
  std::vector<double> v(a, a + n), l(n), u(n);
  lower_upper_lemire(v, n, r, l, u);
  for (int i = 0; i < n; ++i) { lower[i] = l[i]; upper[i] = u[i]; }
}

// ED matrix profile with exclusion zone m: mp = z-normalised Euclidean
// distance, mpi = 1-based index of the nearest neighbour (reference layout).
void ref_mpx(const double* a, long n, int m, double* mp, int* mpi) {
  std::vector<double> v(a, a + n);
  RETURN_MPX r;
  capture_stdout([&] { r = mpx_v2(v, m, m); });
  for (size_t i = 0; i < r.matrixProfile.size(); ++i) {
    mp[i] = r.matrixProfile[i];
    mpi[i] = r.matrixProfileIdx[i];
  }
}

// One full reference join (mpx_v2 + new_dtw_motifGUI).  Outputs 0-based pair
// indices, the distance as printed (%f), the distance recomputed at full FP64
// precision with the reference's own z-normalisation and MON_dtw, the
// reference's own join time (clock() t1->t2) and the wall time of the call.
// Returns 0 on success, 1 if the reference's output could not be parsed.
int ref_join(const double* x, long n, int m, int w, const char* timefile,
             long long* i_out, long long* j_out, double* dist_printed,
             double* dist_full, double* join_seconds, double* wall_seconds) {
  std::vector<double> ts(x, x + n);
  auto t0 = std::chrono::steady_clock::now();
  std::string out = capture_stdout([&] { DTWMotifDiscoveryGUI(ts, m, w, timefile); });
  auto t1 = std::chrono::steady_clock::now();
  *wall_seconds = std::chrono::duration<double>(t1 - t0).count();
  double fm = 0, sm = 0, dist = 0, secs = 0;
  size_t p = out.rfind("first min is ");
  if (p == std::string::npos ||
      sscanf(out.c_str() + p, "first min is %lf sec min is %lf", &fm, &sm) != 2)
    return 1;
  if (!find_double_after(out, "final distance :", &dist)) return 1;
  if (!find_double_after(out, "total time is ", &secs)) secs = -1;
  long long i0 = (long long)llround(fm) - 1, j0 = (long long)llround(sm) - 1;
  *i_out = i0;
  *j_out = j0;
  *dist_printed = dist;
  *join_seconds = secs;
  // Full-precision distance of the reported pair, z-normalised exactly as
  // new_dtw_motifGUI does ((a - mu) / sig with mvmean's statistics).
  long s = n - m + 1;
  std::vector<double> mu(s), sig(s);
  mvmean(ts, m, mu, sig);
  *dist_full = NAN;
  if (i0 >= 0 && j0 >= 0 && i0 < s && j0 < s) {
    std::vector<double> q(m), t(m), cb((size_t)m + w + 2, 0.0);
    for (int k = 0; k < m; ++k) {
      q[k] = (ts[i0 + k] - mu[i0]) / sig[i0];
      t[k] = (ts[j0 + k] - mu[j0]) / sig[j0];
    }
    *dist_full = std::sqrt(MON_dtw(q, t, cb, m, w, 1e300));
  }
  return 0;
}

// The reference's global mask of series a (n samples, windows m, band w), set
// up as new_dtw_motifGUI does: mvmean statistics, z-normalised subsequences
// and their lower_upper_lemire envelopes (:29-45), the CDF table length from
// the largest |z| (:155-197), then the two reference functions (:201-207).
// Writes mask[n] (0/1) and the table length; returns 0.
int ref_mask(const double* x, long n, int m, int w, double* mask, int* table_len) {
  std::vector<double> a(x, x + n);
  const long s = n - m + 1;
  std::vector<double> mu(s), sig(s);
  mvmean(a, m, mu, sig);
  vector<vector<DOUBLE>> subs((size_t)s, vector<DOUBLE>(m)), U((size_t)s, vector<DOUBLE>(m)),
      L((size_t)s, vector<DOUBLE>(m));
  DOUBLE vmax = 0, vmin = 0;
  for (long i = 0; i < s; ++i) {
    for (int j = 0; j < m; ++j) subs[i][j] = (a[i + j] - mu[i]) / sig[i];
    lower_upper_lemire(subs[i], m, w, L[i], U[i]);
  }
  vmax = vmin = subs[0][0];
  for (const auto& r : subs)
    for (auto v : r) {
      if (v > vmax) vmax = v;
      if (v < vmin) vmin = v;
    }
  DOUBLE mrv = floor(MAX(std::abs(vmax), std::abs(vmin))) * 2 * 100;
  int lt = static_cast<int>(MAX(INITIAL_LEN_OF_TABLE, mrv));
  vector<vector<DOUBLE>> table((size_t)m, vector<DOUBLE>((size_t)lt, 0.0));
  compute_shared_data_global(a, m, subs, lt, table);
  vector<DOUBLE> M((size_t)n, 0.0);
  compute_MASK_global(a, m, subs, lt, table, U, L, M);
  for (long p = 0; p < n; ++p) mask[p] = M[p];
  *table_len = lt;
  return 0;
}

// The reference's loaders: format 0 loadfile, 1 loadfile_apart(param),
// 2 loadfile_2(path, path2), 3 loadfile_.  Writes up to cap values, returns
// how many the loader produced.  (The reference exits on a file it cannot
// open: call it with readable files only.)
long ref_load(const char* path, const char* path2, int format, int param, double* out,
              long cap) {
  vector<DOUBLE> v;
  if (format == 0) v = loadfile(path);
  else if (format == 1) v = loadfile_apart(path, param);
  else if (format == 2) v = loadfile_2(path, path2);
  else v = loadfile_(path);
  for (long k = 0; k < (long)v.size() && k < cap; ++k) out[k] = (double)v[(size_t)k];
  return (long)v.size();
}

}  // extern "C"
