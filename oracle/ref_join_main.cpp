// Test infrastructure only: runs ONE reference join (CPU_version1's
// DTWMotifDiscoveryGUI through ref_shim.cpp) on a series read from a file and
// prints one JSON line.  bench.py's reference arm starts one such process per
// host core.
//
//   ref_join <series.f64 | series.txt> <m> <w>
//
// A file ending in .txt is read as whitespace-separated ASCII (the reference's
// own format, CPU_version1/loadfile.cpp:14); anything else as raw
// little-endian float64.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <unistd.h>

extern "C" int ref_join(const double* x, long n, int m, int w, const char* timefile,
                        long long* i_out, long long* j_out, double* dist_printed,
                        double* dist_full, double* join_seconds, double* wall_seconds);

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s <series> <m> <w>\n", argv[0]);
    return 2;
  }
  std::string path = argv[1];
  int m = atoi(argv[2]);
  int w = atoi(argv[3]);
  std::vector<double> x;
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) { fprintf(stderr, "cannot open %s\n", path.c_str()); return 2; }
  if (path.size() > 4 && path.compare(path.size() - 4, 4, ".txt") == 0) {
    double v;
    while (fscanf(f, "%lf", &v) == 1) x.push_back(v);
  } else {
    double buf[4096];
    size_t k;
    while ((k = fread(buf, sizeof(double), 4096, f)) > 0) x.insert(x.end(), buf, buf + k);
  }
  fclose(f);
  char timefile[] = "/tmp/dtwj_ref_time_XXXXXX";
  int fd = mkstemp(timefile);
  if (fd >= 0) close(fd);
  long long i = -1, j = -1;
  double dp = 0, df = 0, js = 0, ws = 0;
  int rc = ref_join(x.data(), (long)x.size(), m, w, timefile, &i, &j, &dp, &df, &js, &ws);
  unlink(timefile);
  printf("{\"rc\": %d, \"n\": %zu, \"m\": %d, \"w\": %d, \"i\": %lld, \"j\": %lld, "
         "\"dist_printed\": %.6f, \"dist\": %.17g, \"join_seconds\": %.6f, "
         "\"wall_seconds\": %.6f}\n",
         rc, x.size(), m, w, i, j, dp, df, js, ws);
  return rc;
}
