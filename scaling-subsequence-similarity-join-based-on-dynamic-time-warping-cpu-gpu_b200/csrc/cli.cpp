// dtwj — drop-in for the reference executables GPU_dtw.exe / CPU_dtw.exe.
//
//   dtwj <data_path> <time_out_path> <m> <ratio> [options]
//
// argv[1..4] mean what they mean for the reference (README.md:15-34,
// GPU_version1/src/AAAA.cu:17-36): the series file (whitespace-separated
// ASCII, read like loadfile, GPU_version1/src/loadfile.cu:14-33), the file
// the join time is appended to ("%lf\n", new_dtw_motifGUI_malloc.cu:750-753),
// the subsequence length and the band ratio.  Like the reference, an
// unopenable data file prints "Error opening file: <path>" and exits with 0.
//
// Options:
//   --band-rounding=ceil|round  w = ceil(ratio*m) (default) or the reference
//                               executables' max(round(ratio*m), 1)
//   --band=W                    explicit band, overrides the ratio
//   --format=values|every|first-column|rows|binary
//                               how the data file is read (dtwj_load): every
//                               number (default, loadfile), every N-th
//                               (loadfile_apart), the first number of each line
//                               (loadfile_2, with --data2 as its second file),
//                               a matrix row by row (loadfile_), raw float64
//   --every=N                   N for --format=every
//   --data2=PATH                second file for --format=first-column
//   --binary                    same as --format=binary
//   --json=PATH                 also write the full result as JSON
//   --masked-cascade            the reference's masked diagonal bound and
//                               endpoint bound as the run filter
//   --petitjean                 LB_Petitjean between LB_Keogh and DTW
//   --no-masked, --no-seed      disable the masked bound (with
//                               --masked-cascade) / ED seeding
//   --verbose                   phase timings on stderr
#include "../../include/dtwj.h"

#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

int main(int argc, char** argv) {
  if (argc < 5) {
    fprintf(stderr,
            "usage: %s <data_path> <time_out_path> <m> <ratio> [--band-rounding=ceil|round]"
            " [--band=W] [--format=values|every|first-column|rows|binary] [--every=N]"
            " [--data2=PATH] [--binary] [--json=PATH] [--masked-cascade] [--petitjean]"
            " [--no-masked] [--no-seed] [--verbose]\n",
            argv[0]);
    return 2;
  }
  const char* data = argv[1];
  const char* time_out = argv[2];
  const int m = atoi(argv[3]);
  const double ratio = atof(argv[4]);
  int rounding = 0, band = -1, format = DTWJ_LOAD_VALUES, every = 1;
  std::string data2;
  std::string json;
  uint32_t flags = 0;
  for (int k = 5; k < argc; ++k) {
    const char* a = argv[k];
    if (!strcmp(a, "--band-rounding=round")) rounding = 1;
    else if (!strcmp(a, "--band-rounding=ceil")) rounding = 0;
    else if (!strncmp(a, "--band=", 7)) band = atoi(a + 7);
    else if (!strcmp(a, "--binary") || !strcmp(a, "--format=binary")) format = DTWJ_LOAD_BINARY;
    else if (!strcmp(a, "--format=values")) format = DTWJ_LOAD_VALUES;
    else if (!strcmp(a, "--format=every")) format = DTWJ_LOAD_EVERY;
    else if (!strcmp(a, "--format=first-column")) format = DTWJ_LOAD_FIRST_COLUMN;
    else if (!strcmp(a, "--format=rows")) format = DTWJ_LOAD_ROWS;
    else if (!strncmp(a, "--every=", 8)) every = atoi(a + 8);
    else if (!strncmp(a, "--data2=", 8)) data2 = a + 8;
    else if (!strncmp(a, "--json=", 7)) json = a + 7;
    else if (!strcmp(a, "--masked-cascade")) flags |= DTWJ_F_MASKED_CASCADE;
    else if (!strcmp(a, "--petitjean")) flags |= DTWJ_F_PETITJEAN;
    else if (!strcmp(a, "--no-masked")) flags |= DTWJ_F_NO_MASKED;
    else if (!strcmp(a, "--no-seed")) flags |= DTWJ_F_NO_SEED;
    else if (!strcmp(a, "--verbose")) flags |= DTWJ_F_VERBOSE;
    else {
      fprintf(stderr, "unknown option %s\n", a);
      return 2;
    }
  }
  std::vector<double> x;
  int64_t n = 0;
  const char* d2 = data2.empty() ? nullptr : data2.c_str();
  int lrc = dtwj_load(data, d2, format, every, nullptr, 0, &n);
  if (lrc == DTWJ_OK) {
    x.resize((size_t)n);
    lrc = dtwj_load(data, d2, format, every, x.data(), n, &n);
  }
  if (lrc == DTWJ_ERR_IO) {
    // as the reference: report and exit with 0 (GPU_version1/src/loadfile.cu:17-21)
    fprintf(stderr, "Error opening file: %s\n", data);
    return 0;
  }
  if (lrc != DTWJ_OK) {
    fprintf(stderr, "dtwj: %s\n", dtwj_strerror(lrc));
    return 2;
  }
  const int w = band >= 0 ? band : dtwj_band(m, ratio, rounding);
  printf("buffer_length: %d, maxwarp: %d\n", m, w);
  printf("the buffer_length of TS is %zu\n", x.size());
  dtwj_result r;
  const int rc = dtwj_join(x.data(), (int64_t)x.size(), m, w, flags, &r);
  if (rc != DTWJ_OK) {
    fprintf(stderr, "dtwj: %s\n", dtwj_strerror(rc));
    return 1;
  }
  // reference output lines (1-based indices, new_dtw_motifGUI.cpp:575-579)
  printf("first min is %" PRId64 " sec min is %" PRId64 "\n", r.i + 1, r.j + 1);
  printf("total time is %fs   input of bsf:%5.3f  ,final distance :%f  \n", r.seconds_join,
         r.seed_bsf, r.dist);
  printf("pair (0-based) %" PRId64 " %" PRId64 "  distance %.17g\n", r.i, r.j, r.dist);
  FILE* op = fopen(time_out, "a");
  if (op) {
    fprintf(op, "%lf", r.seconds_join);
    fprintf(op, "\n");
    fclose(op);
  }
  if (!json.empty()) {
    FILE* jf = fopen(json.c_str(), "w");
    if (!jf) {
      fprintf(stderr, "dtwj: cannot write %s\n", json.c_str());
      return 1;
    }
    fprintf(jf,
            "{\"i\": %" PRId64 ", \"j\": %" PRId64 ", \"dist\": %.17g, \"dist_fp32\": %.9g, "
            "\"seed_bsf\": %.9g, \"n\": %" PRId64 ", \"m\": %d, \"w\": %d, \"pairs\": %llu, "
            "\"pruned_fast\": %llu, \"pruned_kim\": %llu, \"pruned_masked\": %llu, "
            "\"pruned_keogh\": %llu, \"dtw_calls\": %llu, \"dtw_abandoned\": %llu, "
            "\"dtw_cells\": %llu, \"candidates\": %llu, \"seconds_join\": %.6f, "
            "\"seconds_total\": %.6f}\n",
            r.i, r.j, r.dist, r.dist_fp32, r.seed_bsf, r.n, r.m, r.w,
            (unsigned long long)r.pairs, (unsigned long long)r.pruned_fast,
            (unsigned long long)r.pruned_kim, (unsigned long long)r.pruned_masked,
            (unsigned long long)r.pruned_keogh, (unsigned long long)r.dtw_calls,
            (unsigned long long)r.dtw_abandoned, (unsigned long long)r.dtw_cells,
            (unsigned long long)r.candidates, r.seconds_join, r.seconds_total);
    fclose(jf);
  }
  return 0;
}
