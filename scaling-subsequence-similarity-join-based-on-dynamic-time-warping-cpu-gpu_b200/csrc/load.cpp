// Series file readers for the formats of the reference's loaders
// (CPU_version1/loadfile.cpp:14-142, GPU_version1/src/loadfile.cu:13-148),
// host code.  Numbers are read with the C++ stream extraction the reference
// uses, so a token that is not a number ends the read (of the file, or of the
// line for the line formats) as it does there.
#include "../../include/dtwj.h"

#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace {

bool read_values(const char* path, std::vector<double>* out) {
  std::ifstream f(path);
  if (!f.is_open()) return false;
  double v;
  while (f >> v) out->push_back(v);
  return true;
}

// Every line of the file as the numbers it starts with.
bool read_rows(const char* path, std::vector<std::vector<double>>* rows) {
  std::ifstream f(path);
  if (!f.is_open()) return false;
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream iss(line);
    std::vector<double> row;
    double v;
    while (iss >> v) row.push_back(v);
    rows->push_back(std::move(row));
  }
  return true;
}

bool read_binary(const char* path, std::vector<double>* out) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  double buf[8192];
  size_t k;
  while ((k = fread(buf, sizeof(double), 8192, f)) > 0) out->insert(out->end(), buf, buf + k);
  fclose(f);
  return true;
}

}  // namespace

extern "C" int dtwj_load(const char* path, const char* path2, int32_t format, int32_t param,
                         double* out, int64_t cap, int64_t* n) {
  if (!path || !n || (out == nullptr && cap != 0) || cap < 0) return DTWJ_ERR_ARG;
  std::vector<double> x;
  switch (format) {
    case DTWJ_LOAD_VALUES:
      if (!read_values(path, &x)) return DTWJ_ERR_IO;
      break;
    case DTWJ_LOAD_EVERY: {
      if (param < 1) return DTWJ_ERR_ARG;
      std::vector<double> all;
      if (!read_values(path, &all)) return DTWJ_ERR_IO;
      for (size_t k = 0; k < all.size(); k += (size_t)param) x.push_back(all[k]);
      break;
    }
    case DTWJ_LOAD_FIRST_COLUMN: {
      std::vector<std::vector<double>> rows;
      if (!read_rows(path, &rows)) return DTWJ_ERR_IO;
      if (path2 && !read_rows(path2, &rows)) return DTWJ_ERR_IO;
      for (const auto& r : rows)
        if (!r.empty()) x.push_back(r[0]);
      break;
    }
    case DTWJ_LOAD_ROWS: {
      std::vector<std::vector<double>> rows;
      if (!read_rows(path, &rows)) return DTWJ_ERR_IO;
      if (!rows.empty()) {
        const size_t width = rows[0].size();
        for (const auto& r : rows) {
          if (r.size() < width) return DTWJ_ERR_IO;  // ragged: shorter than the first row
          x.insert(x.end(), r.begin(), r.begin() + (long)width);
        }
      }
      break;
    }
    case DTWJ_LOAD_BINARY:
      if (!read_binary(path, &x)) return DTWJ_ERR_IO;
      break;
    default:
      return DTWJ_ERR_ARG;
  }
  *n = (int64_t)x.size();
  for (int64_t k = 0; k < *n && k < cap; ++k) out[k] = x[(size_t)k];
  return DTWJ_OK;
}
