// Allocation-free pair DTW: dtwj_pair_dtw_noalloc (include/dtwj.h).
//
// For callers that must not allocate device memory after start-up - a host
// framework that reserves the whole device at initialisation and fails or
// stalls later cudaMalloc calls, or a latency-bound loop that cannot afford
// the implicit synchronisation of cudaMalloc/cudaFree.  The caller passes
// device pointers for the series, the pair lists and the output; the only
// scratch (the window statistics) lives in one file-scope __device__ array
// of fixed size, which every GPU that loads this library keeps until exit.
#include "../../include/dtwj.h"
#include "dtwj_dev.cuh"

#include <climits>
#include <cstring>

namespace dtwj {
void launch_stats(const DevSeries& S, cudaStream_t st);
void launch_pair_dtw64(const DevSeries& S, const int64_t* pi, const int64_t* pj, int64_t count,
                       bool precise, BandShape band, double* out, cudaStream_t st);
}  // namespace dtwj

using namespace dtwj;

namespace {

// Windows the fixed scratch holds: mean, deviation, inverse deviation (FP64)
// and a flat flag (byte) per window, 25 bytes each -> 6.25 MiB.
constexpr int64_t kMaxWindows = DTWJ_NOALLOC_MAX_WINDOWS;
constexpr size_t kScratchBytes = (size_t)kMaxWindows * 25;

static __device__ __align__(256) unsigned char g_pair_scratch[kScratchBytes];

// Device address of the scratch on the current device.  The host-side name
// of the array is only a stand-in, so the address is looked up on every call
// with the caller's device current: the lookup allocates nothing, and it stays
// right after cudaDeviceReset, when the module may come back elsewhere.
int scratch_address(void** out) {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_pair_scratch) != cudaSuccess || !p) {
    cudaGetLastError();
    return DTWJ_ERR_CUDA;
  }
  *out = p;
  return DTWJ_OK;
}

}  // namespace

extern "C" int dtwj_pair_dtw_noalloc(const double* x_dev, int64_t n, int32_t m, int32_t w,
                                     const int64_t* pi_dev, const int64_t* pj_dev, int64_t count,
                                     int32_t precise, double* dist_dev, void* stream) {
  if (!x_dev || count < 0 || (count > 0 && (!pi_dev || !pj_dev || !dist_dev))) return DTWJ_ERR_ARG;
  if (m < 8 || m > DTWJ_MAX_M || w < 0 || n < 2 * (int64_t)m + 1 || n > (int64_t)INT32_MAX - 4)
    return DTWJ_ERR_ARG;
  const int64_t s = n - m + 1;
  if (s > kMaxWindows) return DTWJ_ERR_SCRATCH;
  if (count == 0) return DTWJ_OK;
  const int we = w > m - 1 ? m - 1 : w;
  BandShape band;
  if (!choose_band_list(we, &band)) return DTWJ_ERR_BAND;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return DTWJ_ERR_NODEVICE;
  }
  void* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  unsigned char* b = static_cast<unsigned char*>(base);
  DevSeries S;
  memset(&S, 0, sizeof S);
  S.a = x_dev;
  S.n = n;
  S.s = s;
  S.m = m;
  S.w = we;
  S.mu = reinterpret_cast<double*>(b);
  S.sig = reinterpret_cast<double*>(b + 8 * kMaxWindows);
  S.isg = reinterpret_cast<double*>(b + 16 * kMaxWindows);
  S.flat = b + 24 * kMaxWindows;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  launch_stats(S, st);
  launch_pair_dtw64(S, pi_dev, pj_dev, count, precise != 0, band, dist_dev, st);
  if (cudaGetLastError() != cudaSuccess) return DTWJ_ERR_CUDA;
  return DTWJ_OK;
}
