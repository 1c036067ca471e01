// Features of the diagonal-sweep tiles for the learned ordering (no
// counterpart in the reference).  One warp per tile, FP64 arithmetic, 64
// values per tile (float):
//
//   [0, 8)    PAA-8 (segment means) of the z-normalised window at the tile's
//             centre row ic = i0 + rows / 2
//   [8, 16)   PAA-8 of the window at the centre column jc = ic + Lc,
//             Lc = the tile's middle lag (clamped to the series)
//   [16, 24)  |PAA(ic) - PAA(jc)|
//   [24, 32)  per eighth of the rows: min over its rows of the row's ED
//             matrix-profile value / sqrt(2m) (nearest neighbour j >= i + m)
//   [32, 40)  per eighth of the rows: fraction of rows whose ED nearest
//             neighbour lies in the tile's lag range
//   [40, 48)  ED / sqrt(2m) of the pairs (r_k, r_k + Lc), r_k = i0 + (2k + 1)
//             rows / 16
//   [48, 56)  sqrt(LB_Keogh) / sqrt(2m) of the same pairs (window r_k against
//             the raw envelope of r_k + Lc, normalised by its window)
//   [56, 64)  L0 / s, i0 / s, rows / kLbRows, lags / kLbLags, m / 1024, w / m,
//             the smallest profile value of the tile's rows / sqrt(2m), 1
//
// The matrix-profile keys are those of the profile pass: high 32 bits of the
// FP64 squared distance with the 3 lowest cleared, low 32 bits the partner
// (ULLONG_MAX: none).
#include "dtwj_dev.cuh"

#include <climits>

namespace dtwj {
namespace {

constexpr int kFeat = 64;

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double wmin(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Profile value of row i as d / sqrt(2m) (+inf when the row has no partner).
__device__ __forceinline__ double mp_value(unsigned long long key, double inv_norm) {
  if (key == ULLONG_MAX) return __longlong_as_double(0x7ff0000000000000LL);
  const double d2 = __longlong_as_double((long long)(key & 0xffffffff00000000ull));
  return sqrt(fmax(d2, 0.0)) * inv_norm;
}

__global__ void k_tile_features(DevSeries S, const Tile* tiles, int ntiles,
                                const unsigned long long* keys, int grid, float* out) {
  const int lane = threadIdx.x & 31;
  const int t = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  if (t >= ntiles) return;
  const Tile T = tiles[t];
  const int m = S.m;
  const double inv_norm = 1.0 / sqrt(2.0 * m);
  const double INF = __longlong_as_double(0x7ff0000000000000LL);
  const int64_t wb = S.sbeg ? S.sbeg[T.series] : 0;  // the series' first window
  const int64_t s = T.send - wb;                        // its window count
  const int64_t lags = (int64_t)T.send - 1 - T.i0 - T.L0 + 1 < kLbLags
                           ? (int64_t)T.send - 1 - T.i0 - T.L0 + 1
                           : kLbLags;
  const int64_t ic = T.i0 + T.rows / 2;
  int64_t Lc = T.L0 + lags / 2;
  if (ic + Lc > T.send - 1) Lc = T.send - 1 - ic;
  if (Lc < m) Lc = m;
  const int64_t jc = ic + Lc;
  float* f = out + (size_t)t * kFeat;

  // PAA-8 of windows ic and jc (segment k: [k m / 8, (k + 1) m / 8))
  double pi_[8], pj_[8];
  const double mi = S.mu[ic], si = S.isg[ic], mj = S.mu[jc], sj = S.isg[jc];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int a = k * m / 8, b = (k + 1) * m / 8;
    double ai = 0.0, aj = 0.0;
    for (int x = a + lane; x < b; x += 32) {
      ai += (S.a[ic + x] - mi) * si;
      aj += (S.a[jc + x] - mj) * sj;
    }
    ai = wsum(ai);
    aj = wsum(aj);
    pi_[k] = b > a ? ai / (b - a) : 0.0;
    pj_[k] = b > a ? aj / (b - a) : 0.0;
  }
  // profile minima and in-range fractions per eighth of the rows
  double mpmin[8], frac[8];
  double tile_min = INF;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int a = k * T.rows / 8, b = (k + 1) * T.rows / 8;
    double mn = INF, cnt = 0.0;
    // only the keyed rows (every row, or the seed profile's grid rows)
    for (int r = (a + grid - 1) / grid * grid + lane * grid; r < b; r += 32 * grid) {
      const int64_t i = T.i0 + r;
      const unsigned long long key = keys[i];
      mn = fmin(mn, mp_value(key, inv_norm));
      if (key != ULLONG_MAX) {
        const int64_t lag = (int64_t)(unsigned int)(key & 0xffffffffu) - i;
        if (lag >= T.L0 && lag < T.L0 + lags) cnt += 1.0;
      }
    }
    mn = wmin(mn);
    cnt = wsum(cnt);
    mpmin[k] = mn;
    // rows that carry a key: every row, or the rows r % grid == 0 of the seed
    // profile's grid (a tile starts on its series' grid)
    const int keyed = (b + grid - 1) / grid - (a + grid - 1) / grid;
    frac[k] = keyed > 0 ? cnt / keyed : 0.0;
    tile_min = fmin(tile_min, mn);
  }
  // ED and LB_Keogh of 8 sample pairs at the middle lag
  double ed[8], lbk[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int64_t r = T.i0 + (int64_t)(2 * k + 1) * T.rows / 16;
    int64_t L = Lc;
    if (r + L > T.send - 1) L = T.send - 1 - r;
    double e = INF, l = INF;
    if (L >= m) {
      const int64_t j = r + L;
      const double mr = S.mu[r], sr = S.isg[r], mc = S.mu[j], sc = S.isg[j];
      double ae = 0.0, al = 0.0;
      for (int x = lane; x < m; x += 32) {
        const double zr = (S.a[r + x] - mr) * sr, zc = (S.a[j + x] - mc) * sc;
        const double u = (S.U[j + x] - mc) * sc, lo = (S.L[j + x] - mc) * sc;
        ae += (zr - zc) * (zr - zc);
        const double d = fmax(fmax(zr - u, lo - zr), 0.0);
        al += d * d;
      }
      e = sqrt(wsum(ae)) * inv_norm;
      l = sqrt(wsum(al)) * inv_norm;
    }
    ed[k] = e;
    lbk[k] = l;
  }
  // a missing value (no sample pair, no partner) is written as 4, above any
  // z-normalised ED / sqrt(2m) (at most 2)
  auto fin = [](double v) { return (float)(v < 1e300 ? v : 4.0); };
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      f[k] = (float)pi_[k];
      f[8 + k] = (float)pj_[k];
      f[16 + k] = (float)fabs(pi_[k] - pj_[k]);
      f[24 + k] = fin(mpmin[k]);
      f[32 + k] = (float)frac[k];
      f[40 + k] = fin(ed[k]);
      f[48 + k] = fin(lbk[k]);
    }
    f[56] = (float)((double)(T.L0) / (double)s);
    f[57] = (float)((double)(T.i0 - wb) / (double)s);
    f[58] = (float)((double)T.rows / kLbRows);
    f[59] = (float)((double)lags / kLbLags);
    f[60] = (float)(m / 1024.0);
    f[61] = (float)((double)S.w / m);
    f[62] = fin(tile_min);
    f[63] = 1.0f;
  }
}

}  // namespace

void launch_tile_features(const DevSeries& S, const Tile* tiles, int ntiles,
                          const unsigned long long* keys, int grid, float* out,
                          cudaStream_t st) {
  if (ntiles <= 0) return;
  const int per_block = 4;  // warps
  k_tile_features<<<(ntiles + per_block - 1) / per_block, 32 * per_block, 0, st>>>(
      S, tiles, ntiles, keys, grid, out);
}

}  // namespace dtwj
