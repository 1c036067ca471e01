// Tile-scoring MLP of the learned ordering: 64 -> 128 -> 128 -> 1 with ReLU,
// mean squared error, Adam.  No counterpart in the reference.
//
// Every layer is a GEMM on the 5th-generation tensor cores (tcgen05.mma,
// BF16 operands staged in shared memory, FP32 accumulator in tensor memory),
// FP32 activations and FP32 master weights; the BF16 copies of W1 and W2 are
// refreshed after every Adam step.  A SIMT FP32 GEMM with the same interface
// is the debug path the gradient check compares against (`precise`).
//
// Parameter layout (FP32, 24,961 values): W1 [128][64], b1 [128],
// W2 [128][128], b2 [128], w3 [128], b3 [1].
//
// Forward, batch X [B][64]:  H1 = relu(X W1^T + b1), H2 = relu(H1 W2^T + b2),
// y = H2 w3 + b3.  Backward of L = mean (y - t)^2:  dy = 2 (y - t) / B,
// dw3 = H2^T dy, db3 = sum dy, dH2 = dy w3^T . [H2 > 0], dW2 = dH2^T H1,
// db2 = colsum dH2, dH1 = dH2 W2 . [H1 > 0], dW1 = dH1^T X, db1 = colsum dH1.
#include "../../include/dtwj.h"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

namespace {

constexpr int kIn = DTWJ_MLP_IN, kHid = DTWJ_MLP_HIDDEN;
constexpr int64_t kOffW1 = 0, kOffB1 = kOffW1 + kHid * kIn, kOffW2 = kOffB1 + kHid,
                  kOffB2 = kOffW2 + kHid * kHid, kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid,
                  kNumParams = kOffB3 + 1;
static_assert(kNumParams == DTWJ_MLP_PARAMS, "parameter layout");
constexpr int kMaxBatch = 8192;
constexpr int kThreads = 256;

using bf16 = __nv_bfloat16;

unsigned grid_for(int64_t n, int t = kThreads) {
  int64_t g = (n + t - 1) / t;
  if (g > 148 * 32) g = 148 * 32;
  return (unsigned)(g < 1 ? 1 : g);
}

// ---- GEMM: C[m][n] (+)= sum_k A(m, k) B(k, n) ----
// A(m, k) = A[m * sam + k * sak], B(k, n) = B[k * sbk + n * sbn], C row-major
// with leading dimension ldc.
//
// BF16 path on the 5th-generation tensor cores: a CTA of 4 warps computes
// 128 rows x N columns (N <= 128, a multiple of 16) in a tensor-memory
// accumulator.  K runs in stages of 64: the 4 warps stage the A and B tiles
// (B transposed, both K-major) in shared memory in the canonical layout
// without swizzle (8-row x 16-byte core matrices; the two core matrices of a
// K-step of 16 are 128 bytes apart, 8-row groups 1024 bytes apart), one
// thread issues the stage's four tcgen05.mma (M = 128, K = 16 each) and
// commits them to an mbarrier, which every thread waits on before the next
// stage overwrites the tiles.  Each warp then reads its 32 rows of the
// accumulator (tcgen05.ld) and writes them to C.  The MLP's operands have
// arbitrary strides (transposed operands in the weight gradients), so the
// tiles are staged with ordinary loads rather than tensor-map copies.

__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
  const uint32_t l = __bfloat16_as_ushort(lo), h = __bfloat16_as_ushort(hi);
  return l | (h << 16);
}

constexpr int kTcRows = 128;   // rows of A (and of the accumulator) per CTA
constexpr int kTcK = 64;       // K per stage
constexpr int kTcCols = 128;   // accumulator columns allocated (N <= 128)
constexpr uint32_t kTcLbo = 128, kTcSbo = 1024;  // canonical K-major strides, bytes
constexpr int kTcWaitLimit = 1 << 24;            // mbarrier polls before giving up

struct TcSmem {
  alignas(1024) bf16 a[kTcRows * kTcK];
  alignas(1024) bf16 b[kTcCols * kTcK];
  alignas(8) uint64_t mbar;
  uint32_t tmem;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, k) of a K-major tile of kTcK columns.
__device__ __forceinline__ uint32_t tc_offset(int r, int k) {
  return (uint32_t)((r & 7) * 16 + (r >> 3) * kTcSbo + (k & 7) * 2 + (k >> 3) * kTcLbo);
}

// Shared-memory matrix descriptor: start address, leading (K) and stride
// (8-row group) byte offsets in 16-byte units, descriptor version 1, no
// swizzle.
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((kTcLbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((kTcSbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// Polls the mbarrier for `phase`; false if it did not complete within the limit.
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t phase) {
  for (int it = 0; it < kTcWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done) : "r"(mbar), "r"(phase) : "memory");
    if (done) return true;
  }
  return false;
}

// Reads 32 accumulator columns of this warp's 32 lanes (one row per thread).
__device__ __forceinline__ void tc_load32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Stages 128 (or N) rows x kTcK columns of op(r, k) into a K-major tile.
template <typename Get>
__device__ __forceinline__ void tc_stage(unsigned char* tile, int rows, int tid, const Get& get) {
  for (int it = tid; it < rows * (kTcK / 8); it += 128) {
    const int r = it / (kTcK / 8), kg = it % (kTcK / 8);
    uint32_t v[4];
#pragma unroll
    for (int h = 0; h < 4; ++h) v[h] = pack2(get(r, kg * 8 + 2 * h), get(r, kg * 8 + 2 * h + 1));
    *reinterpret_cast<uint4*>(tile + tc_offset(r, kg * 8)) = make_uint4(v[0], v[1], v[2], v[3]);
  }
}

__global__ void __launch_bounds__(128) k_gemm_tc(int M, int N, int K, const bf16* __restrict__ A,
                                                 int64_t sam, int64_t sak,
                                                 const bf16* __restrict__ B, int64_t sbk,
                                                 int64_t sbn, float* __restrict__ C, int64_t ldc,
                                                 bool accumulate, int* status) {
  extern __shared__ unsigned char tc_raw[];
  TcSmem& sh = *reinterpret_cast<TcSmem*>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) &
                                          ~static_cast<uintptr_t>(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kTcRows;
  // split K (weight gradients: K = the batch rows): CTA y takes [k_beg, k_end)
  const int k_per = (K + (int)gridDim.y * kTcK - 1) / ((int)gridDim.y * kTcK) * kTcK;
  const int k_beg = (int)blockIdx.y * k_per;
  const int k_end = k_beg + k_per < K ? k_beg + k_per : K;
  const uint32_t a_base = smem_u32(sh.a), b_base = smem_u32(sh.b), mbar = smem_u32(&sh.mbar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&sh.tmem)), "r"(kTcCols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = sh.tmem;
  const uint32_t idesc = tc_idesc(kTcRows, N);
  const bf16 z = __float2bfloat16(0.0f);
  uint32_t phase = 0;
  bool ok = true;
  for (int k0 = k_beg; k0 < k_end && ok; k0 += kTcK) {
    tc_stage(reinterpret_cast<unsigned char*>(sh.a), kTcRows, tid, [&](int r, int k) {
      const int m = m0 + r, kk = k0 + k;
      return (m < M && kk < k_end) ? A[m * sam + kk * sak] : z;
    });
    tc_stage(reinterpret_cast<unsigned char*>(sh.b), N, tid, [&](int n, int k) {
      const int kk = k0 + k;
      return kk < k_end ? B[kk * sbk + n * sbn] : z;
    });
    // the tiles written by ordinary stores become visible to the tensor cores
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int s = 0; s < kTcK / 16; ++s) {
        const uint64_t ad = tc_desc(a_base + s * 2 * kTcLbo), bd = tc_desc(b_base + s * 2 * kTcLbo);
        const uint32_t acc = (k0 > k_beg || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
            :: "r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc) : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   :: "r"(mbar) : "memory");
    }
    // the stage's products are in the accumulator and its tiles free again
    ok = __syncthreads_and(tc_wait(mbar, phase)) != 0;
    phase ^= 1u;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const int row = m0 + warp * 32 + lane;
  // a split-K CTA whose range is empty has no accumulator to add
  for (int c0 = 0; c0 < N && k_beg < k_end; c0 += 32) {
    uint32_t v[32];
    if (ok) tc_load32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
    if (row < M) {
      float* c = C + row * ldc + c0;
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const float x = ok ? __uint_as_float(v[j]) : __int_as_float(0x7fc00000);
        if (gridDim.y > 1) atomicAdd(c + j, x);  // split K: C was cleared or holds the sum
        else c[j] = accumulate ? c[j] + x : x;
      }
    }
  }
  if (!ok && tid == 0) atomicOr(status, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :: "r"(tmem), "r"(kTcCols) : "memory");
  }
}

// FP32 SIMT GEMM with the same meaning (the debug path).
__global__ void k_gemm_f32(int M, int N, int K, const float* __restrict__ A, int64_t sam,
                           int64_t sak, const float* __restrict__ B, int64_t sbk, int64_t sbn,
                           float* __restrict__ C, int64_t ldc, bool accumulate) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= (int64_t)M * N) return;
  const int m = (int)(idx / N), n = (int)(idx % N);
  float acc = 0.f;
  for (int k = 0; k < K; ++k) acc = fmaf(A[m * sam + k * sak], B[k * sbk + n * sbn], acc);
  float* c = C + m * ldc + n;
  *c = accumulate ? *c + acc : acc;
}

__global__ void k_to_bf16(const float* __restrict__ x, bf16* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16(x[i]);
}

// H[r][c] = relu(H[r][c] + b[c]) over rows x cols.
__global__ void k_bias_relu(float* __restrict__ H, const float* __restrict__ b, int rows,
                            int cols) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)rows * cols;
       i += (int64_t)gridDim.x * blockDim.x)
    H[i] = fmaxf(H[i] + b[i % cols], 0.0f);
}

// y[r] = H2[r] . w3 + b3; with targets: dy = 2 (y - t) / rows, loss += (y - t)^2 / rows.
__global__ void k_head(const float* __restrict__ H2, const float* __restrict__ w3,
                       const float* __restrict__ b3, int rows, float* __restrict__ y,
                       const float* __restrict__ t, float* __restrict__ dy, float* loss) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (warp >= rows) return;
  float acc = 0.f;
  for (int c = lane; c < kHid; c += 32) acc = fmaf(H2[warp * kHid + c], w3[c], acc);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) {
    const float v = acc + b3[0];
    if (y) y[warp] = v;
    if (t) {
      const float e = v - t[warp];
      dy[warp] = 2.0f * e / rows;
      atomicAdd(loss, e * e / rows);
    }
  }
}

// dH2[r][c] = dy[r] w3[c] [H2[r][c] > 0]
__global__ void k_dh2(const float* __restrict__ dy, const float* __restrict__ w3,
                      const float* __restrict__ H2, float* __restrict__ dH2, int rows) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)rows * kHid;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / kHid;
    const int c = (int)(i % kHid);
    dH2[i] = H2[i] > 0.0f ? dy[r] * w3[c] : 0.0f;
  }
}

// D[r][c] *= [H[r][c] > 0]
__global__ void k_relu_grad(float* __restrict__ D, const float* __restrict__ H, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (!(H[i] > 0.0f)) D[i] = 0.0f;
}

// out[c] = sum_r X[r][c] * (v ? v[r] : 1), one thread per column.
__global__ void k_colsum(const float* __restrict__ X, const float* __restrict__ v, int rows,
                         int cols, float* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  double acc = 0.0;
  for (int r = 0; r < rows; ++r) acc += (double)X[(int64_t)r * cols + c] * (v ? v[r] : 1.0f);
  out[c] = (float)acc;
}

__global__ void k_sum(const float* __restrict__ v, int n, float* __restrict__ out) {
  __shared__ float red[32];
  float acc = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += v[i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    *out = t;
  }
}

// Adam (bias-corrected), then the BF16 copies of W1 and W2.
__global__ void k_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M1,
                       float* __restrict__ M2, int64_t n, float lr, float b1, float b2,
                       float eps, float c1, float c2, bf16* __restrict__ W1b,
                       bf16* __restrict__ W2b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float g = G[i];
    const float m = b1 * M1[i] + (1.0f - b1) * g;
    const float v = b2 * M2[i] + (1.0f - b2) * g * g;
    M1[i] = m;
    M2[i] = v;
    const float p = P[i] - lr * (m / c1) / (sqrtf(v / c2) + eps);
    P[i] = p;
    if (i < kOffB1) W1b[i - kOffW1] = __float2bfloat16(p);
    else if (i >= kOffW2 && i < kOffB2) W2b[i - kOffW2] = __float2bfloat16(p);
  }
}

}  // namespace

struct dtwj_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  float* P = nullptr;   // master parameters
  float* G = nullptr;   // gradient
  float* M1 = nullptr;  // Adam moments
  float* M2 = nullptr;
  bf16* W1b = nullptr;  // BF16 copies of the GEMM weights
  bf16* W2b = nullptr;
  int64_t step = 0;
  // batch workspace (kMaxBatch rows)
  float *X = nullptr, *T = nullptr, *H1 = nullptr, *H2 = nullptr, *Y = nullptr, *DY = nullptr,
        *DH1 = nullptr, *DH2 = nullptr, *loss = nullptr;
  bf16 *Xb = nullptr, *H1b = nullptr, *DH1b = nullptr, *DH2b = nullptr;
  int* tc_status = nullptr;  // set when a tensor-core GEMM gave up waiting on its mbarrier
};

namespace {

template <typename T>
bool dalloc(T** p, int64_t count) {
  return cudaMalloc((void**)p, (size_t)count * sizeof(T)) == cudaSuccess;
}

// The BF16 path needs N <= 128 and N % 16 == 0 (the MLP's N are 64 and 128).
constexpr int kTcSmemBytes = 48 * 1024;  // also keeps at most 4 CTAs (512 TMEM columns) per SM
static_assert(sizeof(TcSmem) + 1024 <= kTcSmemBytes, "tcgen05 GEMM tiles");

void gemm(bool precise, int M, int N, int K, const void* A, int64_t sam, int64_t sak,
          const void* B, int64_t sbk, int64_t sbn, float* C, int64_t ldc, bool acc,
          int* status, cudaStream_t st) {
  if (precise) {
    k_gemm_f32<<<grid_for((int64_t)M * N), kThreads, 0, st>>>(
        M, N, K, (const float*)A, sam, sak, (const float*)B, sbk, sbn, C, ldc, acc);
  } else {
    // long K on few rows (the weight gradients): split K over CTAs that add
    // their products into C, cleared first unless accumulating
    const int mblocks = (M + kTcRows - 1) / kTcRows;
    int ksplit = 1;
    if (mblocks == 1 && K >= 1024) ksplit = K / 512 < 64 ? K / 512 : 64;
    if (ksplit > 1 && !acc) cudaMemsetAsync(C, 0, (size_t)M * ldc * sizeof(float), st);
    k_gemm_tc<<<dim3((unsigned)mblocks, (unsigned)ksplit), 128, kTcSmemBytes, st>>>(
        M, N, K, (const bf16*)A, sam, sak, (const bf16*)B, sbk, sbn, C, ldc, acc, status);
  }
}

// Forward of `rows` rows staged in net->X; with targets (net->T) also the
// backward into net->G and the loss into *net->loss.  precise: FP32 GEMMs on
// the FP32 parameters; otherwise BF16 operands (weights from the BF16 copies).
void pass(dtwj_mlp* net, int rows, bool train, bool precise) {
  cudaStream_t st = net->stream;
  const float* P = net->P;
  const unsigned gr = grid_for((int64_t)rows * kHid);
  // H1 = relu(X W1^T + b1): A = X [rows][64], B(k, n) = W1[n][k]
  if (!precise) k_to_bf16<<<grid_for((int64_t)rows * kIn), kThreads, 0, st>>>(net->X, net->Xb, (int64_t)rows * kIn);
  gemm(precise, rows, kHid, kIn, precise ? (const void*)net->X : net->Xb, kIn, 1,
       precise ? (const void*)(P + kOffW1) : net->W1b, 1, kIn, net->H1, kHid, false, net->tc_status, st);
  k_bias_relu<<<gr, kThreads, 0, st>>>(net->H1, P + kOffB1, rows, kHid);
  // H2 = relu(H1 W2^T + b2)
  if (!precise) k_to_bf16<<<gr, kThreads, 0, st>>>(net->H1, net->H1b, (int64_t)rows * kHid);
  gemm(precise, rows, kHid, kHid, precise ? (const void*)net->H1 : net->H1b, kHid, 1,
       precise ? (const void*)(P + kOffW2) : net->W2b, 1, kHid, net->H2, kHid, false, net->tc_status, st);
  k_bias_relu<<<gr, kThreads, 0, st>>>(net->H2, P + kOffB2, rows, kHid);
  if (train) cudaMemsetAsync(net->loss, 0, 4, st);
  k_head<<<grid_for((int64_t)rows * 32), kThreads, 0, st>>>(net->H2, P + kOffW3, P + kOffB3, rows,
                                                           net->Y, train ? net->T : nullptr,
                                                           net->DY, net->loss);
  if (!train) return;
  float* G = net->G;
  // head: dw3 = H2^T dy, db3 = sum dy
  k_colsum<<<1, kHid, 0, st>>>(net->H2, net->DY, rows, kHid, G + kOffW3);
  k_sum<<<1, 256, 0, st>>>(net->DY, rows, G + kOffB3);
  // dH2, dW2 = dH2^T H1 [128][128] (K = rows), db2
  k_dh2<<<gr, kThreads, 0, st>>>(net->DY, P + kOffW3, net->H2, net->DH2, rows);
  if (!precise) k_to_bf16<<<gr, kThreads, 0, st>>>(net->DH2, net->DH2b, (int64_t)rows * kHid);
  gemm(precise, kHid, kHid, rows, precise ? (const void*)net->DH2 : net->DH2b, 1, kHid,
       precise ? (const void*)net->H1 : net->H1b, kHid, 1, G + kOffW2, kHid, false, net->tc_status, st);
  k_colsum<<<1, kHid, 0, st>>>(net->DH2, nullptr, rows, kHid, G + kOffB2);
  // dH1 = dH2 W2 . [H1 > 0]: A = dH2 [rows][128], B(k, n) = W2[k][n]
  gemm(precise, rows, kHid, kHid, precise ? (const void*)net->DH2 : net->DH2b, kHid, 1,
       precise ? (const void*)(P + kOffW2) : net->W2b, kHid, 1, net->DH1, kHid, false, net->tc_status, st);
  k_relu_grad<<<gr, kThreads, 0, st>>>(net->DH1, net->H1, (int64_t)rows * kHid);
  // dW1 = dH1^T X [128][64] (K = rows), db1
  if (!precise) k_to_bf16<<<gr, kThreads, 0, st>>>(net->DH1, net->DH1b, (int64_t)rows * kHid);
  gemm(precise, kHid, kIn, rows, precise ? (const void*)net->DH1 : net->DH1b, 1, kHid,
       precise ? (const void*)net->X : net->Xb, kIn, 1, G + kOffW1, kIn, false, net->tc_status, st);
  k_colsum<<<1, kHid, 0, st>>>(net->DH1, nullptr, rows, kHid, G + kOffB1);
}

// After the stream is synchronised: DTWJ_ERR_CUDA if a tensor-core GEMM gave
// up waiting for its products (its outputs are NaN then).
int tc_check(dtwj_mlp* net) {
  int st = 0;
  if (cudaMemcpy(&st, net->tc_status, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return DTWJ_ERR_CUDA;
  return st ? DTWJ_ERR_CUDA : DTWJ_OK;
}

void refresh_bf16(dtwj_mlp* net) {
  k_to_bf16<<<grid_for(kHid * kIn), kThreads, 0, net->stream>>>(net->P + kOffW1, net->W1b, kHid * kIn);
  k_to_bf16<<<grid_for(kHid * kHid), kThreads, 0, net->stream>>>(net->P + kOffW2, net->W2b, kHid * kHid);
}

// splitmix64 -> uniform in [0, 1)
double uniform(uint64_t* s) {
  uint64_t z = (*s += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

int stage(dtwj_mlp* net, const float* x, const float* y, int64_t r0, int rows) {
  if (cudaMemcpyAsync(net->X, x + r0 * kIn, (size_t)rows * kIn * 4, cudaMemcpyHostToDevice,
                      net->stream) != cudaSuccess)
    return DTWJ_ERR_CUDA;
  if (y && cudaMemcpyAsync(net->T, y + r0, (size_t)rows * 4, cudaMemcpyHostToDevice,
                           net->stream) != cudaSuccess)
    return DTWJ_ERR_CUDA;
  return DTWJ_OK;
}

}  // namespace

extern "C" {

int dtwj_mlp_create(int device, uint64_t seed, dtwj_mlp** out) {
  if (!out) return DTWJ_ERR_ARG;
  *out = nullptr;
  if (dtwj_device_count() <= device || device < 0) return DTWJ_ERR_NODEVICE;
  if (cudaSetDevice(device) != cudaSuccess) return DTWJ_ERR_CUDA;
  dtwj_mlp* net = new (std::nothrow) dtwj_mlp();
  if (!net) return DTWJ_ERR_OOM;
  net->device = device;
  const int64_t B = kMaxBatch;
  bool ok = cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking) == cudaSuccess &&
            dalloc(&net->P, kNumParams) && dalloc(&net->G, kNumParams) &&
            dalloc(&net->M1, kNumParams) && dalloc(&net->M2, kNumParams) &&
            dalloc(&net->W1b, kHid * kIn) && dalloc(&net->W2b, kHid * kHid) &&
            dalloc(&net->X, B * kIn) && dalloc(&net->T, B) && dalloc(&net->H1, B * kHid) &&
            dalloc(&net->H2, B * kHid) && dalloc(&net->Y, B) && dalloc(&net->DY, B) &&
            dalloc(&net->DH1, B * kHid) && dalloc(&net->DH2, B * kHid) &&
            dalloc(&net->loss, 1) && dalloc(&net->Xb, B * kIn) && dalloc(&net->H1b, B * kHid) &&
            dalloc(&net->DH1b, B * kHid) && dalloc(&net->DH2b, B * kHid) &&
            dalloc(&net->tc_status, 1) && cudaMemset(net->tc_status, 0, 4) == cudaSuccess;
  if (!ok) {
    dtwj_mlp_destroy(net);
    return DTWJ_ERR_OOM;
  }
  // He-uniform weights, zero biases
  std::vector<float> p((size_t)kNumParams, 0.0f);
  uint64_t s = seed;
  const double a1 = std::sqrt(6.0 / kIn), a2 = std::sqrt(6.0 / kHid);
  for (int64_t i = 0; i < kHid * kIn; ++i) p[kOffW1 + i] = (float)((2 * uniform(&s) - 1) * a1);
  for (int64_t i = 0; i < kHid * kHid; ++i) p[kOffW2 + i] = (float)((2 * uniform(&s) - 1) * a2);
  for (int64_t i = 0; i < kHid; ++i) p[kOffW3 + i] = (float)((2 * uniform(&s) - 1) * a2);
  *out = net;
  return dtwj_mlp_set(net, p.data());
}

void dtwj_mlp_destroy(dtwj_mlp* net) {
  if (!net) return;
  cudaSetDevice(net->device);
  if (net->stream) cudaStreamSynchronize(net->stream);
  void* bufs[] = {net->P,  net->G,  net->M1, net->M2,  net->W1b, net->W2b, net->X,
                  net->T,  net->H1, net->H2, net->Y,   net->DY,  net->DH1, net->DH2,
                  net->loss, net->Xb, net->H1b, net->DH1b, net->DH2b, net->tc_status};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (net->stream) cudaStreamDestroy(net->stream);
  delete net;
}

int dtwj_mlp_set(dtwj_mlp* net, const float* params) {
  if (!net || !params) return DTWJ_ERR_ARG;
  cudaSetDevice(net->device);
  if (cudaMemcpyAsync(net->P, params, kNumParams * 4, cudaMemcpyHostToDevice, net->stream) !=
          cudaSuccess ||
      cudaMemsetAsync(net->M1, 0, kNumParams * 4, net->stream) != cudaSuccess ||
      cudaMemsetAsync(net->M2, 0, kNumParams * 4, net->stream) != cudaSuccess)
    return DTWJ_ERR_CUDA;
  net->step = 0;
  refresh_bf16(net);
  return cudaStreamSynchronize(net->stream) == cudaSuccess ? DTWJ_OK : DTWJ_ERR_CUDA;
}

int dtwj_mlp_get(dtwj_mlp* net, float* params) {
  if (!net || !params) return DTWJ_ERR_ARG;
  cudaSetDevice(net->device);
  if (cudaMemcpyAsync(params, net->P, kNumParams * 4, cudaMemcpyDeviceToHost, net->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(net->stream) != cudaSuccess)
    return DTWJ_ERR_CUDA;
  return DTWJ_OK;
}

int dtwj_mlp_grad(dtwj_mlp* net, const float* x, const float* y, int64_t count, int32_t precise,
                  float* grad, float* loss) {
  if (!net || !x || !y || !grad || count < 1 || count > kMaxBatch) return DTWJ_ERR_ARG;
  cudaSetDevice(net->device);
  int rc = stage(net, x, y, 0, (int)count);
  if (rc) return rc;
  pass(net, (int)count, true, precise != 0);
  if (cudaMemcpyAsync(grad, net->G, kNumParams * 4, cudaMemcpyDeviceToHost, net->stream) !=
      cudaSuccess)
    return DTWJ_ERR_CUDA;
  float l = 0.f;
  if (cudaMemcpyAsync(&l, net->loss, 4, cudaMemcpyDeviceToHost, net->stream) != cudaSuccess ||
      cudaStreamSynchronize(net->stream) != cudaSuccess)
    return DTWJ_ERR_CUDA;
  if (loss) *loss = l;
  return tc_check(net);
}

int dtwj_mlp_train(dtwj_mlp* net, const float* x, const float* y, int64_t count, int32_t epochs,
                   int32_t batch, float lr, uint64_t seed, float* last_loss) {
  if (!net || !x || !y || count < 1 || epochs < 1 || batch < 1 || batch > kMaxBatch || !(lr > 0))
    return DTWJ_ERR_ARG;
  cudaSetDevice(net->device);
  // minibatches of a shuffled copy (Fisher-Yates with splitmix64)
  std::vector<int64_t> perm((size_t)count);
  for (int64_t i = 0; i < count; ++i) perm[i] = i;
  std::vector<float> xs((size_t)batch * kIn), ys((size_t)batch);
  uint64_t s = seed;
  double epoch_loss = 0.0;
  for (int ep = 0; ep < epochs; ++ep) {
    for (int64_t i = count - 1; i > 0; --i) {
      const int64_t j = (int64_t)(uniform(&s) * (double)(i + 1));
      std::swap(perm[i], perm[j < i ? j : i]);
    }
    epoch_loss = 0.0;
    int64_t seen = 0;
    for (int64_t r0 = 0; r0 < count; r0 += batch) {
      const int rows = (int)(count - r0 < batch ? count - r0 : batch);
      for (int r = 0; r < rows; ++r) {
        memcpy(&xs[(size_t)r * kIn], x + perm[r0 + r] * kIn, kIn * 4);
        ys[r] = y[perm[r0 + r]];
      }
      int rc = stage(net, xs.data(), ys.data(), 0, rows);
      if (rc) return rc;
      pass(net, rows, true, false);
      ++net->step;
      const float b1 = 0.9f, b2 = 0.999f;
      const float c1 = 1.0f - std::pow(b1, (float)net->step);
      const float c2 = 1.0f - std::pow(b2, (float)net->step);
      k_adam<<<grid_for(kNumParams), kThreads, 0, net->stream>>>(
          net->P, net->G, net->M1, net->M2, kNumParams, lr, b1, b2, 1e-8f, c1, c2, net->W1b,
          net->W2b);
      float l = 0.f;
      if (cudaMemcpyAsync(&l, net->loss, 4, cudaMemcpyDeviceToHost, net->stream) != cudaSuccess ||
          cudaStreamSynchronize(net->stream) != cudaSuccess)
        return DTWJ_ERR_CUDA;
      epoch_loss += (double)l * rows;
      seen += rows;
    }
    epoch_loss /= (double)seen;
  }
  if (last_loss) *last_loss = (float)epoch_loss;
  return cudaGetLastError() == cudaSuccess ? tc_check(net) : DTWJ_ERR_CUDA;
}

int dtwj_mlp_predict(dtwj_mlp* net, const float* x, int64_t count, float* out) {
  if (!net || !x || !out || count < 0) return DTWJ_ERR_ARG;
  cudaSetDevice(net->device);
  for (int64_t r0 = 0; r0 < count; r0 += kMaxBatch) {
    const int rows = (int)(count - r0 < kMaxBatch ? count - r0 : kMaxBatch);
    int rc = stage(net, x, nullptr, r0, rows);
    if (rc) return rc;
    pass(net, rows, false, false);
    if (cudaMemcpyAsync(out + r0, net->Y, (size_t)rows * 4, cudaMemcpyDeviceToHost,
                        net->stream) != cudaSuccess)
      return DTWJ_ERR_CUDA;
  }
  return cudaStreamSynchronize(net->stream) == cudaSuccess ? tc_check(net) : DTWJ_ERR_CUDA;
}

int dtwj_mlp_save(dtwj_mlp* net, const char* path) {
  if (!net || !path) return DTWJ_ERR_ARG;
  std::vector<float> p((size_t)kNumParams);
  int rc = dtwj_mlp_get(net, p.data());
  if (rc) return rc;
  FILE* f = fopen(path, "wb");
  if (!f) return DTWJ_ERR_IO;
  const char magic[8] = {'D', 'T', 'W', 'J', 'M', 'L', 'P', '1'};
  bool ok = fwrite(magic, 1, 8, f) == 8 && fwrite(p.data(), 4, p.size(), f) == p.size();
  ok = (fclose(f) == 0) && ok;
  return ok ? DTWJ_OK : DTWJ_ERR_IO;
}

int dtwj_mlp_load(int device, const char* path, dtwj_mlp** out) {
  if (!path || !out) return DTWJ_ERR_ARG;
  *out = nullptr;
  FILE* f = fopen(path, "rb");
  if (!f) return DTWJ_ERR_IO;
  char magic[8];
  std::vector<float> p((size_t)kNumParams);
  const bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, "DTWJMLP1", 8) == 0 &&
                  fread(p.data(), 4, p.size(), f) == p.size();
  fclose(f);
  if (!ok) return DTWJ_ERR_IO;
  int rc = dtwj_mlp_create(device, 0, out);
  if (rc) return rc;
  rc = dtwj_mlp_set(*out, p.data());
  if (rc) {
    dtwj_mlp_destroy(*out);
    *out = nullptr;
  }
  return rc;
}

}  // extern "C"

namespace dtwj {

// Scores of `count` feature rows already on the device (x_dev [count][64])
// into y_dev, after the work queued on `st` (which produced x_dev) is done.
int mlp_predict_device(dtwj_mlp* net, const float* x_dev, int64_t count, float* y_dev,
                       cudaStream_t st) {
  if (cudaStreamSynchronize(st) != cudaSuccess) return DTWJ_ERR_CUDA;
  for (int64_t r0 = 0; r0 < count; r0 += kMaxBatch) {
    const int rows = (int)(count - r0 < kMaxBatch ? count - r0 : kMaxBatch);
    if (cudaMemcpyAsync(net->X, x_dev + r0 * kIn, (size_t)rows * kIn * 4,
                        cudaMemcpyDeviceToDevice, net->stream) != cudaSuccess)
      return DTWJ_ERR_CUDA;
    pass(net, rows, false, false);
    if (cudaMemcpyAsync(y_dev + r0, net->Y, (size_t)rows * 4, cudaMemcpyDeviceToDevice,
                        net->stream) != cudaSuccess)
      return DTWJ_ERR_CUDA;
  }
  return cudaStreamSynchronize(net->stream) == cudaSuccess ? tc_check(net) : DTWJ_ERR_CUDA;
}

int mlp_device(const dtwj_mlp* net) { return net->device; }

}  // namespace dtwj
