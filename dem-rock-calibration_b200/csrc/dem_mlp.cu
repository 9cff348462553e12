// Surrogate MLP kernels (the B200 counterpart of the sklearn MLPRegressor that
// NN_MP.py trains on simulation results, NN_MP.py:374-378, 895): BF16 operands,
// FP32 accumulation on the 5th-generation tensor cores.
//
//   k_gemm_tn   C[M x N] = A[M x K] . B[N x K]^T, A and B row-major BF16 (both
//               "K-major"), accumulator in tensor memory: a 128-row tile of A and
//               an N-tile (32..256) of B are staged in shared memory in the
//               canonical no-swizzle core-matrix layout (8 rows x 16 bytes per
//               core matrix), one thread issues tcgen05.mma (M = 128, K = 16 per
//               instruction, kind::f16) into a TMEM accumulator and commits to an
//               mbarrier; the four warps read the accumulator back with
//               tcgen05.ld (32 lanes each) and apply the epilogue: + bias and
//               GELU or ReLU to BF16 (hidden layers, pre-activation kept in
//               FP32), + bias to FP32 (output layer), or plain FP32 (weight and
//               activation gradients).
//   small kernels: input packing, transposes, activation backward, column
//               sums, MSE gradient, Adam.
//
// All waits are bounded: a commit that does not arrive within the poll limit
// sets *err, the block waits once more (bounded) and frees its tensor memory.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "b200dem.h"

namespace dem {
namespace {

constexpr int kTM = 128;   // rows per tile (tcgen05 M)
constexpr int kTK = 32;    // K staged per round (two K = 16 instructions)
constexpr uint32_t kPollLimit = 1u << 22;

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t* b) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(b)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity) {
  const uint32_t a = saddr(b);
  for (uint32_t n = 0; n < kPollLimit; ++n) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor (sm_100): start address, leading-dimension
// byte offset (between the two core matrices along K of one instruction),
// stride byte offset (between 8-row groups), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// exact (erf) GELU and its derivative; ReLU takes 0 as its derivative at 0, as
// sklearn's MLPRegressor does (NN_MP.py:374 uses its default activation)
__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

template <int TN>
struct __align__(128) GemmSmem {
  uint4 a[4 * kTM];   // 4 K-groups of 8 BF16 x 128 rows
  uint4 b[4 * TN];    // 4 K-groups x TN rows
  uint64_t bar;
  uint32_t tmem;
};

template <int TN>
__global__ void __launch_bounds__(128) k_gemm_tn(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ B,
                                                 int M, int N, int K, const float* __restrict__ bias, int mode,
                                                 float* __restrict__ outf, __nv_bfloat16* __restrict__ outh,
                                                 unsigned int* err) {
  constexpr uint32_t kCols = TN <= 32 ? 32 : (TN <= 64 ? 64 : (TN <= 128 ? 128 : 256));
  __shared__ GemmSmem<TN> sm;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kTM, n0 = blockIdx.y * TN;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&sm.tmem)),
                 "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) bar_init(&sm.bar);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem;
  // instruction descriptor: F32 accumulate, BF16 A and B, both K-major, N, M = 128
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(kTM >> 4) << 24);
  const int rounds = K / kTK;
  bool ok = true;
  for (int c = 0; c < rounds; ++c) {
    const int k0 = c * kTK;
    for (int q = tid; q < 4 * kTM; q += 128) {
      const int g = q & 3, r = q >> 2;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (m0 + r < M) v = *reinterpret_cast<const uint4*>(A + (size_t)(m0 + r) * K + k0 + 8 * g);
      sm.a[g * kTM + r] = v;
    }
    for (int q = tid; q < 4 * TN; q += 128) {
      const int g = q & 3, r = q >> 2;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (n0 + r < N) v = *reinterpret_cast<const uint4*>(B + (size_t)(n0 + r) * K + k0 + 8 * g);
      sm.b[g * TN + r] = v;
    }
    // the tensor core reads shared memory through the async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      for (int kk = 0; kk < kTK / 16; ++kk) {
        const uint64_t da = smem_desc(saddr(&sm.a[2 * kk * kTM]), kTM * 16, 128);
        const uint64_t db = smem_desc(saddr(&sm.b[2 * kk * TN]), TN * 16, 128);
        const uint32_t acc = (c > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       saddr(&sm.bar))
                   : "memory");
    }
    ok = bar_wait(&sm.bar, (uint32_t)(c & 1));
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicOr(err, 1u);
      bar_wait(&sm.bar, (uint32_t)(c & 1));
      ok = false;
      break;
    }
  }
  if (ok && rounds > 0) {
    tc_fence_after();
    const int row = m0 + warp * 32 + lane;
    for (int col0 = 0; col0 < TN; col0 += 32) {
      uint32_t r[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
          "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
            "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
            "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
          : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)col0)
          : "memory");
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < M) {
        for (int j = 0; j < 32; ++j) {
          const int n = n0 + col0 + j;
          if (n >= N) break;
          float v = __uint_as_float(r[j]);
          const size_t o = (size_t)row * N + n;
          if (mode == DEM_MLP_BIAS_GELU || mode == DEM_MLP_BIAS_RELU) {
            v += bias[n];
            if (outf) outf[o] = v;
            outh[o] = __float2bfloat16_rn(mode == DEM_MLP_BIAS_GELU ? gelu(v) : fmaxf(v, 0.f));
          } else if (mode == DEM_MLP_BIAS) {
            outf[o] = v + bias[n];
          } else {
            outf[o] = v;
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
}

// x (rows x k FP32) -> BF16 rows of kpad, zero padded; row r of the output is
// row idx[r] of x when idx is given
__global__ void k_pack_bf16(const float* __restrict__ x, const int* __restrict__ idx, int rows, int k, int kpad,
                            __nv_bfloat16* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)rows * kpad;
       i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / kpad), c = (int)(i % kpad);
    const size_t src = idx ? (size_t)idx[r] : (size_t)r;
    out[i] = __float2bfloat16_rn(c < k ? x[src * k + c] : 0.f);
  }
}

// in (rows x cols BF16) -> out (cols x ldo BF16), out[c][r] = in[r][c]; columns r >= rows of out are zeroed
__global__ void k_transpose_bf16(const __nv_bfloat16* __restrict__ in, int rows, int cols, int ldo,
                                 __nv_bfloat16* __restrict__ out) {
  __shared__ __nv_bfloat16 t[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = r0 + y, c = c0 + threadIdx.x;
    t[y][threadIdx.x] = (r < rows && c < cols) ? in[(size_t)r * cols + c] : __float2bfloat16_rn(0.f);
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int c = c0 + y, r = r0 + threadIdx.x;
    if (c < cols && r < ldo) out[(size_t)c * ldo + r] = t[threadIdx.x][y];
  }
}

// dZ = dH * act'(Z) (FP32 in, BF16 and FP32 out)
__global__ void k_act_backward(const float* __restrict__ dh, const float* __restrict__ z, size_t n, int act,
                               __nv_bfloat16* __restrict__ dzh, float* __restrict__ dzf) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float zi = z[i];
    const float g = dh[i] * (act == DEM_MLP_BIAS_GELU ? gelu_grad(zi) : (zi > 0.f ? 1.f : 0.f));
    dzh[i] = __float2bfloat16_rn(g);
    if (dzf) dzf[i] = g;
  }
}

// column sums in two deterministic passes: block (x, s) of 32 x 8 threads sums
// rows s, s + S, s + 2S, ... of 32 columns (S = gridDim.y), the eight row
// phases combined in shared memory in a fixed order, into part[s][c]; then one
// thread per column adds the S partial sums in order
__global__ void k_colsum_part(const float* __restrict__ in, int rows, int cols, float* __restrict__ part) {
  __shared__ float t[8][33];
  const int c = blockIdx.x * 32 + threadIdx.x, S = gridDim.y;
  float acc = 0.f;
  if (c < cols)
    for (int r = blockIdx.y + S * threadIdx.y; r < rows; r += 8 * S) acc += in[(size_t)r * cols + c];
  t[threadIdx.y][threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.y == 0 && c < cols) {
    float s = t[0][threadIdx.x];
    for (int y = 1; y < 8; ++y) s += t[y][threadIdx.x];
    part[(size_t)blockIdx.y * cols + c] = s;
  }
}
__global__ void k_colsum_final(const float* __restrict__ part, int S, int cols, float* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (int k = 0; k < S; ++k) s += part[(size_t)k * cols + c];
  out[c] = s;
}

// out row r = x row idx[r] (FP32, k columns)
__global__ void k_gather(const float* __restrict__ x, const int* __restrict__ idx, int rows, int k,
                         float* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)rows * k;
       i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / k), c = (int)(i % k);
    out[i] = x[(size_t)idx[r] * k + c];
  }
}

__global__ void k_tick(int* step) { *step += 1; }

// mean squared error of y against t (rows x cols): dY = 2 (y - t) / (rows cols),
// BF16 and FP32; loss accumulated into *loss (double)
__global__ void k_mse_grad(const float* __restrict__ y, const float* __restrict__ t, size_t n,
                           __nv_bfloat16* __restrict__ dyh, float* __restrict__ dyf, double* loss) {
  double s = 0.0;
  const float k = 2.0f / (float)n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float d = y[i] - t[i];
    s += (double)d * d;
    dyh[i] = __float2bfloat16_rn(k * d);
    if (dyf) dyf[i] = k * d;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, s / (double)n);
}

// Adam on FP32 master weights (gradient + l2 w, the L2 penalty of sklearn's
// alpha / n_samples); BF16 copy refreshed.  The step number t >= 1 is read from
// the device so that a captured graph of training steps stays valid on replay.
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       size_t n, float lr, float b1, float b2, float eps, const int* __restrict__ step, float l2,
                       __nv_bfloat16* __restrict__ wh) {
  const float t = (float)max(*step, 1);
  const float c1 = 1.f - powf(b1, t), c2 = 1.f - powf(b2, t);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i] + l2 * w[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wh) wh[i] = __float2bfloat16_rn(wi);
  }
}

// per device: a flag set by a GEMM block whose tensor-core commit timed out
constexpr int kMaxDev = 64;
std::mutex g_mu;
unsigned int* g_err[kMaxDev] = {};

int err_flag(unsigned int** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return DEM_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_err[dev]) {
    unsigned int* p = nullptr;
    if (cudaMalloc((void**)&p, sizeof(unsigned int)) != cudaSuccess) return DEM_ERR_CUDA;
    if (cudaMemset(p, 0, sizeof(unsigned int)) != cudaSuccess) return DEM_ERR_CUDA;
    g_err[dev] = p;
  }
  *out = g_err[dev];
  return DEM_OK;
}

uint32_t blocks(size_t n) { return (uint32_t)std::min<size_t>((n + 255) / 256, 148 * 16); }

}  // namespace
}  // namespace dem

using namespace dem;

extern "C" {

int dem_mlp_gemm_tn(const void* A, const void* B, int M, int N, int K, const float* bias, int mode, float* out_f32,
                    void* out_bf16, void* stream) {
  if (!A || !B || M <= 0 || N <= 0 || K <= 0 || (K % 32) != 0) return DEM_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15) return DEM_ERR_ARG;
  if (mode < DEM_MLP_PLAIN || mode > DEM_MLP_BIAS_RELU) return DEM_ERR_ARG;
  if ((mode == DEM_MLP_BIAS_GELU || mode == DEM_MLP_BIAS_RELU) && (!bias || !out_bf16)) return DEM_ERR_ARG;
  if (mode == DEM_MLP_BIAS && (!bias || !out_f32)) return DEM_ERR_ARG;
  if (mode == DEM_MLP_PLAIN && !out_f32) return DEM_ERR_ARG;
  unsigned int* err = nullptr;
  if (err_flag(&err)) return DEM_ERR_CUDA;
  cudaStream_t st = (cudaStream_t)stream;
  const auto* a = static_cast<const __nv_bfloat16*>(A);
  const auto* b = static_cast<const __nv_bfloat16*>(B);
  auto* oh = static_cast<__nv_bfloat16*>(out_bf16);
  const unsigned gx = (unsigned)((M + kTM - 1) / kTM);
  if (N <= 32)
    k_gemm_tn<32><<<dim3(gx, 1), 128, 0, st>>>(a, b, M, N, K, bias, mode, out_f32, oh, err);
  else if (N <= 64)
    k_gemm_tn<64><<<dim3(gx, 1), 128, 0, st>>>(a, b, M, N, K, bias, mode, out_f32, oh, err);
  else if (N <= 128)
    k_gemm_tn<128><<<dim3(gx, 1), 128, 0, st>>>(a, b, M, N, K, bias, mode, out_f32, oh, err);
  else
    k_gemm_tn<256><<<dim3(gx, (unsigned)((N + 255) / 256)), 128, 0, st>>>(a, b, M, N, K, bias, mode, out_f32, oh,
                                                                         err);
  return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

int dem_mlp_status(int* timed_out) {
  if (!timed_out) return DEM_ERR_ARG;
  unsigned int* err = nullptr;
  if (err_flag(&err)) return DEM_ERR_CUDA;
  unsigned int h = 0;
  if (cudaMemcpy(&h, err, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) return DEM_ERR_CUDA;
  *timed_out = (int)h;
  return DEM_OK;
}

int dem_mlp_pack_bf16(const float* x, const int* idx, int rows, int k, int kpad, void* out, void* stream) {
  if (!x || !out || rows <= 0 || k <= 0 || kpad < k) return DEM_ERR_ARG;
  k_pack_bf16<<<blocks((size_t)rows * kpad), 256, 0, (cudaStream_t)stream>>>(x, idx, rows, k, kpad,
                                                                             static_cast<__nv_bfloat16*>(out));
  return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

int dem_mlp_transpose_bf16(const void* in, int rows, int cols, int ldo, void* out, void* stream) {
  if (!in || !out || rows <= 0 || cols <= 0 || ldo < rows) return DEM_ERR_ARG;
  const dim3 g((unsigned)((cols + 31) / 32), (unsigned)((ldo + 31) / 32));
  k_transpose_bf16<<<g, dim3(32, 8), 0, (cudaStream_t)stream>>>(static_cast<const __nv_bfloat16*>(in), rows, cols,
                                                                 ldo, static_cast<__nv_bfloat16*>(out));
  return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

int dem_mlp_act_backward(const float* dh, const float* z, size_t n, int act, void* dz_bf16, float* dz_f32,
                         void* stream) {
  if (!dh || !z || !dz_bf16 || n == 0) return DEM_ERR_ARG;
  if (act != DEM_MLP_BIAS_GELU && act != DEM_MLP_BIAS_RELU) return DEM_ERR_ARG;
  k_act_backward<<<blocks(n), 256, 0, (cudaStream_t)stream>>>(dh, z, n, act, static_cast<__nv_bfloat16*>(dz_bf16),
                                                             dz_f32);
  return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

int dem_mlp_colsum(const float* in, int rows, int cols, float* out, float* scratch, void* stream) {
  if (!in || !out || !scratch || rows <= 0 || cols <= 0) return DEM_ERR_ARG;
  const int S = std::min(DEM_MLP_COLSUM_SPLIT, std::max(1, rows / 64));
  k_colsum_part<<<dim3((unsigned)((cols + 31) / 32), (unsigned)S), dim3(32, 8), 0, (cudaStream_t)stream>>>(
      in, rows, cols, scratch);
  k_colsum_final<<<(unsigned)((cols + 127) / 128), 128, 0, (cudaStream_t)stream>>>(scratch, S, cols, out);
  return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

int dem_mlp_gather(const float* x, const int* idx, int rows, int k, float* out, void* stream) {
  if (!x || !idx || !out || rows <= 0 || k <= 0) return DEM_ERR_ARG;
  k_gather<<<blocks((size_t)rows * k), 256, 0, (cudaStream_t)stream>>>(x, idx, rows, k, out);
  return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

int dem_mlp_tick(int* step, void* stream) {
  if (!step) return DEM_ERR_ARG;
  k_tick<<<1, 1, 0, (cudaStream_t)stream>>>(step);
  return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

int dem_mlp_mse_grad(const float* y, const float* t, size_t n, void* dy_bf16, float* dy_f32, double* loss,
                     void* stream) {
  if (!y || !t || !dy_bf16 || n == 0) return DEM_ERR_ARG;
  k_mse_grad<<<blocks(n), 256, 0, (cudaStream_t)stream>>>(y, t, n, static_cast<__nv_bfloat16*>(dy_bf16), dy_f32,
                                                         loss);
  return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

int dem_mlp_adam(float* w, const float* g, float* m, float* v, size_t n, float lr, float b1, float b2, float eps,
                 float l2, const int* step, void* w_bf16, void* stream) {
  if (!w || !g || !m || !v || !step || n == 0) return DEM_ERR_ARG;
  k_adam<<<blocks(n), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, lr, b1, b2, eps, step, l2,
                                                     static_cast<__nv_bfloat16*>(w_bf16));
  return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

}  // extern "C"
