// Surrogate MLP kernels (the B200 counterpart of the sklearn MLPRegressor that
// NN_MP.py trains on simulation results, NN_MP.py:374-378, 895): BF16 operands,
// FP32 accumulation on the 5th-generation tensor cores.
//
//   k_gemm_tn   C[M x N] = A[M x K] . B[N x K]^T, A and B row-major BF16 (both
//               "K-major"), accumulator in tensor memory.  Warp-specialised:
//               one thread streams 128-row tiles of A and TN-row tiles of B
//               (TN 32..256, narrowed for small grids), 64 of K per stage, with
//               the TMA into a 2-4 stage ring in the 128-byte swizzled layout;
//               one thread issues tcgen05.mma (M = 128, K = 16 per
//               instruction, kind::f16) as each stage lands and commits it
//               back to the producer; the eight warps then read the
//               accumulator with tcgen05.ld (warps w and w + 4 share lanes
//               32 (w % 4) and split the columns) and apply the epilogue in
//               registers: + bias and GELU or ReLU to BF16 (hidden layers,
//               pre-activation kept in FP32 when asked), + bias to FP32
//               (output layer), or plain FP32 (weight and activation
//               gradients), written with 16-byte stores.
//   small kernels: input packing, transposes, activation backward, column
//               sums, MSE gradient, Adam.
//
// All waits are bounded: a commit that does not arrive within the poll limit
// sets *err, the block waits once more (bounded) and frees its tensor memory.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "b200dem.h"

namespace dem {
namespace {

constexpr int kTM = 128;      // rows per tile (tcgen05 M)
constexpr int kThreads = 256; // eight warps: all load, warp 0 lane 0 issues, all eight drain the accumulator
constexpr uint32_t kPollLimit = 1u << 22;

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t* b) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(b)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void bar_init_count(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void bar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(b)) : "memory");
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
// Shared-memory matrix descriptor of a K-major operand in the 128-byte
// swizzled layout the TMA writes: rows of 64 BF16 (128 bytes), 8-row atoms of
// 1024 bytes one after another (stride byte offset 1024; the leading byte
// offset is unused for swizzled K-major operands and set to 16), descriptor
// version 1, layout type 2 (SWIZZLE_128B).  The K = 16 slices of a row start
// 32 bytes apart inside the atom.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}
__device__ __forceinline__ void bar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}
// TMA load of one box (x = K element, y = row) of a 2-D tensor map into shared
// memory, completing on the mbarrier; no multicast
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(saddr(bar))
      : "memory");
}

// GELU in the tanh form of Hendrycks & Gimpel (2016),
//   gelu(z) = z/2 (1 + tanh(u)) = z s,  s = 1 / (1 + exp(-2u)),
//   u = sqrt(2/pi) (z + 0.044715 z^3),
// evaluated as z s with the hardware base-2 exponential (ex2.approx, with
// exp(-2u) = 2^(-2u log2 e) and the three constant factors folded into one)
// and reciprocal (rcp.approx), which keep their relative accuracy in both
// tails (the form 1 + tanh(u) cancels for large negative z); its derivative
//   gelu'(z) = s + 2 z s (1 - s) sqrt(2/pi) (1 + 3 0.044715 z^2).
// ReLU takes 0 as its derivative at 0, as sklearn's MLPRegressor does
// (NN_MP.py:374 uses its default activation).
constexpr float kGeluC = 0.7978845608028654f;   // sqrt(2/pi)
constexpr float kGeluA = 0.044715f;
constexpr float kGeluE = (float)(-2.0 * 0.7978845608028654 * 1.4426950408889634);   // -2 sqrt(2/pi) log2(e)
__device__ __forceinline__ float rcp_hw(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ex2_hw(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu_s(float z) {
  return rcp_hw(1.f + ex2_hw(kGeluE * __fmaf_rn(kGeluA * z * z, z, z)));
}
__device__ __forceinline__ float gelu(float z) { return z * gelu_s(z); }
__device__ __forceinline__ float gelu_grad(float z) {
  const float s = gelu_s(z);
  const float du = kGeluC * __fmaf_rn(3.f * kGeluA, z * z, 1.f);
  return __fmaf_rn(2.f * z * s * (1.f - s), du, s);
}

// Pipeline geometry of a TN-column tile: a stage holds 64 of K (one 128-byte
// swizzled row) for the 128 rows of A and the TN rows of B; as many stages as
// fit in about 100 KB (2..4), so that two blocks share an SM and one block's
// epilogue overlaps the other's main loop.
constexpr int kSK = 64;
template <int TN>
struct GemmCfg {
  static constexpr int kABytes = kTM * 128;
  static constexpr int kStageBytes = (kTM + TN) * 128;
  static constexpr int kStages = (100 * 1024 / kStageBytes) < 2 ? 2 : ((100 * 1024 / kStageBytes) > 4 ? 4 : (100 * 1024 / kStageBytes));
  static constexpr int kSmem = kStages * kStageBytes + 1024 /* alignment */ + 8 * (2 * kStages + 1) + 16;
  static constexpr uint32_t kCols = TN <= 32 ? 32 : (TN <= 64 ? 64 : (TN <= 128 ? 128 : 256));
};

// 32 consecutive FP32 accumulator columns of this thread's row (TMEM address
// taddr: lane quarter of the warp, column), without waiting for them
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Epilogue of one 32-column chunk of an accumulator row, its values r already
// loaded from tensor memory: + bias and the activation to BF16 and/or the
// FP32 values, written with 16-byte stores (scalar stores at a ragged right
// edge or when a row is not a multiple of 16 bytes); rows >= M and columns >=
// N are not written.  kBias4: the bias is a zero-padded shared-memory copy
// read as 16-byte vectors (the same address in every lane: one broadcast per
// vector); otherwise it is read from global memory value by value.
template <bool kBias4 = false>
__device__ __forceinline__ void chunk_out(const uint32_t (&r)[32], int row, int nc, int M, int N,
                                          const float* __restrict__ bias, int mode, bool act,
                                          float* __restrict__ outf, __nv_bfloat16* __restrict__ outh) {
  if (row >= M || nc >= N) return;
  const int cols = min(32, N - nc);
  float v[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
  if (mode != DEM_MLP_PLAIN) {
    if constexpr (kBias4) {
      const float4* b4 = reinterpret_cast<const float4*>(bias + nc);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const float4 b = b4[j];
        v[4 * j] += b.x;
        v[4 * j + 1] += b.y;
        v[4 * j + 2] += b.z;
        v[4 * j + 3] += b.w;
      }
    } else {
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] += (j < cols) ? __ldg(bias + nc + j) : 0.f;
    }
  }
  const size_t o = (size_t)row * N + nc;
  if (outf) {
    if (cols == 32 && (N & 3) == 0) {
      float4* dst = reinterpret_cast<float4*>(outf + o);
#pragma unroll
      for (int j = 0; j < 8; ++j) dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    } else {
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (j < cols) outf[o + j] = v[j];
    }
  }
  if (act) {
    const bool g = mode == DEM_MLP_BIAS_GELU;
    uint32_t h[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const float a0 = g ? gelu(v[2 * j]) : fmaxf(v[2 * j], 0.f);
      const float a1 = g ? gelu(v[2 * j + 1]) : fmaxf(v[2 * j + 1], 0.f);
      const __nv_bfloat162 p = __floats2bfloat162_rn(a0, a1);
      h[j] = *reinterpret_cast<const uint32_t*>(&p);
    }
    if (cols == 32 && (N & 7) == 0) {
      uint4* dst = reinterpret_cast<uint4*>(outh + o);
#pragma unroll
      for (int j = 0; j < 4; ++j) dst[j] = make_uint4(h[4 * j], h[4 * j + 1], h[4 * j + 2], h[4 * j + 3]);
    } else {
      unsigned short* dst = reinterpret_cast<unsigned short*>(outh + o);
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (j < cols) dst[j] = (unsigned short)((j & 1) ? (h[j >> 1] >> 16) : (h[j >> 1] & 0xFFFFu));
    }
  }
}

// One chunk loaded, waited for and written (every lane of the warp takes part
// in the load).
template <bool kBias4 = false>
__device__ __forceinline__ void drain_chunk(uint32_t taddr, int row, int nc, int M, int N,
                                            const float* __restrict__ bias, int mode, bool act,
                                            float* __restrict__ outf, __nv_bfloat16* __restrict__ outh) {
  uint32_t r[32];
  tmem_ld32(taddr, r);
  tmem_wait_ld();
  chunk_out<kBias4>(r, row, nc, M, N, bias, mode, act, outf, outh);
}

// Warp-specialised: warp 0 lane 0 streams the stages with the TMA (A box
// 64 x 128 rows, B box 64 x TN rows, 128-byte swizzle, zero fill past the
// edges), warp 1 allocates the accumulator and its lane 0 issues the MMAs of
// each stage once its bytes have landed and commits the stage back to the
// producer; all eight warps then drain the accumulator.
template <int TN>
__global__ void __launch_bounds__(kThreads) k_gemm_tn(const __grid_constant__ CUtensorMap tmA,
                                                 const __grid_constant__ CUtensorMap tmB, int M, int N, int K,
                                                 const float* __restrict__ bias, int mode, float* __restrict__ outf,
                                                 __nv_bfloat16* __restrict__ outh, unsigned int* err) {
  using Cfg = GemmCfg<TN>;
  constexpr int S = Cfg::kStages;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + S * Cfg::kStageBytes);
  uint64_t* empty = full + S;
  uint64_t* accum = empty + S;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(accum + 1);
  const uint32_t sbase = saddr(base);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kTM, n0 = blockIdx.y * TN;
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tslot)),
                 "r"(Cfg::kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      bar_init(&full[s]);
      bar_init(&empty[s]);
    }
    bar_init(accum);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(kTM >> 4) << 24);
  const int rounds = (K + kSK - 1) / kSK;
  bool ok = true;
  if (warp == 0 && lane == 0) {
    // producer
    int issued = 0;
    for (int c = 0; c < rounds; ++c) {
      const int s = c % S;
      if (c >= S && !bar_wait(&empty[s], (uint32_t)((c / S - 1) & 1))) {
        ok = false;
        break;
      }
      const uint32_t st = sbase + s * Cfg::kStageBytes;
      bar_expect_tx(&full[s], (uint32_t)Cfg::kStageBytes);
      tma_load_2d(st, &tmA, c * kSK, m0, &full[s]);
      tma_load_2d(st + Cfg::kABytes, &tmB, c * kSK, n0, &full[s]);
      issued = c + 1;
    }
    // no load may still be writing shared memory when the block ends
    for (int c = (issued > S ? issued - S : 0); c < issued; ++c)
      if (!bar_wait(&full[c % S], (uint32_t)((c / S) & 1))) ok = false;
    if (!ok) atomicOr(err, 1u);
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    int committed = 0;
    for (int c = 0; c < rounds; ++c) {
      const int s = c % S;
      if (!bar_wait(&full[s], (uint32_t)((c / S) & 1))) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t st = sbase + s * Cfg::kStageBytes;
      for (int kk = 0; kk < kSK / 16; ++kk) {
        const uint64_t da = smem_desc_sw128(st + (uint32_t)(kk * 32));
        const uint64_t db = smem_desc_sw128(st + (uint32_t)(Cfg::kABytes + kk * 32));
        const uint32_t acc = (c > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       saddr(&empty[s]))
                   : "memory");
      committed = c + 1;
    }
    if (ok)
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       saddr(accum))
                   : "memory");
    else if (committed > 0)
      bar_wait(&empty[(committed - 1) % S], (uint32_t)(((committed - 1) / S) & 1));
    if (!ok) atomicOr(err, 1u);
  }
  // everyone: the accumulator is complete when the last commit arrives
  if (rounds > 0) ok = ok && bar_wait(accum, 0u);
  ok = !__syncthreads_or(!ok);
  if (!ok && tid == 0) atomicOr(err, 1u);
  if (ok && rounds > 0) {
    tc_fence_after();
    // epilogue: warp w reads accumulator lanes 32 (w % 4) .. +31 (the lanes its
    // quarter of the warps may access), warps w and w + 4 taking alternate
    // 32-column chunks; a thread holds 32 consecutive columns of one row and
    // writes them with 16-byte stores (scalar stores at a ragged right edge
    // or when a row is not a multiple of 16 bytes)
    const int q4 = warp & 3, half = warp >> 2;
    const int row = m0 + q4 * 32 + lane;
    const bool act = mode == DEM_MLP_BIAS_GELU || mode == DEM_MLP_BIAS_RELU;
    for (int col0 = 32 * half; col0 < TN; col0 += 64)
      drain_chunk(tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)col0, row, n0 + col0, M, N, bias, mode, act, outf,
                  outh);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::kCols) : "memory");
}

// Persistent form for the tall layers (many 128-row tiles, N <= 256, K <= 256,
// the surrogate's forward and inference passes): one block per SM (two when
// the accumulators are narrow) walks the 128-row tiles blockIdx.x,
// blockIdx.x + gridDim.x, ...  The whole B operand (N x K, at most 128 KB)
// is loaded once and stays in shared memory; A streams through a four-stage
// ring.  Tensor memory holds two accumulators, so the epilogue of tile t
// (eight warps draining accumulator t % 2) overlaps the loads and MMAs of
// tile t + 1 (warp 0: TMA producer, warp 1: MMA issuer).
//   full[s] / empty[s]   A stage s loaded / consumed by its MMAs
//   bfull                the resident B has landed
//   tfull[a] / tempty[a] accumulator a complete / drained (eight arrivals)
template <int TN>
struct PersistCfg {
  static constexpr int kStages = 4;
  static constexpr int kABytes = kTM * 128;                     // one 64-wide K slice of a 128-row tile
  static constexpr int kBBlock = TN * 128;                      // one 64-wide K slice of B
  static constexpr int kMaxK = 256;
  static constexpr int kBBytes = (kMaxK / kSK) * kBBlock;
  // mbarriers and the TMEM address slot, rounded to 16 bytes (the bias copy
  // after them is read as 16-byte vectors)
  static constexpr int kBarBytes = (8 * (2 * kStages + 5) + 16 + 15) / 16 * 16;
  static constexpr int kSmem = kStages * kABytes + kBBytes + 1024 + kBarBytes + TN * 4;
  static constexpr uint32_t kCols = 2 * (TN <= 32 ? 32 : (TN <= 64 ? 64 : (TN <= 128 ? 128 : 256)));
  static constexpr int kEpiWarps = 16;
  static_assert((kStages * kABytes + kBBytes) % 1024 == 0, "B and the barriers follow 1024-byte aligned stages");
  static_assert(kSmem <= 227 * 1024, "dynamic shared memory of one block");
  static constexpr int kThreads = 64 + 32 * kEpiWarps;          // producer, MMA, sixteen epilogue warps
};

template <int TN>
__global__ void __launch_bounds__(PersistCfg<TN>::kThreads, 1)
    k_gemm_tn_persist(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M, int N,
                      int K, const float* __restrict__ bias, int mode, float* __restrict__ outf,
                      __nv_bfloat16* __restrict__ outh, unsigned int* err) {
  using Cfg = PersistCfg<TN>;
  constexpr int S = Cfg::kStages;
  constexpr uint32_t kAcc = Cfg::kCols / 2;   // column offset of the second accumulator
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* bres = base + S * Cfg::kABytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(bres + Cfg::kBBytes);
  uint64_t* empty = full + S;
  uint64_t* bfull = empty + S;
  uint64_t* tfull = bfull + 1;
  uint64_t* tempty = tfull + 2;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(tempty + 2);
  float* sbias = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(full) + Cfg::kBarBytes);
  const uint32_t sbase = saddr(base), bbase = saddr(bres);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles = (M + kTM - 1) / kTM;
  const int rounds = (K + kSK - 1) / kSK;
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tslot)),
                 "r"(Cfg::kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      bar_init(&full[s]);
      bar_init(&empty[s]);
    }
    bar_init(bfull);
    for (int a = 0; a < 2; ++a) {
      bar_init(&tfull[a]);
      bar_init_count(&tempty[a], Cfg::kEpiWarps);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(kTM >> 4) << 24);
  bool ok = true;
  if (warp == 0) {
    if (lane == 0) {
      // producer: B once, then the A slices of every tile of this block
      bar_expect_tx(bfull, (uint32_t)(rounds * Cfg::kBBlock));
      for (int c = 0; c < rounds; ++c) tma_load_2d(bbase + c * Cfg::kBBlock, &tmB, c * kSK, 0, bfull);
      int g = 0;
      for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        for (int c = 0; c < rounds; ++c, ++g) {
          const int s = g % S;
          if (g >= S && !bar_wait(&empty[s], (uint32_t)((g / S - 1) & 1))) {
            ok = false;
            break;
          }
          bar_expect_tx(&full[s], (uint32_t)Cfg::kABytes);
          tma_load_2d(sbase + s * Cfg::kABytes, &tmA, c * kSK, t * kTM, &full[s]);
        }
      }
      // no load may still be writing shared memory when the block ends
      for (int q = (g > S ? g - S : 0); q < g; ++q)
        if (!bar_wait(&full[q % S], (uint32_t)((q / S) & 1))) ok = false;
      if (!bar_wait(bfull, 0u)) ok = false;
      if (!ok) atomicOr(err, 1u);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer
      int g = 0, it = 0, last_commit = -1;
      if (!bar_wait(bfull, 0u)) ok = false;
      for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x, ++it) {
        const int a = it & 1;
        if (it >= 2 && !bar_wait(&tempty[a], (uint32_t)(((it >> 1) - 1) & 1))) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)a * kAcc;
        for (int c = 0; c < rounds; ++c, ++g) {
          const int s = g % S;
          if (!bar_wait(&full[s], (uint32_t)((g / S) & 1))) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t st = sbase + s * Cfg::kABytes;
          for (int kk = 0; kk < kSK / 16; ++kk) {
            const uint64_t da = smem_desc_sw128(st + (uint32_t)(kk * 32));
            const uint64_t db = smem_desc_sw128(bbase + (uint32_t)(c * Cfg::kBBlock + kk * 32));
            const uint32_t acc = (c > 0 || kk > 0) ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                ::"r"(d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                : "memory");
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                           saddr(&empty[s]))
                       : "memory");
          last_commit = s;
        }
        if (!ok) break;
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         saddr(&tfull[a]))
                     : "memory");
      }
      // on a timeout, let the MMAs already issued finish before the block ends
      if (!ok && last_commit >= 0) bar_wait(&empty[last_commit], (uint32_t)(((g - 1) / S) & 1));
      if (!ok) atomicOr(err, 1u);
    }
  } else {
    // epilogue warps 2..17: lane quarter warp % 4 (the accumulator lanes this
    // warp may read), column group (warp - 2) / 4 (32-column chunks cg,
    // cg + 4, ...).  The bias goes to shared memory first (zero past N).
    const int q4 = warp & 3, cg = (warp - 2) >> 2;
    const bool act = mode == DEM_MLP_BIAS_GELU || mode == DEM_MLP_BIAS_RELU;
    for (int c = tid - 64; c < TN; c += 32 * Cfg::kEpiWarps)
      sbias[c] = (mode != DEM_MLP_PLAIN && c < N) ? bias[c] : 0.f;
    asm volatile("bar.sync 1, %0;" ::"n"(32 * Cfg::kEpiWarps) : "memory");
    int it = 0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++it) {
      const int a = it & 1;
      if (!bar_wait(&tfull[a], (uint32_t)((it >> 1) & 1))) {
        ok = false;
        break;
      }
      tc_fence_after();
      const int row = t * kTM + q4 * 32 + lane;
      const uint32_t acc = tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)a * kAcc;
      // (loading a warp's two chunks before one wait was measured slower:
      // 23.4 against 21.4 us on the 65,536 x 256 x 256 layer)
      for (int col0 = 32 * cg; col0 < TN; col0 += 128)
        drain_chunk<true>(acc + (uint32_t)col0, row, col0, M, N, sbias, mode, act, outf, outh);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) bar_arrive(&tempty[a]);
    }
    if (!ok && lane == 0) atomicOr(err, 1u);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::kCols) : "memory");
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

// Adam over a list of arrays in one launch: block row y updates array y of
// the descriptor list (grid-stride over its elements), with the same update as
// k_adam.
__global__ void k_adam_multi(const dem_mlp_tensor* __restrict__ list, float lr, float b1, float b2, float eps,
                             const int* __restrict__ step) {
  const dem_mlp_tensor T = list[blockIdx.y];
  const float t = (float)max(*step, 1);
  const float c1 = 1.f - powf(b1, t), c2 = 1.f - powf(b2, t);
  __nv_bfloat16* wh = static_cast<__nv_bfloat16*>(T.w_bf16);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < T.n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = T.g[i] + T.l2 * T.w[i];
    const float mi = b1 * T.m[i] + (1.f - b1) * gi;
    const float vi = b2 * T.v[i] + (1.f - b2) * gi * gi;
    T.m[i] = mi;
    T.v[i] = vi;
    const float wi = T.w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    T.w[i] = wi;
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
    // zeroed before any caller stream uses it (the caller's stream may not be
    // ordered with the legacy default stream)
    if (cudaMemsetAsync(p, 0, sizeof(unsigned int), 0) != cudaSuccess || cudaStreamSynchronize(0) != cudaSuccess)
      return DEM_ERR_CUDA;
    g_err[dev] = p;
  }
  *out = g_err[dev];
  return DEM_OK;
}

uint32_t blocks(size_t n) { return (uint32_t)std::min<size_t>((n + 255) / 256, 148 * 16); }

// Tensor maps of the two operands: row-major BF16 [rows x K], box 64 x rows
// of the tile, 128-byte swizzle, zero fill outside.  cuTensorMapEncodeTiled
// comes from the driver through the runtime (no link against libcuda).
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}
int make_map(CUtensorMap* map, const void* ptr, int rows, int K, int box_rows) {
  auto fn = encode_fn();
  if (!fn) return DEM_ERR_CUDA;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)K * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kSK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? DEM_OK : DEM_ERR_CUDA;
}

// the pipeline needs more than the default 48 KB of dynamic shared memory: the
// limit is raised once per device and tile width (before any graph capture,
// since the first call of every shape comes from eager code)
template <int TN>
int launch_gemm(unsigned gx, unsigned gy, cudaStream_t st, const __nv_bfloat16* a, const __nv_bfloat16* b, int M,
                int N, int K, const float* bias, int mode, float* outf, __nv_bfloat16* oh, unsigned int* err) {
  static bool raised[kMaxDev] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return DEM_ERR_CUDA;
  if (!raised[dev]) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (cudaFuncSetAttribute(k_gemm_tn<TN>, cudaFuncAttributeMaxDynamicSharedMemorySize, GemmCfg<TN>::kSmem) !=
        cudaSuccess)
      return DEM_ERR_CUDA;
    raised[dev] = true;
  }
  CUtensorMap ma, mb;
  if (make_map(&ma, a, M, K, kTM) || make_map(&mb, b, N, K, TN)) return DEM_ERR_CUDA;
  k_gemm_tn<TN><<<dim3(gx, gy), kThreads, GemmCfg<TN>::kSmem, st>>>(ma, mb, M, N, K, bias, mode, outf, oh, err);
  return DEM_OK;
}

template <int TN>
int launch_gemm_persist(unsigned grid, cudaStream_t st, const __nv_bfloat16* a, const __nv_bfloat16* b, int M, int N,
                        int K, const float* bias, int mode, float* outf, __nv_bfloat16* oh, unsigned int* err) {
  static bool raised[kMaxDev] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return DEM_ERR_CUDA;
  if (!raised[dev]) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (cudaFuncSetAttribute(k_gemm_tn_persist<TN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             PersistCfg<TN>::kSmem) != cudaSuccess)
      return DEM_ERR_CUDA;
    raised[dev] = true;
  }
  CUtensorMap ma, mb;
  if (make_map(&ma, a, M, K, kTM) || make_map(&mb, b, N, K, TN)) return DEM_ERR_CUDA;
  k_gemm_tn_persist<TN><<<grid, PersistCfg<TN>::kThreads, PersistCfg<TN>::kSmem, st>>>(ma, mb, M, N, K, bias, mode,
                                                                                       outf, oh, err);
  return DEM_OK;
}

// SM count of the current device (looked up once per device)
int sm_count() {
  static int cached[kMaxDev] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return 0;
  if (cached[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    cached[dev] = n;
  }
  return cached[dev];
}

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
  // tall layers (at least two 128-row tiles per SM, one column tile, B small
  // enough to stay in shared memory): the persistent kernel, one block per SM
  const int sms = sm_count();
  if (sms > 0 && N <= 256 && K <= PersistCfg<256>::kMaxK && gx >= 2u * (unsigned)sms) {
    const unsigned grid = (unsigned)sms;
    int rc;
    if (N <= 32)
      rc = launch_gemm_persist<32>(grid, st, a, b, M, N, K, bias, mode, out_f32, oh, err);
    else if (N <= 64)
      rc = launch_gemm_persist<64>(grid, st, a, b, M, N, K, bias, mode, out_f32, oh, err);
    else if (N <= 128)
      rc = launch_gemm_persist<128>(grid, st, a, b, M, N, K, bias, mode, out_f32, oh, err);
    else
      rc = launch_gemm_persist<256>(grid, st, a, b, M, N, K, bias, mode, out_f32, oh, err);
    if (rc) return rc;
    return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
  }
  // tile width: the widest that covers N, narrowed while the grid would leave
  // most SMs idle (small batches), down to 32 columns
  int tn = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
  while (tn > 32 && (size_t)gx * (size_t)((N + tn - 1) / tn) < 148) tn >>= 1;
  const unsigned gy = (unsigned)((N + tn - 1) / tn);
  int rc;
  if (tn == 32)
    rc = launch_gemm<32>(gx, gy, st, a, b, M, N, K, bias, mode, out_f32, oh, err);
  else if (tn == 64)
    rc = launch_gemm<64>(gx, gy, st, a, b, M, N, K, bias, mode, out_f32, oh, err);
  else if (tn == 128)
    rc = launch_gemm<128>(gx, gy, st, a, b, M, N, K, bias, mode, out_f32, oh, err);
  else
    rc = launch_gemm<256>(gx, gy, st, a, b, M, N, K, bias, mode, out_f32, oh, err);
  if (rc) return rc;
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
  // up to 2048 rows one pass writes the sums directly; beyond, partial sums of
  // row slices are added in order by a second pass
  const int S = rows <= 2048 ? 1 : std::min(DEM_MLP_COLSUM_SPLIT, rows / 256);
  k_colsum_part<<<dim3((unsigned)((cols + 31) / 32), (unsigned)S), dim3(32, 8), 0, (cudaStream_t)stream>>>(
      in, rows, cols, S == 1 ? out : scratch);
  if (S > 1)
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

int dem_mlp_adam_multi(const dem_mlp_tensor* list, int count, size_t max_n, float lr, float b1, float b2,
                       float eps, const int* step, void* stream) {
  if (!list || !step || count <= 0 || count > 65535 || max_n == 0) return DEM_ERR_ARG;
  const dim3 g(std::min<uint32_t>((uint32_t)((max_n + 255) / 256), 148u * 4u), (unsigned)count);
  k_adam_multi<<<g, 256, 0, (cudaStream_t)stream>>>(list, lr, b1, b2, eps, step);
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
