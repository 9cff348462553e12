// Device-side building blocks shared by the B200 DEM kernels.
//
// Arithmetic contract: this library is compiled with -fmad=false, so every
// a*b+c below is two correctly rounded operations, exactly as written; the
// float path uses the correctly rounded intrinsics __frcp_rn/__fsqrt_rn/
// __frsqrt_rn (the ones the reference kernels use), the double path uses IEEE
// division and sqrt.  Evaluation order follows the reference kernels
// (md_calculateforcesdem3.cu, md_compression_hm.cu), so per-bond results are
// reproducible bit for bit by a CPU restatement with the same order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dem {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;

template <class Real>
struct RT;

template <>
struct RT<float> {
  using V4 = float4;
  static __device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }
  static __device__ __forceinline__ float sqrt_rn(float x) { return __fsqrt_rn(x); }
  static __device__ __forceinline__ float rsqrt_rn(float x) { return __frsqrt_rn(x); }
  static __device__ __forceinline__ float fabs_(float x) { return fabsf(x); }
  // a*b+c with one rounding (the contractions the bond kernel chooses; its
  // CPU restatement uses fmaf at the same places)
  static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
  static constexpr float kPi = 3.14159265358979f;    // value of the reference's float pi
  static constexpr float kTwoThirds = 0.6666666667f;  // value of the reference's float 2/3
  static constexpr float kDamp = -1.8257f;
};

template <>
struct RT<double> {
  using V4 = double4;
  static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
  static __device__ __forceinline__ double sqrt_rn(double x) { return sqrt(x); }
  static __device__ __forceinline__ double rsqrt_rn(double x) { return 1.0 / sqrt(x); }
  static __device__ __forceinline__ double fabs_(double x) { return fabs(x); }
  static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
  static constexpr double kPi = 3.1415926535897932384626433832795;
  static constexpr double kTwoThirds = 2.0 / 3.0;
  static constexpr double kDamp = -1.8257;
};

template <class Real>
struct Vec3 {
  Real x, y, z;
};

// Euclidean norm of a pair vector.  float: the squares are exact in double, so
// the double sum and square root rounded once to float give the correctly
// rounded norm (the reference's norm3df is within a few ulp of it); double:
// sqrt of the rounded sum of squares.  A CPU evaluation of the same
// expression gives the same bits.
__device__ __forceinline__ float norm3(float x, float y, float z) {
  const double dx = x, dy = y, dz = z;
  return __double2float_rn(sqrt((dx * dx + dy * dy) + dz * dz));
}
__device__ __forceinline__ double norm3(double x, double y, double z) { return sqrt((x * x + y * y) + z * z); }

// Norm of a history vector for the bond-break test, in the working precision:
// sqrt(z*z + (y*y + x*x)) with the sums fused into the products.  The
// reference's norm3df is not correctly rounded either; a threshold test
// cannot tell the two apart except at exact ties.
__device__ __forceinline__ float norm3_hist(float x, float y, float z) {
  return __fsqrt_rn(__fmaf_rn(z, z, __fmaf_rn(y, y, x * x)));
}
__device__ __forceinline__ double norm3_hist(double x, double y, double z) {
  return sqrt(__fma_rn(z, z, __fma_rn(y, y, x * x)));
}

// 128-bit (float) / 256-bit (double) vector loads and stores through the
// read-only / default paths.
__device__ __forceinline__ float4 ld4(const float4* p) { return __ldg(p); }
__device__ __forceinline__ double4 ld4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = __ldg(q), b = __ldg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 ld4_rw(const float4* p) { return *p; }
__device__ __forceinline__ double4 ld4_rw(const double4* p) { return *p; }
// Streamed pair state (read once and written once per step): evict-first, so
// the particle arrays that every pair gathers stay in L2.
__device__ __forceinline__ float4 ld4_cs(const float4* p) { return __ldcs(p); }
__device__ __forceinline__ double4 ld4_cs(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = __ldcs(q), b = __ldcs(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void st4_cs(float4* p, const float4& v) { __stcs(p, v); }
__device__ __forceinline__ void st4_cs(double4* p, const double4& v) {
  double2* q = reinterpret_cast<double2*>(p);
  __stcs(q, make_double2(v.x, v.y));
  __stcs(q + 1, make_double2(v.z, v.w));
}

__device__ __forceinline__ float4 mk4(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
__device__ __forceinline__ double4 mk4(double a, double b, double c, double d) { return make_double4(a, b, c, d); }

// Accumulation of per-pair contributions into particle force/moment.
// float: one 128-bit vector reduction (sm_90+); double: three scalar atomics.
__device__ __forceinline__ void acc3(float4* p, float x, float y, float z) {
  atomicAdd(p, make_float4(x, y, z, 0.0f));
}
// Deterministic accumulation (dem_options.deterministic, FP32): contributions
// as 64-bit fixed point with a resolution of 2^-40 (an FP32 value of magnitude
// 2^-16 or more converts exactly, smaller ones round to the nearest 2^-40) added
// with integer atomics, so a particle's sum is exact and does not depend on the
// order in which its pairs are processed.  Range +-8.4e6 in engine units.
constexpr float kFixScale = 1099511627776.0f;        // 2^40
constexpr double kFixInv = 1.0 / 1099511627776.0;
__device__ __forceinline__ long long to_fix(float x) { return __float2ll_rn(x * kFixScale); }
__device__ __forceinline__ long long to_fix(double x) { return __double2ll_rn(x * (double)kFixScale); }
__device__ __forceinline__ void acc3q(long long* q, float x, float y, float z) {
  unsigned long long* u = reinterpret_cast<unsigned long long*>(q);
  atomicAdd(u + 0, (unsigned long long)to_fix(x));
  atomicAdd(u + 1, (unsigned long long)to_fix(y));
  atomicAdd(u + 2, (unsigned long long)to_fix(z));
}
// FP64 and sensitivity builds: the same scheme with 2^-50 resolution (range
// +-8192), stored in place of the double accumulators (same width; a zero
// double is a zero integer, so the accumulators reset as before).
constexpr double kFixScaleD = 1125899906842624.0;    // 2^50
constexpr double kFixInvD = 1.0 / 1125899906842624.0;
__device__ __forceinline__ long long fix_of(double x) { return __double2ll_rn(x * kFixScaleD); }
__device__ __forceinline__ void fix_add(double* slot, double x) {
  atomicAdd(reinterpret_cast<unsigned long long*>(slot), (unsigned long long)fix_of(x));
}
__device__ __forceinline__ double fix_val(double slot) { return (double)__double_as_longlong(slot) * kFixInvD; }
__device__ __forceinline__ void acc3(double4* p, double x, double y, double z) {
  double* q = reinterpret_cast<double*>(p);
  atomicAdd(q + 0, x);
  atomicAdd(q + 1, y);
  atomicAdd(q + 2, z);
}
__device__ __forceinline__ void acc3_fix(double4* p, double x, double y, double z) {
  fix_add(&p->x, x);
  fix_add(&p->y, y);
  fix_add(&p->z, z);
}
__device__ __forceinline__ double4 unfix4(const double4& a) {
  return make_double4(fix_val(a.x), fix_val(a.y), fix_val(a.z), 0.0);
}

// Counter-based normal deviates for per-bond properties: splitmix64 mixing of
// (seed, a, b, stream) into two uniforms, then Box-Muller.  Keyed by the
// original particle indices of the bond, so the draw does not depend on the
// thread or storage order.
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ double u01_from(uint64_t h) {
  // 53 random bits -> (0,1)
  return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

__host__ __device__ __forceinline__ double normal_from(uint64_t seed, uint64_t a, uint64_t b, uint64_t stream) {
  uint64_t k = splitmix64(seed ^ splitmix64(a * 0x100000001B3ull + b) ^ (stream * 0xD6E8FEB86659FD93ull));
  double u1 = u01_from(splitmix64(k));
  double u2 = u01_from(splitmix64(k ^ 0x5851F42D4C957F2Dull));
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586476925286766559 * u2);
}

// Bulk prefetch of [p, p + bytes) into L2 by the copy engine (sm_90+);
// p 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void l2_prefetch(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

}  // namespace dem
