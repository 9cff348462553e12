// Forward-mode (tangent-linear) arithmetic for the sensitivity build of the
// engine: a value and its derivatives with respect to K parameters, carried
// through the same templated kernels as float and double.  Every operation
// applies the chain rule to the derivative part; comparisons look at values
// only, so branch decisions are those of the plain FP64 run.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

#include "dem_common.cuh"
#include "dem_step.cuh"

namespace dem {

// Parameters of the sensitivity build (derivative slots; DEM_SENS_* in b200dem.h).
enum SensParam : int { kSensEBond = 0, kSensKnKs = 1, kSensBondRadius = 2, kSensE = 3, kSensMu = 4, kSensCount = 5 };

template <int K>
struct Dual {
  double v;
  double d[K];
  __host__ __device__ Dual() {}
  __host__ __device__ Dual(double x) : v(x) {
    for (int k = 0; k < K; ++k) d[k] = 0.0;
  }
  __host__ __device__ explicit operator double() const { return v; }
  __host__ __device__ explicit operator float() const { return (float)v; }
  __host__ __device__ explicit operator unsigned int() const { return (unsigned int)v; }
  __host__ __device__ Dual& operator+=(const Dual& b) {
    v += b.v;
    for (int k = 0; k < K; ++k) d[k] += b.d[k];
    return *this;
  }
  __host__ __device__ Dual& operator-=(const Dual& b) {
    v -= b.v;
    for (int k = 0; k < K; ++k) d[k] -= b.d[k];
    return *this;
  }
  __host__ __device__ Dual& operator*=(const Dual& b) { return *this = *this * b; }
};

template <int K>
__host__ __device__ inline Dual<K> operator-(const Dual<K>& a) {
  Dual<K> r;
  r.v = -a.v;
  for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
  return r;
}
template <int K>
__host__ __device__ inline Dual<K> operator+(const Dual<K>& a, const Dual<K>& b) {
  Dual<K> r;
  r.v = a.v + b.v;
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <int K>
__host__ __device__ inline Dual<K> operator-(const Dual<K>& a, const Dual<K>& b) {
  Dual<K> r;
  r.v = a.v - b.v;
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <int K>
__host__ __device__ inline Dual<K> operator*(const Dual<K>& a, const Dual<K>& b) {
  Dual<K> r;
  r.v = a.v * b.v;
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
template <int K>
__host__ __device__ inline Dual<K> operator/(const Dual<K>& a, const Dual<K>& b) {
  Dual<K> r;
  const double q = a.v / b.v;
  r.v = q;
  for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - q * b.d[k]) / b.v;
  return r;
}
// mixed forms (a double is a constant)
template <int K>
__host__ __device__ inline Dual<K> operator+(const Dual<K>& a, double b) { return a + Dual<K>(b); }
template <int K>
__host__ __device__ inline Dual<K> operator+(double a, const Dual<K>& b) { return Dual<K>(a) + b; }
template <int K>
__host__ __device__ inline Dual<K> operator-(const Dual<K>& a, double b) { return a - Dual<K>(b); }
template <int K>
__host__ __device__ inline Dual<K> operator-(double a, const Dual<K>& b) { return Dual<K>(a) - b; }
template <int K>
__host__ __device__ inline Dual<K> operator*(const Dual<K>& a, double b) {
  Dual<K> r;
  r.v = a.v * b;
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b;
  return r;
}
template <int K>
__host__ __device__ inline Dual<K> operator*(double a, const Dual<K>& b) { return b * a; }
template <int K>
__host__ __device__ inline Dual<K> operator/(const Dual<K>& a, double b) {
  Dual<K> r;
  r.v = a.v / b;
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] / b;
  return r;
}
template <int K>
__host__ __device__ inline Dual<K> operator/(double a, const Dual<K>& b) { return Dual<K>(a) / b; }

#define DEM_DUAL_CMP(op)                                                                            \
  template <int K>                                                                                  \
  __host__ __device__ inline bool operator op(const Dual<K>& a, const Dual<K>& b) { return a.v op b.v; } \
  template <int K>                                                                                  \
  __host__ __device__ inline bool operator op(const Dual<K>& a, double b) { return a.v op b; }     \
  template <int K>                                                                                  \
  __host__ __device__ inline bool operator op(double a, const Dual<K>& b) { return a op b.v; }
DEM_DUAL_CMP(<)
DEM_DUAL_CMP(>)
DEM_DUAL_CMP(<=)
DEM_DUAL_CMP(>=)
DEM_DUAL_CMP(==)
DEM_DUAL_CMP(!=)
#undef DEM_DUAL_CMP

template <int K>
__host__ __device__ inline Dual<K> sqrt(const Dual<K>& a) {
  Dual<K> r;
  r.v = ::sqrt(a.v);
  const double h = r.v > 0.0 ? 0.5 / r.v : 0.0;
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * h;
  return r;
}
template <int K>
__host__ __device__ inline Dual<K> fabs(const Dual<K>& a) {
  return a.v < 0.0 ? -a : a;
}
template <int K>
__host__ __device__ inline Dual<K> floor(const Dual<K>& a) {
  return Dual<K>(::floor(a.v));
}

template <int K>
__host__ __device__ inline Dual<K> frozen(const Dual<K>& a) {
  return Dual<K>(a.v);
}

template <int K>
struct Dual4 {
  Dual<K> x, y, z, w;
};

template <int K>
struct RT<Dual<K>> {
  using V4 = Dual4<K>;
  static __host__ __device__ Dual<K> rcp(const Dual<K>& x) { return 1.0 / x; }
  static __host__ __device__ Dual<K> sqrt_rn(const Dual<K>& x) { return sqrt(x); }
  static __host__ __device__ Dual<K> rsqrt_rn(const Dual<K>& x) { return 1.0 / sqrt(x); }
  static __host__ __device__ Dual<K> fabs_(const Dual<K>& x) { return fabs(x); }
  static __host__ __device__ Dual<K> fma(const Dual<K>& a, const Dual<K>& b, const Dual<K>& c) { return a * b + c; }
  static constexpr double kPi = 3.1415926535897932384626433832795;
  static constexpr double kTwoThirds = 2.0 / 3.0;
  static constexpr double kDamp = -1.8257;
};

template <int K>
__device__ __forceinline__ Dual4<K> ld4(const Dual4<K>* p) { return *p; }
template <int K>
__device__ __forceinline__ Dual4<K> ld4_rw(const Dual4<K>* p) { return *p; }
template <int K>
__device__ __forceinline__ Dual4<K> ld4_cs(const Dual4<K>* p) { return *p; }
template <int K>
__device__ __forceinline__ void st4_cs(Dual4<K>* p, const Dual4<K>& v) { *p = v; }
template <int K>
__host__ __device__ __forceinline__ Dual4<K> mk4(const Dual<K>& a, const Dual<K>& b, const Dual<K>& c,
                                                 const Dual<K>& d) {
  return Dual4<K>{a, b, c, d};
}
template <int K>
__device__ __forceinline__ void acc1(Dual<K>* p, const Dual<K>& a) {
  atomicAdd(&p->v, a.v);
  for (int k = 0; k < K; ++k)
    if (a.d[k] != 0.0) atomicAdd(&p->d[k], a.d[k]);
}
template <int K>
__device__ __forceinline__ void acc3(Dual4<K>* p, const Dual<K>& a, const Dual<K>& b, const Dual<K>& c) {
  acc1(&p->x, a);
  acc1(&p->y, b);
  acc1(&p->z, c);
}
// deterministic mode: every value and derivative slot in 2^-50 fixed point
template <int K>
__device__ __forceinline__ void acc1_fix(Dual<K>* p, const Dual<K>& a) {
  fix_add(&p->v, a.v);
  for (int k = 0; k < K; ++k)
    if (a.d[k] != 0.0) fix_add(&p->d[k], a.d[k]);
}
template <int K>
__device__ __forceinline__ void acc3_fix(Dual4<K>* p, const Dual<K>& a, const Dual<K>& b, const Dual<K>& c) {
  acc1_fix(&p->x, a);
  acc1_fix(&p->y, b);
  acc1_fix(&p->z, c);
}
template <int K>
__device__ __forceinline__ Dual<K> unfix1(const Dual<K>& a) {
  Dual<K> r;
  r.v = fix_val(a.v);
  for (int k = 0; k < K; ++k) r.d[k] = fix_val(a.d[k]);
  return r;
}
template <int K>
__device__ __forceinline__ Dual4<K> unfix4(const Dual4<K>& a) {
  return Dual4<K>{unfix1(a.x), unfix1(a.y), unfix1(a.z), Dual<K>(0.0)};
}
template <int K>
__host__ __device__ __forceinline__ Dual<K> norm3(const Dual<K>& x, const Dual<K>& y, const Dual<K>& z) {
  return sqrt((x * x + y * y) + z * z);
}
template <int K>
__host__ __device__ __forceinline__ Dual<K> norm3_hist(const Dual<K>& x, const Dual<K>& y, const Dual<K>& z) {
  return sqrt((x * x + y * y) + z * z);
}

// Sensitivity hooks of the step kernels.  Per sample, sfl_tan holds 4K + 2
// doubles: the running platen-force tangents of this step (bottom K, top K),
// the last completed step's tangents (2K) and its platen force sums (2).
template <int K>
__device__ __forceinline__ void tangent_wall(const StepArgs<Dual<K>>& A, uint32_t s, int which, const Dual<K>& f) {
  double* t = A.sfl_tan + (size_t)s * (4 * K + 2) + which * K;
  for (int k = 0; k < K; ++k)
    if (f.d[k] != 0.0) {
      if (A.det)
        fix_add(t + k, -f.d[k]);
      else
        atomicAdd(t + k, -f.d[k]);
    }
}
template <int K>
__device__ __forceinline__ void tangent_step_end(const StepArgs<Dual<K>>& A, const SampleCtl& C, uint32_t s) {
  double* t = A.sfl_tan + (size_t)s * (4 * K + 2);
  for (int k = 0; k < 2 * K; ++k) {
    t[2 * K + k] = A.det ? fix_val(t[k]) : t[k];
    t[k] = 0.0;
  }
  t[4 * K] = C.sFL[0];
  t[4 * K + 1] = C.sFL[1];
}

// Host helpers: set a derivative slot (no-op for plain float / double).
template <class Real>
struct DualK {
  static constexpr int K = 0;
};
template <int K_>
struct DualK<Dual<K_>> {
  static constexpr int K = K_;
};
template <class Real>
inline void set_d(Real&, int, double) {}
template <int K>
inline void set_d(Dual<K>& x, int k, double dv) {
  x.d[k] = dv;
}

}  // namespace dem
