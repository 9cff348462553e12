// Sample preparation kernels: soft repulsion, FIRE relaxation and the
// cylinder confinement of the reference's h_CreateCylinderSample
// (md_createcylindersample.cu:184-439):
//
//   k_soft_pairs      pair force of d_CalculateForces (md_calculateforces.cu:20-67):
//                     F_i += -D (a^2/r^2) (x_j - x_i) for r < a, a = s (r_i + r_j),
//                     or a linear overlap spring (packing by radius growth)
//   k_fire_power      P = sum F.v per sample (d_FdotVEntire, md_firerelaxation.cu:375-494);
//                     the last block adapts dt and alpha on the device (the host
//                     logic of md_createcylindersample.cu:368-397)
//   k_fire_move       half step back on P <= 0 (d_CalculateDecrementsHalfStepFIRE),
//                     FIRE velocity mix and move (d_CalculateIncrementsFIRE,
//                     md_firerelaxation.cu:18-70), cylinder confinement
//                     (d_CylinderRestrictionZ, md_cylinderrestriction.cu:190-234)
#pragma once

#include "dem_common.cuh"

namespace dem {

struct FireCtl {
  double P;            // F.v of the current step (accumulated)
  double dt, alpha;    // current FIRE time step and mixing
  double dt0, dtmax, dtmin, dtgrow, dtshrink, alpha0, alphashrink;
  uint32_t Npos, Nneg, Ndelay, back;  // back: this step moves half a step back and zeroes v
  unsigned long long step;
  float max_overlap;   // largest relative overlap seen by the pair kernel this step
  float pad;
};

template <class Real>
struct PackArgs {
  using V4 = typename RT<Real>::V4;
  V4* pos;        // x, y, z, target radius
  V4* vel;        // v, dt0/m (reference Po.dt_d_m)
  V4* frc;
  const uint32_t* sid;
  uint32_t np;
  const uint2* c_ij;
  const uint32_t* nc;
  const Real* scale;   // per sample: radius scale during growth
  const Real* D;       // per sample: soft-force constant (reference Po.D) or spring stiffness
  int linear;          // 0: reference soft force, 1: linear overlap spring
  FireCtl* fire;       // per sample
  const Real* cyl;     // per sample: centre x,y,z, radius R, half height H (5 values)
  uint32_t nsamples;
  unsigned int* blocks_done;
  int viscous;         // 1: viscous step of the pre-relaxation instead of FIRE
  Real vis;            // viscous coefficient (reference Po.vism)
};

template <class Real>
__global__ void __launch_bounds__(256) k_soft_pairs(PackArgs<Real> A) {
  using V4 = typename RT<Real>::V4;
  const uint32_t nc = *A.nc;
  float worst = 0.f;
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    const uint2 e = A.c_ij[c];
    const uint32_t i = e.x, j = e.y & 0x7FFFFFFFu;
    const uint32_t s = A.sid[i];
    const V4 xi = ld4(A.pos + i), xj = ld4(A.pos + j);
    const Real dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
    const Real rr = (dx * dx + dy * dy) + dz * dz;
    const Real a = A.scale[s] * (xi.w + xj.w);
    const Real aa = a * a;
    if (!(rr < aa) || !(rr > Real(0))) continue;
    Real fm;
    if (!A.linear) {
      // d_CalculateForces: fm = -D * (aa / rr)
      const Real aa_d_rr = aa * RT<Real>::rcp(rr);
      fm = (-A.D[s]) * aa_d_rr;
    } else {
      const Real r = RT<Real>::sqrt_rn(rr);
      fm = -A.D[s] * (a - r) / r;
    }
    acc3(A.frc + i, fm * dx, fm * dy, fm * dz);
    acc3(A.frc + j, -fm * dx, -fm * dy, -fm * dz);
    const float ov = (float)((a - RT<Real>::sqrt_rn(rr)) / a);
    worst = fmaxf(worst, ov);
  }
  // block max of the relative overlap, then one atomic per block
  for (int o = 16; o > 0; o >>= 1) worst = fmaxf(worst, __shfl_xor_sync(0xFFFFFFFFu, worst, o));
  if ((threadIdx.x & 31) == 0 && worst > 0.f && A.nsamples == 1)
    atomicMax(reinterpret_cast<int*>(&A.fire[0].max_overlap), __float_as_int(worst));
}

template <class Real>
__global__ void __launch_bounds__(256) k_fire_power(PackArgs<Real> A) {
  using V4 = typename RT<Real>::V4;
  __shared__ int s_last;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < A.np; p += gridDim.x * blockDim.x) {
    const V4 f = A.frc[p], v = A.vel[p];
    const double pw = (double)((f.x * v.x + f.y * v.y) + f.z * v.z);
    if (pw != 0.0) atomicAdd(&A.fire[A.sid[p]].P, pw);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(A.blocks_done, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  for (uint32_t s = threadIdx.x; s < A.nsamples; s += blockDim.x) {
    FireCtl& F = A.fire[s];
    // md_createcylindersample.cu:374-397
    if (F.P > 0) {
      ++F.Npos;
      F.Nneg = 0;
      if (F.Npos > F.Ndelay) {
        F.dt = (F.dt * F.dtgrow < F.dtmax) ? F.dt * F.dtgrow : F.dtmax;
        F.alpha *= F.alphashrink;
      }
      F.back = 0;
    } else {
      F.Npos = 0;
      ++F.Nneg;
      if (F.step > F.Ndelay) {
        F.dt = (F.dt * F.dtshrink > F.dtmin) ? F.dt * F.dtshrink : F.dtmin;
        F.alpha = F.alpha0;
      }
      F.back = 1;
    }
    F.P = 0.0;
    ++F.step;
  }
  if (threadIdx.x == 0) *A.blocks_done = 0;
}

template <class Real>
__global__ void __launch_bounds__(256) k_fire_move(PackArgs<Real> A) {
  using T = RT<Real>;
  using V4 = typename T::V4;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < A.np; p += gridDim.x * blockDim.x) {
    const uint32_t s = A.sid[p];
    V4 x = A.pos[p], v = A.vel[p], f = A.frc[p];
    const Real dtm = v.w;
    if (A.viscous) {
      // d_CalculateIncrementsViscos: v += (F - v vis) dt/m, x += v dt
      const Real dt = (Real)A.fire[s].dt0;
      v.x += (f.x - v.x * A.vis) * dtm;
      v.y += (f.y - v.y * A.vis) * dtm;
      v.z += (f.z - v.z * A.vis) * dtm;
      x.x += v.x * dt;
      x.y += v.y * dt;
      x.z += v.z * dt;
    } else {
      const FireCtl& F = A.fire[s];
      const Real dt = (Real)F.dt, alpha = (Real)F.alpha;
      if (F.back) {
        const Real h = Real(0.5) * dt;
        x.x -= v.x * h;
        x.y -= v.y * h;
        x.z -= v.z * h;
      }
      // the reference recomputes v from the current force only (md_firerelaxation.cu:28-44)
      Real vx = f.x * dtm, vy = f.y * dtm, vz = f.z * dtm;
      const Real vv = (vx * vx + vy * vy) + vz * vz;
      const Real ff = (f.x * f.x + f.y * f.y) + f.z * f.z;
      Real vdf;
      if (ff > Real(1e-12f))
        vdf = alpha * T::sqrt_rn(vv * T::rcp(ff));
      else
        vdf = alpha * T::sqrt_rn(vv) * Real(1e6);
      vx = (Real(1) - alpha) * vx + vdf * f.x;
      vy = (Real(1) - alpha) * vy + vdf * f.y;
      vz = (Real(1) - alpha) * vz + vdf * f.z;
      v.x = vx;
      v.y = vy;
      v.z = vz;
      x.x += vx * dt;
      x.y += vy * dt;
      x.z += vz * dt;
    }
    // cylinder confinement of the particle centre (radius R - r_i, half height H - r_i)
    const Real* c = A.cyl + 5 * s;
    const Real R0 = c[3] - A.scale[s] * x.w, H0 = c[4] - A.scale[s] * x.w;
    const Real dx = x.x - c[0], dy = x.y - c[1], dz = x.z - c[2];
    Real rr = dx * dx + dy * dy;
    if (rr > R0 * R0) {
      const Real q = R0 * T::rsqrt_rn(rr) - Real(1);
      x.x += dx * q;
      x.y += dy * q;
      v.x = -v.x;
      v.y = -v.y;
    }
    if (dz > H0) {
      x.z += H0 - dz;
      v.z = -v.z;
    }
    if (dz < -H0) {
      x.z += -H0 - dz;
      v.z = -v.z;
    }
    A.pos[p] = x;
    A.vel[p] = v;
    A.frc[p] = mk4(Real(0), Real(0), Real(0), Real(0));
  }
}

}  // namespace dem
