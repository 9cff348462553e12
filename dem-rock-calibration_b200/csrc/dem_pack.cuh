// Sample preparation kernels: soft repulsion, FIRE relaxation and the
// cylinder confinement of the reference's h_CreateCylinderSample
// (md_createcylindersample.cu:184-439):
//
//   k_soft_pairs      pair force of d_CalculateForces (md_calculateforces.cu:20-67):
//                     F_i += -D (a^2/r^2) (x_j - x_i) for r < a, a = s (r_i + r_j),
//                     or a linear overlap spring (packing by radius growth)
//   k_fire_power      cylinder walls as linear springs of the pair stiffness (the
//                     confinement of d_CylinderRestrictionZ, md_cylinderrestriction.cu:190-234,
//                     as a force so FIRE sees it), then P = F.v, |v|^2, |F|^2 per
//                     sample, reduced per block (d_FdotVEntire, md_firerelaxation.cu:375-494);
//                     the last block adapts dt and alpha on the device (the host
//                     logic of md_createcylindersample.cu:368-397)
//   k_fire_move       one FIRE move; a centre that crossed a wall is put back.
//                     Variant 0 is inertial FIRE 2.0 (Guenole et al., Comput. Mater.
//                     Sci. 175 (2020) 109584: half step back and v = 0 on P <= 0,
//                     semi-implicit Euler, velocity mixing); variant 1 is the
//                     reference's update (d_CalculateDecrementsHalfStepFIRE +
//                     d_CalculateIncrementsFIRE, md_firerelaxation.cu:18-70), which
//                     rebuilds v from the current force alone each step.
#pragma once

#include "dem_common.cuh"

namespace dem {

struct FireCtl {
  double P;            // F.v of the current step (accumulated)
  double dt, alpha;    // current FIRE time step and mixing
  double dt0, dtmax, dtmin, dtgrow, dtshrink, alpha0, alphashrink;
  uint32_t Npos, Nneg, Ndelay, back;  // back: this step moves half a step back and zeroes v
  unsigned long long step;
  double vv, ff;       // |v|^2 and |F|^2 of the current step (accumulated)
  float max_overlap;   // largest relative overlap seen by the pair kernel this step
  float vmax2;         // largest |v|^2 after a move (since the host reset it)
  float dmax2;         // largest squared displacement since the last list build (last move)
  uint32_t variant;    // 0: inertial FIRE 2.0, 1: the reference's force-only update
};

template <class Real>
struct PackArgs {
  using V4 = typename RT<Real>::V4;
  V4* pos;        // x, y, z, target radius
  V4* vel;        // v, dt0/m (reference Po.dt_d_m)
  V4* frc;
  const V4* ref;  // positions at the last list build
  const uint32_t* sid;
  uint32_t np;
  const uint2* c_ij;
  const uint32_t* nc;
  const Real* scale;   // per sample: radius scale during growth
  const Real* D;       // per sample: soft-force constant (reference Po.D) or spring stiffness
  int linear;          // 0: reference soft force, 1: linear overlap spring
  FireCtl* fire;       // per sample
  float* povl;         // per particle: largest relative overlap of the step (null: not tracked)
  const Real* cyl;     // per sample: centre x,y,z, radius R, half height H (5 values)
  uint32_t nsamples;
  unsigned int* blocks_done;
  int viscous;         // 1: viscous step of the pre-relaxation instead of FIRE
  Real vis;            // viscous coefficient (reference Po.vism)
  // Determinism: pair forces in exact fixed point (4 per particle, see acc3q),
  // and the FIRE power / norms as per-block partial sums (3 per block) that the
  // last block adds in block order; a seeded packing then repeats exactly.
  long long* frcq;
  double* part;
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
    acc3q(A.frcq + 4 * (size_t)i, fm * dx, fm * dy, fm * dz);
    acc3q(A.frcq + 4 * (size_t)j, -fm * dx, -fm * dy, -fm * dz);
    const float ov = (float)((a - RT<Real>::sqrt_rn(rr)) / a);
    worst = fmaxf(worst, ov);
    if (A.povl && ov > 0.f) {
      atomicMax(reinterpret_cast<int*>(A.povl + i), __float_as_int(ov));
      atomicMax(reinterpret_cast<int*>(A.povl + j), __float_as_int(ov));
    }
  }
  // block max of the relative overlap, then one atomic per block
  for (int o = 16; o > 0; o >>= 1) worst = fmaxf(worst, __shfl_xor_sync(0xFFFFFFFFu, worst, o));
  if ((threadIdx.x & 31) == 0 && worst > 0.f && A.nsamples == 1)
    atomicMax(reinterpret_cast<int*>(&A.fire[0].max_overlap), __float_as_int(worst));
}

// Block sum of three doubles (256 threads); result valid in thread 0.
__device__ __forceinline__ void block_sum3(double& a, double& b, double& c) {
  __shared__ double sh[3][8];
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
    b += __shfl_xor_sync(0xFFFFFFFFu, b, o);
    c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sh[0][w] = a;
    sh[1][w] = b;
    sh[2][w] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    a = b = c = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      a += sh[0][k];
      b += sh[1][k];
      c += sh[2][k];
    }
  }
}

// One sample (the packer relaxes one specimen per call).
template <class Real>
__global__ void __launch_bounds__(256) k_fire_power(PackArgs<Real> A) {
  using V4 = typename RT<Real>::V4;
  __shared__ int s_last;
  double pw = 0.0, vv = 0.0, ff = 0.0;
  float worst = 0.f;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < A.np; p += gridDim.x * blockDim.x) {
    const uint32_t s = A.sid[p];
    const V4 x = A.pos[p], v = A.vel[p];
    long long* q = A.frcq + 4 * (size_t)p;
    V4 f = mk4((Real)((double)q[0] * kFixInv), (Real)((double)q[1] * kFixInv), (Real)((double)q[2] * kFixInv),
               Real(0));
    q[0] = q[1] = q[2] = 0;
    // walls: radius R - r_i, caps at +-(H - r_i), force D * penetration
    const Real* c = A.cyl + 5 * s;
    const Real r = A.scale[s] * x.w, D = A.D[s];
    const Real R0 = c[3] - r, H0 = c[4] - r;
    const Real dx = x.x - c[0], dy = x.y - c[1], dz = x.z - c[2];
    const Real rr = dx * dx + dy * dy;
    Real pen = Real(0);
    if (rr > R0 * R0) {
      const Real rho = RT<Real>::sqrt_rn(rr);
      pen = rho - R0;
      const Real q = -D * pen / rho;
      f.x += q * dx;
      f.y += q * dy;
    }
    if (dz > H0) {
      f.z -= D * (dz - H0);
      pen = fmax(pen, dz - H0);
    }
    if (dz < -H0) {
      f.z += D * (-H0 - dz);
      pen = fmax(pen, -H0 - dz);
    }
    A.frc[p] = f;
    if (pen > Real(0)) worst = fmaxf(worst, (float)(pen / (Real(2) * r)));
    pw += (double)((f.x * v.x + f.y * v.y) + f.z * v.z);
    vv += (double)((v.x * v.x + v.y * v.y) + v.z * v.z);
    ff += (double)((f.x * f.x + f.y * f.y) + f.z * f.z);
  }
  for (int o = 16; o > 0; o >>= 1) worst = fmaxf(worst, __shfl_xor_sync(0xFFFFFFFFu, worst, o));
  if ((threadIdx.x & 31) == 0 && worst > 0.f)
    atomicMax(reinterpret_cast<int*>(&A.fire[0].max_overlap), __float_as_int(worst));
  block_sum3(pw, vv, ff);
  FireCtl& F = A.fire[0];
  if (A.viscous) return;
  if (threadIdx.x == 0) {
    A.part[3 * blockIdx.x + 0] = pw;
    A.part[3 * blockIdx.x + 1] = vv;
    A.part[3 * blockIdx.x + 2] = ff;
    __threadfence();
    s_last = (atomicAdd(A.blocks_done, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  for (uint32_t b = 0; b < gridDim.x; ++b) {
    F.P += __ldcg(A.part + 3 * b);
    F.vv += __ldcg(A.part + 3 * b + 1);
    F.ff += __ldcg(A.part + 3 * b + 2);
  }
  // md_createcylindersample.cu:374-397 (the same adaptation drives FIRE 2.0)
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
  F.vv = 0.0;
  F.ff = 0.0;
  ++F.step;
  *A.blocks_done = 0;
}

template <class Real>
__global__ void __launch_bounds__(256) k_fire_move(PackArgs<Real> A) {
  using T = RT<Real>;
  using V4 = typename T::V4;
  float my_v2 = 0.f, my_d2 = 0.f;
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
    } else if (A.fire[s].variant == 1) {
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
    } else {
      // FIRE 2.0: on P <= 0 half a step back and v = 0; then v += dt F/m,
      // v = (1 - alpha) v + alpha |v| F/|F| (per particle), x += dt v
      const FireCtl& F = A.fire[s];
      const Real dt = (Real)F.dt, alpha = (Real)F.alpha;
      if (F.back) {
        const Real h = Real(0.5) * dt;
        x.x -= v.x * h;
        x.y -= v.y * h;
        x.z -= v.z * h;
        v.x = v.y = v.z = Real(0);
      }
      const Real k = dtm * (Real)(F.dt / F.dt0);  // dt / m
      v.x += f.x * k;
      v.y += f.y * k;
      v.z += f.z * k;
      const Real ff = (f.x * f.x + f.y * f.y) + f.z * f.z;
      if (ff > Real(0)) {
        const Real vn = T::sqrt_rn((v.x * v.x + v.y * v.y) + v.z * v.z);
        const Real c = alpha * vn * T::rsqrt_rn(ff);
        v.x = (Real(1) - alpha) * v.x + c * f.x;
        v.y = (Real(1) - alpha) * v.y + c * f.y;
        v.z = (Real(1) - alpha) * v.z + c * f.z;
      }
      x.x += v.x * dt;
      x.y += v.y * dt;
      x.z += v.z * dt;
    }
    // a centre that crossed a wall surface is put back on it with its normal
    // velocity removed (the wall springs keep everything else inside)
    const Real* c = A.cyl + 5 * s;
    const Real R1 = c[3], H1 = c[4];
    const Real dx = x.x - c[0], dy = x.y - c[1], dz = x.z - c[2];
    const Real rr = dx * dx + dy * dy;
    if (rr > R1 * R1) {
      const Real rinv = T::rsqrt_rn(rr);
      const Real q = R1 * rinv - Real(1);
      x.x += dx * q;
      x.y += dy * q;
      const Real vn = (v.x * dx + v.y * dy) * rinv;
      if (vn > Real(0)) {
        v.x -= vn * dx * rinv;
        v.y -= vn * dy * rinv;
      }
    }
    if (dz > H1) {
      x.z += H1 - dz;
      if (v.z > Real(0)) v.z = Real(0);
    }
    if (dz < -H1) {
      x.z += -H1 - dz;
      if (v.z < Real(0)) v.z = Real(0);
    }
    A.pos[p] = x;
    A.vel[p] = v;
    A.frc[p] = mk4(Real(0), Real(0), Real(0), Real(0));
    const V4 r0 = A.ref[p];
    const Real ex = x.x - r0.x, ey = x.y - r0.y, ez = x.z - r0.z;
    my_v2 = fmaxf(my_v2, (float)((v.x * v.x + v.y * v.y) + v.z * v.z));
    my_d2 = fmaxf(my_d2, (float)((ex * ex + ey * ey) + ez * ez));
  }
  for (int o = 16; o > 0; o >>= 1) {
    my_v2 = fmaxf(my_v2, __shfl_xor_sync(0xFFFFFFFFu, my_v2, o));
    my_d2 = fmaxf(my_d2, __shfl_xor_sync(0xFFFFFFFFu, my_d2, o));
  }
  if ((threadIdx.x & 31) == 0) {
    // non-negative floats order as their bit patterns
    if (my_v2 > 0.f) atomicMax(reinterpret_cast<int*>(&A.fire[0].vmax2), __float_as_int(my_v2));
    if (my_d2 > 0.f) atomicMax(reinterpret_cast<int*>(&A.fire[0].dmax2), __float_as_int(my_d2));
  }
}

}  // namespace dem
