// Per-step kernels of the B200 DEM engine:
//
//   k_pairs     one thread per bond or contact pair: BPM bond force/moment with
//               break test, Hertz-Mindlin contact for broken bonds and unbonded
//               pairs; contributions scattered to both particles with 128-bit
//               vector reductions.  Replaces the reference's d_CalculateForcesDEM_22
//               + d_CalculateForcesDEM_21 (md_calculateforcesdem3.cu:341-486), which
//               compute every pair twice, once per direction.
//   k_particles one thread per particle: platen contacts (d_UniaxialCompression_hm /
//               d_BrazilCompression_hm, md_compression_hm.cu:156-449), integration
//               (d_CalculateIncrementsDEM, md_calculateincrementsdem.cu:128-158), escape
//               parking (d_ParallelepipedCutRestriction, md_parallelepipedrestriction.cu:254),
//               accumulator reset, neighbour-list validity, platen force sums; the
//               last block to finish runs the loading controller of every sample
//               (SumForces{U,B}Loading + Compress{U,B}_S3, md_results.cu:56-145,
//               md_data_types.h:347-494) on the device, so a step needs no host sync.
#pragma once

#include "dem_common.cuh"
#include "dem_types.h"

namespace dem {

template <class Real>
struct StepArgs {
  using V4 = typename RT<Real>::V4;
  V4* pos;
  V4* vel;
  V4* omg;
  V4* frc;
  V4* mom;
  V4* wallO;
  uint8_t* wflag;  // per particle: 1 = wallO may be non-zero (it touched the lower platen last step)
  V4* pos_ref;
  const Real* mass;
  const uint32_t* sid;
  uint32_t np;
  // bonds
  const uint2* b_ij;
  V4* b_s0;
  V4* b_s1;
  V4* b_s2;
  V4* b_par;
  uint32_t nb;
  // contacts
  uint2* c_ij;
  V4* c_o;
  const uint32_t* nc;  // device count
  // samples
  const SampleParams<Real>* sp;
  SampleCtl* ctl;
  uint32_t nsamples;
  unsigned int* blocks_done;
  int keep_forces;  // 1: leave the step's total force/moment in frc/mom (parity checks)
  unsigned long long* touching;  // non-null: count touching contacts (algorithmic-byte accounting)
  float* stat;      // running maxima of |v|^2 and displacement^2 over blocks and steps (reset by the host)
  const uint8_t* lat;  // per particle: 1 = on the lateral surface near mid-height (or null)
  double* sfl_tan;     // sensitivity build only: per sample the platen-force tangents (see dem_dual.cuh)
  // deterministic mode (FP32 only): fixed-point force and moment accumulators,
  // 4 per particle (x, y, z, unused), used instead of frc / mom
  long long* frcq;
  long long* momq;
  int det;
  // batched runs: when set, the pair kernel visits only the listed bond tiles
  // (tiles holding a bond of an unfinished sample); ntiles on the device
  const uint32_t* tiles;
  const uint32_t* ntiles;
  // per bond tile (blockDim.x bonds): the sample all its bonds belong to, or
  // ~0u when the tile spans two samples; lets a bond find its sample's state
  // without first loading the sample id of its particle
  const uint32_t* tile_s;
};

// Scatter of one contribution to a particle's force or moment accumulator:
// a 128-bit float reduction, or in deterministic mode three fixed-point adds.
template <class Real>
__device__ __forceinline__ void acc_f(const StepArgs<Real>& A, uint32_t p, const Real& x, const Real& y,
                                      const Real& z) {
  if (A.det) {
    if constexpr (sizeof(Real) == 4)
      acc3q(A.frcq + 4 * (size_t)p, x, y, z);
    else
      acc3_fix(A.frc + p, x, y, z);
    return;
  }
  acc3(A.frc + p, x, y, z);
}
template <class Real>
__device__ __forceinline__ void acc_m(const StepArgs<Real>& A, uint32_t p, const Real& x, const Real& y,
                                      const Real& z) {
  if (A.det) {
    if constexpr (sizeof(Real) == 4)
      acc3q(A.momq + 4 * (size_t)p, x, y, z);
    else
      acc3_fix(A.mom + p, x, y, z);
    return;
  }
  acc3(A.mom + p, x, y, z);
}

// Hooks of the sensitivity build (dem_dual.cuh overloads them for dual
// numbers); for float and double they do nothing.
template <class Real>
__device__ __forceinline__ void tangent_wall(const StepArgs<Real>&, uint32_t, int, const Real&) {}
template <class Real>
__device__ __forceinline__ void tangent_step_end(const StepArgs<Real>&, const SampleCtl&, uint32_t) {}

// A value whose derivative the sensitivity build drops (the identity for float
// and double).  Used for the unit directions of the Coulomb cap and of rolling
// friction (derivative ~ 1/|v| or 1/|w| near rest): rolling friction turns a
// spin that is nearly zero into a moment of fixed size whose direction
// flips from step to step, and the linearised step of that term is
// unstable, so its tangents would grow without bound.  The contact damping
// keeps its full derivative (the overlap factor sqrt(R* overlap) inside
// sqrt(K m) included): on a 20,000-sphere uniaxial run the secant-modulus
// derivatives were 7e-4 to 1.7e-3 (relative) from central differences with
// that factor's derivative dropped, and 8e-5 to 6e-4 with it kept.
template <class Real>
__device__ __forceinline__ Real frozen(const Real& x) {
  return x;
}

// Hertz-Mindlin contact of pair (i, j) seen from i (n points from i to j), in
// the polydisperse form that reduces bit for bit to dd_Calculate_fijn_ppHM_2 /
// dd_Calculate_fijtmijt_ppHM_2 / dd_Calculate_mijroll_ppHM_2
// (md_calculateforcesdem3.cu:202-339) when r_i = r_j is a power of two and the
// masses are equal.  Updates the tangential history o and returns the force on
// i and the moments on i and j (the reference drops the whole contact moment of
// a particle whose spin satisfies |w|^2 <= 1e-18, see md_calculateforcesdem3.cu:333-338).
template <class Real>
__device__ __forceinline__ void hm_pair(const SampleParams<Real>& sp, Real rx, Real ry, Real rz, Real rijm, Real ri,
                                        Real rj, Real mi, Real mj, const typename RT<Real>::V4& vi,
                                        const typename RT<Real>::V4& vj, const typename RT<Real>::V4& wi,
                                        const typename RT<Real>::V4& wj, Real& ox, Real& oy, Real& oz, Real f[3],
                                        Real mI[3], Real mJ[3], bool& dropI, bool& dropJ) {
  using T = RT<Real>;
  const Real half = Real(0.5);
  const Real sumr = ri + rj;
  const Real rinv = T::rcp(rijm);
  const Real n0 = rx * rinv, n1 = ry * rinv, n2 = rz * rinv;
  const Real reff = ri * rj / sumr;
  Real cef1 = T::sqrt_rn(reff * (sumr - rijm));
  const Real Kn = Real(2) * sp.hmE * cef1;
  const Real Kt = Real(8) * sp.hmG * cef1;
  const Real rbar = half * sumr, rdif = half * (rj - ri);
  const Real sw0 = wj.x + wi.x, sw1 = wj.y + wi.y, sw2 = wj.z + wi.z;
  const Real dw0 = wj.x - wi.x, dw1 = wj.y - wi.y, dw2 = wj.z - wi.z;
  const Real v0 = vj.x - vi.x + rbar * (n1 * sw2 - n2 * sw1) + rdif * (n1 * dw2 - n2 * dw1);
  const Real v1 = vj.y - vi.y + rbar * (n2 * sw0 - n0 * sw2) + rdif * (n2 * dw0 - n0 * dw2);
  const Real v2 = vj.z - vi.z + rbar * (n0 * sw1 - n1 * sw0) + rdif * (n0 * dw1 - n1 * dw0);
  const Real vn = n0 * v0 + n1 * v1 + n2 * v2;
  const Real fijnm = (rijm - sumr) * Kn * T::kTwoThirds;
  // 2 m* = m_a (2 m_b / (m_a + m_b)) with m_a the smaller mass: the same bits
  // from either side of the pair, and m_i when the masses are equal
  const Real ma = mi < mj ? mi : mj, mb = mi < mj ? mj : mi;
  const Real m2 = ma * ((mb + mb) / (ma + mb));
  cef1 = T::kDamp * sp.pA * vn * T::sqrt_rn(Kn * half * m2);
  const Real fn0 = n0 * (fijnm + cef1), fn1 = n1 * (fijnm + cef1), fn2 = n2 * (fijnm + cef1);
  const Real vt0 = v0 - n0 * vn, vt1 = v1 - n1 * vn, vt2 = v2 - n2 * vn;
  // rotate the old tangential overlap into the new tangent plane, keep its length
  cef1 = n0 * ox + n1 * oy + n2 * oz;
  Real t0 = ox - n0 * cef1, t1 = oy - n1 * cef1, t2 = oz - n2 * cef1;
  cef1 = (t0 * t0 + t1 * t1) + t2 * t2;
  if (cef1 > Real(1e-18)) {
    cef1 = T::rcp(cef1);
    cef1 *= (ox * ox + oy * oy) + oz * oz;
    cef1 = T::sqrt_rn(cef1);
    t0 *= cef1;
    t1 *= cef1;
    t2 *= cef1;
  }
  const Real dt = sp.dt;
  t0 += vt0 * dt;
  t1 += vt1 * dt;
  t2 += vt2 * dt;
  Real ft0 = t0 * Kt, ft1 = t1 * Kt, ft2 = t2 * Kt;
  const Real ftmm = (ft0 * ft0 + ft1 * ft1) + ft2 * ft2;
  if (ftmm > sp.mu * sp.mu * fijnm * fijnm) {
    cef1 = sp.mu * T::fabs_(fijnm) * frozen(T::rsqrt_rn(ftmm));
    ft0 = frozen(ft0) * cef1;
    ft1 = frozen(ft1) * cef1;
    ft2 = frozen(ft2) * cef1;
    cef1 = T::rcp(Kt);
    t0 = ft0 * cef1;
    t1 = ft1 * cef1;
    t2 = ft2 * cef1;
  } else {
    cef1 = T::kDamp * sp.pA * T::sqrt_rn(Kt * half * m2);
    ft0 += vt0 * cef1;
    ft1 += vt1 * cef1;
    ft2 += vt2 * cef1;
  }
  ox = t0;
  oy = t1;
  oz = t2;
  f[0] = fn0 + ft0;
  f[1] = fn1 + ft1;
  f[2] = fn2 + ft2;
  const Real c0 = n1 * ft2 - n2 * ft1, c1 = n2 * ft0 - n0 * ft2, c2 = n0 * ft1 - n1 * ft0;
  mI[0] = c0 * ri;
  mI[1] = c1 * ri;
  mI[2] = c2 * ri;
  mJ[0] = c0 * rj;
  mJ[1] = c1 * rj;
  mJ[2] = c2 * rj;
  const Real afn = T::fabs_(fijnm);
  const Real wim = (wi.x * wi.x + wi.y * wi.y) + wi.z * wi.z;
  const Real wjm = (wj.x * wj.x + wj.y * wj.y) + wj.z * wj.z;
  dropI = !(wim > Real(1e-18));
  dropJ = !(wjm > Real(1e-18));
  if (!dropI) {
    const Real c = -sp.mur * afn * frozen(T::rsqrt_rn(wim));
    mI[0] += frozen(wi.x) * c;
    mI[1] += frozen(wi.y) * c;
    mI[2] += frozen(wi.z) * c;
  }
  if (!dropJ) {
    const Real c = -sp.mur * afn * frozen(T::rsqrt_rn(wjm));
    mJ[0] += frozen(wj.x) * c;
    mJ[1] += frozen(wj.y) * c;
    mJ[2] += frozen(wj.z) * c;
  }
}

template <class Real>
__device__ __forceinline__ void scatter_pair(const StepArgs<Real>& A, uint32_t i, uint32_t j, const Real f[3],
                                             const Real mI[3], const Real mJ[3], bool dropI, bool dropJ) {
  acc_f(A, i, f[0], f[1], f[2]);
  acc_f(A, j, -f[0], -f[1], -f[2]);
  if (!dropI) acc_m(A, i, mI[0], mI[1], mI[2]);
  if (!dropJ) acc_m(A, j, mJ[0], mJ[1], mJ[2]);
}

// Sum of v over the run of lanes of this warp that share a key (keys sorted
// along the lanes, all 32 lanes active; run_end = the first lane after this
// lane's run): a segmented suffix sum by shuffles; the run's first lane ends
// with the run's total.
template <class T, int N>
__device__ __forceinline__ void warp_run_sum(uint32_t run_end, T (&v)[N]) {
  const uint32_t lane = threadIdx.x & 31;
#pragma unroll
  for (uint32_t d = 1; d < 32; d <<= 1) {
    const bool same = lane + d < run_end;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const T o = __shfl_down_sync(0xFFFFFFFFu, v[k], d);
      if (same) v[k] += o;
    }
  }
}

// The i-side force and moment of an intact bond.  Bonds are stored sorted by
// i, so the lanes of a warp that share i are adjacent: when the whole warp is
// here their contributions are first summed over each run of equal i and the
// run's first lane issues the atomics, which cuts the atomics reaching L2 by
// about a third (float) or a half (fixed point, three per vector).  In
// deterministic mode every lane's contribution is first rounded to fixed point
// and the run is summed as integers, so the sum is the same exact value the
// per-lane fixed-point atomics give.  Otherwise (a partial warp, the
// sensitivity build) every lane adds its own.
template <class Real>
__device__ __forceinline__ void scatter_i_warp(const StepArgs<Real>& A, uint32_t i, Real f0, Real f1, Real f2,
                                               Real m0, Real m1, Real m2) {
  if constexpr (sizeof(Real) == 4 || sizeof(Real) == 8) {
    if (__activemask() == 0xFFFFFFFFu) {
      const uint32_t lane = threadIdx.x & 31;
      // every lane takes part in the shuffle (no short-circuit around it)
      const uint32_t iu = __shfl_up_sync(0xFFFFFFFFu, i, 1);
      const bool head = lane == 0 || iu != i;
      // end of this lane's run: the next run head above it (one ballot
      // instead of a key shuffle per round of the segmented sum)
      const unsigned heads = __ballot_sync(0xFFFFFFFFu, head);
      const unsigned above = lane < 31 ? heads & (~0u << (lane + 1)) : 0u;
      const uint32_t run_end = above ? (uint32_t)(__ffs(above) - 1) : 32u;
      if (A.det) {
        long long q[6];
        if constexpr (sizeof(Real) == 4) {
          q[0] = to_fix(f0); q[1] = to_fix(f1); q[2] = to_fix(f2);
          q[3] = to_fix(m0); q[4] = to_fix(m1); q[5] = to_fix(m2);
        } else {
          q[0] = fix_of(f0); q[1] = fix_of(f1); q[2] = fix_of(f2);
          q[3] = fix_of(m0); q[4] = fix_of(m1); q[5] = fix_of(m2);
        }
        warp_run_sum(run_end, q);
        if (head) {
          unsigned long long* uf;
          unsigned long long* um;
          if constexpr (sizeof(Real) == 4) {
            uf = reinterpret_cast<unsigned long long*>(A.frcq + 4 * (size_t)i);
            um = reinterpret_cast<unsigned long long*>(A.momq + 4 * (size_t)i);
          } else {
            uf = reinterpret_cast<unsigned long long*>(A.frc + i);
            um = reinterpret_cast<unsigned long long*>(A.mom + i);
          }
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            atomicAdd(uf + k, (unsigned long long)q[k]);
            atomicAdd(um + k, (unsigned long long)q[3 + k]);
          }
        }
      } else {
        Real v[6] = {f0, f1, f2, m0, m1, m2};
        warp_run_sum(run_end, v);
        if (head) {
          acc3(A.frc + i, v[0], v[1], v[2]);
          acc3(A.mom + i, v[3], v[4], v[5]);
        }
      }
      return;
    }
  }
  acc_f(A, i, f0, f1, f2);
  acc_m(A, i, m0, m1, m2);
}

// The j-side force and moment of an intact bond.  Deterministic FP32 mode and
// FP64 with the whole warp here: a contribution costs six 64-bit atomics, so
// the lanes whose bonds share j (neighbours of nearby i; they need not be
// adjacent) are found with a warp match and their values summed by a shuffle
// tree over their ranks (in deterministic mode as fixed-point integers: the
// same exact total); the lowest of them issues the atomics.  FP32 float
// atomics cost too little for the match to pay (measured), so every other case
// adds per lane.  The code is compiled only into the pair kernels of
// deterministic FP32 and of FP64 contexts (kDetJ): its registers slowed the
// FP32 float kernel by 12%.
// Sum of v over the lanes of this warp named in peers (this lane among them,
// at rank r of n; maxn the largest n in the warp): a shuffle tree over the
// ranks, rank r adding rank r + s for r = 0 mod 2s, so that rank 0 ends with
// the sum.  Every lane runs every shuffle (maxn is the same in all lanes).
template <class T, int N>
__device__ __forceinline__ void warp_peer_sum(unsigned peers, uint32_t n, uint32_t r, uint32_t maxn, T (&v)[N]) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t s = 1; s < maxn; s <<= 1) {
    uint32_t src = lane;
    if (r % (2 * s) == 0 && r + s < n) {
      unsigned above = lane < 31 ? peers & ~((2u << lane) - 1u) : 0u;
      for (uint32_t t = 1; t < s; ++t) above &= above - 1u;
      if (above) src = __ffs(above) - 1;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const T o = __shfl_sync(0xFFFFFFFFu, v[k], src);
      if (src != lane) v[k] += o;
    }
  }
}

template <class Real, bool kDetJ>
__device__ __forceinline__ void scatter_j_warp(const StepArgs<Real>& A, uint32_t j, Real f0, Real f1, Real f2,
                                               Real m0, Real m1, Real m2) {
  if constexpr ((sizeof(Real) == 4 || sizeof(Real) == 8) && kDetJ) {
    if ((sizeof(Real) == 8 || A.det) && __activemask() == 0xFFFFFFFFu) {
      const uint32_t lane = threadIdx.x & 31;
      const unsigned peers = __match_any_sync(0xFFFFFFFFu, j);
      const uint32_t n = __popc(peers), r = __popc(peers & ((1u << lane) - 1u));
      const uint32_t maxn = __reduce_max_sync(0xFFFFFFFFu, n);
      if (A.det) {
        long long q[6];
        if constexpr (sizeof(Real) == 4) {
          q[0] = to_fix(f0); q[1] = to_fix(f1); q[2] = to_fix(f2);
          q[3] = to_fix(m0); q[4] = to_fix(m1); q[5] = to_fix(m2);
        } else {
          q[0] = fix_of(f0); q[1] = fix_of(f1); q[2] = fix_of(f2);
          q[3] = fix_of(m0); q[4] = fix_of(m1); q[5] = fix_of(m2);
        }
        warp_peer_sum(peers, n, r, maxn, q);
        if (r == 0) {
          unsigned long long* uf;
          unsigned long long* um;
          if constexpr (sizeof(Real) == 4) {
            uf = reinterpret_cast<unsigned long long*>(A.frcq + 4 * (size_t)j);
            um = reinterpret_cast<unsigned long long*>(A.momq + 4 * (size_t)j);
          } else {
            uf = reinterpret_cast<unsigned long long*>(A.frc + j);
            um = reinterpret_cast<unsigned long long*>(A.mom + j);
          }
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            atomicAdd(uf + k, (unsigned long long)q[k]);
            atomicAdd(um + k, (unsigned long long)q[3 + k]);
          }
        }
      } else {
        Real v[6] = {f0, f1, f2, m0, m1, m2};
        warp_peer_sum(peers, n, r, maxn, v);
        if (r == 0) {
          acc3(A.frc + j, v[0], v[1], v[2]);
          acc3(A.mom + j, v[3], v[4], v[5]);
        }
      }
      return;
    }
  }
  acc_f(A, j, f0, f1, f2);
  acc_m(A, j, m0, m1, m2);
}

// One bond (i < j).  The arithmetic is that of d_CalculateForcesDEM_22 for the
// slot i->j (md_calculateforcesdem3.cu:41-200, 427-486); the slot j->i of the
// reference is its exact mirror (all vectors negated, the unsymmetric moment
// equal), so j receives -F, -(Mn + Mt) terms and the same unsymmetric moment.
template <class Real, bool kDetJ>
__device__ __forceinline__ void do_bond_core(const StepArgs<Real>& A, uint32_t b, const uint2 ij,
                                             typename RT<Real>::V4 par, typename RT<Real>::V4 s0,
                                             typename RT<Real>::V4 s1, typename RT<Real>::V4 s2, uint32_t ts,
                                             const typename RT<Real>::V4& pi, const typename RT<Real>::V4& pj,
                                             const typename RT<Real>::V4& vi, const typename RT<Real>::V4& vj,
                                             const typename RT<Real>::V4& wi, const typename RT<Real>::V4& wj);

template <class Real, bool kDetJ>
__device__ __forceinline__ void do_bond(const StepArgs<Real>& A, uint32_t b, const uint2 ij,
                                        typename RT<Real>::V4 par, typename RT<Real>::V4 s0,
                                        typename RT<Real>::V4 s1, typename RT<Real>::V4 s2, uint32_t ts) {
  using V4 = typename RT<Real>::V4;
  // the gathers depend only on (i, j): all issued before the first branch
  const uint32_t i = ij.x, j = ij.y;
  const V4 pi = ld4(A.pos + i), pj = ld4(A.pos + j);
  const V4 wi = ld4(A.omg + i), wj = ld4(A.omg + j);
  const V4 vi = ld4(A.vel + i), vj = ld4(A.vel + j);
  do_bond_core<Real, kDetJ>(A, b, ij, par, s0, s1, s2, ts, pi, pj, vi, vj, wi, wj);
}

// The bond itself, given the particle states of its two ends.
template <class Real, bool kDetJ>
__device__ __forceinline__ void do_bond_core(const StepArgs<Real>& A, uint32_t b, const uint2 ij,
                                             typename RT<Real>::V4 par, typename RT<Real>::V4 s0,
                                             typename RT<Real>::V4 s1, typename RT<Real>::V4 s2, uint32_t ts,
                                             const typename RT<Real>::V4& pi, const typename RT<Real>::V4& pj,
                                             const typename RT<Real>::V4& vi, const typename RT<Real>::V4& vj,
                                             const typename RT<Real>::V4& wi, const typename RT<Real>::V4& wj) {
  using T = RT<Real>;
  const uint32_t i = ij.x, j = ij.y;
  const uint32_t s = ts != ~0u ? ts : A.sid[i];
  if (A.ctl[s].hold) return;
  const SampleParams<Real>& sp = A.sp[s];
  const Real rx = pj.x - pi.x, ry = pj.y - pi.y, rz = pj.z - pi.z;
  const Real rr = (rx * rx + ry * ry) + rz * rz;
  bool intact = par.x > Real(0);
  if (intact && (rr > sp.aa_far || rr < Real(1e-10))) {
    // d_DeleteFarLinks (md_interaction_list_reconstructbpm.cu:169-181): the slot is
    // emptied with all histories; the pair later interacts only by contact.
    par.x = -par.x;
    st4_cs(A.b_par + b, par);
    const Real z = Real(0);
    st4_cs(A.b_s0 + b, mk4(z, z, z, z));
    st4_cs(A.b_s1 + b, mk4(z, z, z, z));
    st4_cs(A.b_s2 + b, mk4(z, z, z, z));
    atomicSub(&A.ctl[s].bonds, 1);
    return;
  }
  const Real rijm = norm3(rx, ry, rz);
  Real ox = s0.w, oy = s1.x, oz = s1.y;
  if (intact) {
    // The reference's operation order (dd_*_bpm_2, md_calculateforcesdem3.cu:41-200)
    // with chosen products fused into their sums (T::fma, one rounding); the CPU
    // oracle fuses the same ones, so both stay identical bit for bit.
    const Real one = Real(1), half = Real(0.5), dt = sp.dt, E = sp.E, G = sp.G, pi_ = T::kPi;
    const Real il = par.x, br = par.w;
    const Real rinv = T::rcp(rijm);
    const Real n0 = rx * rinv, n1 = ry * rinv, n2 = rz * rinv;
    // normal force (dd_Calculate_fijn_bpm_2)
    Real cef = E * (rijm - T::rcp(il)) * il;
    Real Sc = cef;
    cef *= br * br * pi_;
    const Real fn0 = n0 * cef, fn1 = n1 * cef, fn2 = n2 * cef;
    // incremental rotation (dd_Calculate_M123_bpm_2)
    const Real tp0 = T::fma(s0.y, n2, -(s0.z * n1)), tp1 = T::fma(s0.z, n0, -(s0.x * n2)),
               tp2 = T::fma(s0.x, n1, -(s0.y * n0));
    cef = T::fma(wj.z + wi.z, n2, T::fma(wj.y + wi.y, n1, (wj.x + wi.x) * n0)) * dt * half;
    const Real ph0 = n0 * cef, ph1 = n1 * cef, ph2 = n2 * cef;
    s0.x = n0;
    s0.y = n1;
    s0.z = n2;
    const Real M10 = T::fma(tp1, ph1, T::fma(tp2, ph2, one));
    const Real M11 = T::fma(-tp1, ph0, ph2 - tp2);
    const Real M12 = T::fma(-tp2, ph0, -ph1) + tp1;
    const Real M20 = T::fma(-tp0, ph1, tp2 - ph2);
    const Real M21 = T::fma(tp0, ph0, T::fma(tp2, ph2, one));
    const Real M22 = T::fma(-tp2, ph1, ph0) - tp0;
    const Real M30 = T::fma(-tp0, ph2, -tp1) + ph1;
    const Real M31 = T::fma(-tp1, ph2, tp0) - ph0;
    const Real M32 = T::fma(tp0, ph0, tp1 * ph1) + one;
    // twisting moment (dd_Calculate_mijn_bpm_2)
    const Real dwx = wj.x - wi.x, dwy = wj.y - wi.y, dwz = wj.z - wi.z;
    const Real wn = T::fma(n2, dwz, T::fma(n1, dwy, n0 * dwx));
    Real cef1 = wn * (dt * half * G * il);
    const Real Nx = s1.z, Ny = s1.w, Nz = s2.x;
    const Real mn0 = T::fma(n0, cef1, T::fma(M12, Nz, T::fma(M11, Ny, M10 * Nx)));
    const Real mn1 = T::fma(n1, cef1, T::fma(M22, Nz, T::fma(M21, Ny, M20 * Nx)));
    const Real mn2 = T::fma(n2, cef1, T::fma(M32, Nz, T::fma(M31, Ny, M30 * Nx)));
    cef1 = pi_ * br * br * br * br;
    const Real tn0 = mn0 * cef1, tn1 = mn1 * cef1, tn2 = mn2 * cef1;
    // bending moment (dd_Calculate_mijt_bpm_2)
    Real cef2 = dt * Real(0.25) * E * il;
    const Real Tx = s2.y, Ty = s2.z, Tz = s2.w;
    const Real mt0 = T::fma(T::fma(-n0, wn, dwx), cef2, T::fma(M12, Tz, T::fma(M11, Ty, M10 * Tx)));
    const Real mt1 = T::fma(T::fma(-n1, wn, dwy), cef2, T::fma(M22, Tz, T::fma(M21, Ty, M20 * Tx)));
    const Real mt2 = T::fma(T::fma(-n2, wn, dwz), cef2, T::fma(M32, Tz, T::fma(M31, Ty, M30 * Tx)));
    cef2 *= pi_ * br * br * br * br;
    const Real tt0 = mt0 * cef2, tt1 = mt1 * cef2, tt2 = mt2 * cef2;
    // shear force and unsymmetric moment (dd_Calculate_fijt_mijunsym_bpm_2)
    const Real ws0 = half * (wj.x + wi.x), ws1 = half * (wj.y + wi.y), ws2 = half * (wj.z + wi.z);
    const Real v0 = T::fma(ws2, ry, T::fma(-ws1, rz, vj.x - vi.x));
    const Real v1 = T::fma(ws0, rz, T::fma(-ws2, rx, vj.y - vi.y));
    const Real v2 = T::fma(ws1, rx, T::fma(-ws0, ry, vj.z - vi.z));
    cef = T::fma(n2, v2, T::fma(n1, v1, n0 * v0));
    const Real ot0 = T::fma(T::fma(-n0, cef, v0), dt, T::fma(M12, oz, T::fma(M11, oy, M10 * ox)));
    const Real ot1 = T::fma(T::fma(-n1, cef, v1), dt, T::fma(M22, oz, T::fma(M21, oy, M20 * ox)));
    const Real ot2 = T::fma(T::fma(-n2, cef, v2), dt, T::fma(M32, oz, T::fma(M31, oy, M30 * ox)));
    cef = G * il;
    Real Mc = cef;
    cef *= br * br * pi_;
    const Real ft0 = ot0 * cef, ft1 = ot1 * cef, ft2 = ot2 * cef;
    const Real mu0 = half * T::fma(ry, ot2, -(rz * ot1)) * cef;
    const Real mu1 = half * T::fma(rz, ot0, -(rx * ot2)) * cef;
    const Real mu2 = half * T::fma(rx, ot1, -(ry * ot0)) * cef;
    // contributions: i gets (F, Mn+Mt+Mu), j gets (-F, -(Mn+Mt)+Mu)
    scatter_j_warp<Real, kDetJ>(A, j, -(fn0 + ft0), -(fn1 + ft1), -(fn2 + ft2), mu0 - (tn0 + tt0), mu1 - (tn1 + tt1),
                         mu2 - (tn2 + tt2));
    scatter_i_warp<Real>(A, i, fn0 + ft0, fn1 + ft1, fn2 + ft2, (tn0 + tt0) + mu0, (tn1 + tt1) + mu1,
                         (tn2 + tt2) + mu2);
    // break test (dd_CheckBreakConditionDEM_2)
    bool broke = false;
    if (!sp.nobreak) {
      Mc *= norm3_hist(ot0, ot1, ot2);
      Sc += norm3_hist(mt0, mt1, mt2) * Real(4) * br;
      Mc += norm3_hist(mn0, mn1, mn2) * Real(2) * br;
      broke = (Sc > par.y) || (Mc > par.z);
    }
    if (!broke) {
      s0.w = ot0;
      s1 = mk4(ot1, ot2, mn0, mn1);
      s2 = mk4(mn2, mt0, mt1, mt2);
      st4_cs(A.b_s0 + b, s0);
      st4_cs(A.b_s1 + b, s1);
      st4_cs(A.b_s2 + b, s2);
      return;
    }
    // broken: histories cleared; the pair is a contact from now on and, as in the
    // reference (DEM_21 runs after DEM_22 in the same step), already this step.
    par.x = -par.x;
    st4_cs(A.b_par + b, par);
    atomicSub(&A.ctl[s].bonds, 1);
    ox = oy = oz = Real(0);
    const Real z = Real(0);
    s1.z = z;
    s1.w = z;
    s2 = mk4(z, z, z, z);
  }
  // Hertz-Mindlin contact of a broken bond
  const Real ri = pi.w, rj = pj.w;
  if (rr > Real(1e-10) && rijm < ri + rj) {
    Real f[3], mI[3], mJ[3];
    bool dI, dJ;
    hm_pair<Real>(sp, rx, ry, rz, rijm, ri, rj, A.mass[i], A.mass[j], vi, vj, wi, wj, ox, oy, oz, f, mI, mJ, dI, dJ);
    scatter_pair<Real>(A, i, j, f, mI, mJ, dI, dJ);
    if (A.touching) atomicAdd(A.touching, 1ull);
  } else {
    ox = oy = oz = Real(0);
  }
  s0.w = ox;
  s1.x = oy;
  s1.y = oz;
  st4_cs(A.b_s0 + b, s0);
  st4_cs(A.b_s1 + b, s1);
  if (intact) st4_cs(A.b_s2 + b, s2);
}

// One unbonded contact-list pair (i < j).  Bit 31 of j flags a non-zero
// tangential history, so separated pairs cost only the position gathers.
template <class Real>
__device__ __forceinline__ void do_contact(const StepArgs<Real>& A, uint32_t c) {
  using T = RT<Real>;
  using V4 = typename T::V4;
  uint2 ij = A.c_ij[c];
  const uint32_t i = ij.x, j = ij.y & 0x7FFFFFFFu;
  const bool has_hist = (ij.y >> 31) != 0;
  const uint32_t s = A.sid[i];
  if (A.ctl[s].hold) return;
  const V4 pi = ld4(A.pos + i), pj = ld4(A.pos + j);
  const Real rx = pj.x - pi.x, ry = pj.y - pi.y, rz = pj.z - pi.z;
  const Real rr = (rx * rx + ry * ry) + rz * rz;
  const Real ri = pi.w, rj = pj.w;
  const Real rijm = norm3(rx, ry, rz);
  if (!(rr > Real(1e-10) && rijm < ri + rj)) {
    if (has_hist) {
      const Real z = Real(0);
      A.c_o[c] = mk4(z, z, z, z);
      A.c_ij[c] = make_uint2(i, j);
    }
    return;
  }
  const SampleParams<Real>& sp = A.sp[s];
  V4 o = has_hist ? ld4_rw(A.c_o + c) : mk4(Real(0), Real(0), Real(0), Real(0));
  const V4 wi = ld4(A.omg + i), wj = ld4(A.omg + j);
  const V4 vi = ld4(A.vel + i), vj = ld4(A.vel + j);
  Real f[3], mI[3], mJ[3];
  bool dI, dJ;
  Real ox = o.x, oy = o.y, oz = o.z;
  hm_pair<Real>(sp, rx, ry, rz, rijm, ri, rj, A.mass[i], A.mass[j], vi, vj, wi, wj, ox, oy, oz, f, mI, mJ, dI, dJ);
  scatter_pair<Real>(A, i, j, f, mI, mJ, dI, dJ);
  if (A.touching) atomicAdd(A.touching, 1ull);
  A.c_o[c] = mk4(ox, oy, oz, Real(0));
  if (!has_hist) A.c_ij[c] = make_uint2(i, j | 0x80000000u);
}

// Pair kernel: one thread per bond, then one per contact-list pair, grid
// stride.  A block's bonds of one pass are a contiguous tile of blockDim
// bonds; while the block works on it, one thread asks the copy engine to
// prefetch the block's next tile of bond state into L2 (four bulk prefetches),
// so the next pass finds its streamed loads in L2, and every thread already
// holds the next tile's pair indices.  Bond arrays are padded to whole
// 256-bond tiles.
template <class Real, int kMinBlocks = (sizeof(Real) == 4 ? 4 : 2), int kBlock = 256, bool kDetJ = false>
__global__ void __launch_bounds__(kBlock, kMinBlocks) k_pairs(StepArgs<Real> A) {
  using V4 = typename RT<Real>::V4;
  const uint32_t nb = A.nb;
  const uint32_t tile = blockDim.x, stride = gridDim.x * tile;
  const uint32_t ntl = A.tiles ? *A.ntiles : (nb + tile - 1) / tile;
  // software pipeline over the block's tiles: the pair indices and the sample
  // of the next tile are loaded before this tile's gathers, so a pass starts
  // its particle gathers at once instead of after an index round trip
  uint32_t k = blockIdx.x;
  uint32_t base = 0, ts = ~0u;
  uint2 ij = make_uint2(0, 0);
  if (k < ntl) {
    base = (A.tiles ? A.tiles[k] : k) * tile;
    if (A.tile_s) ts = __ldg(A.tile_s + base / tile);
    if (base + threadIdx.x < nb) ij = __ldcs(A.b_ij + base + threadIdx.x);
  }
  for (; k < ntl; k += gridDim.x) {
    const uint32_t kn = k + gridDim.x;
    uint32_t nbase = 0, nts = ~0u;
    uint2 nij = make_uint2(0, 0);
    if (kn < ntl) {
      nbase = (A.tiles ? A.tiles[kn] : kn) * tile;
      if (threadIdx.x == 0) {
        l2_prefetch(A.b_par + nbase, tile * sizeof(V4));
        l2_prefetch(A.b_s0 + nbase, tile * sizeof(V4));
        l2_prefetch(A.b_s1 + nbase, tile * sizeof(V4));
        l2_prefetch(A.b_s2 + nbase, tile * sizeof(V4));
      }
      if (A.tile_s) nts = __ldg(A.tile_s + nbase / tile);
      if (nbase + threadIdx.x < nb) nij = __ldcs(A.b_ij + nbase + threadIdx.x);
    }
    const uint32_t b = base + threadIdx.x;
    if (b < nb)
      do_bond<Real, kDetJ>(A, b, ij, ld4_cs(A.b_par + b), ld4_cs(A.b_s0 + b), ld4_cs(A.b_s1 + b), ld4_cs(A.b_s2 + b), ts);
    base = nbase;
    ts = nts;
    ij = nij;
  }
  const uint32_t nc = *A.nc;
  for (uint32_t c = blockIdx.x * tile + threadIdx.x; c < nc; c += stride) do_contact<Real>(A, c);
}

// Particle-platen contact (dd_Calculate_fijn_pwHM_2 + dd_Calculate_fijtmijt_pwHM_2,
// md_compression_hm.cu:20-154) with radius ri and mass mi.  Returns the normal
// force component along the platen axis.
template <class Real>
__device__ __forceinline__ Real wall_contact(const SampleParams<Real>& sp, int axis, Real sgn, Real wallvel,
                                             Real riwm, Real ri, Real mi, const typename RT<Real>::V4& v,
                                             const typename RT<Real>::V4& w, Real o[3], Real F[3], Real M[3]) {
  using T = RT<Real>;
  // the platen normal and velocity lie along the loading axis, y (Brazilian)
  // or z (uniaxial); selects instead of an indexed store keep them in registers
  const bool a1 = axis == 1, a2 = axis == 2;
  const Real zero = Real(0);
  const Real niw[3] = {zero, a1 ? sgn : zero, a2 ? sgn : zero};
  const Real wv[3] = {zero, a1 ? wallvel : zero, a2 ? wallvel : zero};
  Real cef1 = T::sqrt_rn(ri * T::fabs_(ri - riwm));
  const Real Kn = Real(2) * sp.wallE * cef1;
  const Real Kt = Real(8) * sp.wallG * cef1;
  Real viw[3];
  viw[0] = wv[0] - v.x + ri * (niw[1] * w.z - niw[2] * w.y);
  viw[1] = wv[1] - v.y + ri * (niw[2] * w.x - niw[0] * w.z);
  viw[2] = wv[2] - v.z + ri * (niw[0] * w.y - niw[1] * w.x);
  const Real vn = niw[0] * viw[0] + niw[1] * viw[1] + niw[2] * viw[2];
  const Real fiwnm = (riwm - ri) * Kn * T::kTwoThirds;
  cef1 = T::kDamp * sp.pA * vn * T::sqrt_rn(Kn * mi);
  const Real fiwn[3] = {niw[0] * (fiwnm + cef1), niw[1] * (fiwnm + cef1), niw[2] * (fiwnm + cef1)};
  const Real vt[3] = {viw[0] - niw[0] * vn, viw[1] - niw[1] * vn, viw[2] - niw[2] * vn};
  cef1 = niw[0] * o[0] + niw[1] * o[1] + niw[2] * o[2];
  Real ot[3] = {o[0] - niw[0] * cef1, o[1] - niw[1] * cef1, o[2] - niw[2] * cef1};
  cef1 = (ot[0] * ot[0] + ot[1] * ot[1]) + ot[2] * ot[2];
  if (cef1 > Real(1e-18)) {
    cef1 = T::rcp(cef1);
    // md_compression_hm.cu:91 multiplies the x and y components in the first term
    cef1 *= (o[0] * o[1] + o[1] * o[1]) + o[2] * o[2];
    cef1 = T::sqrt_rn(cef1);
    ot[0] *= cef1;
    ot[1] *= cef1;
    ot[2] *= cef1;
  }
  const Real dt = sp.dt;
  ot[0] += vt[0] * dt;
  ot[1] += vt[1] * dt;
  ot[2] += vt[2] * dt;
  Real ft[3] = {ot[0] * Kt, ot[1] * Kt, ot[2] * Kt};
  const Real ftmm = (ft[0] * ft[0] + ft[1] * ft[1]) + ft[2] * ft[2];
  if (ftmm > sp.mu * sp.mu * fiwnm * fiwnm) {
    cef1 = sp.mu * T::fabs_(fiwnm) * frozen(T::rsqrt_rn(ftmm));
    ft[0] = frozen(ft[0]) * cef1;
    ft[1] = frozen(ft[1]) * cef1;
    ft[2] = frozen(ft[2]) * cef1;
    cef1 = T::rcp(Kt);
    ot[0] = ft[0] * cef1;
    ot[1] = ft[1] * cef1;
    ot[2] = ft[2] * cef1;
  } else {
    cef1 = T::kDamp * sp.pA * T::sqrt_rn(Kt * mi);
    ft[0] += vt[0] * cef1;
    ft[1] += vt[1] * cef1;
    ft[2] += vt[2] * cef1;
  }
  o[0] = ot[0];
  o[1] = ot[1];
  o[2] = ot[2];
  const Real mt[3] = {(niw[1] * ft[2] - niw[2] * ft[1]) * ri, (niw[2] * ft[0] - niw[0] * ft[2]) * ri,
                      (niw[0] * ft[1] - niw[1] * ft[0]) * ri};
  const Real wim = (w.x * w.x + w.y * w.y) + w.z * w.z;
  Real madd[3] = {0, 0, 0};
  if (wim > Real(1e-18)) {
    cef1 = -sp.mur * T::fabs_(fiwnm) * frozen(T::rsqrt_rn(wim));
    madd[0] = frozen(w.x) * cef1;
    madd[1] = frozen(w.y) * cef1;
    madd[2] = frozen(w.z) * cef1;
  }
  F[0] += fiwn[0] + ft[0];
  F[1] += fiwn[1] + ft[1];
  F[2] += fiwn[2] + ft[2];
  M[0] += mt[0] + madd[0];
  M[1] += mt[1] + madd[1];
  M[2] += mt[2] + madd[2];
  return a2 ? fiwn[2] : fiwn[1];
}

// Loading controller of one sample after its platen force sums are complete:
// SumInteractions + SumForces{U,B}Loading + Compress{U,B}_S3.
__device__ inline void controller_step(SampleCtl& C) {
  const int ax = C.brazil ? 1 : 2;
  const unsigned long long n = C.step;
  const double sF0 = C.sFL[0], sF1 = C.sFL[1];
  const bool save = C.dNsave && (n % C.dNsave == 0);
  // SumInteractions (md_results.cu:198-203): bonded directed slots
  if (save && C.stepsave < C.Nsave) C.rec_bonds[C.stepsave] = 2u * (uint32_t)max(C.bonds, 0);
  // SumForces{U,B}Loading (md_results.cu:56-145)
  if (save && C.stepsave < C.Nsave) {
    C.rec[3 * C.stepsave] = (C.size_d[ax] - C.sz0) / C.sz0;
    C.rec[3 * C.stepsave + 1] = sF0 * C.inv_Area;
    C.rec[3 * C.stepsave + 2] = sF1 * C.inv_Area;
    if (C.rec_lat) C.rec_lat[C.stepsave] = C.lat_count ? C.lat_sum / C.lat_count : 0.0;
    if (fabs(C.V) > 1e-9) ++C.stepsave;
  }
  C.Stress = 0.5 * (fabs(sF0) + fabs(sF1)) * C.inv_Area;
  if (!C.Loading && C.Stress > C.MinStress) C.Loading = 1;
  if (!C.brazil) {
    if (C.FractureStress < C.Stress) {
      C.FractureStress = C.Stress;
      C.FractureStrain = (C.sz0 - C.size_d[ax]) / C.sz0;
    }
    if (C.Loading && (C.Stress < C.ZeroStress || C.Stress < C.ConditionFracture * C.FractureStress)) C.Fracture = 1;
  } else {
    if (C.FractureStress < C.Stress || C.Stress < C.ConditionFracture * C.FractureStress) {
      C.FractureStress = C.Stress;
      C.FractureStrain = (C.sz0 - C.size_d[ax]) / C.sz0;
    }
    if (C.Loading && C.Stress < C.ZeroStress) C.Fracture = 1;
  }
  // Compress{U,B}_S3 (md_data_types.h:347-379, 462-494)
  const double pS = C.brazil ? 0.5 * (-sF0 + sF1) : 0.5 * fabs(-sF0 + sF1);
  const double pD = fabs(sF0 + sF1);
  if (pS * C.inv_Area < 1e-9) {
    C.V = 10.0 * C.VLoad;
  } else if (pD > 0.20 * pS && pS * C.inv_Area > 2.0e+6 / 1e9) {
    if (fabs(C.V) > 1e-15) C.StepsStop = 0;
    C.V = 0;
    ++C.StepsStop;
    if (C.StepsStop > 30000) C.Fracture = 1;
  } else {
    C.V = C.VLoad;
  }
  C.size_d[ax] += C.V * C.dt;
  C.Top += 0.5 * C.V * C.dt;
  C.Bottom -= 0.5 * C.V * C.dt;
  C.Strain = (C.size_d[ax] - C.Size0) / C.Size0;
  C.sFL[0] = 0.0;
  C.sFL[1] = 0.0;
  C.lat_sum = 0.0;
  ++C.step;
  // loop condition of h_Calculation{UniaxialCompression,BrazilTest}; a sample
  // whose state went non-finite also stops
  if (!(fabs(C.Strain) < C.MaxStrain) || C.Fracture || C.step >= C.max_steps || C.numeric) C.done = 1;
  C.hold = (C.done || C.stale || C.step >= C.stop_at) ? 1u : 0u;
}

// After the host has cleared the rebuild flags or moved the stop: the hold
// flag of every sample again (stop_steps: new stop_at = step + stop_steps,
// saturating; 0 keeps stop_at).
__global__ void k_set_hold(SampleCtl* ctl, uint32_t S, unsigned long long stop_steps, int clear_rebuild) {
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
    SampleCtl& C = ctl[s];
    if (clear_rebuild) {
      C.rebuild = 0;
      C.stale = 0;
    }
    if (stop_steps) C.stop_at = C.step + stop_steps < C.step ? ~0ull : C.step + stop_steps;
    C.hold = (C.done || C.stale || C.step >= C.stop_at) ? 1u : 0u;
  }
}

// The controllers of all samples, run by the last block of the particle
// kernel once every block's platen sums are in.  Not inlined: its private
// copy of a sample's state (one load, one store back instead of a chain of
// dependent global accesses) lives in this function's frame, not in the
// particle loop's registers.
template <class Real>
__device__ __noinline__ void run_controllers(const StepArgs<Real> A) {
  for (uint32_t s = threadIdx.x; s < A.nsamples; s += blockDim.x) {
    if (A.ctl[s].hold) continue;
    SampleCtl C = A.ctl[s];
    // fixed-point platen and lateral sums of the deterministic mode (zero otherwise)
    C.sFL[0] += (double)C.sFLq[0] * kFixInv;
    C.sFL[1] += (double)C.sFLq[1] * kFixInv;
    C.lat_sum += (double)C.lat_q * kFixInv;
    C.sFLq[0] = C.sFLq[1] = C.lat_q = 0;
    tangent_step_end(A, C, s);
    controller_step(C);
    A.ctl[s] = C;
  }
  if (threadIdx.x == 0) *A.blocks_done = 0;
}

template <class Real>
__global__ void __launch_bounds__(256, sizeof(Real) == 4 ? 4 : 1) k_particles(StepArgs<Real> A) {
  using T = RT<Real>;
  using V4 = typename T::V4;
  __shared__ int s_last;
  // The constants and this step's controller state of every sample (up to
  // kCacheSamples; FP32 and FP64), copied into shared memory once per block:
  // a particle's sample id then costs one shared lookup instead of two
  // dependent global loads (controller flags, then the sample's constants).
  // The controller updates the global state only after every block is done.
  constexpr uint32_t kCacheSamples = 16;
  constexpr bool kCacheable = sizeof(Real) <= 8;
  __shared__ SampleParams<Real> c_sp[kCacheable ? kCacheSamples : 1];
  __shared__ float c_wall[kCacheable ? kCacheSamples : 1][3];   // platen top, bottom, velocity (as float)
  __shared__ uint32_t c_flag[kCacheable ? kCacheSamples : 1];   // bit 0: held (done, stale, at its stop); bit 1: a lateral-record step
  const bool cached = kCacheable && A.nsamples <= kCacheSamples;
  if (cached) {
    for (uint32_t s = threadIdx.x; s < A.nsamples; s += blockDim.x) {
      c_sp[s] = A.sp[s];
      const SampleCtl& C = A.ctl[s];
      c_wall[s][0] = (float)C.Top;
      c_wall[s][1] = (float)C.Bottom;
      c_wall[s][2] = (float)C.V;
      c_flag[s] = (C.hold ? 1u : 0u) | ((C.dNsave && C.step % C.dNsave == 0) ? 2u : 0u);
    }
    __syncthreads();
  }
  // platen force partial sums of this block are kept per sample in registers and
  // flushed with one double atomic per (sample, warp) run
  float my_v2 = 0.f, my_d2 = 0.f;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < A.np; p += gridDim.x * blockDim.x) {
    // the particle's own state is loaded before its sample's flags arrive (the
    // loads do not depend on them; a finished sample's values go unused)
    // (FP32 only: the wider types would hold too many registers across the wait)
    V4 x, v, w, f, m, xref;
    if constexpr (sizeof(Real) == 4) {
      x = A.pos[p];
      v = A.vel[p];
      w = A.omg[p];
      xref = ld4_rw(A.pos_ref + p);
      if (!A.det) {
        f = A.frc[p];
        m = A.mom[p];
      }
    }
    const uint32_t s = A.sid[p];
    SampleCtl& C = A.ctl[s];
    double sb = 0.0, st = 0.0, sl = 0.0;
    const uint32_t flag = cached ? c_flag[s] : ((C.hold ? 1u : 0u) | ((C.dNsave && C.step % C.dNsave == 0) ? 2u : 0u));
    if (!(flag & 1u)) {
      const SampleParams<Real>& sp = cached ? c_sp[s] : A.sp[s];
      if constexpr (sizeof(Real) == 4) {
        if (A.det) {
          const longlong2 q0 = *reinterpret_cast<const longlong2*>(A.frcq + 4 * (size_t)p);
          const long long q2 = A.frcq[4 * (size_t)p + 2];
          const longlong2 u0 = *reinterpret_cast<const longlong2*>(A.momq + 4 * (size_t)p);
          const long long u2 = A.momq[4 * (size_t)p + 2];
          f = mk4((Real)((double)q0.x * kFixInv), (Real)((double)q0.y * kFixInv), (Real)((double)q2 * kFixInv),
                  Real(0));
          m = mk4((Real)((double)u0.x * kFixInv), (Real)((double)u0.y * kFixInv), (Real)((double)u2 * kFixInv),
                  Real(0));
        }
      } else {
        x = A.pos[p];
        v = A.vel[p];
        w = A.omg[p];
        xref = ld4_rw(A.pos_ref + p);
        if (A.det) {
          f = unfix4(A.frc[p]);    // FP64 / sensitivity build: fixed point in place
          m = unfix4(A.mom[p]);
        } else {
          f = A.frc[p];
          m = A.mom[p];
        }
      }
      Real F[3] = {f.x, f.y, f.z}, M[3] = {m.x, m.y, m.z};
      if (sp.axis >= 0) {
        // d_UniaxialCompression_hm / d_BrazilCompression_hm (md_compression_hm.cu:167-239)
        const int ax = sp.axis;
        Real r[3];
        r[0] = x.x - Real(sp.wall_c[0]);
        if (ax == 2) {
          r[1] = x.y - Real(sp.wall_c[1]);
          r[2] = x.z;
        } else {
          r[1] = x.y;
          r[2] = x.z - Real(sp.wall_c[2]);
        }
        const Real lat = (ax == 2) ? (r[0] * r[0] + r[1] * r[1]) : (r[0] * r[0] + r[2] * r[2]);
        // The history ends zero unless the sphere touches the lower platen (the
        // branch of the platen it does not touch clears it), so a sphere of the
        // platen zone that touches neither platen and had no history keeps a zero
        // one: nothing to read or write.
        if (lat < Real(sp.wall_RR) && r[2] < Real(sp.zcut)) {
          const Real wtop = Real(cached ? c_wall[s][0] : (float)C.Top), wbot = Real(cached ? c_wall[s][1] : (float)C.Bottom);
          const Real rax = ax == 2 ? r[2] : r[1];   // coordinate along the loading axis
          const bool top = wtop - rax < x.w, bot = rax - wbot < x.w;
          const uint8_t had = A.wflag[p];
          if (top || bot || had) {
            const Real wvel = Real(cached ? c_wall[s][2] : (float)C.V);
            V4 o4 = had ? A.wallO[p] : mk4(Real(0), Real(0), Real(0), Real(0));
            Real o[3] = {o4.x, o4.y, o4.z};
            const Real ri = x.w, mi = A.mass[p];
            if (top) {
              const Real f = wall_contact<Real>(sp, ax, Real(1), wvel, T::fabs_(wtop - rax), ri, mi, v, w, o, F, M);
              st = -(double)f;
              tangent_wall(A, s, 1, f);
            } else {
              o[0] = o[1] = o[2] = Real(0);
            }
            if (bot) {
              const Real f =
                  wall_contact<Real>(sp, ax, Real(-1), -wvel, T::fabs_(wbot - rax), ri, mi, v, w, o, F, M);
              sb = -(double)f;
              tangent_wall(A, s, 0, f);
            } else {
              o[0] = o[1] = o[2] = Real(0);
            }
            A.wallO[p] = mk4(o[0], o[1], o[2], Real(0));
            if (had != (uint8_t)bot) A.wflag[p] = bot ? 1 : 0;
          }
        }
      }
      // d_CalculateIncrementsDEM: v += F dt/m, x += v dt, w += M dt/I
      const Real dtm = v.w, dtI = w.w, dt = sp.dt;
      v.x += F[0] * dtm;
      v.y += F[1] * dtm;
      v.z += F[2] * dtm;
      x.x += v.x * dt;
      x.y += v.y * dt;
      x.z += v.z * dt;
      w.x += M[0] * dtI;
      w.y += M[1] * dtI;
      w.z += M[2] * dtI;
      // d_ParallelepipedCutRestriction: park escaped particles at the hidden point
      const Real d0 = x.x - sp.space_c[0], d1 = x.y - sp.space_c[1], d2 = x.z - sp.space_c[2];
      bool parked = false;
      if (d0 - sp.space_h[0] > Real(0) || d0 + sp.space_h[0] < Real(0) || d1 - sp.space_h[1] > Real(0) ||
          d1 + sp.space_h[1] < Real(0) || d2 - sp.space_h[2] > Real(0) || d2 + sp.space_h[2] < Real(0)) {
        x.x = sp.hide[0];
        x.y = sp.hide[1];
        x.z = sp.hide[2];
        v.x = v.y = v.z = Real(0);
        parked = true;
      }
      // a non-finite position, velocity or spin (the sum of the nine values is
      // NaN or infinite exactly when one of them is, barring an overflow of the
      // sum itself) stops the sample: the controller marks it done and the host
      // reports DEM_ERR_NUMERIC
      if (!isfinite((double)x.x + (double)x.y + (double)x.z + (double)v.x + (double)v.y + (double)v.z + (double)w.x +
                    (double)w.y + (double)w.z))
        C.numeric = 1u;
      A.pos[p] = x;
      A.vel[p] = v;
      A.omg[p] = w;
      const Real z = Real(0);
      if (A.keep_forces) {
        A.frc[p] = mk4(F[0], F[1], F[2], z);
        A.mom[p] = mk4(M[0], M[1], M[2], z);
      } else if (!A.det || sizeof(Real) != 4) {
        A.frc[p] = mk4(z, z, z, z);   // (a zero double is also a zero fixed-point value)
        A.mom[p] = mk4(z, z, z, z);
      }
      if constexpr (sizeof(Real) == 4) {
        if (A.det) {
          *reinterpret_cast<longlong4*>(A.frcq + 4 * (size_t)p) = make_longlong4(0, 0, 0, 0);
          *reinterpret_cast<longlong4*>(A.momq + 4 * (size_t)p) = make_longlong4(0, 0, 0, 0);
        }
      }
      // neighbour-list validity: displacement since the last build.  A parked
      // particle interacts with nothing (all parked particles coincide, and
      // pairs closer than 1e-10 are ignored), so it restarts its reference.
      // lateral surface particles on record steps: radial distance from the axis
      if (A.lat && A.lat[p] && !parked && (flag & 2u)) {
        const double ex = (double)x.x - sp.wall_c[0], ey = (double)x.y - sp.wall_c[1];
        sl = sqrt(ex * ex + ey * ey);
      }
      if (parked) {
        A.pos_ref[p] = x;
      } else {
        const V4 x0 = xref;
        const Real e0 = x.x - x0.x, e1 = x.y - x0.y, e2 = x.z - x0.z;
        const Real d2s = (e0 * e0 + e1 * e1) + e2 * e2;
        if (d2s > Real(0.25) * sp.skin_half2) C.rebuild = 1;  // past a quarter of the skin: rebuild soon
        if (d2s > sp.skin_half2) C.stale = 1;                 // past half the skin: the list is no longer valid
        my_d2 = fmaxf(my_d2, (float)d2s);
        my_v2 = fmaxf(my_v2, (float)((v.x * v.x + v.y * v.y) + v.z * v.z));
      }
    }
    // per-sample double sums: a full warp of one sample reduces with shuffles and
    // issues one atomic; otherwise each contributing lane adds its own value.  In
    // deterministic mode every particle's terms are first rounded to fixed point
    // and summed as integers (exact, independent of the warp a particle falls in).
    // Most warps hold no platen or lateral-record sphere: a full warp with
    // nothing to add skips the reduction.
    {
      const unsigned am = __activemask();
      if (am == 0xFFFFFFFFu && !__any_sync(am, sb != 0.0 || st != 0.0 || sl != 0.0)) continue;
    }
    if (A.det) {
      long long qb = to_fix(sb), qt = to_fix(st), ql = to_fix(sl);
      const unsigned fm = __activemask();
      bool uni = false;
      if (fm == 0xFFFFFFFFu) {
        const uint32_t s0 = __shfl_sync(fm, s, 0);
        uni = __all_sync(fm, s == s0);
      }
      if (uni) {
        for (int off = 16; off > 0; off >>= 1) {
          qb += __shfl_xor_sync(fm, qb, off);
          qt += __shfl_xor_sync(fm, qt, off);
          ql += __shfl_xor_sync(fm, ql, off);
        }
      }
      if (!uni || (threadIdx.x & 31) == 0) {
        unsigned long long* q = reinterpret_cast<unsigned long long*>(A.ctl[s].sFLq);
        if (qb) atomicAdd(q + 0, (unsigned long long)qb);
        if (qt) atomicAdd(q + 1, (unsigned long long)qt);
        if (ql) atomicAdd(reinterpret_cast<unsigned long long*>(&A.ctl[s].lat_q), (unsigned long long)ql);
      }
      continue;
    }
    const unsigned full = __activemask();
    bool uniform = false;
    if (full == 0xFFFFFFFFu) {
      const uint32_t s0 = __shfl_sync(full, s, 0);
      uniform = __all_sync(full, s == s0);
    }
    if (uniform) {
      for (int off = 16; off > 0; off >>= 1) {
        sb += __shfl_xor_sync(full, sb, off);
        st += __shfl_xor_sync(full, st, off);
        sl += __shfl_xor_sync(full, sl, off);
      }
      if ((threadIdx.x & 31) == 0) {
        if (sb != 0.0 || st != 0.0) {
          atomicAdd(&A.ctl[s].sFL[0], sb);
          atomicAdd(&A.ctl[s].sFL[1], st);
        }
        if (sl != 0.0) atomicAdd(&A.ctl[s].lat_sum, sl);
      }
    } else {
      if (sb != 0.0 || st != 0.0) {
        atomicAdd(&A.ctl[s].sFL[0], sb);
        atomicAdd(&A.ctl[s].sFL[1], st);
      }
      if (sl != 0.0) atomicAdd(&A.ctl[s].lat_sum, sl);
    }
  }
  // block maxima of speed and displacement (the host sizes the next chunk of
  // steps from them so no particle outruns the contact-list skin)
  __shared__ float s_v2[32], s_d2[32];
  for (int o = 16; o > 0; o >>= 1) {
    my_v2 = fmaxf(my_v2, __shfl_xor_sync(0xFFFFFFFFu, my_v2, o));
    my_d2 = fmaxf(my_d2, __shfl_xor_sync(0xFFFFFFFFu, my_d2, o));
  }
  if ((threadIdx.x & 31) == 0) {
    s_v2[threadIdx.x >> 5] = my_v2;
    s_d2[threadIdx.x >> 5] = my_d2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float a = 0.f, b = 0.f;
    for (uint32_t w = 0; w < (blockDim.x + 31) / 32; ++w) {
      a = fmaxf(a, s_v2[w]);
      b = fmaxf(b, s_d2[w]);
    }
    // running maxima since the host last reset them (non-negative floats order
    // as their bit patterns)
    atomicMax(reinterpret_cast<int*>(A.stat), __float_as_int(a));
    atomicMax(reinterpret_cast<int*>(A.stat) + 1, __float_as_int(b));
  }
  // the last block to finish runs the controllers.  The barrier orders the
  // block's flag stores and sum atomics before thread 0's fence and count
  // (one fence per block, as a grid barrier does; a fence in every thread
  // would also wait for the particle-state stores, which no controller reads)
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = (atomicAdd(A.blocks_done, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  run_controllers<Real>(A);
}

}  // namespace dem
