// Device-resident data layout of the B200 DEM engine (host+device visible).
//
// Particles of all specimens ("samples") are stored back to back, each
// sample's particles sorted along a Morton curve of its cell grid.  Every
// per-particle field is one 128-bit vector (256-bit in FP64 builds) so a
// warp reads it with fully coalesced vector loads:
//
//   pos  x, y, z, radius          vel  vx, vy, vz, dt/m
//   omg  wx, wy, wz, dt/I         frc/mom  force and moment accumulators
//   wallO  platen tangential history (the reference's Oiwt)
//
// Bonds are stored once per undirected pair (i < j) in (i, j) order, as four
// vector streams:
//
//   s0 = (prev-direction xyz, Ot.x)   s1 = (Ot.y, Ot.z, Mn.x, Mn.y)
//   s2 = (Mn.z, Mt.x, Mt.y, Mt.z)     par = (1/L0, sigma_c, tau_c, b_r)
//
// with 1/L0 < 0 marking a broken bond (the pair then interacts by Hertz-Mindlin
// contact, history in Ot).  Unbonded pairs within contact range + skin form
// the contact list (ij, tangential history), rebuilt from the cell grid when
// a particle has moved more than half the skin.
#pragma once
#include <stdint.h>

namespace dem {

// Per-sample constants read by the kernels (one entry per specimen).
template <class Real>
struct SampleParams {
  Real dt;          // time step
  Real E, G;        // bond Young and shear modulus
  Real hmE, hmG;    // particle-particle Hertz-Mindlin equivalent moduli (reference hm_E, hm_G)
  Real wallE, wallG;  // particle-platen moduli (2*hm_E, 2*hm_G uniaxial; hm_E, hm_G Brazilian)
  Real pA, mu, mur; // damping coefficient ln e/sqrt(pi^2+ln^2 e), sliding and rolling friction
  Real aa_far;      // squared far cut-off: bonds beyond it are deleted (reference aa_farcut)
  Real skin_half2;  // (skin/2)^2: neighbour-list validity radius
  Real space_c[3], space_h[3], hide[3];  // escape box centre, half size, hidden point
  float wall_c[3];  // platen frame centre (reference Compress.center)
  float wall_RR;    // squared lateral radius of the platen contact zone
  float zcut;       // hidden-particle cut (reference S.center.z + S.spacesized2.z)
  int axis;         // 2: uniaxial (z platens), 1: Brazilian (y platens), -1: none
  int nobreak;      // 1: bonds never break (elastic stage)
  uint32_t p_begin, p_end;  // particle range
};

// Per-sample loading controller (the reference's compression_data and
// result_data, md_data_types.h:190-495), in double like the reference host.
struct SampleCtl {
  double Top, Bottom, V, VLoad;
  double size_d[3];
  double Size0, sz0, inv_Area, p_r;
  double MinStress, ZeroStress, MaxStrain, ConditionFracture;
  double Stress, Strain, FractureStress, FractureStrain;
  double sFL[2];            // platen force sums of the current step
  double dt;
  unsigned long long step, max_steps;
  int32_t bonds;            // intact undirected bonds
  uint32_t StepsStop, Loading, Fracture, done, brazil;
  uint32_t stepsave, Nsave, dNsave;
  uint32_t rebuild;         // neighbour list must be rebuilt before the next force pass
  uint32_t stale;           // a particle moved more than the skin allows: list was stale
  double* rec;              // 3*Nsave: strain, sigma_bottom, sigma_top (reference h_sFL)
  uint32_t* rec_bonds;      // Nsave: bonded directed slots (reference h_sSI)
  // lateral surface of a uniaxial specimen (Poisson ratio): sum of the radial
  // distances of the marked particles on record steps, and its record
  double lat_sum;
  double* rec_lat;          // Nsave: mean radial distance of the marked particles
  uint32_t lat_count;       // marked particles (0: no lateral record)
  uint32_t numeric;         // a particle's position, velocity or spin became NaN or infinite
  // deterministic mode: the platen and lateral sums of the step in 2^-40 fixed
  // point, folded into sFL / lat_sum by the controller
  long long sFLq[2];
  long long lat_q;
  long long q_pad;
  // The step kernels skip a sample while `hold` is set: finished (done), its
  // contact list no longer valid (stale: a particle moved past half the skin,
  // so the next step would miss contacts until the host rebuilds the list),
  // or at the step the current host call asked for (stop_at).  The controller
  // sets it at the end of each step; the host refreshes it when it clears
  // stale or sets stop_at.
  unsigned long long stop_at;
  uint32_t hold;
  uint32_t hold_pad;
};

}  // namespace dem
