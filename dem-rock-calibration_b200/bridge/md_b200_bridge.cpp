// md_b200_bridge.cpp - the reference's loading drivers over libb200dem.
//
// Added to the reference's sources in place of md_calculationuniaxialcompression.cu
// and md_calculationbraziltest.cu, it defines the two driver entry points the
// reference declares in mp.h (h_CalculationUniaxialCompression,
// h_CalculationBrazilTest; mp.h:21-22) over dem_calculation_test, with the
// reference's inputs (md_task_data, SoA host positions h_R in mm) and outputs
// (the Compress and result fields its callers read, mp_calculateonesample.cu:165-168,
// and the Uniaxial_<n>.txt / Brazil_<n>.txt loading records, md_results.cu:168-180).
// Build: compile with the reference's headers on the include path and link
// with -lb200dem.
// the reference headers use memset and DBL_MAX without including their headers
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <vector>

#include "md_data_types.h"
#include "mp.h"
#include "b200dem.h"

static void fill(const md_task_data& td, bool brazil, dem_material& m, dem_loading& L) {
  m = dem_material{};
  m.E = td.Po.m_E;  m.nu = td.Po.m_nu;  m.Ec = td.Po.m_Ec;  m.Gc = td.Po.m_Gc;
  m.b_r = td.Po.b_r;  m.gap = td.Po.b_d - 2.0 * td.Po.p_r;  m.rho = td.Po.m_ro;
  m.p_r = td.Po.p_r;  m.p_e = td.Po.p_e;  m.mu = td.Po.p_mu;  m.mur = td.Po.p_mur;
  m.farcut = td.Po.a_farcut / td.Po.p_r;
  L = dem_loading{};
  L.test = brazil ? DEM_TEST_BRAZIL : DEM_TEST_UNIAXIAL;
  const float3 c = td.S.center, h = td.S.spacesized2, hp = td.S.hidenpoint;
  L.space_center[0] = c.x;  L.space_center[1] = c.y;  L.space_center[2] = c.z;
  L.space_half[0] = h.x;    L.space_half[1] = h.y;    L.space_half[2] = h.z;
  L.hidden_point[0] = hp.x; L.hidden_point[1] = hp.y; L.hidden_point[2] = hp.z;
  L.zcut = td.S.center.z + td.S.spacesized2.z;
  L.size_real[0] = td.S.size_real.x;  L.size_real[1] = td.S.size_real.y;  L.size_real[2] = td.S.size_real.z;
  L.center_real[0] = td.S.center_real.x;  L.center_real[1] = td.S.center_real.y;
  L.center_real[2] = td.S.center_real.z;
  L.velocity = td.Compress.VLoad;  L.min_stress = td.Compress.MinStress;
  L.max_strain = td.Compress.MaxStrain;  L.cond_fracture = td.Compress.ConditionFracture;
  L.dNsave = td.R.dNsave;
}

static void run(md_task_data& td, float* h_R, bool brazil) {
  dem_material m; dem_loading L; dem_result r;
  fill(td, brazil, m, L);
  const uint32_t cap = 1u << 22;
  std::vector<double> rec(3 * (size_t)cap);
  std::vector<uint32_t> bonds(cap);
  uint32_t nrec = 0;
  int rc = dem_calculation_test(nullptr, &m, &L, h_R, nullptr, td.P.N, &r, rec.data(), bonds.data(), cap, &nrec);
  if (rc) std::fprintf(stderr, "libb200dem: %s\n", dem_strerror(rc));   // the reference prints and continues
  td.Compress.FractureStress = r.FractureStress;
  td.Compress.FractureStrain = r.FractureStrain;
  td.Compress.LinearityDeviation = r.LinearityDeviation;
  td.Compress.Strain = r.Strain;
  td.R.Destruction = r.Destruction;
  char name[256];
  std::snprintf(name, sizeof name, brazil ? "./result/Brazil_%i.txt" : "./result/Uniaxial_%i.txt", td.R.fileN);
  dem_save_sum_forces_loading(name, rec.data(), nrec < cap ? nrec : cap);
}

void h_CalculationUniaxialCompression(md_task_data& td, float* h_R) { run(td, h_R, false); }
void h_CalculationBrazilTest(md_task_data& td, float* h_R) { run(td, h_R, true); }
