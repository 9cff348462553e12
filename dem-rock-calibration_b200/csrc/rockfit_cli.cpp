// rockfit-dem: the reference's command line and stdout contract (kernel.cu:23-123,
// CalculateOneSample in mp_calculateonesample.cu:17-250) over libb200dem, so a
// caller such as NN_MP.py can spawn it unchanged:
//
//   rockfit-dem G<d> M(E,Ec,Gc,br,gap,poros) [CS][U][B] I<idx> [FUSC] [FBSC]
//
// E, Ec, Gc in Pa, br and gap in m, poros the sample porosity.  CS creates the
// samples (./result/Sample_0_<i>.txt uniaxial, Sample_1_<i>.txt Brazilian) before
// testing, U / B select the uniaxial / Brazilian test, FUSC / FBSC force the
// creation of one sample.  stdout carries "There are <n> GPUs", "Correct GPU
// request! Requested: <d>", "INDEX <idx>" and the result line
// ResultCalculateOneSample[E,Ec,Gc,br,gap,poros,epsU,sigmaU,LD,destrU,epsB,sigmaB,0,destrB]
// with stresses in Pa; diagnostics go to stderr.  DCG and TSS (the calibration
// drivers) are served by dem-rock-calibration_b200.calibrate / .sweep instead.
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "b200dem.h"

namespace {

constexpr double kLength = 1e-3, kMass = 1e-6, kTime = 1e-6;
const double kStress = (kMass * kLength / (kTime * kTime)) / (kLength * kLength);
const double kVelocity = kLength / kTime;
constexpr double kPi = 3.14159265358979323846;

struct Geometry {
  double lsi[3], space[3];
};
// mp_calculateonesample.cu:86-87: uniaxial 25 x 25 x 50 mm in a 40 x 40 x 60 mm
// space, Brazilian 50 x 50 x 20 mm in 65 x 65 x 30 mm
const Geometry kGeo[2] = {{{0.025, 0.025, 0.05}, {0.04, 0.04, 0.06}}, {{0.05, 0.05, 0.02}, {0.065, 0.065, 0.03}}};
constexpr double kPr = 0.5;       // SetInitialParameters: p_r = 0.5 mm
constexpr double kFarcut = 3.2;   // a_farcut = 3.2 p_r
int g_device = 0;                 // G<d>

bool parse_material(const std::string& s, double v[6]) {
  size_t a = s.find('(');
  if (a == std::string::npos) return false;
  for (int k = 0; k < 6; ++k) {
    const size_t b = s.find_first_of(",)", a + 1);
    if (b == std::string::npos) return false;
    try {
      v[k] = std::stod(s.substr(a + 1, b - a - 1));
    } catch (...) {
      return false;
    }
    a = b;
  }
  return true;
}

dem_material material(const double v[6]) {
  dem_material m{};
  m.E = v[0] / kStress;
  m.Ec = v[1] / kStress;
  m.Gc = v[2] / kStress;
  m.b_r = v[3] / kLength;
  m.gap = v[4] / kLength;
  m.nu = 0.247;
  m.rho = 2610.0 * (kLength * kLength * kLength) / kMass;
  m.p_r = kPr;
  m.p_e = 0.6;
  m.mu = 0.45;
  m.mur = 0.05;
  m.farcut = kFarcut;
  return m;
}

// sample volume of SetLSi/CalculateParameters: pi (L0/2 + p_r)^2 (L2 + 2 p_r)
double vext(const Geometry& g) {
  const double L0 = g.lsi[0] / kLength - 2 * kPr, L2 = g.lsi[2] / kLength - 2 * kPr;
  return kPi * (0.5 * L0 + kPr) * (0.5 * L0 + kPr) * (L2 + 2 * kPr);
}

// h_CreateCylinderSample: N = (1 - porosity) Vext / p_V spheres of radius p_r,
// relaxed until no overlap exceeds 1e-4 of the diameter, removing the spheres
// of the worst overlaps as needed; returns the porosity reached.
int create_sample(int which, int index, double porosity, double* porosity_out) {
  const Geometry& g = kGeo[which];
  const double pV = 4.0 / 3.0 * kPi * kPr * kPr * kPr;
  const uint32_t n = (uint32_t)((1.0 - porosity) * vext(g) / pV);
  dem_loading box{};
  int rc = dem_reference_space(g.space, g.lsi, kPr, kFarcut, &box);
  if (rc) return rc;
  dem_pack_params p{};
  for (int d = 0; d < 3; ++d) p.center[d] = box.space_center[d];
  p.radius = 0.5 * g.lsi[0] / kLength;
  p.half_height = 0.5 * g.lsi[2] / kLength;
  p.r_min = p.r_max = kPr;
  p.E = 30.0;
  p.nu = 0.247;
  p.rho = 2.61;
  p.overlap_tol = 1e-4;
  p.n = n;
  p.growth_stages = 40;
  p.steps_per_stage = 200;
  p.max_fire_steps = 20000;
  p.seed = 1000003ull * (uint64_t)(index + 1) + (uint64_t)which;
  p.max_removed = n / 10;
  p.device = g_device;
  std::vector<float> xyz(3 * (size_t)n), rad(n);
  uint32_t kept = 0;
  dem_pack_report rep{};
  rc = dem_create_cylinder_sample(&p, xyz.data(), rad.data(), n, &kept, &rep);
  if (rc) return rc;
  std::cerr << "Sample " << which << " created: " << kept << " spheres (" << rep.removed << " removed), largest overlap "
            << rep.max_overlap << "\n";
  char name[256];
  std::snprintf(name, sizeof name, "./result/Sample_%d_%d.txt", which, index);
  rc = dem_save_cylinder_sample(name, xyz.data(), kept, box.hidden_point);
  *porosity_out = 1.0 - kept * pV / vext(g);
  return rc;
}

struct TestOut {
  double strain = 1e-2, stress = 1e6 / kStress, ld = 1.0, destruction = 1.0;
};

int run_test(int which, int index, const dem_material& m, TestOut* out) {
  const Geometry& g = kGeo[which];
  char name[256];
  std::snprintf(name, sizeof name, "./result/Sample_%d_%d.txt", which, index);
  uint32_t n = 0;
  int rc = dem_load_cylinder_sample(name, kPr, nullptr, 0, &n, nullptr, nullptr);
  if (rc) return rc;
  std::vector<float> xyz(3 * (size_t)n);
  dem_loading L{};
  rc = dem_load_cylinder_sample(name, kPr, xyz.data(), n, &n, L.size_real, L.center_real);
  if (rc) return rc;
  rc = dem_reference_space(g.space, g.lsi, kPr, kFarcut, &L);
  if (rc) return rc;
  L.test = which == 0 ? DEM_TEST_UNIAXIAL : DEM_TEST_BRAZIL;
  L.velocity = -5.0 * 0.02 / kVelocity;  // mp_calculateonesample.cu:130-131
  if (which == 0) {
    L.min_stress = 10e6 / kStress;
    L.max_strain = 0.01;
    L.cond_fracture = 0.1;
    L.dNsave = 100;
  } else {
    L.min_stress = 2.1e6 / kStress;
    L.max_strain = 0.03;
    L.cond_fracture = 0.1;
    L.dNsave = 1000;
  }
  const uint32_t cap = 1u << 22;
  std::vector<double> rec(3 * (size_t)cap);
  std::vector<uint32_t> bonds(cap);
  uint32_t nrec = 0;
  dem_result r{};
  dem_options opt{};
  opt.device = g_device;
  rc = dem_calculation_test(&opt, &m, &L, xyz.data(), nullptr, n, &r, rec.data(), bonds.data(), cap, &nrec);
  if (rc) return rc;
  std::snprintf(name, sizeof name, which == 0 ? "./result/Uniaxial_%d.txt" : "./result/Brazil_%d.txt", index);
  dem_save_sum_forces_loading(name, rec.data(), nrec < cap ? nrec : cap);
  out->strain = r.FractureStrain;
  out->stress = r.FractureStress;
  out->ld = r.LinearityDeviation;
  out->destruction = r.Destruction;
  std::cerr << (which == 0 ? "RU " : "RB ") << r.FractureStrain << " " << r.FractureStress * kStress << "\n";
  return DEM_OK;
}

}  // namespace

int main(int argc, char** argv) {
  int ndev = 0;
  dem_device_count(&ndev);
  std::cout << "There are " << ndev << " GPUs" << std::endl;
  bool one = false, create = false, U = false, B = false, fusc = false, fbsc = false;
  std::string mat, index = "0";
  for (int i = 1; i < argc; ++i) {
    const std::string a(argv[i]);
    size_t shift = 0;
    if (a.compare(0, 1, "G") == 0 && a.size() >= 2) {
      const int d = a[1] - '0';
      if (d < 0 || d >= ndev) {
        std::cerr << "Incorrect GPU request! Requested:" << d << "\n";
        return 1;
      }
      std::cout << "Correct GPU request! Requested: " << d << "\n";
      g_device = d;
    }
    if (a.compare(0, 1, "M") == 0) {
      mat = a;
      one = true;
    }
    if (a.size() >= 2 && a.compare(0, 2, "CS") == 0) {
      create = true;
      shift = 2;
    }
    if (a.size() >= shift + 1 && a.compare(shift, 1, "U") == 0) {
      U = true;
      ++shift;
    }
    if (a.size() >= shift + 1 && a.compare(shift, 1, "B") == 0) B = true;
    if (a.compare(0, 4, "FUSC") == 0) fusc = true;
    if (a.compare(0, 4, "FBSC") == 0) fbsc = true;
    if (a.compare(0, 1, "I") == 0) {
      index = a.substr(1);
      std::cout << "INDEX " << index << "\n";
    }
    if (a.compare(0, 3, "DCG") == 0 || a.compare(0, 3, "TSS") == 0)
      std::cerr << "calibration drivers: use dem-rock-calibration_b200.calibrate / .sweep\n";
  }
  if (!one) return 0;
  double v[6];
  if (!parse_material(mat, v)) {
    std::cerr << "bad material string " << mat << "\n";
    return 1;
  }
  const int idx = std::atoi(index.c_str());
  mkdir("result", 0755);
  const dem_material m = material(v);
  double pu = v[5], pb = v[5];
  TestOut tu, tb;
  int rc = 0;
  if ((U && create) || fusc) rc = create_sample(0, idx, v[5], &pu);
  if (!rc && U) rc = run_test(0, idx, m, &tu);
  if (!rc && ((B && create) || fbsc)) rc = create_sample(1, idx, std::max(v[5], pu), &pb);
  if (!rc && B) rc = run_test(1, idx, m, &tb);
  if (rc) {
    std::cerr << "libb200dem: " << dem_strerror(rc) << " " << dem_last_error_detail() << "\n";
    return 2;
  }
  // CalculateOneSample reports the larger of the requested and reached porosities
  const double porosity = std::max(v[5], std::max(pu, pb));
  std::cout << "ResultCalculateOneSample[" << v[0] << "," << v[1] << "," << v[2] << "," << v[3] << "," << v[4] << ","
            << porosity << "," << tu.strain << "," << tu.stress * kStress << "," << tu.ld << "," << tu.destruction << ","
            << tb.strain << "," << tb.stress * kStress << "," << 0 << "," << tb.destruction << "]\n";
  return 0;
}
