// Host-side derivation of the kernel constants from the micro-parameters, in
// double precision with the same formulas and the same float conversions as
// the reference (potential_data::CalculateParameters md_data_types.h:155-187,
// cell_data::CalculateParameters :42-55, sample_data :87-123,
// compression_data::Calculate{U,B}Parameters :212-242, :380-409), so that a
// monodisperse specimen gets bit-identical kernel arguments.
#pragma once

#include <cmath>
#include <cstdint>

namespace dem {

constexpr double kPiD = 3.1415926535897932384626433832795;
constexpr double kStressConst = 1e9;   // GPa per Pa (reference stress_const)
constexpr double kLengthConst = 1e-3;  // m per mm
constexpr double kDensityConst = 1e3;  // (mg/mm^3) per (kg/m^3)... reference density_const = 1e-6/1e-9
constexpr double kVelocityConst = 1e3; // (m/s) per (mm/us)

struct Potential {
  // inputs
  double m_E, m_nu, m_Ec, m_Gc, b_r, b_d, p_r, m_ro, p_e, p_mu, p_mur, a_farcut;
  // derived
  double m_G, b_S, p_V, p_m, b_dd, p_1d_m, p_I, hm_E, hm_G, p_A, aa_farcut, Trayleigh, Tsim, dt, dt_d_m, dt_d_I;

  void calculate() {
    m_G = 0.5 * m_E / (1.0 + m_nu);
    b_S = kPiD * b_r * b_r;
    p_V = 4.0 * (1.0 / 3.0) * kPiD * p_r * p_r * p_r;
    p_m = m_ro * p_V;
    b_dd = b_d * b_d;
    p_1d_m = 1.0 / p_m;
    p_I = 0.4 * p_m * p_r * p_r;
    hm_E = 0.5 * m_E / (1.0 - m_nu * m_nu);
    hm_G = 0.5 * m_G / (2.0 - m_nu);
    const double le = std::log(p_e);
    p_A = le / std::sqrt(kPiD * kPiD + le * le);
    aa_farcut = a_farcut * a_farcut;
    Trayleigh = kPiD * p_r * std::sqrt(2.0 * m_ro * (1.0 + m_nu)) / (std::sqrt(m_E) * (0.163 * m_nu + 0.8766));
    const double t0 = m_E * b_S / (2.0 * p_r), t1 = m_G * b_S / (2.0 * p_r);
    Tsim = (t0 > t1) ? 2.0 * std::sqrt(p_m / t0) : 2.0 * std::sqrt(p_m / t1);
    dt = (Trayleigh < Tsim) ? 0.05 * Trayleigh : 0.05 * Tsim;
    dt_d_m = p_1d_m * dt;
    dt_d_I = dt / p_I;
  }
};

// Per-particle integration constants with the reference's formulas for a
// particle of radius r (p_V, p_m, p_1d_m, p_I, dt_d_m, dt_d_I).
#ifdef __CUDACC__
__host__ __device__
#endif
inline void particle_constants(double r, double m_ro, double dt, double& mass, double& dtm, double& dtI) {
  const double V = 4.0 * (1.0 / 3.0) * kPiD * r * r * r;
  mass = m_ro * V;
  const double inv_m = 1.0 / mass;
  const double I = 0.4 * mass * r * r;
  dtm = inv_m * dt;
  dtI = dt / I;
}

// Rayleigh time of a particle of radius r (the reference's Trayleigh).
inline double rayleigh_time(double r, double m_ro, double m_E, double m_nu) {
  return kPiD * r * std::sqrt(2.0 * m_ro * (1.0 + m_nu)) / (std::sqrt(m_E) * (0.163 * m_nu + 0.8766));
}

inline float F32(double x) { return (float)x; }

}  // namespace dem
