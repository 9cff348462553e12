/*
 * CPU oracle for the bonded-particle DEM time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * kernels of MSMS-LAB/DEM-Rock-Calibration, kept in the reference's own data
 * layout (SoA positions x[0..N) y[N..2N) z[2N..3N), IonP neighbour slots per
 * particle, per-slot float3 histories), so that the CUDA product can be
 * checked against it.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load it; the product never calls it.
 *
 * Parity pin: the oracle is checked against golden vectors produced by the
 * reference's own CUDA kernels (compiled from the reference sources by
 * oracle/Makefile into oracle/_ref/, run on a B200 by
 * tests/golden/make_golden.py).
 *
 * Arithmetic contract.  Every floating-point operation is rounded separately
 * (compiled with -ffp-contract=off): the reference's __fmul_rn / __frcp_rn /
 * __fsqrt_rn are correctly rounded and map to a*b, 1/x and sqrt; __frsqrt_rn
 * maps to orc_rsqrt_rn (correctly rounded 1/sqrt, see dem_oracle.c); the
 * reference's norm3df(x,y,z) is restated as sqrt(x*x+y*y+z*z) with each
 * operation rounded (norm3df itself is a CUDA library routine and is not
 * reproduced; the two agree to a few ulp).
 *
 * Each function cites the reference file:line it restates.
 */
#ifndef DEM_ORACLE_H
#define DEM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_EMPTY 0xFFFFFFFFu

/* Correctly rounded reciprocal square root (restates the IEEE semantics of
 * __frsqrt_rn used at md_boundinteractions_construct.cu:65). */
float orc_rsqrt_rn_f(float x);
double orc_rsqrt_rn_d(double x);

void orc_set_threads(int nthreads);
int orc_get_threads(void);

/* Functions below exist in two precisions: suffix _f (float) and _d (double).
 * Optional arrays may be NULL, which selects the reference's scalar value.   */
#define ORC_DECLARE(REAL, SFX)                                                                  \
  /* md_calculate_cell.cu:13-41 + md_cell_distribution.cu:130-172 + md_calculate_cell.cu:43-75 */ \
  void orc_cell_distribution_##SFX(const REAL* R, uint32_t N, REAL inv_a, uint32_t nx, uint32_t ny, \
                                   uint32_t nz, uint32_t* CI, uint32_t* CIs, uint32_t* pnC);       \
  /* md_interaction_list_construct.cu:204-317 ; returns number of slot overflows */                \
  int64_t orc_il_construct_##SFX(const REAL* R, uint32_t N, const uint32_t* CIs, const uint32_t* pnC, \
                                 uint32_t* IL, uint32_t IonP, REAL a, REAL inv_a, REAL aacut,      \
                                 uint32_t nx, uint32_t ny, uint32_t nz);                           \
  /* md_interaction_list_reconstructbpm.cu:13-46, 80-139 ; returns overflows */                     \
  int64_t orc_il_reconstruct_bpm_##SFX(const REAL* R, uint32_t N, const uint32_t* CIs,              \
                                       const uint32_t* pnC, uint32_t* IL, uint32_t* ILtype,         \
                                       uint32_t IonP, REAL a, REAL inv_a, REAL aacut, uint32_t nx,  \
                                       uint32_t ny, uint32_t nz);                                   \
  /* md_interaction_list_reconstructbpm.cu:141-186 */                                              \
  void orc_delete_far_links_##SFX(const REAL* R, uint32_t N, uint32_t* IL, uint32_t* ILtype,        \
                                  REAL* Rij, REAL* Oijt, REAL* Mijn, REAL* Mijt, uint32_t IonP,     \
                                  REAL aacut);                                                      \
  /* md_boundinteractions_construct.cu:35-106.  rad/gap: per-particle radii and absolute gap     \
   * for polydisperse samples (bond if r^2 < (r_i+r_j+gap)^2); rad==NULL uses aa_create. */        \
  void orc_construct_bonds_##SFX(const REAL* R, uint32_t N, const uint32_t* IL, uint32_t* ILtype,   \
                                 REAL* inv_L0, REAL* Rij, REAL* Oijt, REAL* Mijn, REAL* Mijt,       \
                                 uint32_t IonP, REAL aa_create, const REAL* rad, double gap);       \
  /* md_calculateforcesdem3.cu:20-200, 427-547.  slot_br/slot_sn/slot_st: per-slot bond radius,  \
   * normal and shear strength (NULL = scalars b_r, Ec, Gc).  Fabs/Mabs (optional) receive the    \
   * per-particle sum of |contribution| used for reordering tolerances; Fsens (optional, one     \
   * value per particle) the sum over its pairs of normal stiffness times one ulp of the pair    \
   * distance, the forward error of rounding the distance.  nobreak=1 selects the                \
   * _ncb variant. */                                                                              \
  void orc_forces_bpm_##SFX(const REAL* R, const REAL* V, const REAL* W, uint32_t N,                 \
                            const uint32_t* IL, uint32_t* ILtype, const REAL* inv_L0, REAL* Rij,    \
                            REAL* Oijt, REAL* Mijn, REAL* Mijt, REAL* F, REAL* M, uint32_t IonP,    \
                            REAL dt, REAL E, REAL G, REAL b_r, REAL Ec, REAL Gc,                    \
                            const REAL* slot_br, const REAL* slot_sn, const REAL* slot_st,          \
                            REAL* Fabs, REAL* Mabs, REAL* Fsens, int nobreak);                      \
  /* md_calculateforcesdem3.cu:202-425.  rad==NULL: reference (monodisperse rP, mP) formulas;    \
   * otherwise the polydisperse generalisation with per-particle masses. */                              \
  void orc_forces_hm_##SFX(const REAL* R, const REAL* V, const REAL* W, uint32_t N,                  \
                           const uint32_t* IL, const uint32_t* ILtype, REAL* Oijt, REAL* F, REAL* M, \
                           uint32_t IonP, REAL dt, REAL hmE, REAL hmG, REAL pA, REAL mu, REAL mur,  \
                           REAL mP, REAL rP, const REAL* rad, const REAL* mass, REAL* Fabs,         \
                           REAL* Mabs, REAL* Fsens);                                                \
  /* md_compression_hm.cu:20-449.  axis=2: uniaxial (platens normal to z), axis=1: Brazilian    \
   * (platens normal to y).  Block partials of 64 threads are reproduced exactly; FL receives  \
   * 2*nblocks floats (bottom sums then top sums) and sFL their double sums. */                    \
  void orc_platen_##SFX(int axis, const REAL* R, const REAL* V, const REAL* W, REAL* Oiwt, REAL* F,  \
                        REAL* M, uint32_t N, REAL dt, REAL wE, REAL wG, REAL pA, REAL mu, REAL mur, \
                        REAL mP, REAL rP, const REAL* rad, const REAL* mass, const REAL* center,   \
                        REAL wall_RR, REAL wall_top, REAL wall_bot, REAL wall_V, REAL Zcut,        \
                        REAL* FL, double* sFL);                                                    \
  /* Order-independent sums (the engine's deterministic mode): the same per-slot values as      \
   * orc_forces_bpm / orc_forces_hm, each slot's force and moment rounded to fixed point (2^-40   \
   * in float, 2^-50 in double) and added into 64-bit accumulators Fq, Mq (3N each, SoA, added   \
   * to, not cleared); orc_fix_to_real converts them back.  orc_platen_q sums the platen forces  \
   * of the spheres in fixed point (2^-40) into sFL. */                                            \
  void orc_forces_bpm_q_##SFX(const REAL* R, const REAL* V, const REAL* W, uint32_t N,               \
                              const uint32_t* IL, uint32_t* ILtype, const REAL* inv_L0, REAL* Rij,  \
                              REAL* Oijt, REAL* Mijn, REAL* Mijt, uint32_t IonP, REAL dt, REAL E,   \
                              REAL G, REAL b_r, REAL Ec, REAL Gc, const REAL* slot_br,              \
                              const REAL* slot_sn, const REAL* slot_st, int nobreak, int64_t* Fq,   \
                              int64_t* Mq);                                                         \
  void orc_forces_hm_q_##SFX(const REAL* R, const REAL* V, const REAL* W, uint32_t N,                \
                             const uint32_t* IL, const uint32_t* ILtype, REAL* Oijt, uint32_t IonP, \
                             REAL dt, REAL hmE, REAL hmG, REAL pA, REAL mu, REAL mur, REAL mP,      \
                             REAL rP, const REAL* rad, const REAL* mass, int64_t* Fq, int64_t* Mq); \
  void orc_fix_to_real_##SFX(const int64_t* q, REAL* out, uint64_t n);                              \
  void orc_platen_q_##SFX(int axis, const REAL* R, const REAL* V, const REAL* W, REAL* Oiwt,          \
                          REAL* F, REAL* M, uint32_t N, REAL dt, REAL wE, REAL wG, REAL pA, REAL mu, \
                          REAL mur, REAL mP, REAL rP, const REAL* rad, const REAL* mass,           \
                          const REAL* center, REAL wall_RR, REAL wall_top, REAL wall_bot,          \
                          REAL wall_V, REAL Zcut, double* sFL);                                    \
  /* md_calculateincrementsdem.cu:128-158 ; dtm_i/dtI_i per particle (NULL = scalars) */          \
  void orc_increments_##SFX(const REAL* F, REAL* V, REAL* R, const REAL* M, REAL* W, uint32_t N,     \
                            REAL dtm, REAL dt, REAL dtI, const REAL* dtm_i, const REAL* dtI_i);    \
  /* md_parallelepipedrestriction.cu:254-342 */                                                   \
  void orc_cut_restriction_##SFX(REAL* R, REAL* V, REAL* F, uint32_t N, const REAL* center,          \
                                 const REAL* sized2, const REAL* hp);                               \
  /* md_calculateforces.cu:20-67 (soft repulsion of the sample-preparation stage).  rad!=NULL:    \
   * a_ij = r_i + r_j replaces the scalar cut a. */                                                 \
  void orc_soft_forces_##SFX(const REAL* R, REAL* F, uint32_t N, const uint32_t* IL, REAL* Rijm,     \
                             uint32_t IonP, REAL D, REAL aa, const REAL* rad);                      \
  /* md_firerelaxation.cu:18-56 */                                                                 \
  void orc_fire_increments_##SFX(const REAL* F, REAL* V, REAL* R, uint32_t N, REAL dtm, REAL dt,     \
                                 REAL alpha, const REAL* dtm_i);                                    \
  /* md_firerelaxation.cu:58-70 */                                                                 \
  void orc_fire_half_step_back_##SFX(const REAL* V, REAL* R, uint32_t N, REAL dt_d2);               \
  /* md_firerelaxation.cu:375-494 (block partials of 64 threads x 4 elements, summed in double) */ \
  double orc_fdotv_##SFX(const REAL* V, const REAL* F, uint32_t N);                                 \
  /* md_calculateincrements.cu:105-122 */                                                          \
  void orc_increments_viscous_##SFX(const REAL* F, REAL* V, REAL* R, uint32_t N, REAL dtm, REAL dt,  \
                                    REAL vis, const REAL* dtm_i);                                   \
  /* md_cylinderrestriction.cu:190-234 */                                                          \
  void orc_cylinder_restriction_z_##SFX(REAL* V, REAL* R, uint32_t N, const REAL* center, REAL R0,   \
                                        REAL H0, REAL HideZ);

ORC_DECLARE(float, f)
ORC_DECLARE(double, d)

/* md_results.cu:207-272 + 189-205: number of bonded directed slots */
uint64_t orc_count_bonds(const uint32_t* IL, const uint32_t* ILtype, uint64_t nslots);

/* Loading controller and stress bookkeeping (host logic in double):
 * compression_data (md_data_types.h:203-495) and result_data (:190-201). */
typedef struct {
  int brazil;              /* 0: uniaxial (z), 1: Brazilian (y)        */
  double size_d[3], center_d[3];
  double Top, Bottom, TopR, BottomR, Size0;
  double V, VLoad, Area, inv_Area;
  double MinStress, ZeroStress, MaxStrain, ConditionFracture;
  double Stress, Strain, FractureStress, FractureStrain, LinearityDeviation;
  uint32_t StepsStop;
  int Loading, Fracture;
  /* result_data */
  double sFL[2], sz0;
  uint32_t dNsave, Nsave, stepsave;
  double* h_sFL;           /* 3*Nsave: strain, sigma_bottom, sigma_top */
  uint32_t* h_sSI;         /* Nsave bond counts */
} orc_compress;

/* md_data_types.h:212-242 (CalculateUParameters) / :380-409 (CalculateBParameters) */
void orc_compress_init(orc_compress* C, int brazil, const double* size_real, const double* center_real,
                       double p_r, double minstress, double maxstrain, double condfract, double vload);
/* md_results.cu:56-99 (SumForcesULoading) / :101-145 (SumForcesBLoading), with sFL given */
void orc_sum_forces(orc_compress* C, uint32_t step);
/* md_results.cu:189-205 (SumInteractions) given the slot count */
void orc_sum_interactions(orc_compress* C, uint64_t count, uint32_t step);
/* md_data_types.h:347-379 (CompressU_S3) / :462-494 (CompressB_S3) */
void orc_compress_s3(orc_compress* C, double dt, double p_r);
/* md_results.cu:147-166 */
double orc_linearity_deviation(orc_compress* C);
/* md_results.cu:182-187 */
double orc_destruction(const orc_compress* C);

/* Seeded sample creation restated from the engine's packer (dem_pack_oracle.c):
 * same fill, growth, FIRE and contact-list schedule, fixed-point pair sums, so
 * the packing equals the GPU's bit for bit.  Fields as the engine's
 * dem_pack_params (max_removed must be 0).  fire_trace (optional) receives
 * (dt, alpha, half-step-back flag) after every FIRE step. */
typedef struct {
  double center[3];
  double radius, half_height;
  double r_min, r_max;
  double E, nu, rho;
  double overlap_tol;
  uint32_t n, growth_stages, steps_per_stage, max_fire_steps;
  uint64_t seed;
  int device, fire_variant;
  uint32_t max_removed, reserved;
} orc_pack_params;
typedef struct {
  uint64_t steps;
  double max_overlap, packing_fraction;
  uint32_t rebuilds, removed;
} orc_pack_report;
int orc_pack_cylinder(const orc_pack_params* p, float* xyz, float* radii, uint32_t cap, uint32_t* n,
                      orc_pack_report* rep, double* fire_trace, uint32_t trace_cap, uint32_t* ntrace);

#ifdef __cplusplus
}
#endif
#endif
