/*
 * CPU oracle of the bonded-particle DEM step (test infrastructure only; see
 * dem_oracle.h).  Build: oracle/Makefile (gcc -O2 -ffp-contract=off -fopenmp).
 */
#include "dem_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#if defined(__FP_FAST_FMA) && !defined(ORC_ALLOW_CONTRACT)
/* fine: contraction is controlled by -ffp-contract=off, not by FMA availability */
#endif

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Correctly rounded 1/sqrt(x) for float.  A double evaluation is within about
 * 2^-52 of the exact value; the candidate is then corrected by comparing the
 * exact value against the midpoints to its float neighbours, using the exact
 * integer test  1/sqrt(x) > m  <=>  m*m*x < 1  on the significands. */
static int cmp_mid2x_with_one(double mid, float x) {
  /* returns sign(mid^2 * x - 1) computed exactly */
  int em, ex;
  double fm = frexp(mid, &em); /* mid = fm * 2^em, fm in [0.5,1) */
  double fx = frexp((double)x, &ex);
  unsigned long long Mm = (unsigned long long)ldexp(fm, 26); /* 26 bits cover a float midpoint */
  unsigned long long Mx = (unsigned long long)ldexp(fx, 24);
  /* mid^2*x = Mm^2 * Mx * 2^(2(em-26) + ex-24) */
  unsigned __int128 P = (unsigned __int128)Mm * Mm * Mx;
  int e = 2 * (em - 26) + (ex - 24);
  /* compare P * 2^e with 1 */
  if (e >= 0) return P > 0 ? 1 : -1; /* P>=1 and e>=0 means >= 1; equality impossible here */
  int sh = -e;
  if (sh >= 127) return -1;
  unsigned __int128 one = (unsigned __int128)1 << sh;
  if (P > one) return 1;
  if (P < one) return -1;
  return 0;
}

float orc_rsqrt_rn_f(float x) {
  if (!(x > 0)) {
    if (x == 0) return copysignf(INFINITY, x);
    return NAN;
  }
  if (isinf(x)) return 0.0f;
  float y = (float)(1.0 / sqrt((double)x));
  float up = nextafterf(y, INFINITY), dn = nextafterf(y, 0.0f);
  double hi = 0.5 * ((double)y + (double)up);
  double lo = 0.5 * ((double)y + (double)dn);
  /* exact value > hi  <=> hi^2 x < 1 */
  if (cmp_mid2x_with_one(hi, x) < 0) return up;
  if (cmp_mid2x_with_one(lo, x) > 0) return dn;
  return y;
}

/* FP64 builds define the reciprocal square root as 1/sqrt(x) with two IEEE
 * roundings, identically in the CUDA product and here. */
double orc_rsqrt_rn_d(double x) { return 1.0 / sqrt(x); }

/* Correctly rounded Euclidean norm of three floats: the sum of squares is
 * exact in double (each square has 48 bits, the sum < 2^-53 relative error)
 * and the double square root then the rounding to float is correctly rounded
 * except in cases within 2^-29 ulp of a midpoint. */
static inline float orc_norm3_f(float x, float y, float z) {
  double s = (double)x * x + (double)y * y + (double)z * z;
  return (float)sqrt(s);
}
/* FP64 builds: sqrt of the rounded sum of squares, as in the CUDA product */
static inline double orc_norm3_d(double x, double y, double z) { return sqrt((x * x + y * y) + z * z); }

/* ---- float instantiation ---- */
#define REAL float
#define SFX f
#define ONE 1.0f
#define TWO 2.0f
#define FOUR 4.0f
#define EIGHT 8.0f
#define HALF 0.5f
#define QUARTER 0.25f
#define PI 3.14159265358979f   /* MCf_pi, md_math_constants.h:170 */
#define TWO_THIRDS 0.6666666667f /* MCf_2d3, md_math_constants.h:146 */
#define DAMP (-1.8257f)
#define SQRT sqrtf
#define FMA fmaf
#define FABS fabsf
#define FLOOR floorf
#define COPYSIGN copysignf
#define RSQRT_RN orc_rsqrt_rn_f
#define NORM3_RN orc_norm3_f
#define ULP(x) (nextafterf(fabsf(x), INFINITY) - fabsf(x))
/* fixed-point sums of the engine's deterministic FP32 mode: multiples of 2^-40,
 * the product x * 2^40 exact in float, rounded to the nearest integer (ties to
 * even), converted back through double */
#define FIXQ(x) llrintf((x) * 0x1p40f)
#define UNFIXQ(q) ((float)((double)(q) * 0x1p-40))
#include "dem_oracle_impl.h"
#undef REAL
#undef SFX
#undef ONE
#undef TWO
#undef FOUR
#undef EIGHT
#undef HALF
#undef QUARTER
#undef PI
#undef TWO_THIRDS
#undef DAMP
#undef SQRT
#undef FMA
#undef FABS
#undef FLOOR
#undef COPYSIGN
#undef RSQRT_RN
#undef NORM3_RN
#undef ULP
#undef FIXQ
#undef UNFIXQ

/* ---- double instantiation (FP64 build extension) ---- */
#define REAL double
#define SFX d
#define ONE 1.0
#define TWO 2.0
#define FOUR 4.0
#define EIGHT 8.0
#define HALF 0.5
#define QUARTER 0.25
#define PI 3.1415926535897932384626433832795 /* MC_pi, md_math_constants.h:127 */
#define TWO_THIRDS (2.0 / 3.0)
#define DAMP (-1.8257)
#define SQRT sqrt
#define FMA fma
#define FABS fabs
#define FLOOR floor
#define COPYSIGN copysign
#define RSQRT_RN orc_rsqrt_rn_d
#define NORM3_RN orc_norm3_d
#define ULP(x) (nextafter(fabs(x), INFINITY) - fabs(x))
/* FP64 deterministic mode: multiples of 2^-50 */
#define FIXQ(x) llrint((x) * 0x1p50)
#define UNFIXQ(q) ((double)(q) * 0x1p-50)
#include "dem_oracle_impl.h"

/* md_results.cu:207-272 with the host sum of :189-205 */
uint64_t orc_count_bonds(const uint32_t* IL, const uint32_t* ILtype, uint64_t nslots) {
  uint64_t s = 0;
#pragma omp parallel for schedule(static) reduction(+ : s)
  for (int64_t k = 0; k < (int64_t)nslots; ++k)
    if (IL[k] != ORC_EMPTY && ILtype[k] == 1) ++s;
  return s;
}

static const double kPi = 3.1415926535897932384626433832795;
static const double kStress = 1e9; /* stress_const, md_phys_constants.h:12 */

void orc_compress_init(orc_compress* C, int brazil, const double* size_real, const double* center_real,
                       double p_r, double minstress, double maxstrain, double condfract, double vload) {
  memset(C, 0, sizeof(*C));
  C->brazil = brazil;
  for (int d = 0; d < 3; ++d) {
    C->size_d[d] = size_real[d];
    C->center_d[d] = center_real[d];
  }
  const int ax = brazil ? 1 : 2;
  float sized2x = (float)(0.5 * C->size_d[0]);
  float sized2z = (float)(0.5 * C->size_d[2]);
  float sizez = (float)C->size_d[2];
  C->Size0 = C->size_d[ax];
  C->Bottom = C->center_d[ax] - 0.5 * C->size_d[ax];
  C->BottomR = C->Bottom + p_r;
  C->Top = C->center_d[ax] + 0.5 * C->size_d[ax];
  C->TopR = C->Top - p_r;
  float area;
  if (!brazil) {
    /* md_data_types.h:227-228 (float Area, float _1d_Area) */
    area = (float)(kPi * (sized2x + p_r) * (sized2x + p_r));
    C->ZeroStress = 0.33 * minstress;
  } else {
    /* md_data_types.h:395-396 */
    area = (float)(0.5 * 2 * kPi * (sized2x) * (sizez));
    C->ZeroStress = 0.5 * minstress;
  }
  (void)sized2z;
  C->Area = area;
  C->inv_Area = (float)(1.0 / area);
  C->MinStress = minstress;
  C->MaxStrain = maxstrain;
  C->ConditionFracture = condfract;
  C->VLoad = vload;
  C->V = 0;
  /* ResultsUInit/ResultsBInit, md_results.cu:21,36: sz0 is the float size */
  C->sz0 = (double)(float)C->size_d[ax];
}

void orc_sum_forces(orc_compress* C, uint32_t n) {
  const int ax = C->brazil ? 1 : 2;
  if (C->dNsave && n % C->dNsave == 0 && C->h_sFL && C->stepsave < C->Nsave) {
    C->h_sFL[3 * C->stepsave] = (C->size_d[ax] - C->sz0) / C->sz0;
    C->h_sFL[3 * C->stepsave + 1] = C->sFL[0] * C->inv_Area;
    C->h_sFL[3 * C->stepsave + 2] = C->sFL[1] * C->inv_Area;
    if (fabs(C->V) > 1e-9) ++C->stepsave;
  }
  C->Stress = 0.5 * (fabs(C->sFL[0]) + fabs(C->sFL[1])) * C->inv_Area;
  if (!C->Loading && C->Stress > C->MinStress) C->Loading = 1;
  if (!C->brazil) {
    if (C->FractureStress < C->Stress) {
      C->FractureStress = C->Stress;
      C->FractureStrain = (C->sz0 - C->size_d[ax]) / C->sz0;
    }
    if (C->Loading && (C->Stress < C->ZeroStress || C->Stress < C->ConditionFracture * C->FractureStress))
      C->Fracture = 1;
  } else {
    /* md_results.cu:130-134: the Brazilian peak also resets when the stress
     * drops below ConditionFracture times the peak */
    if (C->FractureStress < C->Stress || C->Stress < C->ConditionFracture * C->FractureStress) {
      C->FractureStress = C->Stress;
      C->FractureStrain = (C->sz0 - C->size_d[ax]) / C->sz0;
    }
    if (C->Loading && C->Stress < C->ZeroStress) C->Fracture = 1;
  }
}

void orc_sum_interactions(orc_compress* C, uint64_t count, uint32_t n) {
  if (C->dNsave && n % C->dNsave == 0 && C->h_sSI && C->stepsave < C->Nsave)
    C->h_sSI[C->stepsave] = (uint32_t)count;
}

void orc_compress_s3(orc_compress* C, double dt, double p_r) {
  const int ax = C->brazil ? 1 : 2;
  double pS = C->brazil ? 0.5 * (-C->sFL[0] + C->sFL[1]) : 0.5 * fabs(-C->sFL[0] + C->sFL[1]);
  double pD = fabs(C->sFL[0] + C->sFL[1]);
  if (pS * C->inv_Area < 1e-9) {
    C->V = 10.0 * C->VLoad;
  } else if (pD > 0.20 * pS && pS * C->inv_Area > 2.0e+6 / kStress) {
    if (fabs(C->V) > 1e-15) C->StepsStop = 0;
    C->V = 0;
    ++C->StepsStop;
    if (C->StepsStop > 30000) C->Fracture = 1;
  } else {
    C->V = C->VLoad;
  }
  C->size_d[ax] += C->V * dt;
  C->Top += 0.5 * C->V * dt;
  C->TopR = C->Top - p_r;
  C->Bottom -= 0.5 * C->V * dt;
  C->BottomR = C->Bottom + p_r;
  C->Strain = (C->size_d[ax] - C->Size0) / C->Size0;
}

double orc_linearity_deviation(orc_compress* C) {
  double l_eps = 0, l_deps = 0, l_A = C->FractureStress / C->FractureStrain, l_dS = 0, LD = 0;
  uint32_t i = 0;
  const double* h = C->h_sFL;
  /* the record buffer holds Nsave+2 zeroed entries, so the look-ahead of
   * md_results.cu:157 stays inside it */
  do {
    LD += l_deps * l_dS * l_dS;
    ++i;
    l_eps = -h[3 * i];
    l_deps = -0.5 * (h[3 * (i + 1)] - h[3 * (i - 1)]);
    l_dS = (l_A * l_eps - 0.5 * (h[3 * i + 2] - h[3 * i + 1]));
  } while (l_eps < C->FractureStrain - 2 * l_deps && i < C->stepsave);
  LD /= (C->FractureStrain * C->FractureStress * C->FractureStress);
  LD += 1.0;
  C->LinearityDeviation = LD;
  return LD;
}

double orc_destruction(const orc_compress* C) {
  if (C->stepsave == 0 || C->h_sSI[0] == 0) return 0.0;
  return C->h_sSI[C->stepsave - 1] / (double)C->h_sSI[0];
}
