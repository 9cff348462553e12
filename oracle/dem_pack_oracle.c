/*
 * CPU restatement of the engine's seeded sample creation (the role of the
 * reference's h_CreateCylinderSample, md_createcylindersample.cu:184-439).
 *
 * TEST INFRASTRUCTURE ONLY.  It restates, step for step and operation for
 * operation, what dem_create_cylinder_sample runs on the GPU: the seeded
 * fill of a z-axis cylinder, radius growth with viscous relaxation, then
 * FIRE relaxation (FIRE 2.0, or the reference's FIRE update of
 * md_firerelaxation.cu:18-70 with the dt / alpha adaptation of
 * md_createcylindersample.cu:368-397) of linear overlap springs and spring
 * walls, with the same contact-list and chunk schedule.  Pair forces are
 * summed in 2^-40 fixed point as on the GPU, so a particle's force does not
 * depend on the summation order and the packing comes out bit for bit the
 * same as the GPU's.  It is used by the GPU parity test of the packer and
 * by the benchmark's reference leg, which must build its specimens without
 * the product library.
 *
 * Compiled with -ffp-contract=off: every float operation is rounded
 * separately, as in the product (built with -fmad=false).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "dem_oracle.h"

#ifdef _OPENMP
#include <omp.h>
#endif

static const double kPi = 3.1415926535897932384626433832795;
static const float kFixScale = 1099511627776.0f; /* 2^40 */
static const double kFixInv = 1.0 / 1099511627776.0;

static uint64_t sm64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static double u01(uint64_t h) { return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
static double rng_uniform(uint64_t* s) {
  *s = sm64(*s);
  return u01(*s);
}
static long long to_fix(float x) { return llrintf(x * kFixScale); }

typedef struct {
  float x, y, z, w;
} f4;

typedef struct {
  double P, dt, alpha, dt0, dtmax, dtmin, dtgrow, dtshrink, alpha0, alphashrink;
  uint32_t Npos, Nneg, Ndelay, back;
  uint64_t step;
  float max_overlap, vmax2, dmax2;
  uint32_t variant;
} fire_t;

typedef struct {
  orc_pack_params p;
  uint32_t n;
  f4 *pos, *vel, *ref;
  float* frc;            /* 3 per particle */
  long long* q;          /* 3 per particle, fixed point */
  uint32_t *nb_start, *nb;   /* contact list: partners j > i of each i (CSR) */
  uint32_t *in_start, *in_pair; /* the same pairs by their higher index j: pair numbers (CSR) */
  long long* pf;             /* per pair: fixed-point force on the lower index (3 values) */
  size_t nb_cap;
  float scale, D, vis;
  float cyl[5];
  double skin;
  fire_t F;
  uint32_t rebuilds;
  float last_overlap;
} packer_t;

/* the engine's particle constants (dt/m) for a sphere of radius r */
static double dt_over_m(double r, double rho, double dt) {
  const double V = 4.0 * (1.0 / 3.0) * kPi * r * r * r;
  const double m = rho * V;
  return (1.0 / m) * dt;
}

static double rayleigh(double r, double rho, double E, double nu) {
  return kPi * r * sqrt(2.0 * rho * (1.0 + nu)) / (sqrt(E) * (0.163 * nu + 0.8766));
}

/* Contact list: every pair within r_i + r_j + skin (final radii), from its
 * lower index (the GPU's list), and the transposed index by the higher one. */
static int rebuild(packer_t* S) {
  const uint32_t n = S->n;
  const double a = (2.0 * S->p.r_max + S->skin) * 1.0001;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (uint32_t i = 0; i < n; ++i) {
    const float c[3] = {S->pos[i].x, S->pos[i].y, S->pos[i].z};
    for (int d = 0; d < 3; ++d) {
      if (c[d] < lo[d]) lo[d] = c[d];
      if (c[d] > hi[d]) hi[d] = c[d];
    }
  }
  uint32_t g[3];
  for (int d = 0; d < 3; ++d) g[d] = (uint32_t)((hi[d] - lo[d]) / a) + 1;
  const size_t ncell = (size_t)g[0] * g[1] * g[2];
  uint32_t* cnt = calloc(ncell + 1, sizeof(uint32_t));
  uint32_t* cell = malloc((size_t)n * sizeof(uint32_t));
  uint32_t* list = malloc((size_t)n * sizeof(uint32_t));
  uint32_t* cnb = calloc((size_t)n + 1, sizeof(uint32_t));
  if (!cnt || !cell || !list || !cnb) return -1;
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t c[3];
    const float v[3] = {S->pos[i].x, S->pos[i].y, S->pos[i].z};
    for (int d = 0; d < 3; ++d) {
      double t = floor((v[d] - lo[d]) / a);
      c[d] = t < 0 ? 0 : (t >= g[d] ? g[d] - 1 : (uint32_t)t);
    }
    cell[i] = c[0] + g[0] * (c[1] + g[1] * c[2]);
    ++cnt[cell[i] + 1];
  }
  for (size_t c = 0; c < ncell; ++c) cnt[c + 1] += cnt[c];
  {
    uint32_t* cur = malloc(ncell * sizeof(uint32_t));
    if (!cur) return -1;
    memcpy(cur, cnt, ncell * sizeof(uint32_t));
    for (uint32_t i = 0; i < n; ++i) list[cur[cell[i]]++] = i;
    free(cur);
  }
  const float skin = (float)S->skin;
  /* two passes: count, then fill */
  for (int pass = 0; pass < 2; ++pass) {
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
      const uint32_t i = (uint32_t)ii;
      const f4 xi = S->pos[i];
      const uint32_t ci = cell[i];
      const int cx = (int)(ci % g[0]), cy = (int)((ci / g[0]) % g[1]), cz = (int)(ci / g[0] / g[1]);
      uint32_t k = pass ? S->nb_start[i] : 0;
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            const int x = cx + dx, y = cy + dy, z = cz + dz;
            if (x < 0 || y < 0 || z < 0 || x >= (int)g[0] || y >= (int)g[1] || z >= (int)g[2]) continue;
            const uint32_t c = (uint32_t)x + g[0] * ((uint32_t)y + g[1] * (uint32_t)z);
            for (uint32_t t = cnt[c]; t < cnt[c + 1]; ++t) {
              const uint32_t j = list[t];
              if (j <= i) continue;
              const f4 xj = S->pos[j];
              const float ex = xj.x - xi.x, ey = xj.y - xi.y, ez = xj.z - xi.z;
              const float rr = (ex * ex + ey * ey) + ez * ez;
              const float cut = xi.w + xj.w + skin;
              if (!(rr > 1e-10f && rr < cut * cut)) continue;
              if (pass) S->nb[k] = j;
              ++k;
            }
          }
      if (!pass) cnb[i + 1] = k;
    }
    if (!pass) {
      for (uint32_t i = 0; i < n; ++i) cnb[i + 1] += cnb[i];
      memcpy(S->nb_start, cnb, ((size_t)n + 1) * sizeof(uint32_t));
      if (cnb[n] > S->nb_cap) {
        free(S->nb);
        free(S->in_pair);
        free(S->pf);
        S->nb_cap = (size_t)cnb[n] + cnb[n] / 2 + 1024;
        S->nb = malloc(S->nb_cap * sizeof(uint32_t));
        S->in_pair = malloc(S->nb_cap * sizeof(uint32_t));
        S->pf = malloc(3 * S->nb_cap * sizeof(long long));
        if (!S->nb || !S->in_pair || !S->pf) return -1;
      }
    }
  }
  /* transpose: the pairs of each higher index j */
  memset(S->in_start, 0, ((size_t)n + 1) * sizeof(uint32_t));
  for (uint32_t t = 0; t < S->nb_start[n]; ++t) ++S->in_start[S->nb[t] + 1];
  for (uint32_t j = 0; j < n; ++j) S->in_start[j + 1] += S->in_start[j];
  {
    uint32_t* cur = malloc(((size_t)n + 1) * sizeof(uint32_t));
    if (!cur) return -1;
    memcpy(cur, S->in_start, ((size_t)n + 1) * sizeof(uint32_t));
    for (uint32_t i = 0; i < n; ++i)
      for (uint32_t t = S->nb_start[i]; t < S->nb_start[i + 1]; ++t) S->in_pair[cur[S->nb[t]]++] = t;
    free(cur);
  }
  memcpy(S->ref, S->pos, (size_t)n * sizeof(f4));
  free(cnt);
  free(cell);
  free(list);
  free(cnb);
  ++S->rebuilds;
  return 0;
}

/* k_soft_pairs: linear overlap springs fm = -D (a - r) / r on the pair vector
 * from the lower to the higher index, a = scale (r_i + r_j), summed in fixed
 * point (the higher index receives the negated contribution: rounding to
 * fixed point is symmetric); the largest relative overlap (a - r) / a of the
 * step. */
static float soft_pairs(packer_t* S) {
  const uint32_t n = S->n;
  float worst = 0.f;
#pragma omp parallel for schedule(static) reduction(max : worst)
  for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
    const uint32_t i = (uint32_t)ii;
    const f4 xi = S->pos[i];
    long long acc[3] = {0, 0, 0};
    for (uint32_t t = S->nb_start[i]; t < S->nb_start[i + 1]; ++t) {
      const uint32_t j = S->nb[t];
      const f4 xj = S->pos[j];
      long long* pf = S->pf + 3 * (size_t)t;
      pf[0] = pf[1] = pf[2] = 0;
      const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
      const float rr = (dx * dx + dy * dy) + dz * dz;
      const float a = S->scale * (xi.w + xj.w);
      const float aa = a * a;
      if (!(rr < aa) || !(rr > 0.f)) continue;
      const float r = sqrtf(rr);
      const float fm = -S->D * (a - r) / r;
      pf[0] = to_fix(fm * dx);
      pf[1] = to_fix(fm * dy);
      pf[2] = to_fix(fm * dz);
      acc[0] += pf[0];
      acc[1] += pf[1];
      acc[2] += pf[2];
      const float ov = (a - sqrtf(rr)) / a;
      if (ov > worst) worst = ov;
    }
    S->q[3 * (size_t)i] += acc[0];
    S->q[3 * (size_t)i + 1] += acc[1];
    S->q[3 * (size_t)i + 2] += acc[2];
  }
#pragma omp parallel for schedule(static)
  for (int64_t jj = 0; jj < (int64_t)n; ++jj) {
    const uint32_t j = (uint32_t)jj;
    long long acc[3] = {0, 0, 0};
    for (uint32_t t = S->in_start[j]; t < S->in_start[j + 1]; ++t) {
      const long long* pf = S->pf + 3 * (size_t)S->in_pair[t];
      acc[0] -= pf[0];
      acc[1] -= pf[1];
      acc[2] -= pf[2];
    }
    S->q[3 * (size_t)j] += acc[0];
    S->q[3 * (size_t)j + 1] += acc[1];
    S->q[3 * (size_t)j + 2] += acc[2];
  }
  return worst;
}

/* k_fire_power: pair force out of fixed point, spring walls, F.v, and (FIRE
 * steps) the dt / alpha adaptation of md_createcylindersample.cu:374-397. */
static void fire_power(packer_t* S, int viscous) {
  const uint32_t n = S->n;
  const float* c = S->cyl;
  const float D = S->D;
  double pw = 0.0;
  float worst = 0.f;
#pragma omp parallel for schedule(static) reduction(+ : pw) reduction(max : worst)
  for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
    const uint32_t p = (uint32_t)ii;
    const f4 x = S->pos[p], v = S->vel[p];
    long long* q = S->q + 3 * (size_t)p;
    float f[3] = {(float)((double)q[0] * kFixInv), (float)((double)q[1] * kFixInv), (float)((double)q[2] * kFixInv)};
    q[0] = q[1] = q[2] = 0;
    const float r = S->scale * x.w;
    const float R0 = c[3] - r, H0 = c[4] - r;
    const float dx = x.x - c[0], dy = x.y - c[1], dz = x.z - c[2];
    const float rr = dx * dx + dy * dy;
    float pen = 0.f;
    if (rr > R0 * R0) {
      const float rho = sqrtf(rr);
      pen = rho - R0;
      const float qq = -D * pen / rho;
      f[0] += qq * dx;
      f[1] += qq * dy;
    }
    if (dz > H0) {
      f[2] -= D * (dz - H0);
      pen = fmaxf(pen, dz - H0);
    }
    if (dz < -H0) {
      f[2] += D * (-H0 - dz);
      pen = fmaxf(pen, -H0 - dz);
    }
    S->frc[3 * (size_t)p] = f[0];
    S->frc[3 * (size_t)p + 1] = f[1];
    S->frc[3 * (size_t)p + 2] = f[2];
    if (pen > 0.f) {
      const float w = pen / (2.0f * r);
      if (w > worst) worst = w;
    }
    pw += (double)((f[0] * v.x + f[1] * v.y) + f[2] * v.z);
  }
  if (worst > S->F.max_overlap) S->F.max_overlap = worst;
  if (viscous) return;
  fire_t* F = &S->F;
  F->P += pw;
  if (F->P > 0) {
    ++F->Npos;
    F->Nneg = 0;
    if (F->Npos > F->Ndelay) {
      F->dt = (F->dt * F->dtgrow < F->dtmax) ? F->dt * F->dtgrow : F->dtmax;
      F->alpha *= F->alphashrink;
    }
    F->back = 0;
  } else {
    F->Npos = 0;
    ++F->Nneg;
    if (F->step > F->Ndelay) {
      F->dt = (F->dt * F->dtshrink > F->dtmin) ? F->dt * F->dtshrink : F->dtmin;
      F->alpha = F->alpha0;
    }
    F->back = 1;
  }
  F->P = 0.0;
  ++F->step;
}

/* k_fire_move: the viscous or FIRE 2.0 move, then the wall put-back; speed
 * and displacement maxima (the reference's FIRE move: fire_move_reference). */
static void fire_move(packer_t* S, int viscous) {
  const uint32_t n = S->n;
  const float* c = S->cyl;
  const fire_t F = S->F;
  float v2max = 0.f, d2max = 0.f;
#pragma omp parallel for schedule(static) reduction(max : v2max, d2max)
  for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
    const uint32_t p = (uint32_t)ii;
    f4 x = S->pos[p], v = S->vel[p];
    const float f[3] = {S->frc[3 * (size_t)p], S->frc[3 * (size_t)p + 1], S->frc[3 * (size_t)p + 2]};
    const float dtm = v.w;
    if (viscous) {
      const float dt = (float)F.dt0;
      v.x += (f[0] - v.x * S->vis) * dtm;
      v.y += (f[1] - v.y * S->vis) * dtm;
      v.z += (f[2] - v.z * S->vis) * dtm;
      x.x += v.x * dt;
      x.y += v.y * dt;
      x.z += v.z * dt;
    } else {
      /* FIRE 2.0 (Guenole et al. 2020): half step back and v = 0 on P <= 0,
       * semi-implicit Euler, velocity mixing */
      const float dt = (float)F.dt, alpha = (float)F.alpha;
      if (F.back) {
        const float h = 0.5f * dt;
        x.x -= v.x * h;
        x.y -= v.y * h;
        x.z -= v.z * h;
        v.x = v.y = v.z = 0.f;
      }
      const float k = dtm * (float)(F.dt / F.dt0);
      v.x += f[0] * k;
      v.y += f[1] * k;
      v.z += f[2] * k;
      const float ff = (f[0] * f[0] + f[1] * f[1]) + f[2] * f[2];
      if (ff > 0.f) {
        const float vn = sqrtf((v.x * v.x + v.y * v.y) + v.z * v.z);
        const float cc = alpha * vn * orc_rsqrt_rn_f(ff);
        v.x = (1.0f - alpha) * v.x + cc * f[0];
        v.y = (1.0f - alpha) * v.y + cc * f[1];
        v.z = (1.0f - alpha) * v.z + cc * f[2];
      }
      x.x += v.x * dt;
      x.y += v.y * dt;
      x.z += v.z * dt;
    }
    const float R1 = c[3], H1 = c[4];
    const float dx = x.x - c[0], dy = x.y - c[1], dz = x.z - c[2];
    const float rr = dx * dx + dy * dy;
    if (rr > R1 * R1) {
      const float rinv = orc_rsqrt_rn_f(rr);
      const float qq = R1 * rinv - 1.0f;
      x.x += dx * qq;
      x.y += dy * qq;
      const float vn = (v.x * dx + v.y * dy) * rinv;
      if (vn > 0.f) {
        v.x -= vn * dx * rinv;
        v.y -= vn * dy * rinv;
      }
    }
    if (dz > H1) {
      x.z += H1 - dz;
      if (v.z > 0.f) v.z = 0.f;
    }
    if (dz < -H1) {
      x.z += -H1 - dz;
      if (v.z < 0.f) v.z = 0.f;
    }
    S->pos[p] = x;
    S->vel[p] = v;
    const f4 r0 = S->ref[p];
    const float ex = x.x - r0.x, ey = x.y - r0.y, ez = x.z - r0.z;
    const float a = (v.x * v.x + v.y * v.y) + v.z * v.z, b = (ex * ex + ey * ey) + ez * ez;
    if (a > v2max) v2max = a;
    if (b > d2max) d2max = b;
  }
  if (v2max > S->F.vmax2) S->F.vmax2 = v2max;
  if (d2max > S->F.dmax2) S->F.dmax2 = d2max;
}

/* The reference's FIRE move (fire_variant 1) through the oracle's own
 * restatements of its kernels: d_CalculateDecrementsHalfStepFIRE
 * (orc_fire_half_step_back, md_firerelaxation.cu:58-70) when the power was
 * not positive, then d_CalculateIncrementsFIRE (orc_fire_increments,
 * md_firerelaxation.cu:18-56) with the per-sphere dt0/m; then the engine's
 * wall put-back as in fire_move.  The GPU packer's variant 1 must match this
 * bit for bit. */
static void fire_move_reference(packer_t* S) {
  const uint32_t n = S->n;
  float* R = malloc(3 * (size_t)n * sizeof(float));
  float* V = malloc(3 * (size_t)n * sizeof(float));
  float* Fs = malloc(3 * (size_t)n * sizeof(float));
  float* am = malloc((size_t)n * sizeof(float));
  for (uint32_t p = 0; p < n; ++p) {
    R[p] = S->pos[p].x;
    R[n + p] = S->pos[p].y;
    R[2 * (size_t)n + p] = S->pos[p].z;
    V[p] = S->vel[p].x;
    V[n + p] = S->vel[p].y;
    V[2 * (size_t)n + p] = S->vel[p].z;
    for (int d = 0; d < 3; ++d) Fs[(size_t)d * n + p] = S->frc[3 * (size_t)p + d];
    am[p] = S->vel[p].w;
  }
  const float dt = (float)S->F.dt, alpha = (float)S->F.alpha;
  if (S->F.back) orc_fire_half_step_back_f(V, R, n, 0.5f * dt);
  orc_fire_increments_f(Fs, V, R, n, 0.f, dt, alpha, am);
  const float* c = S->cyl;
  float v2max = 0.f, d2max = 0.f;
  for (uint32_t p = 0; p < n; ++p) {
    f4 x = {R[p], R[n + p], R[2 * (size_t)n + p], S->pos[p].w};
    f4 v = {V[p], V[n + p], V[2 * (size_t)n + p], S->vel[p].w};
    const float R1 = c[3], H1 = c[4];
    const float dx = x.x - c[0], dy = x.y - c[1], dz = x.z - c[2];
    const float rr = dx * dx + dy * dy;
    if (rr > R1 * R1) {
      const float rinv = orc_rsqrt_rn_f(rr);
      const float qq = R1 * rinv - 1.0f;
      x.x += dx * qq;
      x.y += dy * qq;
      const float vn = (v.x * dx + v.y * dy) * rinv;
      if (vn > 0.f) {
        v.x -= vn * dx * rinv;
        v.y -= vn * dy * rinv;
      }
    }
    if (dz > H1) {
      x.z += H1 - dz;
      if (v.z > 0.f) v.z = 0.f;
    }
    if (dz < -H1) {
      x.z += -H1 - dz;
      if (v.z < 0.f) v.z = 0.f;
    }
    S->pos[p] = x;
    S->vel[p] = v;
    const f4 r0 = S->ref[p];
    const float ex = x.x - r0.x, ey = x.y - r0.y, ez = x.z - r0.z;
    const float a = (v.x * v.x + v.y * v.y) + v.z * v.z, b = (ex * ex + ey * ey) + ez * ez;
    if (a > v2max) v2max = a;
    if (b > d2max) d2max = b;
  }
  if (v2max > S->F.vmax2) S->F.vmax2 = v2max;
  if (d2max > S->F.dmax2) S->F.dmax2 = d2max;
  free(R);
  free(V);
  free(Fs);
  free(am);
}

static void step(packer_t* S, int viscous) {
  const float w = soft_pairs(S);
  if (w > S->F.max_overlap) S->F.max_overlap = w;
  fire_power(S, viscous);
  if (!viscous && S->F.variant == 1)
    fire_move_reference(S);
  else
    fire_move(S, viscous);
}

/* Relaxation loop with the GPU's list and chunk schedule (Packer::relax). */
static int relax(packer_t* S, int viscous, uint32_t max_steps, double tol, uint64_t* steps, double* trace,
                 uint32_t trace_cap, uint32_t* ntrace) {
  const double quarter = 0.25 * S->skin;
  const uint32_t kMaxChunk = 50;
  uint32_t done = 0;
  int need_build = 1;
  double vmax = 0.0, dmax = 0.0;
  while (done < max_steps) {
    if (need_build || dmax > quarter) {
      if (rebuild(S)) return -1;
      dmax = 0.0;
      need_build = 0;
    }
    const double dt_bound = viscous ? S->F.dt0 : S->F.dtmax;
    uint32_t m;
    if (vmax > 0.0) {
      const double k = 0.5 * (quarter - dmax) / (vmax * dt_bound);
      double mm = floor(k);
      if (mm > (double)kMaxChunk) mm = kMaxChunk;
      if (!(mm >= 1.0)) mm = 1.0;
      m = (uint32_t)mm;
    } else {
      m = 10 < kMaxChunk ? 10 : kMaxChunk;
    }
    if (m > max_steps - done) m = max_steps - done;
    S->F.vmax2 = 0.f;
    for (uint32_t k = 0; k < m; ++k) {
      if (k == m - 1) {
        S->F.max_overlap = 0.f;
        S->F.dmax2 = 0.f;
      }
      step(S, viscous);
      if (!viscous && trace && *ntrace < trace_cap) {
        trace[3 * *ntrace] = S->F.dt;
        trace[3 * *ntrace + 1] = S->F.alpha;
        trace[3 * *ntrace + 2] = S->F.back;
        ++*ntrace;
      }
    }
    S->last_overlap = S->F.max_overlap;
    vmax = sqrt((double)S->F.vmax2);
    dmax = sqrt((double)S->F.dmax2);
    done += m;
    *steps += m;
    if (tol > 0 && S->F.max_overlap < tol) break;
  }
  return 0;
}

int orc_pack_cylinder(const orc_pack_params* P, float* xyz, float* radii, uint32_t cap, uint32_t* n_out,
                      orc_pack_report* rep, double* fire_trace, uint32_t trace_cap, uint32_t* ntrace) {
  const uint32_t n = P->n;
  if (n == 0 || n > cap || !(P->r_max >= P->r_min) || !(P->r_min > 0) || !(P->radius > P->r_max) ||
      !(P->half_height > P->r_max) || P->max_removed)
    return -1;
  packer_t S;
  memset(&S, 0, sizeof S);
  S.p = *P;
  S.n = n;
  S.pos = malloc((size_t)n * sizeof(f4));
  S.vel = malloc((size_t)n * sizeof(f4));
  S.ref = malloc((size_t)n * sizeof(f4));
  S.frc = calloc(3 * (size_t)n, sizeof(float));
  S.q = calloc(3 * (size_t)n, sizeof(long long));
  S.nb_start = calloc((size_t)n + 1, sizeof(uint32_t));
  S.in_start = calloc((size_t)n + 1, sizeof(uint32_t));
  if (!S.pos || !S.vel || !S.ref || !S.frc || !S.q || !S.nb_start || !S.in_start) return -2;
  /* fill: radii uniform in [r_min, r_max], centres uniform in the cylinder shrunk by r */
  uint64_t rs = P->seed ^ 0x5DEECE66Dull;
  const double rho = P->rho > 0 ? P->rho : 2.65;
  const double dt0 = 0.05 * rayleigh(P->r_min, rho, P->E, P->nu);
  for (uint32_t i = 0; i < n; ++i) {
    const double r = P->r_min + (P->r_max - P->r_min) * rng_uniform(&rs);
    double x, y;
    do {
      x = 2 * rng_uniform(&rs) - 1;
      y = 2 * rng_uniform(&rs) - 1;
    } while (x * x + y * y > 1.0);
    const double Rin = P->radius - r, Hin = P->half_height - r;
    const double z = (2 * rng_uniform(&rs) - 1) * Hin;
    S.pos[i].x = (float)(P->center[0] + x * Rin);
    S.pos[i].y = (float)(P->center[1] + y * Rin);
    S.pos[i].z = (float)(P->center[2] + z);
    S.pos[i].w = (float)r;
    S.vel[i].x = S.vel[i].y = S.vel[i].z = 0.f;
    S.vel[i].w = (float)dt_over_m(r, rho, dt0);
  }
  S.skin = 0.5 * P->r_min;
  S.cyl[0] = (float)P->center[0];
  S.cyl[1] = (float)P->center[1];
  S.cyl[2] = (float)P->center[2];
  S.cyl[3] = (float)P->radius;
  S.cyl[4] = (float)P->half_height;
  const double k = P->E * 0.5 * (P->r_min + P->r_max);
  S.D = (float)k;
  fire_t* F = &S.F;
  F->dt0 = dt0;
  F->dt = dt0;
  F->dtgrow = 1.1;
  F->dtshrink = 0.5;
  F->alphashrink = 0.99;
  F->Ndelay = 20;
  F->variant = P->fire_variant == 1 ? 1u : 0u;
  if (F->variant == 1) {
    F->dtmax = 100.0 * dt0; /* SetFIREData, md_firerelaxation.cu:74-86 */
    F->dtmin = 0.001 * dt0;
    F->alpha0 = 0.1;
  } else {
    F->dtmax = 4.0 * dt0;
    F->dtmin = 0.02 * dt0;
    F->alpha0 = 0.25;
  }
  F->alpha = F->alpha0;
  const uint32_t stages = P->growth_stages > 0 ? P->growth_stages : 1;
  const double s0 = cbrt(0.3);
  const double m_mean = rho * 4.0 / 3.0 * kPi * pow(0.5 * (P->r_min + P->r_max), 3);
  S.vis = (float)(2.0 * sqrt(k * m_mean) * 0.5);
  uint64_t steps = 0;
  if (ntrace) *ntrace = 0;
  int rc = 0;
  for (uint32_t sg = 1; sg <= stages && !rc; ++sg) {
    S.scale = (float)(s0 + (1.0 - s0) * sg / stages);
    rc = relax(&S, 1, P->steps_per_stage, 0.0, &steps, NULL, 0, ntrace);
  }
  if (!rc) {
    S.scale = 1.0f;
    rc = relax(&S, 0, P->max_fire_steps, P->overlap_tol, &steps, fire_trace, trace_cap, ntrace);
  }
  if (!rc) {
    for (uint32_t i = 0; i < n; ++i) {
      xyz[i] = S.pos[i].x;
      xyz[n + i] = S.pos[i].y;
      xyz[2 * (size_t)n + i] = S.pos[i].z;
      if (radii) radii[i] = S.pos[i].w;
    }
    *n_out = n;
    if (rep) {
      memset(rep, 0, sizeof *rep);
      rep->steps = steps;
      rep->max_overlap = S.last_overlap;
      double vs = 0;
      for (uint32_t i = 0; i < n; ++i) vs += 4.0 / 3.0 * kPi * pow((double)S.pos[i].w, 3);
      rep->packing_fraction = vs / (kPi * P->radius * P->radius * 2.0 * P->half_height);
      rep->rebuilds = S.rebuilds;
      rep->removed = 0;
    }
  }
  free(S.pos);
  free(S.vel);
  free(S.ref);
  free(S.frc);
  free(S.q);
  free(S.nb_start);
  free(S.nb);
  free(S.in_start);
  free(S.in_pair);
  free(S.pf);
  return rc ? -2 : 0;
}
