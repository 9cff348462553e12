// C ABI of the B200 DEM engine (declarations and reference mapping in
// include/b200dem.h).  No exception crosses this boundary.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <new>
#include <string>
#include <vector>

#include "b200dem.h"
#include "dem_engine.h"

struct dem_ctx {
  dem::EngineBase* e = nullptr;
};

#define GUARD(...)                    \
  try {                               \
    __VA_ARGS__                       \
  } catch (const std::bad_alloc&) {   \
    return DEM_ERR_NOMEM;             \
  } catch (...) {                     \
    return DEM_ERR_STATE;             \
  }

extern "C" {

const char* dem_strerror(int code) {
  switch (code) {
    case DEM_OK: return "ok";
    case DEM_ERR_ARG: return "invalid argument";
    case DEM_ERR_CUDA: return "CUDA error";
    case DEM_ERR_STATE: return "call not valid in the current state";
    case DEM_ERR_CAPACITY: return "capacity exceeded (too many neighbours or pairs)";
    case DEM_ERR_STALE: return "a particle moved further than the contact-list skin between rebuilds";
    case DEM_ERR_IO: return "file error";
    case DEM_ERR_NOMEM: return "out of host memory";
    case DEM_ERR_NUMERIC: return "non-finite state";
    case DEM_ERR_TIMEOUT: return "timed out";
    default: return "unknown error";
  }
}

const char* dem_last_error_detail(void) { return dem::last_error_detail(); }

int dem_reference_space(const double space_si[3], const double lsi_si[3], double p_r, double farcut, dem_loading* out) {
  if (!space_si || !lsi_si || !out || !(p_r > 0) || !(farcut > 0)) return DEM_ERR_ARG;
  // sample_data::SetSpaceSizeSi / SetLSi / CalculateParameters (md_data_types.h:87-123):
  // float members, cell edge C.a = 2 a_farcut; the escape box does not depend on LSi
  const float Ca = (float)(2.0 * farcut * p_r);
  float size[3], half[3], A[3], Bv[3];
  for (int d = 0; d < 3; ++d) {
    size[d] = (float)(space_si[d] / 1e-3);
    half[d] = (float)(0.5 * (double)size[d]);
    A[d] = (float)(1.01 * (double)Ca);
    Bv[d] = A[d] + size[d];
    out->space_center[d] = (float)(0.5 * (double)(float)(A[d] + Bv[d]));
    out->space_half[d] = half[d];
  }
  out->hidden_point[0] = (float)((double)A[0] + 0.5 * (double)size[0]);
  out->hidden_point[1] = (float)((double)A[1] + 0.5 * (double)size[1]);
  out->hidden_point[2] = (float)(((double)(float)std::floor((float)((double)Bv[2] / (double)Ca)) + 3 - 0.5) * (double)Ca);
  out->zcut = (float)((float)out->space_center[2] + half[2]);
  return DEM_OK;
}

int dem_device_count(int* n) {
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) c = 0;
  if (n) *n = c;
  return DEM_OK;
}

int dem_create(const dem_options* opt, dem_ctx** out) {
  if (!out) return DEM_ERR_ARG;
  GUARD({
    dem_options o{};
    if (opt) o = *opt;
    if (o.precision < 0 || o.precision > 2) return DEM_ERR_ARG;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0 || o.device < 0 || o.device >= n) return DEM_ERR_CUDA;
    int err = DEM_OK;
    dem::EngineBase* e = dem::make_engine(o, &err);
    if (!e) return err ? err : DEM_ERR_CUDA;
    dem_ctx* c = new dem_ctx;
    c->e = e;
    *out = c;
    return DEM_OK;
  })
}

void dem_destroy(dem_ctx* ctx) {
  if (!ctx) return;
  delete ctx->e;
  delete ctx;
}

int dem_release_cached_memory(void) { GUARD(return dem::release_cached_memory();) }

#define CTX_CALL(expr)                          \
  do {                                          \
    if (!ctx || !ctx->e) return DEM_ERR_ARG;    \
    GUARD(return (expr);)                       \
  } while (0)

int dem_add_sample(dem_ctx* ctx, const dem_material* mat, const dem_loading* load, const float* xyz,
                   const float* radii, uint32_t n, int32_t* sample) {
  CTX_CALL(ctx->e->add_sample(mat, load, xyz, radii, n, sample));
}
int dem_setup(dem_ctx* ctx) { CTX_CALL(ctx->e->setup()); }
int dem_run(dem_ctx* ctx, uint64_t max_steps, uint64_t* steps_done) {
  CTX_CALL(ctx->e->run_until_done(max_steps, steps_done));
}
int dem_step(dem_ctx* ctx, uint32_t nsteps) { CTX_CALL(ctx->e->step(nsteps)); }
int dem_step_stages(dem_ctx* ctx, int stages) { CTX_CALL(ctx->e->step_stages(stages)); }
int dem_sync(dem_ctx* ctx) { CTX_CALL(ctx->e->sync()); }
int dem_counts(dem_ctx* ctx, uint32_t* p, uint32_t* b, uint32_t* c, uint32_t* s) {
  CTX_CALL(ctx->e->counts(p, b, c, s));
}
int dem_sample_result(dem_ctx* ctx, int32_t sample, dem_result* out) { CTX_CALL(ctx->e->result(sample, out)); }
int dem_get_record(dem_ctx* ctx, int32_t sample, double* rec, uint32_t* bonds, uint32_t cap, uint32_t* n) {
  CTX_CALL(ctx->e->get_record(sample, rec, bonds, cap, n));
}
int dem_save_lammps_data(dem_ctx* ctx, int32_t sample, const char* path, int with_energy) {
  CTX_CALL(ctx->e->save_lammps(sample, path, with_energy));
}
int dem_sensitivities(dem_ctx* ctx, int32_t sample, dem_sensitivity* out) {
  CTX_CALL(ctx->e->sensitivities(sample, out));
}
int dem_get_lateral_record(dem_ctx* ctx, int32_t sample, double* lat, uint32_t cap, uint32_t* n) {
  CTX_CALL(ctx->e->get_lateral_record(sample, lat, cap, n));
}
int dem_get_particles(dem_ctx* ctx, int32_t s, float* R, float* V, float* W, float* F, float* M, float* O) {
  CTX_CALL(ctx->e->get_particles(s, R, V, W, F, M, O));
}
int dem_get_particles_d(dem_ctx* ctx, int32_t s, double* R, double* V, double* W, double* F, double* M, double* O) {
  CTX_CALL(ctx->e->get_particles_d(s, R, V, W, F, M, O));
}
int dem_set_particles(dem_ctx* ctx, int32_t s, const float* R, const float* V, const float* W, const float* O) {
  CTX_CALL(ctx->e->set_particles(s, R, V, W, O));
}
int dem_get_pairs(dem_ctx* ctx, int32_t s, uint32_t cap, uint32_t* i, uint32_t* j, uint32_t* kind, float* st,
                  uint32_t* n) {
  CTX_CALL(ctx->e->get_pairs(s, cap, i, j, kind, st, n));
}
int dem_get_pairs_d(dem_ctx* ctx, int32_t s, uint32_t cap, uint32_t* i, uint32_t* j, uint32_t* kind, double* st,
                    uint32_t* n) {
  CTX_CALL(ctx->e->get_pairs_d(s, cap, i, j, kind, st, n));
}
int dem_set_pairs(dem_ctx* ctx, int32_t s, uint32_t n, const uint32_t* i, const uint32_t* j, const uint32_t* kind,
                  const float* st) {
  CTX_CALL(ctx->e->set_pairs(s, n, i, j, kind, st));
}
int dem_set_platens(dem_ctx* ctx, int32_t s, double top, double bottom, double v) {
  CTX_CALL(ctx->e->set_platens(s, top, bottom, v));
}
int dem_rebuild_contacts(dem_ctx* ctx) { CTX_CALL(ctx->e->rebuild_contacts()); }
int dem_run_timed(dem_ctx* ctx, uint64_t nsteps, double* ms) { CTX_CALL(ctx->e->run_timed(nsteps, ms)); }
int dem_profile(dem_ctx* ctx, uint32_t nsteps, double* pair_ms, double* particle_ms, double* touching) {
  CTX_CALL(ctx->e->profile(nsteps, pair_ms, particle_ms, touching));
}
int dem_autotune(dem_ctx* ctx, uint32_t steps, dem_tune_report* report) {
  CTX_CALL(ctx->e->autotune(steps, report));
}

int dem_ref_cells(const float* xyz, uint32_t n, float a, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t* CI,
                  uint32_t* CIs, uint32_t* pnC) {
  if (!xyz || n == 0 || !(a > 0) || !nx || !ny || !nz) return DEM_ERR_ARG;
  GUARD(return dem::ref_cells(xyz, n, a, nx, ny, nz, CI, CIs, pnC);)
}

int dem_ref_neighbor_sets(const float* xyz, uint32_t n, float a, uint32_t nx, uint32_t ny, uint32_t nz,
                          float add_thr, float del_thr, uint32_t cap, uint32_t* sets, uint32_t* overflow) {
  if (!xyz || n == 0 || !(a > 0) || !sets || cap == 0 || cap > 48) return DEM_ERR_ARG;
  GUARD(return dem::ref_neighbor_sets(xyz, n, a, nx, ny, nz, add_thr, del_thr, cap, sets, overflow);)
}

int dem_calculation_test(const dem_options* opt, const dem_material* mat, const dem_loading* load, const float* h_R,
                         const float* radii, uint32_t n, dem_result* out, double* rec, uint32_t* rec_bonds,
                         uint32_t rec_cap, uint32_t* rec_n) {
  if (!mat || !load || !h_R || n == 0 || load->test == DEM_TEST_NONE) return DEM_ERR_ARG;
  dem_ctx* ctx = nullptr;
  int rc = dem_create(opt, &ctx);
  if (rc) return rc;
  int32_t sid = 0;
  rc = dem_add_sample(ctx, mat, load, h_R, radii, n, &sid);
  if (!rc) rc = dem_setup(ctx);
  uint64_t steps = 0;
  if (!rc) rc = dem_run(ctx, load->max_steps ? load->max_steps : ~0ull, &steps);
  if (!rc || rc == DEM_ERR_STALE || rc == DEM_ERR_NUMERIC) {
    int rc2 = out ? dem_sample_result(ctx, sid, out) : DEM_OK;
    if (!rc2 && (rec || rec_bonds)) rc2 = dem_get_record(ctx, sid, rec, rec_bonds, rec_cap, rec_n);
    if (!rc) rc = rc2;
  }
  dem_destroy(ctx);
  return rc;
}

int dem_load_cylinder_sample(const char* path, double p_r, float* xyz, uint32_t cap, uint32_t* n, double size_real[3],
                             double center_real[3]) {
  if (!path || !n) return DEM_ERR_ARG;
  GUARD({
    std::ifstream f(path);
    if (!f) return DEM_ERR_IO;
    long long m = 0;
    if (!(f >> m) || m < 0) return DEM_ERR_IO;
    *n = (uint32_t)m;
    if (!xyz) return DEM_OK;
    if ((uint64_t)m > cap) return DEM_ERR_CAPACITY;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (long long i = 0; i < m; ++i) {
      double x, y, z;
      if (!(f >> x >> y >> z)) return DEM_ERR_IO;
      if (!std::isfinite(x) || !std::isfinite(y) || !std::isfinite(z)) return DEM_ERR_IO;
      xyz[i] = (float)(x * (1.0 / 1e-3));
      xyz[m + i] = (float)(y * (1.0 / 1e-3));
      xyz[2 * m + i] = (float)(z * (1.0 / 1e-3));
      const float v[3] = {xyz[i], xyz[m + i], xyz[2 * m + i]};
      for (int d = 0; d < 3; ++d) {
        lo[d] = std::fmin(lo[d], (double)v[d]);
        hi[d] = std::fmax(hi[d], (double)v[d]);
      }
    }
    for (int d = 0; d < 3; ++d) {
      if (size_real) size_real[d] = hi[d] - lo[d] + 2.0 * p_r;
      if (center_real) center_real[d] = 0.5 * (hi[d] + lo[d]);
    }
    return DEM_OK;
  })
}

int dem_save_cylinder_sample(const char* path, const float* xyz, uint32_t n, const double hidden_point[3]) {
  if (!path || !xyz) return DEM_ERR_ARG;
  GUARD({
    std::ofstream f(path);
    if (!f) return DEM_ERR_IO;
    auto hidden = [&](uint32_t i) {
      if (!hidden_point) return false;
      const double d0 = xyz[i] - hidden_point[0], d1 = xyz[n + i] - hidden_point[1], d2 = xyz[2 * n + i] - hidden_point[2];
      return d0 * d0 + d1 * d1 + d2 * d2 < 1e-10;
    };
    uint32_t keep = 0;
    for (uint32_t i = 0; i < n; ++i) keep += hidden(i) ? 0 : 1;
    f << keep << "\n";
    f.precision(9);
    for (uint32_t i = 0; i < n; ++i) {
      if (hidden(i)) continue;
      f << xyz[i] * 1e-3 << " " << xyz[n + i] * 1e-3 << " " << xyz[2 * n + i] * 1e-3 << "\n";
    }
    return f ? DEM_OK : DEM_ERR_IO;
  })
}

int dem_save_sum_forces_loading(const char* path, const double* rec, uint32_t n) {
  if (!path || (!rec && n)) return DEM_ERR_ARG;
  GUARD({
    std::ofstream f(path);
    if (!f) return DEM_ERR_IO;
    f << "EpsZ StressZ_bottom StressZ_top\n";
    for (uint32_t i = 0; i < n; ++i)
      f << rec[3 * i] << " " << rec[3 * i + 1] * 1e9 << " " << rec[3 * i + 2] * 1e9 << "\n";
    return f ? DEM_OK : DEM_ERR_IO;
  })
}

}  // extern "C"
