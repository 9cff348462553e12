// Engine interface behind the C ABI (include/b200dem.h); one implementation
// per precision (dem_engine.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "b200dem.h"

namespace dem {

// Thread-local text of the last CUDA error seen by the library (name, message,
// source location), for dem_last_error_detail.
void note_cuda_error(cudaError_t e, const char* file, int line);
const char* last_error_detail();


class EngineBase {
 public:
  virtual ~EngineBase() = default;
  virtual int precision() const = 0;
  virtual int add_sample(const dem_material* mat, const dem_loading* load, const float* xyz, const float* radii,
                         uint32_t n, int32_t* id) = 0;
  virtual int setup() = 0;
  virtual int run_until_done(uint64_t max_steps, uint64_t* done) = 0;
  virtual int step(uint32_t n) = 0;
  virtual int step_stages(int stages) = 0;
  virtual int sync() = 0;
  virtual int counts(uint32_t* p, uint32_t* b, uint32_t* c, uint32_t* s) = 0;
  virtual int result(int32_t sample, dem_result* out) = 0;
  virtual int get_record(int32_t sample, double* rec, uint32_t* bonds, uint32_t cap, uint32_t* n) = 0;
  virtual int get_lateral_record(int32_t sample, double* lat, uint32_t cap, uint32_t* n) = 0;
  virtual int sensitivities(int32_t sample, dem_sensitivity* out) = 0;
  virtual int save_lammps(int32_t sample, const char* path, int with_energy) = 0;
  virtual int get_particles(int32_t s, float* R, float* V, float* W, float* F, float* M, float* O) = 0;
  virtual int get_particles_d(int32_t s, double* R, double* V, double* W, double* F, double* M, double* O) = 0;
  virtual int set_particles(int32_t s, const float* R, const float* V, const float* W, const float* O) = 0;
  virtual int get_pairs(int32_t s, uint32_t cap, uint32_t* i, uint32_t* j, uint32_t* kind, float* st,
                        uint32_t* n) = 0;
  virtual int get_pairs_d(int32_t s, uint32_t cap, uint32_t* i, uint32_t* j, uint32_t* kind, double* st,
                        uint32_t* n) = 0;
  virtual int set_pairs(int32_t s, uint32_t n, const uint32_t* i, const uint32_t* j, const uint32_t* kind,
                        const float* st) = 0;
  virtual int set_platens(int32_t s, double top, double bottom, double v) = 0;
  virtual int rebuild_contacts() = 0;
  virtual cudaError_t last_cuda() const = 0;
  virtual uint64_t rebuilds() const = 0;
  virtual uint32_t num_sms() const = 0;
  virtual void launch_raw(int stages) = 0;
  virtual void* stream() = 0;
  // nsteps steps replayed from the step graph, timed with CUDA events on the engine stream
  virtual int run_timed(uint64_t nsteps, double* ms) = 0;
  // nsteps steps launched one by one with events around each kernel: average
  // per-launch durations and the mean number of touching contacts per step
  virtual int profile(uint32_t nsteps, double* pair_ms, double* particle_ms, double* touching) = 0;
  virtual int autotune(uint32_t steps, dem_tune_report* rep) = 0;
};

EngineBase* make_engine(const dem_options& o, int* err);
// device blocks kept for reuse after their contexts closed go back to the driver
int release_cached_memory();
int ref_cells(const float* xyz, uint32_t n, float a, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t* CI,
              uint32_t* CIs, uint32_t* pnC);
int ref_neighbor_sets(const float* xyz, uint32_t n, float a, uint32_t nx, uint32_t ny, uint32_t nz, float add_thr,
                      float del_thr, uint32_t cap, uint32_t* sets, uint32_t* overflow);

}  // namespace dem
