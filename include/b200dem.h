/*
 * b200dem: C ABI of the B200-native bonded-particle DEM step for rock
 * calibration (uniaxial compression and Brazilian tests).
 *
 * Units are the reference's (md_phys_constants.h:5-14): length mm, mass mg,
 * time us, so stresses are in GPa, forces in kN, velocities in mm/us.
 * Positions are SoA: x[0..n) y[n..2n) z[2n..3n), as the reference's h_R.
 *
 * Every function returns 0 or a negative DEM_ERR_* code (dem_strerror names
 * it); no exception crosses the ABI.  A context owns all its device memory
 * and one CUDA stream; a context is not thread-safe.
 *
 * Entry points and the reference interfaces they replace:
 *   dem_calculation_test      h_CalculationUniaxialCompression(md_task_data&, float* h_R)
 *                             md_calculationuniaxialcompression.cu:126-340 and
 *                             h_CalculationBrazilTest(md_task_data&, float* h_R)
 *                             md_calculationbraziltest.cu:116-265 (declared mp.h:21-22)
 *   dem_create_cylinder_sample  h_CreateCylinderSample(mp_mdparameters_data&, md_task_data&, uint, char[])
 *                             md_createcylindersample.cu:184-439 (mp.h:16)
 *   dem_load_cylinder_sample  h_LoadCylinderSample(mp_mdparameters_data&, uint, char[])
 *                             md_createcylindersample.cu:441-466 (mp.h:17)
 *   dem_save_sum_forces_loading  SaveSumForcesLoading(result_data&, char*) md_results.cu:168-180
 *   dem_create/dem_add_sample/dem_setup/dem_run/dem_step and the getters expose the
 *   same step pipeline at finer grain (set-up, stepping, state export), which the
 *   reference keeps inside its drivers (md_calculationuniaxialcompression.cu:143-324).
 *   dem_ref_cells / dem_ref_neighbor_sets reproduce CellDistribution
 *   (md_cell_distribution.cu:130-172) and the interaction sets of
 *   InteractionListConstruct/ReConstructBPM (md_interaction_list_construction.cu:382-404)
 *   for parity checks.
 */
#ifndef B200DEM_H
#define B200DEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DEM_OK 0
#define DEM_ERR_ARG (-1)
#define DEM_ERR_CUDA (-2)
#define DEM_ERR_STATE (-3)
#define DEM_ERR_CAPACITY (-4)
#define DEM_ERR_STALE (-5)
#define DEM_ERR_IO (-6)
#define DEM_ERR_NOMEM (-7)
#define DEM_ERR_NUMERIC (-8)
#define DEM_ERR_TIMEOUT (-9)

#define DEM_TEST_NONE 0
#define DEM_TEST_UNIAXIAL 1
#define DEM_TEST_BRAZIL 2

#define DEM_EMPTY 0xFFFFFFFFu

typedef struct dem_ctx dem_ctx;

typedef struct {
  int precision;          /* 0: FP32, 1: FP64, 2: FP64 with tangents (dem_sensitivities) */
  int device;             /* CUDA device ordinal */
  uint32_t pair_block;    /* ignored: set from pair_min_blocks (256 threads, 128 for 5..8) */
  uint32_t pair_grid;     /* blocks of the pair kernel (0: all co-resident blocks) */
  uint32_t particle_block;/* threads per block of the particle kernel (0: 256) */
  uint32_t graph_steps;   /* steps per captured CUDA graph (0: 100) */
  double skin_factor;     /* contact-list skin as a multiple of the smallest radius (0: 0.1) */
  uint32_t pair_min_blocks; /* register budget of the pair kernel: blocks per SM it must fit
                               (1..4 of 256 threads, FP32 also 5..8 of 128 threads;
                               0: 7 for FP32, 2 for FP64, 1 for the sensitivity build) */
  uint32_t deterministic; /* 1: FP32 force and platen sums in exact 64-bit fixed point
                             (2^-40 resolution), so a run is bit-reproducible and a
                             sample's results do not depend on the other samples of
                             its context; 0: floating-point atomics (faster) */
} dem_options;

/* Micro-parameters of one specimen.  The first block is the reference's
 * parameter set (SetInitialParameters, mp_determineconjgradient.cu:15-47);
 * the second block holds the extensions (zero keeps the reference rule). */
typedef struct {
  double E;       /* Young modulus of particles and (by default) bonds, GPa */
  double nu;      /* Poisson ratio (reference 0.247) */
  double Ec, Gc;  /* bond normal / shear strength, GPa */
  double b_r;     /* bond radius, mm (<= 0: bond_radius_factor * min(r_i, r_j)) */
  double gap;     /* bond creation gap, mm: bond if r < r_i + r_j + gap */
  double rho;     /* density, mg/mm^3 (reference 2.61) */
  double p_r;     /* particle radius, mm, when no per-particle radii are given */
  double p_e;     /* restitution coefficient (reference 0.6) */
  double mu;      /* sliding friction (reference 0.45) */
  double mur;     /* rolling friction (reference 0.05) */
  double farcut;  /* far cut-off as a multiple of p_r (reference 3.2) */
  /* extensions */
  double E_bond;             /* > 0: bond Young modulus, separate from particle E */
  double kn_ks;              /* > 0: bond normal/shear stiffness ratio (G_bond = E_bond / kn_ks) */
  double Ec_sd, Gc_sd;       /* > 0: per-bond strengths drawn from N(Ec, Ec_sd), N(Gc, Gc_sd) */
  double bond_radius_factor; /* used when b_r <= 0 */
  double dt;                 /* > 0: time step, us (else the reference rule 0.05*min(T_R, T_bond)) */
  double dt_rayleigh_factor; /* > 0: dt = factor * min(Rayleigh time, bond time 2 sqrt(m/k)) of the
                                smallest particle (the reference's rule with this factor for its 0.05) */
  uint64_t seed;             /* per-bond strength draws */
  int nobreak;               /* 1: bonds never break (elastic stage, d_CalculateForcesDEM_22_ncb) */
  int reserved;
} dem_material;

/* Loading set-up of one specimen: the reference's sample_data and
 * compression_data inputs (md_data_types.h:79-124, 203-495). */
typedef struct {
  int test;                  /* DEM_TEST_* */
  int reserved;
  double space_center[3];    /* escape box centre (reference S.center) */
  double space_half[3];      /* escape box half size (reference S.spacesized2) */
  double hidden_point[3];    /* where escaped particles are parked (reference S.hidenpoint) */
  double zcut;               /* platen zone cut (reference S.center.z + S.spacesized2.z) */
  double size_real[3];       /* specimen extent incl. radius (reference S.size_real) */
  double center_real[3];     /* specimen centre (reference S.center_real) */
  double velocity;           /* platen speed VLoad, mm/us (negative compresses) */
  double min_stress;         /* GPa (reference UMinStress/BMinStress) */
  double max_strain;         /* stop strain (reference UMaxStrain/BMaxStrain) */
  double cond_fracture;      /* stop when stress < cond_fracture * peak (reference ConditionFracture) */
  double p_r_platen;         /* radius used by the platen-area formula (0: material p_r or mean radius) */
  uint32_t dNsave;           /* record every dNsave steps (reference dNSaveU/dNSaveB) */
  uint32_t reserved2;
  uint64_t max_steps;        /* safety bound on the loading loop (0: unlimited) */
} dem_loading;

typedef struct {
  double FractureStress;     /* peak stress, GPa */
  double FractureStrain;     /* strain at peak */
  double LinearityDeviation; /* reference CalculateLinearityDeviation (uniaxial) */
  double Destruction;        /* surviving bond fraction (reference CalculateDestruction) */
  double Strain, Stress, dt;
  double platen_top, platen_bottom, platen_velocity;
  uint64_t steps;
  uint32_t stepsave;         /* number of records */
  uint32_t bonds_initial, bonds_now;  /* intact undirected bonds */
  /* stale: events in which a particle moved past half the contact-list skin
   * within a chunk of steps; the specimen then waited, without stepping,
   * until the list was rebuilt, so no step ran on a list that could miss a
   * contact (the count is informative: results do not depend on it) */
  int fracture, done, stale;
  int rebuilds;              /* contact-list builds of the context so far (all samples) */
  /* extensions (the reference outputs neither): chord Young modulus (GPa)
   * between 10% and 50% of the peak stress, and the Poisson ratio over the
   * same interval from the lateral record; NaN when undefined */
  double E_chord, nu;
  /* 1 when a particle's position, velocity or spin became NaN or infinite:
   * the specimen was stopped at that step (done = 1) and the dem_run /
   * dem_step call in which it happened returned DEM_ERR_NUMERIC.  The
   * reference has no such check (its loop runs on with NaN state). */
  int numeric;
  int reserved_r;
} dem_result;

/* --- context and specimens --- */
int dem_create(const dem_options* opt, dem_ctx** out);
/* Device memory of a destroyed context stays with the library for reuse by
 * later contexts of this process (a calibration creates many of similar
 * sizes; a fresh allocation costs far more than reuse), up to 40% of the
 * device's memory.  It goes back to the driver when an allocation would
 * otherwise fail, and on
 * dem_release_cached_memory() (no counterpart in the reference), for a host
 * that needs the memory for something else. */
void dem_destroy(dem_ctx* ctx);
int dem_release_cached_memory(void);
const char* dem_strerror(int code);
/* Text of the last CUDA error the library saw on this host thread (error name,
 * message, source location), "" if none; kept until the next CUDA error. */
const char* dem_last_error_detail(void);
int dem_device_count(int* n);

/* Adds one specimen.  xyz: 3n floats (mm, SoA); radii: n floats or NULL
 * (all mat->p_r).  All specimens of a context advance together (one launch
 * per kernel for all of them).  Returns the specimen id in *sample. */
int dem_add_sample(dem_ctx* ctx, const dem_material* mat, const dem_loading* load, const float* xyz,
                   const float* radii, uint32_t n, int32_t* sample);
/* Uploads, Morton-sorts, creates bonds and the contact list. */
int dem_setup(dem_ctx* ctx);
/* Advances every specimen max_steps steps or until it met its stop
 * condition (a specimen that is ahead waits for the others); *steps_done:
 * the largest number of steps a specimen advanced. */
int dem_run(dem_ctx* ctx, uint64_t max_steps, uint64_t* steps_done);
/* Advances every specimen exactly nsteps steps (finished specimens stay frozen). */
int dem_step(dem_ctx* ctx, uint32_t nsteps);
/* Stage control for parity checks: one step of the given stages, bit 0 pair
 * forces, bit 1 platens + integration; bit 2 keeps the total force/moment of
 * the step readable by dem_get_particles instead of clearing the
 * accumulators.  The contact list is rebuilt first when dem_run would rebuild
 * it. */
int dem_step_stages(dem_ctx* ctx, int stages);
int dem_sync(dem_ctx* ctx);

int dem_counts(dem_ctx* ctx, uint32_t* particles, uint32_t* bonds, uint32_t* contacts, uint32_t* samples);
int dem_sample_result(dem_ctx* ctx, int32_t sample, dem_result* out);
/* Loading record: 3 doubles per entry (strain, sigma_bottom, sigma_top in GPa)
 * and bonded directed-slot counts, as the reference's h_sFL / h_sSI. */
int dem_get_record(dem_ctx* ctx, int32_t sample, double* rec, uint32_t* bonds, uint32_t cap, uint32_t* n);
/* Secant modulus and secant Poisson ratio of a uniaxial specimen at the last
 * completed step (no counterpart in the reference).  With precision 2 (the
 * sensitivity build: FP64 values carried with their derivatives with respect
 * to DEM_SENS_COUNT micro-parameters, forward mode) also their derivatives;
 * other precisions leave the derivative arrays zero.  The time step is held
 * fixed: set dem_material.dt explicitly when comparing with finite
 * differences. */
#define DEM_SENS_E_BOND 0        /* dem_material.E_bond */
#define DEM_SENS_KN_KS 1         /* dem_material.kn_ks */
#define DEM_SENS_BOND_RADIUS 2   /* bond_radius_factor (or the absolute b_r when b_r > 0) */
#define DEM_SENS_E 3             /* particle E (contacts, platens) */
#define DEM_SENS_MU 4            /* sliding friction coefficient mu (pairs and platens) */
#define DEM_SENS_COUNT 5
typedef struct {
  double strain;                 /* axial strain at the last step, compression positive */
  double stress;                 /* platen stress of the last step, GPa */
  double E_secant;               /* stress / strain */
  double nu_secant;              /* lateral / axial strain (uniaxial specimens; NaN otherwise) */
  double dstress[DEM_SENS_COUNT];
  double dE[DEM_SENS_COUNT];
  double dnu[DEM_SENS_COUNT];
} dem_sensitivity;
int dem_sensitivities(dem_ctx* ctx, int32_t sample, dem_sensitivity* out);

/* Lateral record of a uniaxial specimen (no counterpart in the reference): per
 * loading-record entry the mean radial distance (mm) of the particles on the
 * lateral surface near mid-height; *n = 0 for specimens without one. */
int dem_get_lateral_record(dem_ctx* ctx, int32_t sample, double* lat, uint32_t cap, uint32_t* n);

/* Particle state in the caller's original order, SoA (3n each, NULL skips). */
int dem_get_particles(dem_ctx* ctx, int32_t sample, float* R, float* V, float* W, float* F, float* M,
                      float* Oiwt);
int dem_get_particles_d(dem_ctx* ctx, int32_t sample, double* R, double* V, double* W, double* F, double* M,
                        double* Oiwt);
int dem_set_particles(dem_ctx* ctx, int32_t sample, const float* R, const float* V, const float* W,
                      const float* Oiwt);
/* Pair state: for every bond and contact-list pair, original indices (i < j),
 * kind (1 intact bond, 2 broken bond, 3 contact) and 16 floats
 * (1/L0, prev-direction xyz, tangential xyz, twisting xyz, bending xyz,
 * normal strength, shear strength, bond radius). */
int dem_get_pairs(dem_ctx* ctx, int32_t sample, uint32_t cap, uint32_t* i, uint32_t* j, uint32_t* kind,
                  float* state, uint32_t* n);
/* The same in double (the FP64 builds' pair state without rounding). */
int dem_get_pairs_d(dem_ctx* ctx, int32_t sample, uint32_t cap, uint32_t* i, uint32_t* j, uint32_t* kind,
                    double* state, uint32_t* n);
/* Overwrites the state of listed pairs (the first 13 values of the record
 * layout; kind 1/2 sets a bond intact/broken, contacts take only the
 * tangential history). */
int dem_set_pairs(dem_ctx* ctx, int32_t sample, uint32_t n, const uint32_t* i, const uint32_t* j,
                  const uint32_t* kind, const float* state);
/* Platen state of a specimen (top, bottom position in mm; velocity mm/us). */
int dem_set_platens(dem_ctx* ctx, int32_t sample, double top, double bottom, double velocity);
/* Rebuilds the contact list now (normally automatic). */
int dem_rebuild_contacts(dem_ctx* ctx);
/* Advances nsteps steps from the captured step graphs; *ms = device time of
 * the steps (CUDA events on the context's stream, from the first step's
 * launch to the end of the last step: rebuilds and host checks between
 * chunks of steps included, the state read-back at either end of the call
 * not). */
int dem_run_timed(dem_ctx* ctx, uint64_t nsteps, double* ms);
/* Advances nsteps steps as one captured graph with a CUDA event record node
 * before, between and after the two step kernels of every step (the way the
 * timed steps run): average per-launch times of the pair kernel and the
 * particle kernel, and the mean number of touching contacts per step. */
int dem_profile(dem_ctx* ctx, uint32_t nsteps, double* pair_ms, double* particle_ms, double* touching);
/* Launch-schedule autotuner (no counterpart in the reference): after
 * dem_setup, advances the run by `steps` steps per candidate schedule (real
 * steps: the state moves on as under dem_run), times each with CUDA events
 * and keeps the fastest for the rest of the context's life.  Candidates: the
 * pair kernel's register budget / block size (dem_options.pair_min_blocks)
 * crossed with particle-kernel blocks of 128 and 256 threads; then the
 * contact-list skin (dem_options.skin_factor 0.1, 0.2, 0.3, 0.4; only when
 * the context was created with skin_factor 0), each run for 4 x `steps`
 * steps with its list rebuilds included (two passes in opposite orders).
 * The skin changes only which separated pairs are listed, not the forces. */
#define DEM_TUNE_MAX 16
typedef struct {
  int candidates;
  uint32_t pair_min_blocks[DEM_TUNE_MAX];
  uint32_t particle_block[DEM_TUNE_MAX];
  double ms_per_step[DEM_TUNE_MAX];
  uint32_t chosen_pair_min_blocks, chosen_particle_block;
  double chosen_ms_per_step;
  int skin_candidates;
  double skin_factor[8];
  double skin_ms_per_step[8];    /* measured step time at that skin, list rebuilds included */
  double skin_rebuild_ms[8];     /* one contact-list rebuild at that skin */
  double chosen_skin_factor;
} dem_tune_report;
int dem_autotune(dem_ctx* ctx, uint32_t steps, dem_tune_report* report);

/* --- reference-layout parity exports (stateless, run on the current device) --- */
/* CellDistribution: CI[n], CIs[2n] (sorted keys then particle indices), pnC[2*nx*ny*nz]. */
int dem_ref_cells(const float* xyz, uint32_t n, float a, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t* CI,
                  uint32_t* CIs, uint32_t* pnC);
/* Interaction sets: for each particle the sorted partners j != i with
 * r^2 < add_thr, !(r^2 > del_thr), !(r^2 < 1e-10), padded with DEM_EMPTY to cap. */
int dem_ref_neighbor_sets(const float* xyz, uint32_t n, float a, uint32_t nx, uint32_t ny, uint32_t nz,
                          float add_thr, float del_thr, uint32_t cap, uint32_t* sets, uint32_t* overflow);

/* dem_ref_cells for callers that cannot allocate GPU memory (no counterpart
 * in the reference, whose CellDistribution bins into buffers its driver
 * allocated).  cudaMalloc and cudaFree may synchronise the whole device and so
 * stall every other stream of a serving process, they fail once another
 * framework's caching allocator holds most of the device memory, and some
 * host frameworks do not let a plug-in allocate on its own; such callers use
 * this entry point.  Same arguments and outputs as dem_ref_cells, and it calls
 * no allocating routine: the device work runs out of one file-scope device
 * array of DEM_STATIC_SCRATCH_BYTES (4.5 MiB), which every GPU that loads the
 * library holds until the process exits.  The first call on a device looks
 * up that array's device address (cudaGetSymbolAddress, with that device
 * current) and keeps it for the device's current context (a context reset
 * makes the next call look it up again); make that first call before any
 * stream capture.  Every call issues its work on the legacy default stream
 * and waits for it, so it also waits for the device's other blocking streams
 * and must not run while another thread captures in global mode.
 * Returns DEM_ERR_CAPACITY, before any device work, when n >
 * DEM_STATIC_MAX_PARTICLES or nx*ny*nz > DEM_STATIC_MAX_CELLS.  All calls on
 * a device share the array: calls that overlap on the GPU (several host
 * threads) race on it and must be serialised by the caller. */
#define DEM_STATIC_MAX_PARTICLES 65536u
#define DEM_STATIC_MAX_CELLS 65536u
#define DEM_STATIC_SCRATCH_BYTES 4718592u /* 4.5 MiB */
int dem_ref_cells_static(const float* xyz, uint32_t n, float a, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t* CI,
                         uint32_t* CIs, uint32_t* pnC);

/* --- surrogate MLP on the tensor cores (the role of NN_MP.py's MLPRegressor,
 * NN_MP.py:374-378, 895; the reference trains it with sklearn on the CPU) ---
 * Device pointers, an optional cudaStream_t (NULL: the default stream).
 * dem_mlp_gemm_tn: C[M x N] = A[M x K] B[N x K]^T, A and B row-major BF16,
 * 16-byte aligned, K a multiple of 32, FP32 accumulation on tcgen05; epilogue
 * DEM_MLP_PLAIN (out_f32 = C), DEM_MLP_BIAS (out_f32 = C + bias),
 * DEM_MLP_BIAS_GELU / DEM_MLP_BIAS_RELU (out_bf16 = act(C + bias), and
 * out_f32 = C + bias when given).  dem_mlp_status reports a tensor-core commit
 * that timed out (the GEMM then leaves its output tile unwritten). */
#define DEM_MLP_PLAIN 0
#define DEM_MLP_BIAS 1
#define DEM_MLP_BIAS_GELU 2
#define DEM_MLP_BIAS_RELU 3
int dem_mlp_gemm_tn(const void* A, const void* B, int M, int N, int K, const float* bias, int mode, float* out_f32,
                    void* out_bf16, void* stream);
int dem_mlp_status(int* timed_out);
/* x (rows x k FP32) -> BF16 rows of kpad elements, zero padded; output row r is
 * row idx[r] of x when idx (device int array of rows entries) is given */
int dem_mlp_pack_bf16(const float* x, const int* idx, int rows, int k, int kpad, void* out_bf16, void* stream);
/* out row r = row idx[r] of x (FP32, k columns) */
int dem_mlp_gather(const float* x, const int* idx, int rows, int k, float* out, void* stream);
/* out (cols x ldo BF16) = transpose of in (rows x cols BF16), columns >= rows zeroed */
int dem_mlp_transpose_bf16(const void* in, int rows, int cols, int ldo, void* out, void* stream);
/* dZ = dH * act'(Z), act DEM_MLP_BIAS_GELU or DEM_MLP_BIAS_RELU; BF16 (and FP32 when dz_f32 is given) */
int dem_mlp_act_backward(const float* dh, const float* z, size_t n, int act, void* dz_bf16, float* dz_f32,
                         void* stream);
/* out[c] = sum over rows of in[r][c] (FP32, a fixed summation order);
 * scratch holds DEM_MLP_COLSUM_SPLIT * cols floats (used above 2048 rows) */
#define DEM_MLP_COLSUM_SPLIT 32
int dem_mlp_colsum(const float* in, int rows, int cols, float* out, float* scratch, void* stream);
/* dY = 2 (y - t) / n (BF16, and FP32 when given); *loss (double, device) += mean squared error */
int dem_mlp_mse_grad(const float* y, const float* t, size_t n, void* dy_bf16, float* dy_f32, double* loss, void* stream);
/* one Adam step on FP32 weights with gradient g + l2 w and the step number
 * read from *step (device int, >= 1; bias corrections 1 - b^t); BF16 copy
 * refreshed when w_bf16 is given.  dem_mlp_tick adds 1 to *step on the stream. */
int dem_mlp_adam(float* w, const float* g, float* m, float* v, size_t n, float lr, float b1, float b2, float eps,
                 float l2, const int* step, void* w_bf16, void* stream);
int dem_mlp_tick(int* step, void* stream);
/* The same Adam step over `count` arrays in one launch: `list` is a device
 * array of descriptors (n elements each, at most max_n), per-array l2. */
typedef struct {
  float* w;
  const float* g;
  float* m;
  float* v;
  void* w_bf16;      /* BF16 copy to refresh, or NULL */
  uint64_t n;
  float l2;
  float pad;
} dem_mlp_tensor;
int dem_mlp_adam_multi(const dem_mlp_tensor* list, int count, size_t max_n, float lr, float b1, float b2, float eps,
                       const int* step, void* stream);

/* --- reference entry points --- */
/* One loading test of one specimen from host positions to macro results and
 * the loading record (h_Calculation{UniaxialCompression,BrazilTest}). */
int dem_calculation_test(const dem_options* opt, const dem_material* mat, const dem_loading* load,
                         const float* h_R, const float* radii, uint32_t n, dem_result* out, double* rec,
                         uint32_t* rec_bonds, uint32_t rec_cap, uint32_t* rec_n);
/* Sample text file (first line n, then "x y z" in metres per line):
 * LoadParticleDATAtxt / SaveParticleDATAtxt, md_createcylindersample.cu:144-182.
 * dem_load_cylinder_sample also returns the bounding box of h_LoadCylinderSample
 * (size_real incl. 2*p_r, center_real). */
int dem_load_cylinder_sample(const char* path, double p_r, float* xyz, uint32_t cap, uint32_t* n,
                             double size_real[3], double center_real[3]);
int dem_save_cylinder_sample(const char* path, const float* xyz, uint32_t n, const double hidden_point[3]);
/* LAMMPS data file of one specimen (SaveLammpsDATASimple, md_savelammpsdata.cpp:9-75):
 * atoms in metres, per-atom kinetic energies when with_energy != 0, intact
 * bonds once per direction (type 2). */
int dem_save_lammps_data(dem_ctx* ctx, int32_t sample, const char* path, int with_energy);
/* "EpsZ StressZ_bottom StressZ_top" file of SaveSumForcesLoading (stresses in Pa). */
int dem_save_sum_forces_loading(const char* path, const double* rec, uint32_t n);

/* Escape box of the reference's sample set-up (sample_data::SetSpaceSizeSi,
 * SetLSi, CalculateParameters, md_data_types.h:87-123, cell edge 2 farcut p_r):
 * fills out->space_center, space_half, hidden_point and zcut (mm), rounded to
 * float as the reference stores them; the rest of *out is left as it is
 * (lsi_si is accepted for the reference's argument order; the box does not
 * depend on it). */
int dem_reference_space(const double space_si[3], const double lsi_si[3], double p_r, double farcut, dem_loading* out);

/* Seeded sample creation (the role of h_CreateCylinderSample): n spheres with
 * radii uniform in [r_min, r_max] filled at random into a z-axis cylinder
 * (a column for the uniaxial test, a disc for the Brazilian test), grown from
 * 30% of the final packing fraction with damped soft-sphere relaxation, then
 * FIRE-relaxed until the largest overlap / (r_i + r_j) is below overlap_tol.
 * fire_variant 0: inertial FIRE 2.0; 1: the reference's FIRE update
 * (md_firerelaxation.cu:18-70, velocity rebuilt from the force each step). */
typedef struct {
  double center[3];          /* cylinder centre, mm */
  double radius;             /* cylinder radius, mm */
  double half_height;        /* cylinder half height, mm */
  double r_min, r_max;       /* particle radii, mm */
  double E, nu, rho;         /* particle material (GPa, -, mg/mm^3): stiffness and time step */
  double overlap_tol;        /* target largest relative overlap */
  uint32_t n;                /* number of particles */
  uint32_t growth_stages;    /* radius increments */
  uint32_t steps_per_stage;  /* relaxation steps after each increment */
  uint32_t max_fire_steps;   /* FIRE steps at the final radii */
  uint64_t seed;
  int device;
  int fire_variant;
  uint32_t max_removed;      /* > 0: remove up to this many spheres of the worst overlaps while the largest
                                overlap stays >= overlap_tol (the reference's d_ReduceParticleNumber);
                                *n then returns the spheres kept */
  uint32_t reserved;
} dem_pack_params;

typedef struct {
  uint64_t steps;
  double max_overlap;        /* largest relative overlap at the end */
  double packing_fraction;   /* sphere volume / cylinder volume */
  uint32_t rebuilds;
  uint32_t removed;          /* spheres removed (max_removed) */
} dem_pack_report;

int dem_create_cylinder_sample(const dem_pack_params* p, float* xyz, float* radii, uint32_t cap, uint32_t* n,
                               dem_pack_report* rep);

#ifdef __cplusplus
}
#endif
#endif
