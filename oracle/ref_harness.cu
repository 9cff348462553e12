// Test harness around the reference's OWN CUDA kernels and host drivers
// (test infrastructure only).  oracle/Makefile compiles the reference sources
// from the reference tree together with this file into oracle/_ref/libdemref.so;
// tests/golden/make_golden.py and the GPU tests load it with ctypes on a GPU box
// to produce golden vectors, run the reference's drivers and time its kernels.
// Nothing here is part of the product.
//
// Every entry point takes and returns host arrays in the reference layout
// (SoA x[0..N) y[N..2N) z[2N..3N); IonP slots per particle; float3 per slot)
// and launches the reference kernels exactly as its drivers do
// (md_calculationuniaxialcompression.cu:155-314, md_calculationbraziltest.cu:144-231).
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <fcntl.h>
#include <unistd.h>
#include <sys/stat.h>

#include "md.h"
#include "mp.h"
#include "mp_task.h"

namespace {

int g_err = 0;
void chk(cudaError_t e) {
  if (e != cudaSuccess && g_err == 0) g_err = (int)e;
}

struct DevArrays {
  float *R = nullptr, *V = nullptr, *W = nullptr, *F = nullptr, *M = nullptr, *Oiwt = nullptr;
  uint *IL = nullptr, *ILtype = nullptr;
  float* invL0 = nullptr;
  float3 *Rij = nullptr, *Oijt = nullptr, *Mijn = nullptr, *Mijt = nullptr, *Fijn = nullptr, *Fijt = nullptr,
         *Mijadd = nullptr;
};

template <class T>
T* dalloc(size_t n) {
  T* p = nullptr;
  chk(cudaMalloc((void**)&p, n * sizeof(T) + 64));
  chk(cudaMemset(p, 0, n * sizeof(T) + 64));
  return p;
}

void dfree(void* p) {
  if (p) cudaFree(p);
}

// cell_data set-up identical to cuc_createCD (md_calculationuniaxialcompression.cu:65-74)
void cells_create(md_task_data& td) {
  chk(cudaMalloc((void**)&td.C.d_IP, td.P.N * sizeof(uint)));
  d_FillIndex<<<td.A.bloks, SMEMDIM>>>(td.C.d_IP, td.P.N);
  chk(cudaMalloc((void**)&td.C.d_CI, td.P.N * sizeof(uint)));
  chk(cudaMalloc((void**)&td.C.d_CIs, 2 * td.P.N * sizeof(uint) + 64));
  chk(cudaMemset(td.C.d_CIs, 0xFF, 2 * td.P.N * sizeof(uint) + 64));
  chk(cudaMalloc((void**)&td.C.d_pnC, 2 * td.C.N * sizeof(uint)));
  td.C.dtmpN_old = 128;
  chk(cudaMalloc((void**)&td.C.d_tmp_old, td.C.dtmpN_old));
}

void cells_free(md_task_data& td) {
  dfree(td.C.d_IP);
  dfree(td.C.d_CI);
  dfree(td.C.d_CIs);
  dfree(td.C.d_pnC);
  dfree(td.C.d_tmp_old);
  td.C.d_IP = td.C.d_CI = td.C.d_CIs = td.C.d_pnC = nullptr;
  td.C.d_tmp_old = td.C.d_tmp = nullptr;
}

void setup_task(md_task_data& td, uint32_t N, float a, uint32_t nx, uint32_t ny, uint32_t nz) {
  initArrays(td.A, td.P, td.C, td.IL, td.R);
  td.P.N = N;
  td.C.a = a;
  td.C._1d_a = 1.0 / double(a);
  td.C.Nr = make_uint3(nx, ny, nz);
  td.C.N = nx * ny * nz;
  td.A.CalculateParameters(N, N * 32);
}

}  // namespace

// The definition in md_calculateforcesbpm_cpu.cu:20-24 (per directed slot, with
// the slot and particle indices and the bond type) differs from the overload
// md.h:134 declares (never defined); this prototype matches the definition.
void h_CalculateForceElastic(const float* R, const float* V, const float* W, float* F, float* M, const float* ab_r,
                             const float* _1d_iL, const float* AxialMoment, float3* Rij, float3* OverlapTau,
                             float3* Mijn, float3* Mijt, float3* Fij, const uint N, const uint idx, const uint jdx,
                             const uint kdx, const float dt, const float m_E, const float m_G, const float m_Gcritn,
                             const float m_Gcritt, uint type);

extern "C" {

int refh_last_error(void) { return g_err; }

// CellDistribution (md_cell_distribution.cu:130-179) on given positions.
int refh_cell_distribution(const float* hR, uint32_t N, float a, uint32_t nx, uint32_t ny, uint32_t nz,
                           uint32_t* CI, uint32_t* CIs, uint32_t* pnC) {
  g_err = 0;
  md_task_data td;
  setup_task(td, N, a, nx, ny, nz);
  td.P.d_R = dalloc<float>(3 * N);
  chk(cudaMemcpy(td.P.d_R, hR, 3 * N * sizeof(float), cudaMemcpyHostToDevice));
  cells_create(td);
  CellDistribution(td.P, td.A, td.S, td.C);
  chk(cudaDeviceSynchronize());
  chk(cudaMemcpy(CI, td.C.d_CI, N * sizeof(uint), cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(CIs, td.C.d_CIs, 2 * N * sizeof(uint), cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(pnC, td.C.d_pnC, 2 * td.C.N * sizeof(uint), cudaMemcpyDeviceToHost));
  cells_free(td);
  dfree(td.P.d_R);
  td.P.d_R = nullptr;
  return g_err;
}

// Set-up of a loading test: CellDistribution + InteractionListConstruct +
// d_ConstructBoundInteractions + d_DeleteFarLinks
// (md_calculationuniaxialcompression.cu:155-157, 212-213).
int refh_setup_bonds(const float* hR, uint32_t N, float a, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t IonP,
                     float il_aacut, float aa_farcut, float b_dd, float b_r, uint32_t* IL, uint32_t* ILtype,
                     float* invL0) {
  g_err = 0;
  md_task_data td;
  setup_task(td, N, a, nx, ny, nz);
  size_t S = (size_t)N * IonP;
  DevArrays d;
  td.P.d_R = dalloc<float>(3 * N);
  td.P.d_V = dalloc<float>(3 * N);
  td.P.d_W = dalloc<float>(3 * N);
  chk(cudaMemcpy(td.P.d_R, hR, 3 * N * sizeof(float), cudaMemcpyHostToDevice));
  td.IL.IonP = IonP;
  td.IL.N = S;
  td.IL.aacut = il_aacut;
  td.IL.d_IL = dalloc<uint>(S);
  td.IL.d_ILtype = dalloc<uint>(S);
  td.IL.d_1d_iL = dalloc<float>(S);
  td.IL.d_rij = dalloc<float3>(S);
  td.IL.d_Oijt = dalloc<float3>(S);
  td.IL.d_Fijn = dalloc<float3>(S);
  td.IL.d_Fijt = dalloc<float3>(S);
  td.IL.d_Mijn = dalloc<float3>(S);
  td.IL.d_Mijt = dalloc<float3>(S);
  td.IL.d_Mijadd = dalloc<float3>(S);
  cells_create(td);
  CellDistribution(td.P, td.A, td.S, td.C);
  InteractionListConstruct(td.P, td.A, td.S, td.IL, td.C);
  d_ConstructBoundInteractions<<<td.A.bloks, SMEMDIM>>>(td.P.d_R, td.P.d_V, td.P.d_W, td.IL.d_IL, td.IL.d_ILtype,
                                                        td.IL.d_1d_iL, td.IL.d_rij, td.IL.d_Oijt, td.IL.d_Fijn,
                                                        td.IL.d_Fijt, td.IL.d_Mijn, td.IL.d_Mijt, td.IL.d_Mijadd,
                                                        N, IonP, b_dd, b_r);
  d_DeleteFarLinks<<<td.A.bloks, SMEMDIM>>>(td.P.d_R, N, td.IL.d_IL, td.IL.d_ILtype, td.IL.d_1d_iL, td.IL.d_rij,
                                            td.IL.d_Oijt, td.IL.d_Fijn, td.IL.d_Fijt, td.IL.d_Mijn, td.IL.d_Mijt,
                                            td.IL.d_Mijadd, IonP, aa_farcut);
  chk(cudaDeviceSynchronize());
  chk(cudaMemcpy(IL, td.IL.d_IL, S * sizeof(uint), cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(ILtype, td.IL.d_ILtype, S * sizeof(uint), cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(invL0, td.IL.d_1d_iL, S * sizeof(float), cudaMemcpyDeviceToHost));
  cells_free(td);
  dfree(td.P.d_R);
  dfree(td.P.d_V);
  dfree(td.P.d_W);
  dfree(td.IL.d_IL);
  dfree(td.IL.d_ILtype);
  dfree(td.IL.d_1d_iL);
  dfree(td.IL.d_rij);
  dfree(td.IL.d_Oijt);
  dfree(td.IL.d_Fijn);
  dfree(td.IL.d_Fijt);
  dfree(td.IL.d_Mijn);
  dfree(td.IL.d_Mijt);
  dfree(td.IL.d_Mijadd);
  return g_err;
}

// Scalars of one loading step.  All float, as the reference passes them to its
// kernels (md_calculationuniaxialcompression.cu:269-310).
typedef struct {
  float a;
  uint32_t nx, ny, nz, IonP;
  float il_aacut, aa_farcut;
  float dt, m_E, m_G, b_r, m_Ec, m_Gc;
  float hm_E, hm_G, p_A, p_mu, p_mur, p_m, p_r;
  float wall_E, wall_G;        // 2*hm_E, 2*hm_G (uniaxial) or hm_E, hm_G (Brazilian)
  float center[3];             // Compress.center
  float wall_RR, wall_top, wall_bot, wall_V, Zcut;
  float dt_d_m, dt_d_I;
  float s_center[3], s_spacesized2[3], hidenpoint[3];  // S.center, S.spacesized2, S.hidenpoint
  int brazil;
  int stages;                  // bit 0: rebuild IL; 1: forces; 2: platen; 3: increments; 4: cut; 5: delete far
} refh_step_params;

// One pass of the hot loop body (cells, IL rebuild, forces, platen, increments,
// escape restriction, far-link deletion) on a full state; FL returns the
// per-block platen partials (2*bloks floats).
int refh_step(const refh_step_params* p, uint32_t N, float* R, float* V, float* W, float* F, float* M, float* Oiwt,
              uint32_t* IL, uint32_t* ILtype, float* invL0, float* Rij, float* Oijt, float* Mijn, float* Mijt,
              float* FL) {
  g_err = 0;
  md_task_data td;
  setup_task(td, N, p->a, p->nx, p->ny, p->nz);
  const uint32_t IonP = p->IonP;
  size_t S = (size_t)N * IonP;
  td.P.d_R = dalloc<float>(3 * N);
  td.P.d_V = dalloc<float>(3 * N);
  td.P.d_W = dalloc<float>(3 * N);
  td.P.d_F = dalloc<float>(3 * N);
  td.P.d_M = dalloc<float>(3 * N);
  td.P.d_Oiwt = dalloc<float>(3 * N);
  td.IL.IonP = IonP;
  td.IL.N = S;
  td.IL.aacut = p->il_aacut;
  td.IL.d_IL = dalloc<uint>(S);
  td.IL.d_ILtype = dalloc<uint>(S);
  td.IL.d_1d_iL = dalloc<float>(S);
  td.IL.d_rij = dalloc<float3>(S);
  td.IL.d_Oijt = dalloc<float3>(S);
  td.IL.d_Fijn = dalloc<float3>(S);
  td.IL.d_Fijt = dalloc<float3>(S);
  td.IL.d_Mijn = dalloc<float3>(S);
  td.IL.d_Mijt = dalloc<float3>(S);
  td.IL.d_Mijadd = dalloc<float3>(S);
  td.R.d_FL = dalloc<float>(2 * td.A.bloks);
  chk(cudaMemcpy(td.P.d_R, R, 3 * N * 4, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.P.d_V, V, 3 * N * 4, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.P.d_W, W, 3 * N * 4, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.P.d_F, F, 3 * N * 4, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.P.d_M, M, 3 * N * 4, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.P.d_Oiwt, Oiwt, 3 * N * 4, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.IL.d_IL, IL, S * 4, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.IL.d_ILtype, ILtype, S * 4, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.IL.d_1d_iL, invL0, S * 4, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.IL.d_rij, Rij, S * 12, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.IL.d_Oijt, Oijt, S * 12, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.IL.d_Mijn, Mijn, S * 12, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.IL.d_Mijt, Mijt, S * 12, cudaMemcpyHostToDevice));
  cells_create(td);
  const uint bl = td.A.bloks;
  if (p->stages & 1) {
    CellDistribution(td.P, td.A, td.S, td.C);
    InteractionListReConstructBPM(td.P, td.A, td.S, td.IL, td.C);
  }
  if (p->stages & 2) {
    chk(cudaMemset(td.P.d_F, 0, 3 * N * sizeof(float)));
    chk(cudaMemset(td.P.d_M, 0, 3 * N * sizeof(float)));
    if (p->brazil)
      d_CalculateForcesDEM_22<<<4 * bl, 256>>>(td.P.d_R, td.P.d_V, td.P.d_W, td.IL.d_IL, td.IL.d_ILtype,
                                               td.IL.d_1d_iL, td.IL.d_rij, td.IL.d_Oijt, td.IL.d_Mijn, td.IL.d_Mijt,
                                               td.P.d_F, td.P.d_M, N, IonP, p->dt, p->m_E, p->m_G, p->b_r, p->m_Ec,
                                               p->m_Gc);
    else
      d_CalculateForcesDEM_22<<<bl, SMEMDIM>>>(td.P.d_R, td.P.d_V, td.P.d_W, td.IL.d_IL, td.IL.d_ILtype,
                                               td.IL.d_1d_iL, td.IL.d_rij, td.IL.d_Oijt, td.IL.d_Mijn, td.IL.d_Mijt,
                                               td.P.d_F, td.P.d_M, N, IonP, p->dt, p->m_E, p->m_G, p->b_r, p->m_Ec,
                                               p->m_Gc);
    d_CalculateForcesDEM_21<<<bl, SMEMDIM>>>(td.P.d_R, td.P.d_V, td.P.d_W, td.IL.d_IL, td.IL.d_ILtype,
                                             td.IL.d_1d_iL, td.IL.d_rij, td.IL.d_Oijt, td.P.d_F, td.P.d_M, N, IonP,
                                             p->dt, p->hm_E, p->hm_G, p->p_A, p->p_mu, p->p_mur, p->p_m, p->p_r);
  }
  if (p->stages & 4) {
    float3 c = make_float3(p->center[0], p->center[1], p->center[2]);
    if (p->brazil)
      d_BrazilCompression_hm<<<bl, SMEMDIM>>>(td.P.d_R, td.P.d_V, td.P.d_W, td.P.d_Oiwt, td.P.d_F, td.P.d_M, N, p->dt,
                                              p->wall_E, p->wall_G, p->p_A, p->p_mu, p->p_mur, p->p_m, p->p_r,
                                              td.R.d_FL, c, p->wall_RR, p->wall_top, p->wall_bot, p->wall_V, p->Zcut);
    else
      d_UniaxialCompression_hm<<<bl, SMEMDIM>>>(td.P.d_R, td.P.d_V, td.P.d_W, td.P.d_Oiwt, td.P.d_F, td.P.d_M, N,
                                                p->dt, p->wall_E, p->wall_G, p->p_A, p->p_mu, p->p_mur, p->p_m,
                                                p->p_r, td.R.d_FL, c, p->wall_RR, p->wall_top, p->wall_bot, p->wall_V,
                                                p->Zcut);
  }
  if (p->stages & 8)
    d_CalculateIncrementsDEM<<<bl, SMEMDIM>>>(td.P.d_F, td.P.d_V, td.P.d_R, td.P.d_M, td.P.d_W, N, p->dt_d_m, p->dt,
                                              p->dt_d_I);
  if (p->stages & 16) {
    float3 c = make_float3(p->s_center[0], p->s_center[1], p->s_center[2]);
    float3 s2 = make_float3(p->s_spacesized2[0], p->s_spacesized2[1], p->s_spacesized2[2]);
    float3 hp = make_float3(p->hidenpoint[0], p->hidenpoint[1], p->hidenpoint[2]);
    d_ParallelepipedCutRestriction<<<bl, SMEMDIM>>>(td.P.d_R, td.P.d_V, td.P.d_F, N, c, s2, hp);
  }
  if (p->stages & 32)
    d_DeleteFarLinks<<<bl, SMEMDIM>>>(td.P.d_R, N, td.IL.d_IL, td.IL.d_ILtype, td.IL.d_1d_iL, td.IL.d_rij,
                                      td.IL.d_Oijt, td.IL.d_Fijn, td.IL.d_Fijt, td.IL.d_Mijn, td.IL.d_Mijt,
                                      td.IL.d_Mijadd, IonP, p->aa_farcut);
  chk(cudaDeviceSynchronize());
  chk(cudaGetLastError());
  chk(cudaMemcpy(R, td.P.d_R, 3 * N * 4, cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(V, td.P.d_V, 3 * N * 4, cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(W, td.P.d_W, 3 * N * 4, cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(F, td.P.d_F, 3 * N * 4, cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(M, td.P.d_M, 3 * N * 4, cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(Oiwt, td.P.d_Oiwt, 3 * N * 4, cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(IL, td.IL.d_IL, S * 4, cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(ILtype, td.IL.d_ILtype, S * 4, cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(invL0, td.IL.d_1d_iL, S * 4, cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(Rij, td.IL.d_rij, S * 12, cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(Oijt, td.IL.d_Oijt, S * 12, cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(Mijn, td.IL.d_Mijn, S * 12, cudaMemcpyDeviceToHost));
  chk(cudaMemcpy(Mijt, td.IL.d_Mijt, S * 12, cudaMemcpyDeviceToHost));
  if (FL) chk(cudaMemcpy(FL, td.R.d_FL, 2 * bl * 4, cudaMemcpyDeviceToHost));
  cells_free(td);
  void* ps[] = {td.P.d_R, td.P.d_V, td.P.d_W, td.P.d_F, td.P.d_M, td.P.d_Oiwt, td.IL.d_IL, td.IL.d_ILtype,
                td.IL.d_1d_iL, td.IL.d_rij, td.IL.d_Oijt, td.IL.d_Fijn, td.IL.d_Fijt, td.IL.d_Mijn, td.IL.d_Mijt,
                td.IL.d_Mijadd, td.R.d_FL};
  for (void* q : ps) dfree(q);
  return g_err;
}

// Device time of nsteps passes of the reference's loop body on one state
// (test infrastructure: the reference-GPU baseline).  Each pass launches the
// kernels of md_calculationuniaxialcompression.cu:265-314 selected by
// p->stages, in that order, and - when sync_fl is set - copies the platen
// partial sums to the host as SumForcesULoading does every step
// (md_results.cu:56-100).  *ms = CUDA-event time of the whole loop.
int refh_time_steps(const refh_step_params* p, uint32_t N, const float* R, const float* V, const float* W,
                    const uint32_t* IL, const uint32_t* ILtype, const float* invL0, uint32_t nsteps, int sync_fl,
                    double* ms) {
  g_err = 0;
  md_task_data td;
  setup_task(td, N, p->a, p->nx, p->ny, p->nz);
  const uint32_t IonP = p->IonP;
  size_t S = (size_t)N * IonP;
  td.P.d_R = dalloc<float>(3 * N);
  td.P.d_V = dalloc<float>(3 * N);
  td.P.d_W = dalloc<float>(3 * N);
  td.P.d_F = dalloc<float>(3 * N);
  td.P.d_M = dalloc<float>(3 * N);
  td.P.d_Oiwt = dalloc<float>(3 * N);
  td.IL.IonP = IonP;
  td.IL.N = S;
  td.IL.aacut = p->il_aacut;
  td.IL.d_IL = dalloc<uint>(S);
  td.IL.d_ILtype = dalloc<uint>(S);
  td.IL.d_1d_iL = dalloc<float>(S);
  td.IL.d_rij = dalloc<float3>(S);
  td.IL.d_Oijt = dalloc<float3>(S);
  td.IL.d_Fijn = dalloc<float3>(S);
  td.IL.d_Fijt = dalloc<float3>(S);
  td.IL.d_Mijn = dalloc<float3>(S);
  td.IL.d_Mijt = dalloc<float3>(S);
  td.IL.d_Mijadd = dalloc<float3>(S);
  td.R.d_FL = dalloc<float>(2 * td.A.bloks);
  chk(cudaMemcpy(td.P.d_R, R, 3 * N * 4, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.P.d_V, V, 3 * N * 4, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.P.d_W, W, 3 * N * 4, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.IL.d_IL, IL, S * 4, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.IL.d_ILtype, ILtype, S * 4, cudaMemcpyHostToDevice));
  chk(cudaMemcpy(td.IL.d_1d_iL, invL0, S * 4, cudaMemcpyHostToDevice));
  cells_create(td);
  const uint bl = td.A.bloks;
  float* hFL = new float[2 * bl];
  const float3 c = make_float3(p->center[0], p->center[1], p->center[2]);
  const float3 sc = make_float3(p->s_center[0], p->s_center[1], p->s_center[2]);
  const float3 s2 = make_float3(p->s_spacesized2[0], p->s_spacesized2[1], p->s_spacesized2[2]);
  const float3 hp = make_float3(p->hidenpoint[0], p->hidenpoint[1], p->hidenpoint[2]);
  cudaEvent_t e0, e1;
  chk(cudaEventCreate(&e0));
  chk(cudaEventCreate(&e1));
  chk(cudaDeviceSynchronize());
  chk(cudaEventRecord(e0));
  for (uint32_t k = 0; k < nsteps; ++k) {
    if (p->stages & 1) {
      CellDistribution(td.P, td.A, td.S, td.C);
      InteractionListReConstructBPM(td.P, td.A, td.S, td.IL, td.C);
    }
    if (p->stages & 2) {
      chk(cudaMemset(td.P.d_F, 0, 3 * N * sizeof(float)));
      chk(cudaMemset(td.P.d_M, 0, 3 * N * sizeof(float)));
      d_CalculateForcesDEM_22<<<bl, SMEMDIM>>>(td.P.d_R, td.P.d_V, td.P.d_W, td.IL.d_IL, td.IL.d_ILtype,
                                               td.IL.d_1d_iL, td.IL.d_rij, td.IL.d_Oijt, td.IL.d_Mijn, td.IL.d_Mijt,
                                               td.P.d_F, td.P.d_M, N, IonP, p->dt, p->m_E, p->m_G, p->b_r, p->m_Ec,
                                               p->m_Gc);
      d_CalculateForcesDEM_21<<<bl, SMEMDIM>>>(td.P.d_R, td.P.d_V, td.P.d_W, td.IL.d_IL, td.IL.d_ILtype,
                                               td.IL.d_1d_iL, td.IL.d_rij, td.IL.d_Oijt, td.P.d_F, td.P.d_M, N, IonP,
                                               p->dt, p->hm_E, p->hm_G, p->p_A, p->p_mu, p->p_mur, p->p_m, p->p_r);
    }
    if (p->stages & 4) {
      if (p->brazil)
        d_BrazilCompression_hm<<<bl, SMEMDIM>>>(td.P.d_R, td.P.d_V, td.P.d_W, td.P.d_Oiwt, td.P.d_F, td.P.d_M, N,
                                                p->dt, p->wall_E, p->wall_G, p->p_A, p->p_mu, p->p_mur, p->p_m,
                                                p->p_r, td.R.d_FL, c, p->wall_RR, p->wall_top, p->wall_bot, p->wall_V,
                                                p->Zcut);
      else
        d_UniaxialCompression_hm<<<bl, SMEMDIM>>>(td.P.d_R, td.P.d_V, td.P.d_W, td.P.d_Oiwt, td.P.d_F, td.P.d_M, N,
                                                  p->dt, p->wall_E, p->wall_G, p->p_A, p->p_mu, p->p_mur, p->p_m,
                                                  p->p_r, td.R.d_FL, c, p->wall_RR, p->wall_top, p->wall_bot,
                                                  p->wall_V, p->Zcut);
      if (sync_fl) chk(cudaMemcpy(hFL, td.R.d_FL, 2 * bl * sizeof(float), cudaMemcpyDeviceToHost));
    }
    if (p->stages & 8)
      d_CalculateIncrementsDEM<<<bl, SMEMDIM>>>(td.P.d_F, td.P.d_V, td.P.d_R, td.P.d_M, td.P.d_W, N, p->dt_d_m,
                                                p->dt, p->dt_d_I);
    if (p->stages & 16) d_ParallelepipedCutRestriction<<<bl, SMEMDIM>>>(td.P.d_R, td.P.d_V, td.P.d_F, N, sc, s2, hp);
    if (p->stages & 32)
      d_DeleteFarLinks<<<bl, SMEMDIM>>>(td.P.d_R, N, td.IL.d_IL, td.IL.d_ILtype, td.IL.d_1d_iL, td.IL.d_rij,
                                        td.IL.d_Oijt, td.IL.d_Fijn, td.IL.d_Fijt, td.IL.d_Mijn, td.IL.d_Mijt,
                                        td.IL.d_Mijadd, IonP, p->aa_farcut);
  }
  chk(cudaEventRecord(e1));
  chk(cudaEventSynchronize(e1));
  float t = 0.f;
  chk(cudaEventElapsedTime(&t, e0, e1));
  *ms = t;
  chk(cudaGetLastError());
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  delete[] hFL;
  cells_free(td);
  void* ps[] = {td.P.d_R, td.P.d_V, td.P.d_W, td.P.d_F, td.P.d_M, td.P.d_Oiwt, td.IL.d_IL, td.IL.d_ILtype,
                td.IL.d_1d_iL, td.IL.d_rij, td.IL.d_Oijt, td.IL.d_Fijn, td.IL.d_Fijt, td.IL.d_Mijn, td.IL.d_Mijt,
                td.IL.d_Mijadd, td.R.d_FL};
  for (void* q : ps) dfree(q);
  return g_err;
}

// Full reference loading test through the reference's own entry points:
// h_LoadCylinderSample + compression_data::Calculate{U,B}Parameters +
// h_Calculation{UniaxialCompression,BrazilTest} (mp_calculateonesample.cu:151-214).
// The sample file ./result/Sample_<isample><part>.txt must exist under workdir.
typedef struct {
  double E, Ec, Gc, b_r, gap;      // SI units, as mp_calculateonesample.cu:47-51 receives them
  double p_r_m, rho, nu, p_e, p_mu, p_mur, farcut_factor;
  double space_si[3], lsi[3];      // SpaceSize and LSi (metres), mp_calculateonesample.cu:91
  double velocity_si, minstress_si, maxstrain, condfract;
  uint32_t dNsave, fileN, isample;
} refh_test_params;

typedef struct {
  double FractureStress, FractureStrain, LinearityDeviation, Destruction, Strain;
  double dt, seconds;
  uint64_t steps_hint;
  uint32_t N, stepsave;
} refh_test_result;

int refh_run_test(int brazil, const char* workdir, const char* part, const refh_test_params* q,
                  refh_test_result* out) {
  g_err = 0;
  char cwd[4096];
  if (!getcwd(cwd, sizeof cwd)) return -1;
  if (chdir(workdir) != 0) return -2;
  mkdir("result", 0755);
  {
    mp_mdparameters_data mpMDP;
    md_task_data& td = mpMDP.mdTD[0];
    initArrays(td.A, td.P, td.C, td.IL, td.R);
    // SetInitialParameters (mp_determineconjgradient.cu:15-47) with caller values
    td.IL.IonP = 32;
    td.Po.m_nu = q->nu;
    td.Po.m_E = q->E / stress_const;
    td.Po.m_Ec = q->Ec / stress_const;
    td.Po.m_Gc = q->Gc / stress_const;
    td.Po.m_ro = q->rho / density_const;
    td.Po.b_r = q->b_r / length_const;
    td.Po.p_r = q->p_r_m / length_const;
    td.Po.b_d = 2.0 * td.Po.p_r + q->gap / length_const;
    td.Po.p_e = q->p_e;
    td.Po.p_mu = q->p_mu;
    td.Po.p_mur = q->p_mur;
    td.Po.nuV = 1e-5;
    td.Po.nuW = 1e-3;
    td.Po.a_farcut = q->farcut_factor * td.Po.p_r;
    td.C.a = 2.0 * td.Po.a_farcut;
    td.Po.CalculateParameters();
    const uint i = q->isample;
    mpMDP.S[i].SetSpaceSizeSi(q->space_si[0], q->space_si[1], q->space_si[2]);
    mpMDP.S[i].SetLSi(q->lsi[0], q->lsi[1], q->lsi[2], td.Po.p_r);
    mpMDP.S[i].SetAxis(0.0, 0.0, 1.0);
    mpMDP.S[i].CalculateParameters(td.C.a, td.Po.p_r);
    std::string pt(part);
    h_LoadCylinderSample(mpMDP, i, (char*)pt.c_str());
    td.S = mpMDP.S[i];
    td.P.N = mpMDP.PN[i];
    td.Compress.VLoad = q->velocity_si / velocity_const;
    if (brazil)
      td.Compress.CalculateBParameters(td.S.size_real, td.S.center_real, td.Po, q->minstress_si / stress_const,
                                       q->maxstrain, q->condfract);
    else
      td.Compress.CalculateUParameters(td.S.size_real, td.S.center_real, td.Po, q->minstress_si / stress_const,
                                       q->maxstrain, q->condfract);
    td.R.dNsave = q->dNsave;
    td.R.fileN = q->fileN;
    auto t0 = std::chrono::steady_clock::now();
    if (brazil)
      h_CalculationBrazilTest(td, mpMDP.h_R[i]);
    else
      h_CalculationUniaxialCompression(td, mpMDP.h_R[i]);
    cudaDeviceSynchronize();
    auto t1 = std::chrono::steady_clock::now();
    out->FractureStress = td.Compress.FractureStress;
    out->FractureStrain = td.Compress.FractureStrain;
    out->LinearityDeviation = td.Compress.LinearityDeviation;
    out->Destruction = td.R.Destruction;
    out->Strain = td.Compress.Strain;
    out->dt = td.Po.dt;
    out->seconds = std::chrono::duration<double>(t1 - t0).count();
    out->N = td.P.N;
    out->stepsave = td.R.stepsave;
    out->steps_hint = 0;
  }
  chk(cudaGetLastError());
  if (chdir(cwd) != 0) return -3;
  return g_err;
}

// CalculateStartParameters (mp_task.h:129-145): weights and the first
// variation table from params[5], goal[4], multiplier[4]; goal updated in place.
int refh_cg_start_parameters(const double* params, double* goal, const double* multiplier, int calc_u, int calc_b,
                             int type, double delta, double* weight, double* variation) {
  mp_task_data t;
  t.NSteps = 2;
  t.NParam = 5;
  t.NResult = 4;
  t.createarrays();
  t.Step = 0;
  t.ParameterVariationType = (uint8_t)type;
  t.MaterialDeltaFactor = delta;
  t.CalculateUTest = calc_u != 0;
  t.CalculateBTest = calc_b != 0;
  for (int i = 0; i < 5; ++i) t.MaterialParametersSteps[i] = params[i];
  for (int j = 0; j < 4; ++j) {
    t.ResultsGoal[j] = goal[j];
    t.FunctionalParametersWeightMultiplier[j] = multiplier[j];
  }
  t.CalculateStartParameters();
  for (int j = 0; j < 4; ++j) {
    goal[j] = t.ResultsGoal[j];
    weight[j] = t.FunctionalParametersWeight[j];
  }
  for (int i = 0; i < 30; ++i) variation[i] = t.ParameterVariation[i];
  return 0;
}

// One conjugate-gradient parameter update of the reference's calibration
// driver: mp_task_data::CalculateNewParameters2 (mp_task.h:223-311) on the
// caller's arrays (NParam = 5, NResult = 4).  In: params[5] (the current
// step's parameters), variation[30] (ParameterVariation), rfun[24]
// (RFunction), goal[4], weight[4] (FunctionalParametersWeight),
// dfun[6] / ddfun[6] (previous gradient and direction), type
// (ParameterVariationType), delta (MaterialDeltaFactor).  Out: new_params[5],
// variation, dfun, ddfun updated in place, functional[4].  Host-only.
int refh_cg_new_parameters2(const double* params, double* variation, const double* rfun, const double* goal,
                            const double* weight, double* dfun, double* ddfun, int type, double delta,
                            double* new_params, double* functional) {
  mp_task_data t;
  t.NSteps = 2;
  t.NParam = 5;
  t.NResult = 4;
  t.createarrays();
  t.Step = 0;
  t.ParameterVariationType = (uint8_t)type;
  t.MaterialDeltaFactor = delta;
  for (int i = 0; i < 5; ++i) t.MaterialParametersSteps[i] = params[i];
  for (int i = 0; i < 30; ++i) t.ParameterVariation[i] = variation[i];
  for (int i = 0; i < 24; ++i) t.RFunction[i] = rfun[i];
  for (int j = 0; j < 4; ++j) {
    t.ResultsGoal[j] = goal[j];
    t.FunctionalParametersWeight[j] = weight[j];
  }
  for (int i = 0; i < 6; ++i) {
    t.dFunctional[i] = dfun[i];
    t.ddFunctional[i] = ddfun[i];
  }
  t.CalculateNewParameters2();
  for (int i = 0; i < 5; ++i) new_params[i] = t.MaterialParametersSteps[5 + i];
  for (int i = 0; i < 30; ++i) variation[i] = t.ParameterVariation[i];
  for (int i = 0; i < 6; ++i) {
    dfun[i] = t.dFunctional[i];
    ddfun[i] = t.ddFunctional[i];
  }
  for (int j = 0; j < 4; ++j) functional[j] = t.Functional[j];
  return 0;
}

// Times the reference's CPU BPM routine h_CalculateForceElastic
// (md_calculateforcesbpm_cpu.cu:20-262, declared md.h:134) on one host thread:
// one call per directed bonded slot (i -> j and j -> i for every bond of bi/bj),
// repeated over the bond list until at least min_seconds have passed.  The
// routine prints several lines per call (printf and std::cerr), so stdout and
// stderr are sent to /dev/null for the timed loop and restored afterwards.  Slot state starts as a fresh bond:
// previous direction = current direction, 1/L0 from the positions, zero
// histories; br is the bond radius per bond, the axial moment pi br^4 / 2.
// Returns the directed-slot evaluations per second and the seconds spent.
int refh_time_bpm_cpu(const float* R, const float* V, const float* W, uint32_t N, const uint32_t* bi,
                      const uint32_t* bj, const float* br, uint32_t nb, float dt, float m_E, float m_G, float Gcn,
                      float Gct, double min_seconds, double* evals_per_s, double* seconds) {
  if (!R || !V || !W || !bi || !bj || !br || nb == 0 || N == 0) return -1;
  const size_t ns = 2 * (size_t)nb;
  std::vector<float> F(3 * (size_t)N, 0.f), M(3 * (size_t)N, 0.f), ab_r(ns), inv_l(ns), axial(ns);
  std::vector<float3> Rij(ns), Ot(ns), Mn(ns), Mt(ns), Fij(ns);
  std::vector<uint32_t> idx(ns), jdx(ns);
  for (size_t b = 0; b < nb; ++b) {
    for (int d = 0; d < 2; ++d) {
      const size_t k = 2 * b + d;
      const uint32_t i = d ? bj[b] : bi[b], j = d ? bi[b] : bj[b];
      idx[k] = i;
      jdx[k] = j;
      const float x = R[j] - R[i], y = R[j + N] - R[i + N], z = R[j + 2 * N] - R[i + 2 * N];
      const float r = std::sqrt(x * x + y * y + z * z);
      const float ir = r > 0.f ? 1.f / r : 0.f;
      Rij[k] = make_float3(x * ir, y * ir, z * ir);
      inv_l[k] = ir;
      ab_r[k] = br[b];
      axial[k] = 0.5f * 3.14159265f * br[b] * br[b] * br[b] * br[b];
      Ot[k] = Mn[k] = Mt[k] = Fij[k] = make_float3(0.f, 0.f, 0.f);
    }
  }
  fflush(stdout);
  fflush(stderr);
  const int saved = dup(1), saved2 = dup(2);
  const int devnull = open("/dev/null", O_WRONLY);
  if (saved < 0 || saved2 < 0 || devnull < 0) return -2;
  dup2(devnull, 1);
  dup2(devnull, 2);
  size_t calls = 0;
  const auto t0 = std::chrono::steady_clock::now();
  double el = 0.0;
  do {
    for (size_t k = 0; k < ns; ++k)
      h_CalculateForceElastic(R, V, W, F.data(), M.data(), ab_r.data(), inv_l.data(), axial.data(), Rij.data(),
                              Ot.data(), Mn.data(), Mt.data(), Fij.data(), N, idx[k], jdx[k], (uint)k, dt, m_E,
                              m_G, Gcn, Gct, 1u);
    calls += ns;
    el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  } while (el < min_seconds);
  fflush(stdout);
  fflush(stderr);
  dup2(saved, 1);
  dup2(saved2, 2);
  close(saved);
  close(saved2);
  close(devnull);
  *evals_per_s = (double)calls / el;
  *seconds = el;
  return 0;
}

}  // extern "C"
