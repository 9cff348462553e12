// Seeded sample creation: random fill of a cylinder (disc or column), radius
// growth with damped soft-sphere relaxation, then FIRE relaxation of the
// remaining overlaps - the role of the reference's h_CreateCylinderSample
// (md_createcylindersample.cu:184-439), whose cuRAND fill is seeded with
// time(NULL); here every draw comes from the caller's seed.  All relaxation
// work runs on the device; the host only schedules stages and reads the
// largest overlap every few steps.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "b200dem.h"
#include "dem_build.cuh"
#include "dem_engine.h"
#include "dem_pack.cuh"
#include "dem_params.h"

namespace dem {
namespace {

template <class T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  ~Buf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t k) {
    if (p) cudaFree(p);
    p = nullptr;
    n = k;
    if (!k) return cudaSuccess;
    cudaError_t e = cudaMalloc((void**)&p, k * sizeof(T));
    if (e) return e;
    // zero-filled before returning: the fill runs on the legacy default
    // stream, which is not ordered with the packer's non-blocking stream
    e = cudaMemsetAsync(p, 0, k * sizeof(T), 0);
    return e ? e : cudaStreamSynchronize(0);
  }
};

#define CKP(x)                                 \
  do {                                         \
    cudaError_t e_ = (x);                      \
    if (e_ != cudaSuccess) {                   \
      note_cuda_error(e_, __FILE__, __LINE__); \
      return DEM_ERR_CUDA;                     \
    }                                          \
  } while (0)

uint32_t cdiv(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

struct Rng {
  uint64_t s;
  double uniform() {
    s = splitmix64(s);
    return u01_from(s);
  }
};

class Packer {
 public:
  explicit Packer(const dem_pack_params& p) : P(p) {}

  int run(float* xyz, float* radii, uint32_t cap, uint32_t* n_out, dem_pack_report* rep) {
    n_ = P.n;
    CKP(cudaSetDevice(P.device));
    CKP(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, P.device);
    nsm = (uint32_t)sms;
    const uint32_t n = n_;
    if (n == 0 || n > cap || !(P.r_max >= P.r_min) || !(P.r_min > 0) || !(P.radius > P.r_max) ||
        !(P.half_height > P.r_max))
      return DEM_ERR_ARG;
    // radii and a uniform fill of the cylinder (particle centres inside R - r, H - r)
    Rng rng{P.seed ^ 0x5DEECE66Dull};
    std::vector<float4> hp(n);
    std::vector<float4> hv(n);
    const double rho = P.rho > 0 ? P.rho : 2.65;
    // the reference's time step for the smallest particle (potential_data::CalculateParameters)
    const double dt0 = 0.05 * rayleigh_time(P.r_min, rho, P.E, P.nu);
    for (uint32_t i = 0; i < n; ++i) {
      const double r = P.r_min + (P.r_max - P.r_min) * rng.uniform();
      double x, y;
      do {
        x = 2 * rng.uniform() - 1;
        y = 2 * rng.uniform() - 1;
      } while (x * x + y * y > 1.0);
      const double Rin = P.radius - r, Hin = P.half_height - r;
      const double z = (2 * rng.uniform() - 1) * Hin;
      hp[i] = make_float4((float)(P.center[0] + x * Rin), (float)(P.center[1] + y * Rin), (float)(P.center[2] + z),
                          (float)r);
      double m, dtm, dtI;
      particle_constants(r, rho, dt0, m, dtm, dtI);
      hv[i] = make_float4(0.f, 0.f, 0.f, (float)dtm);
    }
    CKP(pos.alloc(n));
    CKP(vel.alloc(n));
    CKP(frc.alloc(n));
    CKP(frcq.alloc(4 * (size_t)n));
    CKP(cudaMemsetAsync(frcq.p, 0, 4 * (size_t)n * sizeof(long long), st));
    CKP(part.alloc(3 * (size_t)nsm * 8));
    CKP(ref.alloc(n));
    CKP(sid.alloc(n));
    CKP(cudaMemcpy(pos.p, hp.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    CKP(cudaMemcpy(vel.p, hv.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    // grid over the cylinder
    skin = 0.5 * P.r_min;
    const double a = (2.0 * P.r_max + skin) * 1.0001;
    Grid<float> g;
    g.ox = (float)(P.center[0] - P.radius - a);
    g.oy = (float)(P.center[1] - P.radius - a);
    g.oz = (float)(P.center[2] - P.half_height - a);
    g.inv_a = (float)(1.0 / a);
    g.nx = (uint32_t)std::ceil((2 * P.radius + 2 * a) / a) + 1;
    g.ny = g.nx;
    g.nz = (uint32_t)std::ceil((2 * P.half_height + 2 * a) / a) + 1;
    g.off = 0;
    g.hx = g.hy = g.hz = 0.f;
    g.skip_hidden = 0;  // nothing is parked while packing
    ncell = g.nx * g.ny * g.nz;
    CKP(grid.alloc(1));
    CKP(cudaMemcpy(grid.p, &g, sizeof(g), cudaMemcpyHostToDevice));
    CKP(cell_of.alloc(n));
    CKP(cell_count.alloc(ncell + 1));
    CKP(cell_start.alloc(ncell + 1));
    CKP(cursor.alloc(ncell + 1));
    CKP(cell_list.alloc(n));
    CKP(cnt.alloc(n + 1));
    CKP(offs.alloc(n + 1));
    CKP(brow.alloc(n + 1));
    CKP(ovf.alloc(1));
    CKP(nc_dev.alloc(1));
    CKP(skin_d.alloc(1));
    CKP(cudaMemcpy(skin_d.p, &skin, sizeof(double), cudaMemcpyHostToDevice));
    CKP(scale.alloc(1));
    CKP(Dk.alloc(1));
    CKP(cyl.alloc(5));
    const float cy[5] = {(float)P.center[0], (float)P.center[1], (float)P.center[2], (float)P.radius,
                         (float)P.half_height};
    CKP(cudaMemcpy(cyl.p, cy, sizeof(cy), cudaMemcpyHostToDevice));
    CKP(fire.alloc(1));
    CKP(povl.alloc(n));
    CKP(blocks_done.alloc(1));
    CKP(scan_tmp.alloc(2 * cdiv(std::max(ncell, n), kScanBlock) + 2048));
    // linear repulsion stiffness ~ E * r (force per overlap)
    const double k = P.E * 0.5 * (P.r_min + P.r_max);
    const float kf = (float)k;
    CKP(cudaMemcpy(Dk.p, &kf, sizeof(float), cudaMemcpyHostToDevice));
    FireCtl F{};
    F.dt0 = dt0;
    F.dt = dt0;
    F.dtgrow = 1.1;
    F.dtshrink = 0.5;
    F.alphashrink = 0.99;
    F.Ndelay = 20;
    F.variant = P.fire_variant == 1 ? 1u : 0u;
    if (F.variant == 1) {
      F.dtmax = 100.0 * dt0;  // SetFIREData, md_firerelaxation.cu:74-86
      F.dtmin = 0.001 * dt0;
      F.alpha0 = 0.1;
    } else {
      // FIRE 2.0 defaults scaled to this time step: dt0 is about a tenth of the
      // stability limit of the stiffest particle, so dt stays within 4 dt0
      F.dtmax = 4.0 * dt0;
      F.dtmin = 0.02 * dt0;
      F.alpha0 = 0.25;
    }
    F.alpha = F.alpha0;
    CKP(cudaMemcpy(fire.p, &F, sizeof(F), cudaMemcpyHostToDevice));
    // radius growth: from the scale whose packing fraction is 30% of the final
    // one to 1, with damped relaxation after every increment
    const uint32_t stages = std::max(1u, P.growth_stages);
    const double s0 = std::cbrt(0.3);
    const double m_mean = rho * 4.0 / 3.0 * kPiD * std::pow(0.5 * (P.r_min + P.r_max), 3);
    const float vis = (float)(2.0 * std::sqrt(k * m_mean) * 0.5);  // about half of critical damping
    uint64_t steps = 0;
    for (uint32_t sg = 1; sg <= stages; ++sg) {
      const float s = (float)(s0 + (1.0 - s0) * sg / stages);
      CKP(cudaMemcpy(scale.p, &s, sizeof(float), cudaMemcpyHostToDevice));
      int rc = relax(true, vis, P.steps_per_stage, 0.0, steps);
      if (rc) return rc;
    }
    // FIRE on the final radii until the largest overlap is below the tolerance
    float one = 1.0f;
    CKP(cudaMemcpy(scale.p, &one, sizeof(float), cudaMemcpyHostToDevice));
    int rc = relax(false, 0.f, P.max_fire_steps, P.overlap_tol, steps);
    if (rc) return rc;
    // the reference's d_ReduceParticleNumber (md_reduceparticlenumber.cu:18-38,
    // md_createcylindersample.cu:323-338, 402-417): while the largest overlap
    // stays above the tolerance, remove the spheres of the worst overlaps and
    // relax again
    uint32_t removed = 0;
    while (P.max_removed && last_overlap >= P.overlap_tol && removed < P.max_removed) {
      const uint32_t before = removed;
      rc = remove_worst(P.max_removed - removed, removed);
      if (rc) return rc;
      if (removed == before) break;
      rc = relax(false, 0.f, std::max(P.max_fire_steps / 4, 500u), P.overlap_tol, steps);
      if (rc) return rc;
    }
    // results (the spheres kept, first nf entries of each SoA block)
    const uint32_t nf = n_;
    hp.resize(nf);
    CKP(cudaMemcpy(hp.data(), pos.p, nf * sizeof(float4), cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < nf; ++i) {
      xyz[i] = hp[i].x;
      xyz[nf + i] = hp[i].y;
      xyz[2 * nf + i] = hp[i].z;
      if (radii) radii[i] = hp[i].w;
    }
    *n_out = nf;
    if (rep) {
      std::memset(rep, 0, sizeof(*rep));
      rep->steps = steps;
      rep->max_overlap = last_overlap;
      double vs = 0;
      for (uint32_t i = 0; i < nf; ++i) vs += 4.0 / 3.0 * kPiD * std::pow((double)hp[i].w, 3);
      rep->packing_fraction = vs / (kPiD * P.radius * P.radius * 2.0 * P.half_height);
      rep->rebuilds = rebuilds;
      rep->removed = removed;
    }
    cudaStreamDestroy(st);
    return DEM_OK;
  }

 private:
  int scan(const uint32_t* in, uint32_t* out, uint32_t m) {
    const uint32_t nb = cdiv(m, kScanBlock);
    uint32_t* sums = scan_tmp.p;
    uint32_t* ss = scan_tmp.p + nb + 1024;
    if (nb > kScanBlock) return DEM_ERR_CAPACITY;
    k_scan_block<<<std::max(nb, 1u), kScanBlock, 0, st>>>(in, out, m, sums);
    if (nb > 1) {
      k_scan_block<<<1, kScanBlock, 0, st>>>(sums, ss, nb, nullptr);
      k_scan_add<<<nb, kScanBlock, 0, st>>>(out, m, ss);
    }
    k_scan_total<<<1, 1, 0, st>>>(in, out, m);
    return DEM_OK;
  }

  // Removes up to `budget` spheres (at most 0.1% of them per round, worst
  // first): of the spheres whose largest overlap in the last step is above the
  // tolerance, every second one in order of that overlap - both spheres of a
  // pair carry its overlap - by compacting the arrays.
  int remove_worst(uint32_t budget, uint32_t& removed) {
    const uint32_t n = n_;
    std::vector<float> ov(n);
    CKP(cudaMemcpy(ov.data(), povl.p, n * sizeof(float), cudaMemcpyDeviceToHost));
    std::vector<uint32_t> cand;
    for (uint32_t i = 0; i < n; ++i)
      if (ov[i] >= P.overlap_tol) cand.push_back(i);
    if (cand.empty()) return DEM_OK;
    std::stable_sort(cand.begin(), cand.end(), [&](uint32_t a, uint32_t b) { return ov[a] > ov[b]; });
    uint32_t k = (uint32_t)std::max<size_t>(1, cand.size() / 2);
    k = std::min<uint32_t>({k, budget, std::max(1u, n / 1000)});
    std::vector<uint8_t> gone(n, 0);
    for (uint32_t q = 0, t = 0; q < cand.size() && t < k; q += 2, ++t) gone[cand[q]] = 1;
    std::vector<float4> hp(n), hv(n);
    CKP(cudaMemcpy(hp.data(), pos.p, n * sizeof(float4), cudaMemcpyDeviceToHost));
    CKP(cudaMemcpy(hv.data(), vel.p, n * sizeof(float4), cudaMemcpyDeviceToHost));
    uint32_t m = 0;
    for (uint32_t i = 0; i < n; ++i)
      if (!gone[i]) {
        hp[m] = hp[i];
        hv[m] = make_float4(0.f, 0.f, 0.f, hv[i].w);
        ++m;
      }
    removed += n - m;
    n_ = m;
    CKP(cudaMemcpy(pos.p, hp.data(), m * sizeof(float4), cudaMemcpyHostToDevice));
    CKP(cudaMemcpy(vel.p, hv.data(), m * sizeof(float4), cudaMemcpyHostToDevice));
    CKP(cudaMemsetAsync(frc.p, 0, n * sizeof(float4), st));
    CKP(cudaMemsetAsync(frcq.p, 0, 4 * (size_t)n * sizeof(long long), st));
    return DEM_OK;
  }

  int rebuild() {
    const uint32_t n = n_;
    const uint32_t g1 = std::max(1u, std::min(cdiv(n, 256), nsm * 16));
    CKP(cudaMemsetAsync(cell_count.p, 0, (ncell + 1) * sizeof(uint32_t), st));
    k_cell_index<float><<<g1, 256, 0, st>>>(pos.p, sid.p, n, grid.p, cell_of.p, cell_count.p);
    int rc = scan(cell_count.p, cell_start.p, ncell);
    if (rc) return rc;
    CKP(cudaMemcpyAsync(cursor.p, cell_start.p, (ncell + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    k_scatter_cells<<<g1, 256, 0, st>>>(cell_of.p, n, cursor.p, cell_list.p);
    k_sort_cells<<<std::max(1u, std::min(cdiv(ncell, 256), nsm * 16)), 256, 0, st>>>(cell_start.p, ncell,
                                                                                      cell_list.p);
    PairSearch<float> S{};
    S.pos = pos.p;
    S.sid = sid.p;
    S.np = n;
    S.grids = grid.p;
    S.cell_start = cell_start.p;
    S.cell_list = cell_list.p;
    S.mode = kModeContact;
    S.gap = skin_d.p;
    S.b_row = brow.p;  // no bonds: all rows empty
    S.b_ij = nullptr;
    S.count = cnt.p;
    S.offset = offs.p;
    S.cap = 48;
    S.overflow = ovf.p;
    CKP(cudaMemsetAsync(ovf.p, 0, sizeof(uint32_t), st));
    // one search pass (counts and sorted partners in kSearchStride slots per
    // sphere), compacted once the counts are scanned
    if (js.n < (size_t)n * kSearchStride) CKP(js.alloc((size_t)n * kSearchStride));
    S.out_j = js.p;
    k_pair_search<float, 2><<<pair_search_blocks(n), 128, 0, st>>>(S);
    rc = scan(cnt.p, offs.p, n);
    if (rc) return rc;
    uint32_t nc = 0, o = 0;
    CKP(cudaMemcpyAsync(&nc, offs.p + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CKP(cudaMemcpyAsync(&o, ovf.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CKP(cudaStreamSynchronize(st));
    if (o) return DEM_ERR_CAPACITY;
    if (nc + 1 > cij.n) CKP(cij.alloc(nc + nc / 2 + 1024));
    k_expand_stride<<<g1, 256, 0, st>>>(offs.p, n, js.p, cij.p);
    CKP(cudaMemcpyAsync(nc_dev.p, &nc, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    k_copy_pos<float><<<g1, 256, 0, st>>>(pos.p, ref.p, n);
    CKP(cudaGetLastError());
    ++rebuilds;
    return DEM_OK;
  }

  // Relaxation loop.  The pair list holds every pair within r_i + r_j + skin
  // of the final radii; it is rebuilt when a particle has moved more than a
  // quarter of the skin since the last build.  Chunks of steps between host
  // checks are sized so that the fastest particle of the previous chunk cannot
  // use up the rest of that quarter.
  int relax(bool viscous, float vis, uint32_t max_steps, double tol, uint64_t& steps) {
    const uint32_t n = n_;
    PackArgs<float> A{};
    A.pos = pos.p;
    A.vel = vel.p;
    A.frc = frc.p;
    A.frcq = frcq.p;
    A.part = part.p;
    A.ref = ref.p;
    A.sid = sid.p;
    A.np = n;
    A.nc = nc_dev.p;
    A.scale = scale.p;
    A.D = Dk.p;
    A.linear = 1;
    A.fire = fire.p;
    A.povl = P.max_removed ? povl.p : nullptr;
    A.cyl = cyl.p;
    A.nsamples = 1;
    A.blocks_done = blocks_done.p;
    A.viscous = viscous ? 1 : 0;
    A.vis = vis;
    const uint32_t gp = nsm * 8, gn = std::max(1u, std::min(cdiv(n, 256), nsm * 8));
    const double quarter = 0.25 * skin;
    const uint32_t kMaxChunk = 50;
    uint32_t done = 0;
    bool need_build = true;
    FireCtl F{};
    CKP(cudaMemcpyAsync(&F, fire.p, sizeof F, cudaMemcpyDeviceToHost, st));
    CKP(cudaStreamSynchronize(st));
    double vmax = 0.0, dmax = 0.0;
    while (done < max_steps) {
      if (need_build || dmax > quarter) {
        int rc = rebuild();
        if (rc) return rc;
        dmax = 0.0;
        need_build = false;
      }
      A.c_ij = cij.p;
      const double dt_bound = viscous ? F.dt0 : F.dtmax;
      uint32_t m = kMaxChunk;
      if (vmax > 0.0) {
        const double k = 0.5 * (quarter - dmax) / (vmax * dt_bound);
        m = (uint32_t)std::max(1.0, std::min((double)kMaxChunk, std::floor(k)));
      } else {
        m = std::min<uint32_t>(10, kMaxChunk);
      }
      m = std::min(m, max_steps - done);
      const float z = 0.f;
      CKP(cudaMemcpyAsync(&fire.p->vmax2, &z, sizeof(float), cudaMemcpyHostToDevice, st));
      for (uint32_t k = 0; k < m; ++k) {
        if (k == m - 1) {
          CKP(cudaMemcpyAsync(&fire.p->max_overlap, &z, sizeof(float), cudaMemcpyHostToDevice, st));
          CKP(cudaMemcpyAsync(&fire.p->dmax2, &z, sizeof(float), cudaMemcpyHostToDevice, st));
          if (A.povl) CKP(cudaMemsetAsync(povl.p, 0, n * sizeof(float), st));
        }
        k_soft_pairs<float><<<gp, 256, 0, st>>>(A);
        k_fire_power<float><<<gn, 256, 0, st>>>(A);
        k_fire_move<float><<<gn, 256, 0, st>>>(A);
      }
      CKP(cudaGetLastError());
      CKP(cudaMemcpyAsync(&F, fire.p, sizeof F, cudaMemcpyDeviceToHost, st));
      CKP(cudaStreamSynchronize(st));
      last_overlap = F.max_overlap;
      vmax = std::sqrt((double)F.vmax2);
      dmax = std::sqrt((double)F.dmax2);
      done += m;
      steps += m;
      if (tol > 0 && F.max_overlap < tol) break;
    }
    return DEM_OK;
  }

  dem_pack_params P;
  cudaStream_t st = nullptr;
  uint32_t nsm = 148, ncell = 0, n_ = 0;
  double skin = 0;
  float last_overlap = 0.f;
  uint32_t rebuilds = 0;
  Buf<float4> pos, vel, frc, ref;
  Buf<long long> frcq;
  Buf<double> part;
  Buf<uint32_t> sid, cell_of, cell_count, cell_start, cursor, cell_list, cnt, offs, brow, ovf, nc_dev, js, scan_tmp;
  Buf<uint2> cij;
  Buf<Grid<float>> grid;
  Buf<double> skin_d;
  Buf<float> scale, Dk, cyl, povl;
  Buf<FireCtl> fire;
  Buf<unsigned int> blocks_done;
};

}  // namespace
}  // namespace dem

extern "C" int dem_create_cylinder_sample(const dem_pack_params* p, float* xyz, float* radii, uint32_t cap,
                                          uint32_t* n, dem_pack_report* rep) {
  if (!p || !xyz || !n) return DEM_ERR_ARG;
  try {
    dem::Packer pk(*p);
    return pk.run(xyz, radii, cap, n, rep);
  } catch (...) {
    return DEM_ERR_STATE;
  }
}
