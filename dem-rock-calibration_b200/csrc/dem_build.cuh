// Set-up and rebuild kernels of the B200 DEM engine: cell binning as a stable
// counting sort, an exclusive scan, and a 27-cell pair search used for three
// pair sets (the reference's interaction sets, the bond list, the contact
// list).  They replace the reference's CellDistribution
// (md_cell_distribution.cu:130-172 with CUB radix sort), its cell pointer scan
// (md_calculate_cell.cu:43-75), d_ConstructInteractionList / the BPM rebuild
// (md_interaction_list_construct.cu, md_interaction_list_reconstructbpm.cu) and
// d_ConstructBoundInteractions (md_boundinteractions_construct.cu:35-106).
#pragma once

#include "dem_common.cuh"
#include "dem_params.h"
#include "dem_types.h"

namespace dem {

// Uniform cell grid of one sample: cell (ix,iy,iz) = floor((x - origin) / a),
// global id = off + ix + iy*nx + iz*nx*ny.  With origin 0 and the reference's
// edge this is the reference's cell numbering (md_calculate_cell.cu:24-35).
template <class Real>
struct Grid {
  Real ox, oy, oz, inv_a;
  uint32_t nx, ny, nz, off;
  // the sample's hidden point: escaped particles are all parked there and,
  // when skip_hidden is set, take part in no pair search (they interact with
  // nothing anyway, and thousands of them in one cell would make the search
  // quadratic)
  Real hx, hy, hz;
  uint32_t skip_hidden;
};

template <class Real, class V>
__device__ __forceinline__ bool at_hidden(const Grid<Real>& g, const V& x) {
  return g.skip_hidden && x.x == g.hx && x.y == g.hy && x.z == g.hz;
}

template <class Real>
__device__ __forceinline__ uint32_t cell_coord(Real x, Real o, Real inv_a, uint32_t n) {
  const Real f = floor((x - o) * inv_a);
  if (!(f > Real(0))) return 0u;
  const uint32_t u = (uint32_t)f;
  return u < n ? u : n - 1u;
}

template <class Real>
__global__ void k_cell_index(const typename RT<Real>::V4* __restrict__ pos, const uint32_t* __restrict__ sid,
                             uint32_t np, const Grid<Real>* __restrict__ grids, uint32_t* __restrict__ cell_of,
                             uint32_t* __restrict__ cell_count) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
    const auto x = ld4(pos + p);
    const Grid<Real> g = grids[sid[p]];
    const uint32_t ix = cell_coord<Real>(x.x, g.ox, g.inv_a, g.nx);
    const uint32_t iy = cell_coord<Real>(x.y, g.oy, g.inv_a, g.ny);
    const uint32_t iz = cell_coord<Real>(x.z, g.oz, g.inv_a, g.nz);
    const uint32_t c = g.off + ix + iy * g.nx + iz * g.ny * g.nx;
    cell_of[p] = c;
    atomicAdd(cell_count + c, 1u);
  }
}

// --- exclusive scan of uint32 (three passes, recursive over block sums)
constexpr int kScanBlock = 1024;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31) >= (unsigned)o) v += t;
  }
  return v;
}

// each block scans kScanBlock elements; block totals go to sums[blockIdx]
static __global__ void __launch_bounds__(kScanBlock) k_scan_block(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                          uint32_t n, uint32_t* __restrict__ sums) {
  __shared__ uint32_t warp_tot[32];
  const uint32_t i = blockIdx.x * kScanBlock + threadIdx.x;
  const uint32_t v = i < n ? in[i] : 0u;
  const uint32_t inc = warp_incl_scan(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 31) warp_tot[w] = inc;
  __syncthreads();
  if (w == 0) {
    const uint32_t t = warp_incl_scan(warp_tot[lane]);
    warp_tot[lane] = t;
  }
  __syncthreads();
  const uint32_t base = w > 0 ? warp_tot[w - 1] : 0u;
  if (i < n) out[i] = base + inc - v;  // exclusive
  if (threadIdx.x == kScanBlock - 1 && sums) sums[blockIdx.x] = base + inc;
}

static __global__ void k_scan_add(uint32_t* __restrict__ out, uint32_t n, const uint32_t* __restrict__ offs) {
  const uint32_t i = blockIdx.x * kScanBlock + threadIdx.x;
  if (i < n && blockIdx.x > 0) out[i] += offs[blockIdx.x];
}

// out[n] receives the total
static __global__ void k_scan_total(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t n) {
  if (threadIdx.x == 0 && blockIdx.x == 0) out[n] = (n ? out[n - 1] + in[n - 1] : 0u);
}

static __global__ void k_scatter_cells(const uint32_t* __restrict__ cell_of, uint32_t np, uint32_t* __restrict__ cursor,
                                uint32_t* __restrict__ cell_list) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
    const uint32_t slot = atomicAdd(cursor + cell_of[p], 1u);
    cell_list[slot] = p;
  }
}

// Restore ascending particle order inside each cell, so the binning equals a
// stable sort of (cell, particle) pairs (the reference's CUB radix sort).
static __global__ void k_sort_cells(const uint32_t* __restrict__ cell_start, uint32_t ncell, uint32_t* __restrict__ cell_list) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
    const uint32_t b = cell_start[c], e = cell_start[c + 1];
    for (uint32_t k = b + 1; k < e; ++k) {
      const uint32_t v = cell_list[k];
      uint32_t q = k;
      while (q > b && cell_list[q - 1] > v) {
        cell_list[q] = cell_list[q - 1];
        --q;
      }
      cell_list[q] = v;
    }
  }
}

// --- per-particle state at set-up, built on the device from the caller's
// arrays: stage = [x | y | z | r | perm] of all samples (each sample's block
// of x (and y, z, r, perm) at its p_begin, caller order, perm[k] = the
// caller index stored at position p_begin + k); integration constants with the
// host's double formulas (particle_constants), so the values are those the
// host would compute.
struct InitSample {
  uint32_t p_begin, n;
  double m_ro, dt;
};

template <class Real>
__global__ void k_init_particles(const float* __restrict__ stage, uint32_t np, const InitSample* __restrict__ smp,
                                 uint32_t nsamples, typename RT<Real>::V4* __restrict__ pos,
                                 typename RT<Real>::V4* __restrict__ vel, typename RT<Real>::V4* __restrict__ omg,
                                 Real* __restrict__ mass, uint32_t* __restrict__ sid, uint32_t* __restrict__ orig) {
  const float* X = stage;
  const float* Y = stage + np;
  const float* Z = stage + 2 * (size_t)np;
  const float* R = stage + 3 * (size_t)np;
  const uint32_t* P = reinterpret_cast<const uint32_t*>(stage + 4 * (size_t)np);
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
    // the sample of position p: the last one with p_begin <= p
    uint32_t lo = 0, hi = nsamples;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (smp[mid].p_begin <= p) lo = mid;
      else hi = mid;
    }
    const InitSample S = smp[lo];
    const uint32_t q = P[p];                  // caller index within the sample
    const size_t c = (size_t)S.p_begin + q;  // its entry in the stage
    const double r = (double)R[c];
    double m, dtm, dtI;
    particle_constants(r, S.m_ro, S.dt, m, dtm, dtI);
    typename RT<Real>::V4 v4;
    v4.x = (Real)X[c];
    v4.y = (Real)Y[c];
    v4.z = (Real)Z[c];
    v4.w = (Real)R[c];
    pos[p] = v4;
    v4.x = v4.y = v4.z = Real(0);
    v4.w = (Real)dtm;
    vel[p] = v4;
    v4.w = (Real)dtI;
    omg[p] = v4;
    mass[p] = (Real)m;
    sid[p] = lo;
    orig[p] = q;
  }
}

// out[k] = src[idx[k]]
static __global__ void k_gather_u32(const uint32_t* __restrict__ src, const uint32_t* __restrict__ idx, uint32_t n,
                                    uint32_t* __restrict__ out) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) out[k] = src[idx[k]];
}

// --- Morton order of the particles at set-up (device)

// Interleaves the low 21 bits of x, y, z (x in bit 0).
__host__ __device__ inline uint64_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  auto spread = [](uint64_t v) {
    v &= 0x1FFFFF;
    v = (v | v << 32) & 0x1F00000000FFFFull;
    v = (v | v << 16) & 0x1F0000FF0000FFull;
    v = (v | v << 8) & 0x100F00F00F00F00Full;
    v = (v | v << 4) & 0x10C30C30C30C30C3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
  };
  return spread(x) | (spread(y) << 1) | (spread(z) << 2);
}

// Quantisation frame of one sample: lower corner of its particles and 1/r_min.
struct MortonFrame {
  double lo[3];
  double inv_q;
  uint32_t p_begin, n;
};

// Key of set-up position p (the caller's order, samples one after another):
// the sample's index above mbits, below it the Morton code of the position
// quantised by r_min from the sample's lower corner (the host rule, bit for
// bit); idx[p] = p.
static __global__ void k_morton_keys(const float* __restrict__ stage, uint32_t np, const MortonFrame* __restrict__ fr,
                              uint32_t nsamples, int mbits, uint64_t* __restrict__ keys, uint32_t* __restrict__ idx) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = nsamples;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (fr[mid].p_begin <= p) lo = mid;
      else hi = mid;
    }
    const MortonFrame F = fr[lo];
    uint32_t c[3];
    for (int d = 0; d < 3; ++d) {
      const double v = ((double)stage[(size_t)d * np + p] - F.lo[d]) * F.inv_q;
      c[d] = (uint32_t)fmin(fmax(v, 0.0), 2097151.0);
    }
    keys[p] = ((uint64_t)lo << mbits) | morton3(c[0], c[1], c[2]);
    idx[p] = p;
  }
}

// Stable LSD radix sort of (key, index) pairs, 8-bit digits: each block owns a
// contiguous run of kSortItems items.  Pass 1 counts the block's digits
// (hist[digit * blocks + block]); after an exclusive scan of hist, pass 2
// scatters the block's items tile by tile in input order (within a tile a
// warp match ranks equal digits by lane, warps are ranked by index), so equal
// keys keep their input order.
constexpr uint32_t kSortItems = 4096;

static __global__ void __launch_bounds__(256) k_radix_hist(const uint64_t* __restrict__ keys, uint32_t n, int shift,
                                                    uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t i0 = blockIdx.x * kSortItems, i1 = min(n, i0 + kSortItems);
  for (uint32_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) atomicAdd(&h[(uint32_t)(keys[i] >> shift) & 255u], 1u);
  __syncthreads();
  hist[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = h[threadIdx.x];
}

static __global__ void __launch_bounds__(256) k_radix_scatter(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                       uint32_t n, int shift, const uint32_t* __restrict__ offs,
                                                       uint64_t* __restrict__ kout, uint32_t* __restrict__ vout) {
  __shared__ uint32_t base[256];     // next output slot of each digit for this block
  __shared__ uint32_t wcnt[8][256];  // per warp: digit counts, then the digit's offset of the warp in the tile
  __shared__ uint32_t tot[256];      // digit counts of the tile
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  base[threadIdx.x] = offs[(size_t)threadIdx.x * gridDim.x + blockIdx.x];
  const uint32_t i0 = blockIdx.x * kSortItems, i1 = min(n, i0 + kSortItems);
  for (uint32_t t0 = i0; t0 < i1; t0 += 256) {
    for (uint32_t w = 0; w < 8; ++w) wcnt[w][threadIdx.x] = 0;
    __syncthreads();
    const uint32_t i = t0 + threadIdx.x;
    const bool ok = i < i1;
    const uint64_t k = ok ? kin[i] : 0ull;
    const uint32_t v = ok ? vin[i] : 0u;
    const uint32_t dg = ok ? ((uint32_t)(k >> shift) & 255u) : 256u;   // 256: no item
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, dg);
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    if (ok && rank == 0) wcnt[warp][dg] = __popc(peers);
    __syncthreads();
    {
      uint32_t run = 0;
      for (uint32_t w = 0; w < 8; ++w) {
        const uint32_t c = wcnt[w][threadIdx.x];
        wcnt[w][threadIdx.x] = run;
        run += c;
      }
      tot[threadIdx.x] = run;
    }
    __syncthreads();
    if (ok) {
      const uint32_t o = base[dg] + wcnt[warp][dg] + rank;
      kout[o] = k;
      vout[o] = v;
    }
    __syncthreads();
    base[threadIdx.x] += tot[threadIdx.x];
    __syncthreads();
  }
}

// Storage position k holds set-up position idx[k]: the caller index within its
// sample (the stage's order slot, read by k_init_particles).
static __global__ void k_morton_perm(const uint32_t* __restrict__ idx, uint32_t np, const MortonFrame* __restrict__ fr,
                              uint32_t nsamples, uint32_t* __restrict__ perm) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = nsamples;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (fr[mid].p_begin <= k) lo = mid;
      else hi = mid;
    }
    perm[k] = idx[k] - fr[lo].p_begin;
  }
}

// --- pair search over the 27 surrounding cells
enum PairMode : int {
  kModeRefSet = 0,  // reference interaction set: j != i, r^2 < add && !(r^2 > del) && !(r^2 < 1e-10)
  kModeBond = 1,    // bonds: j > i, 1e-10 <= r^2 < (r_i + r_j + gap)^2
  kModeContact = 2  // contacts: j > i, not bonded, 1e-10 < r^2 < (r_i + r_j + skin)^2
};

template <class Real>
struct PairSearch {
  using V4 = typename RT<Real>::V4;
  const V4* pos;
  const uint32_t* sid;
  uint32_t np;
  const Grid<Real>* grids;
  const uint32_t* cell_start;  // ncell + 1
  const uint32_t* cell_list;
  int mode;
  Real add_thr, del_thr;  // kModeRefSet thresholds (squared)
  const double* gap;      // per sample: bond gap (kModeBond) or skin (kModeContact)
  const uint32_t* b_row;  // kModeContact: bonds of i (CSR over i, j > i, sorted)
  const uint2* b_ij;
  uint32_t* count;        // count pass output (per particle)
  const uint32_t* offset; // fill pass input (per particle)
  uint32_t* out_j;        // fill: partner indices (kModeRefSet: np*cap slots)
  uint32_t cap;           // max pairs per particle kept in registers / slots
  uint32_t* overflow;     // number of particles whose pairs exceeded cap
  const uint32_t* done;   // kModeContact, optional: per sample 1 = finished (its contacts are not listed)
};

template <class Real>
__device__ __forceinline__ bool pair_pred(const PairSearch<Real>& S, uint32_t i, uint32_t j, const typename RT<Real>::V4& xi,
                                          const typename RT<Real>::V4& xj, uint32_t s) {
  const Real dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
  const Real rr = (dx * dx + dy * dy) + dz * dz;
  if (S.mode == kModeRefSet) {
    return j != i && rr < S.add_thr && !(rr > S.del_thr) && !(rr < Real(1e-10));
  }
  if (j <= i) return false;
  if (S.mode == kModeBond) {
    const double r = (double)xi.w + (double)xj.w + (double)S.gap[s];
    // (a gap below -(r_i + r_j) bonds nothing; squaring would bond again)
    return r > 0.0 && !(rr < Real(1e-10)) && rr < Real(r * r);
  }
  // contact: not bonded
  const Real cut = xi.w + xj.w + (Real)S.gap[s];
  if (!(rr > Real(1e-10) && rr < cut * cut)) return false;
  for (uint32_t k = S.b_row[i], e = S.b_row[i + 1]; k < e; ++k)
    if (S.b_ij[k].y == j) return false;
  return true;
}

// One warp per particle; fill=false counts pairs, fill=true writes them in
// ascending partner order at offset[i] (kModeRefSet: at i*cap).
//
// Lane l < 27 holds cell l of the particle's 3 x 3 x 3 neighbourhood (z
// outermost, x innermost) with its range in the cell list; an inclusive scan
// of the ranges' lengths over the lanes numbers the candidates of all 27
// cells consecutively, and the warp takes them 32 at a time (a lane finds its
// candidate's cell by a binary search over the scanned lengths, fetched by
// shuffles).  The candidates are therefore visited in the order of a scan of
// the cells by z, y, x and of each cell in cell-list order; a ballot ranks the
// accepted ones in that order, the first min(cap, 48) are kept in shared
// memory and written out sorted by partner index (each lane places one by
// counting the smaller ones).  With about 60 candidates a sphere this keeps 32
// independent gathers in flight per warp where one thread per sphere walked
// its candidates one dependent load after another.
constexpr uint32_t kSearchWarps = 4;   // warps (spheres in flight) per 128-thread block

inline uint32_t pair_search_blocks(uint32_t np) { return np ? (np + kSearchWarps - 1) / kSearchWarps : 1u; }

// kPass 0 counts, 1 fills the CSR lists at offset[i], 2 does both at once:
// count[i] and up to kSearchStride partners, sorted, at out_j + i *
// kSearchStride (the caller then compacts them with k_expand_stride).
constexpr uint32_t kSearchStride = 48;

template <class Real, int kPass>
__global__ void __launch_bounds__(128) k_pair_search(PairSearch<Real> S) {
  constexpr bool kCount = kPass != 1, kFill = kPass != 0;
  using V4 = typename RT<Real>::V4;
  constexpr uint32_t kMax = 48;
  static_assert(kMax <= kSearchStride, "one-pass slots hold every kept partner");
  constexpr unsigned kFull = 0xFFFFFFFFu;
  __shared__ uint32_t s_buf[kSearchWarps][kMax];
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint32_t* buf = s_buf[wib];
  for (uint32_t i = blockIdx.x * kSearchWarps + wib; i < S.np; i += gridDim.x * kSearchWarps) {
    const V4 xi = ld4(S.pos + i);
    const uint32_t s = S.sid[i];
    const Grid<Real> g = S.grids[s];
    if (at_hidden(g, xi) || (S.done && S.done[s])) {
      if (kCount && lane == 0) S.count[i] = 0;
      continue;
    }
    const int ix = (int)cell_coord<Real>(xi.x, g.ox, g.inv_a, g.nx);
    const int iy = (int)cell_coord<Real>(xi.y, g.oy, g.inv_a, g.ny);
    const int iz = (int)cell_coord<Real>(xi.z, g.oz, g.inv_a, g.nz);
    uint32_t cstart = 0, ccount = 0;
    if (lane < 27) {
      const int cz = iz + (int)(lane / 9) - 1, cy = iy + (int)((lane / 3) % 3) - 1, cx = ix + (int)(lane % 3) - 1;
      if (cx >= 0 && cx < (int)g.nx && cy >= 0 && cy < (int)g.ny && cz >= 0 && cz < (int)g.nz) {
        const uint32_t c = g.off + (uint32_t)cx + (uint32_t)cy * g.nx + (uint32_t)cz * g.ny * g.nx;
        cstart = S.cell_start[c];
        ccount = S.cell_start[c + 1] - cstart;
      }
    }
    uint32_t pe = ccount;   // inclusive scan of the lengths
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(kFull, pe, d);
      if (lane >= d) pe += o;
    }
    const uint32_t pb = pe - ccount;   // exclusive
    const uint32_t total = __shfl_sync(kFull, pe, 31);
    const uint32_t lim = S.cap < kMax ? S.cap : kMax;
    uint32_t n = 0;
    for (uint32_t base = 0; base < total; base += 32) {
      const uint32_t v = base + lane;
      // the cell of candidate v: the first lane c whose inclusive end exceeds v
      uint32_t lo = 0, hi = 26;
#pragma unroll
      for (int step = 0; step < 5; ++step) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t e = __shfl_sync(kFull, pe, mid);
        if (e > v) hi = mid;
        else lo = mid + 1;
      }
      const uint32_t c = lo < hi ? lo : hi;
      const uint32_t st = __shfl_sync(kFull, cstart, c), bf = __shfl_sync(kFull, pb, c);
      bool pass = false;
      uint32_t j = 0;
      if (v < total) {
        j = S.cell_list[st + (v - bf)];
        if (S.mode == kModeRefSet || j > i) {   // each pair once, from its lower index
          const V4 xj = ld4(S.pos + j);
          pass = !at_hidden(g, xj) && pair_pred<Real>(S, i, j, xi, xj, s);
        }
      }
      const unsigned mask = __ballot_sync(kFull, pass);
      if (kFill && pass) {
        const uint32_t r = n + __popc(mask & ((1u << lane) - 1u));
        if (r < lim) buf[r] = j;
      }
      n += __popc(mask);
    }
    __syncwarp();
    if (kCount && lane == 0) {
      S.count[i] = n;
      if (n > S.cap && S.overflow) atomicAdd(S.overflow, 1u);
    }
    if (kFill) {
      const uint32_t m = n < lim ? n : lim;
      uint32_t* o = kPass == 2 ? S.out_j + (size_t)i * kSearchStride
                               : (S.mode == kModeRefSet ? S.out_j + (size_t)i * S.cap : S.out_j + S.offset[i]);
      for (uint32_t e = lane; e < m; e += 32) {
        const uint32_t val = buf[e];
        uint32_t r = 0;
        for (uint32_t f = 0; f < m; ++f) r += buf[f] < val ? 1u : 0u;
        o[r] = val;
      }
      if (S.mode == kModeRefSet)
        for (uint32_t a = m + lane; a < S.cap; a += 32) o[a] = kEmpty;
    }
    __syncwarp();   // the buffer is refilled for the next sphere
  }
}

// The one-pass lists (kPass 2, kSearchStride slots a particle) compacted into
// (i, j) pairs at the scanned offsets.
static __global__ void k_expand_stride(const uint32_t* __restrict__ offset, uint32_t np,
                                       const uint32_t* __restrict__ js, uint2* __restrict__ ij) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    const uint32_t k0 = offset[i], n = offset[i + 1] - k0;
    const uint32_t m = n < kSearchStride ? n : kSearchStride;
    for (uint32_t r = 0; r < m; ++r) ij[k0 + r] = make_uint2(i, js[(size_t)i * kSearchStride + r]);
  }
}

// Bond state at creation (d_ConstructBoundInteractions, md_boundinteractions_construct.cu:57-98):
// 1/L0 = rsqrt(r^2) with r^2 rounded as the reference rounds it, all histories
// zero (the reference zeroes the previous direction too), radius and
// strengths from the sample's law.
template <class Real>
struct BondLaw {
  Real br_abs;      // > 0: absolute bond radius (reference b_r)
  Real br_factor;   // otherwise b_r = factor * min(r_i, r_j)
  Real sn_mean, sn_sd, st_mean, st_sd;  // normal / shear strength distribution
  uint64_t seed;
};

template <class Real>
__global__ void k_bond_init(const uint2* __restrict__ ij, uint32_t nb, const typename RT<Real>::V4* __restrict__ pos,
                            const uint32_t* __restrict__ sid, const uint32_t* __restrict__ orig,
                            const BondLaw<Real>* __restrict__ law, typename RT<Real>::V4* __restrict__ s0,
                            typename RT<Real>::V4* __restrict__ s1, typename RT<Real>::V4* __restrict__ s2,
                            typename RT<Real>::V4* __restrict__ par, int32_t* __restrict__ per_sample_count) {
  using T = RT<Real>;
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const uint2 e = ij[b];
    const auto xi = ld4(pos + e.x), xj = ld4(pos + e.y);
    const Real rx = xj.x - xi.x, ry = xj.y - xi.y, rz = xj.z - xi.z;
    const Real rm2 = (rx * rx + ry * ry) + rz * rz;
    const uint32_t s = sid[e.x];
    const BondLaw<Real> L = law[s];
    const Real br = L.br_abs > Real(0) ? L.br_abs : L.br_factor * (xi.w < xj.w ? xi.w : xj.w);
    const uint32_t oa = orig[e.x], ob = orig[e.y];
    const uint32_t lo = oa < ob ? oa : ob, hi = oa < ob ? ob : oa;
    Real sn = L.sn_mean, st = L.st_mean;
    if (L.sn_sd > Real(0)) sn = Real((double)L.sn_mean + (double)L.sn_sd * normal_from(L.seed, lo, hi, 1));
    if (L.st_sd > Real(0)) st = Real((double)L.st_mean + (double)L.st_sd * normal_from(L.seed, lo, hi, 2));
    if (sn < Real(0)) sn = Real(0);
    if (st < Real(0)) st = Real(0);
    const Real z = Real(0);
    s0[b] = mk4(z, z, z, z);
    s1[b] = mk4(z, z, z, z);
    s2[b] = mk4(z, z, z, z);
    par[b] = mk4(T::rsqrt_rn(rm2), sn, st, br);
    atomicAdd(per_sample_count + s, 1);
  }
}

// History carry-over after a contact-list rebuild: a pair present before keeps
// its tangential history (bit 31 of j marks non-zero history).
template <class Real>
__global__ void k_contact_carry(uint2* __restrict__ ij, uint32_t nc_new, typename RT<Real>::V4* __restrict__ o_new,
                                const uint2* __restrict__ ij_old, const typename RT<Real>::V4* __restrict__ o_old,
                                const uint32_t* __restrict__ row_old) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nc_new; c += gridDim.x * blockDim.x) {
    const uint2 e = ij[c];
    uint32_t lo = row_old[e.x], hi = row_old[e.x + 1];
    auto ov = mk4(Real(0), Real(0), Real(0), Real(0));
    uint32_t flag = 0;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      const uint32_t jm = ij_old[mid].y & 0x7FFFFFFFu;
      if (jm < e.y)
        lo = mid + 1;
      else
        hi = mid;
    }
    if (lo < row_old[e.x + 1] && (ij_old[lo].y & 0x7FFFFFFFu) == e.y && (ij_old[lo].y >> 31)) {
      ov = ld4(o_old + lo);
      flag = 0x80000000u;
    }
    o_new[c] = ov;
    ij[c] = make_uint2(e.x, e.y | flag);
  }
}

template <class Real>
__global__ void k_copy_pos(const typename RT<Real>::V4* __restrict__ pos, typename RT<Real>::V4* __restrict__ ref,
                           uint32_t np) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) ref[p] = pos[p];
}

// CSR row pointer of a pair list sorted by i: row[i] = first pair with first index >= i
static __global__ void k_rows_from_pairs(const uint2* __restrict__ ij, uint32_t n, uint32_t np, uint32_t* __restrict__ row) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k <= n; k += gridDim.x * blockDim.x) {
    const uint32_t a = k > 0 ? ij[k - 1].x + 1 : 0u;
    const uint32_t b = k < n ? ij[k].x : np;
    for (uint32_t i = a; i <= b && i <= np; ++i) row[i] = k;
  }
}

}  // namespace dem
