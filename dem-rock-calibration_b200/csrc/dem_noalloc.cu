// dem_ref_cells_static: the cell binning of dem_ref_cells (CellDistribution,
// md_cell_distribution.cu:130-172) for callers that cannot allocate GPU memory
// - cudaMalloc/cudaFree may synchronise the whole device and stall the other
// streams of a serving process, they fail when another framework's caching
// allocator holds most of the memory, and some host frameworks forbid a
// plug-in its own allocations.  It runs out of one file-scope device array
// instead of per-call buffers and allocates nothing, neither on the device nor
// on the host: the input and the three outputs are copied straight between
// the caller's host buffers and sub-ranges of the array, and the reference
// layouts (CIs, pnC) are produced on the device.
//
// Set-up: host code cannot use the array's name as a device address, so the
// first call on each device looks the address up with cudaGetSymbolAddress
// (that device current) and caches it; that first call should come before
// any stream capture.  The cache is keyed by the device and the unique id of
// its current context: after a context reset (cudaDeviceReset, or a host
// framework that recreates the primary context) the module is loaded again
// at a new address, and the next call looks it up again instead of using the
// stale one.
//
// Stream: every call issues its copies and kernels on the legacy default
// stream and waits for them before returning, so it also waits for the other
// blocking streams of the device, and it must not be called while another
// host thread captures a stream in global capture mode.
//
// Limits: n <= DEM_STATIC_MAX_PARTICLES particles and nx*ny*nz <=
// DEM_STATIC_MAX_CELLS cells; larger calls return DEM_ERR_CAPACITY before any
// device work.  The array keeps the last call's contents and is shared by
// every call on a device: what must start at zero is cleared per call, and
// calls that overlap on the GPU (two host threads) race on it, so callers
// serialise them.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <mutex>

#include "b200dem.h"
#include "dem_build.cuh"

namespace dem {
namespace {

constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }

// Sub-ranges of the scratch array, in bytes, for nmax particles and cmax cells.
struct StaticLayout {
  size_t xyz, pos, sid, cell_of, clist, cis, count, cstart, cursor, pnc, tmp1, tmp2, grid, total;
};

constexpr uint32_t kScanBlocksMax = (DEM_STATIC_MAX_CELLS + kScanBlock - 1) / kScanBlock;

constexpr StaticLayout make_layout(size_t nmax, size_t cmax) {
  StaticLayout L{};
  size_t o = 0;
  L.xyz = o;     o += align_up(3 * nmax * sizeof(float));
  L.pos = o;     o += align_up(nmax * sizeof(float4));
  L.sid = o;     o += align_up(nmax * sizeof(uint32_t));
  L.cell_of = o; o += align_up(nmax * sizeof(uint32_t));
  L.clist = o;   o += align_up(nmax * sizeof(uint32_t));
  L.cis = o;     o += align_up(2 * nmax * sizeof(uint32_t));
  L.count = o;   o += align_up((cmax + 1) * sizeof(uint32_t));
  L.cstart = o;  o += align_up((cmax + 1) * sizeof(uint32_t));
  L.cursor = o;  o += align_up((cmax + 1) * sizeof(uint32_t));
  L.pnc = o;     o += align_up(2 * cmax * sizeof(uint32_t));
  L.tmp1 = o;    o += align_up((kScanBlocksMax + 1) * sizeof(uint32_t));
  L.tmp2 = o;    o += align_up((kScanBlocksMax + 1) * sizeof(uint32_t));
  L.grid = o;    o += align_up(sizeof(Grid<float>));
  L.total = o;
  return L;
}

constexpr StaticLayout kLayout = make_layout(DEM_STATIC_MAX_PARTICLES, DEM_STATIC_MAX_CELLS);
static_assert(kScanBlocksMax <= kScanBlock, "two scan levels cover the cell range");
static_assert(kLayout.total <= DEM_STATIC_SCRATCH_BYTES, "scratch layout exceeds the declared size");

// The scratch: 4.5 MiB, 256-byte aligned, one instance per device.
static __device__ __align__(256) unsigned char g_scratch[DEM_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
unsigned char* g_addr[kMaxDevices] = {};
unsigned long long g_ctx_id[kMaxDevices] = {};   // context the cached address belongs to

// Unique id of the calling thread's current context.  The driver functions
// are reached through the runtime's entry-point query, so the library keeps
// no link-time dependency on the driver library (it loads on hosts without a
// GPU driver, where only its argument checks run).
int current_context_id(unsigned long long* id) {
  static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
  static PFN_cuCtxGetId_v12000 get_id = nullptr;
  if (!get_current || !get_id) {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 4000, cudaEnableDefault, &q1) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || !f1 ||
        cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) != cudaSuccess ||
        q2 != cudaDriverEntryPointSuccess || !f2)
      return DEM_ERR_CUDA;
    get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f1);
    get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(f2);
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, id) != CUDA_SUCCESS) return DEM_ERR_CUDA;
  return DEM_OK;
}

// Device address of g_scratch on the current device: looked up with
// cudaGetSymbolAddress on the first call in the device's current context,
// then cached for that context.
int scratch_address(unsigned char** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return DEM_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_addr_mu);
  // makes the device's primary context current (and creates it if needed),
  // so the driver's current context is the one the runtime calls below use
  if (cudaSetDevice(dev) != cudaSuccess) return DEM_ERR_CUDA;
  unsigned long long id = 0;
  if (current_context_id(&id) != DEM_OK) return DEM_ERR_CUDA;
  if (!g_addr[dev] || g_ctx_id[dev] != id) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) return DEM_ERR_CUDA;
    g_addr[dev] = static_cast<unsigned char*>(p);
    g_ctx_id[dev] = id;
  }
  *out = g_addr[dev];
  return DEM_OK;
}

// SoA float[3n] (x block, y block, z block) -> float4 (x, y, z, 0).
static __global__ void k_static_pack(const float* __restrict__ xyz, uint32_t n, float4* __restrict__ pos) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    pos[i] = make_float4(xyz[i], xyz[n + i], xyz[2 * n + i], 0.f);
}

// Reference layouts: CIs = (cell key of the k-th sorted entry, its particle),
// pnC = (first sorted entry, population) per cell, both zero for empty cells.
static __global__ void k_static_layout(const uint32_t* __restrict__ cell_of, const uint32_t* __restrict__ clist,
                                       const uint32_t* __restrict__ cstart, uint32_t n, uint32_t ncell,
                                       uint32_t* __restrict__ cis, uint32_t* __restrict__ pnc) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
    const uint32_t p = clist[k];
    cis[k] = cell_of[p];
    cis[n + k] = p;
  }
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += stride) {
    const uint32_t b = cstart[c], e = cstart[c + 1];
    pnc[c] = e > b ? b : 0u;
    pnc[ncell + c] = e - b;
  }
}

template <class T>
T* at(unsigned char* base, size_t off) {
  return reinterpret_cast<T*>(base + off);
}

int ref_cells_static(const float* xyz, uint32_t n, float a, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t* CI,
                     uint32_t* CIs, uint32_t* pnC) {
  const uint64_t ncell64 = (uint64_t)nx * ny * nz;
  if (n > DEM_STATIC_MAX_PARTICLES || ncell64 > DEM_STATIC_MAX_CELLS) return DEM_ERR_CAPACITY;
  const uint32_t ncell = (uint32_t)ncell64;
  unsigned char* s = nullptr;
  int rc = scratch_address(&s);
  if (rc) return rc;
  const cudaStream_t st = 0;
  float* d_xyz = at<float>(s, kLayout.xyz);
  float4* pos = at<float4>(s, kLayout.pos);
  uint32_t* sid = at<uint32_t>(s, kLayout.sid);
  uint32_t* cell_of = at<uint32_t>(s, kLayout.cell_of);
  uint32_t* clist = at<uint32_t>(s, kLayout.clist);
  uint32_t* cis = at<uint32_t>(s, kLayout.cis);
  uint32_t* count = at<uint32_t>(s, kLayout.count);
  uint32_t* cstart = at<uint32_t>(s, kLayout.cstart);
  uint32_t* cursor = at<uint32_t>(s, kLayout.cursor);
  uint32_t* pnc = at<uint32_t>(s, kLayout.pnc);
  uint32_t* tmp1 = at<uint32_t>(s, kLayout.tmp1);
  uint32_t* tmp2 = at<uint32_t>(s, kLayout.tmp2);
  Grid<float>* grid = at<Grid<float>>(s, kLayout.grid);
  const Grid<float> g{0.f, 0.f, 0.f, (float)(1.0 / (double)a), nx, ny, nz, 0, 0.f, 0.f, 0.f, 0u};
  // what must start at zero: the per-particle grid id (one grid) and the cell counters
  if (cudaMemsetAsync(sid, 0, n * sizeof(uint32_t), st) != cudaSuccess ||
      cudaMemsetAsync(count, 0, (ncell + 1) * sizeof(uint32_t), st) != cudaSuccess ||
      cudaMemcpyAsync(d_xyz, xyz, 3 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(grid, &g, sizeof g, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return DEM_ERR_CUDA;
  const uint32_t gb = std::max(1u, (n + 255) / 256);
  k_static_pack<<<gb, 256, 0, st>>>(d_xyz, n, pos);
  k_cell_index<float><<<gb, 256, 0, st>>>(pos, sid, n, grid, cell_of, count);
  const uint32_t nb = (ncell + kScanBlock - 1) / kScanBlock;
  k_scan_block<<<nb, kScanBlock, 0, st>>>(count, cstart, ncell, tmp1);
  if (nb > 1) {
    k_scan_block<<<1, kScanBlock, 0, st>>>(tmp1, tmp2, nb, nullptr);
    k_scan_add<<<nb, kScanBlock, 0, st>>>(cstart, ncell, tmp2);
  }
  k_scan_total<<<1, 1, 0, st>>>(count, cstart, ncell);
  if (cudaMemcpyAsync(cursor, cstart, (ncell + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return DEM_ERR_CUDA;
  k_scatter_cells<<<gb, 256, 0, st>>>(cell_of, n, cursor, clist);
  k_sort_cells<<<std::max(1u, (ncell + 255) / 256), 256, 0, st>>>(cstart, ncell, clist);
  k_static_layout<<<std::max(gb, (ncell + 255) / 256), 256, 0, st>>>(cell_of, clist, cstart, n, ncell, cis, pnc);
  if (cudaGetLastError() != cudaSuccess) return DEM_ERR_CUDA;
  if ((CI && cudaMemcpyAsync(CI, cell_of, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess) ||
      (CIs && cudaMemcpyAsync(CIs, cis, 2 * (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess) ||
      (pnC && cudaMemcpyAsync(pnC, pnc, 2 * (size_t)ncell * sizeof(uint32_t), cudaMemcpyDeviceToHost, st) !=
                  cudaSuccess))
    return DEM_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return DEM_ERR_CUDA;
  return DEM_OK;
}

}  // namespace
}  // namespace dem

extern "C" int dem_ref_cells_static(const float* xyz, uint32_t n, float a, uint32_t nx, uint32_t ny, uint32_t nz,
                                    uint32_t* CI, uint32_t* CIs, uint32_t* pnC) {
  if (!xyz || n == 0 || !(a > 0) || !nx || !ny || !nz) return DEM_ERR_ARG;
  // no exception crosses the C ABI (std::mutex::lock may throw)
  try {
    return dem::ref_cells_static(xyz, n, a, nx, ny, nz, CI, CIs, pnC);
  } catch (...) {
    return DEM_ERR_STATE;
  }
}
