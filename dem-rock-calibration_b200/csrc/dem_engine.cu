// B200 DEM engine: device memory, set-up, the per-step pipeline (two kernels
// per step, replayed from a captured CUDA graph), contact-list rebuilds and
// state export.  The C ABI (include/b200dem.h) is a thin layer over
// dem::EngineBase in dem_capi.cpp.
#include "dem_engine.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <unistd.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <functional>
#include <condition_variable>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "dem_build.cuh"
#include "dem_dual.cuh"
#include "dem_params.h"
#include "dem_step.cuh"

namespace dem {

namespace {
thread_local char g_detail[192] = "";
}  // namespace

void note_cuda_error(cudaError_t e, const char* file, int line) {
  const char* base = std::strrchr(file, '/');
  std::snprintf(g_detail, sizeof g_detail, "%s (%s) at %s:%d", cudaGetErrorName(e), cudaGetErrorString(e),
                base ? base + 1 : file, line);
  // the error is reported through the return code: clear the thread's last
  // runtime error, so that a later cudaGetLastError check of another call
  // does not report it again
  (void)cudaGetLastError();
}

const char* last_error_detail() { return g_detail; }

#define CK(x)                                  \
  do {                                         \
    cudaError_t e_ = (x);                      \
    if (e_ != cudaSuccess) {                   \
      last_cuda_ = e_;                         \
      note_cuda_error(e_, __FILE__, __LINE__); \
      return DEM_ERR_CUDA;                     \
    }                                          \
  } while (0)
#define RC(x)                \
  do {                       \
    int r_ = (x);            \
    if (r_ != DEM_OK) return r_; \
  } while (0)

// Time spent in device allocation and release (set-up trace, DEM_TRACE=1).
static std::atomic<uint64_t> g_alloc_ns{0}, g_free_ns{0}, g_alloc_calls{0};
static uint64_t now_ns() {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Device blocks released by a context are kept for reuse by later allocations
// in this process.  Calibration work creates many contexts of similar sizes
// one after another, and a cudaMalloc cost about 230 us on average in the
// set-up of a 490k-sphere context (12 ms of its 28 ms), while cudaFree
// synchronises the device.  Allocations are rounded up to size classes (four
// per octave) and a cached block serves requests of its class.  A block
// enters the cache only after its device has finished all queued work (a
// device synchronisation, the ordering cudaFree gives), so a later user cannot
// race with kernels of the releasing context.  Blocks are kept per CUDA context (its unique id): after a context
// reset none of the old blocks is offered again.  Before a block is handed
// out, the driver must still know it as an allocation of at least its size
// starting at its address (a block that other code freed behind the cache's
// back is dropped).  The cache holds at most 40% of the device's memory.
// When cudaMalloc fails, the cached blocks of the current context go back to
// the driver and the allocation is retried; dem_release_cached_memory()
// returns them all on request.
namespace blockcache {
std::mutex mu;
std::multimap<std::pair<unsigned long long, size_t>, void*> blocks;   // (context id, bytes) -> block
size_t cached_bytes = 0;
std::map<int, size_t> total_mem;   // device -> bytes of device memory

// total memory of a device (cudaDeviceProp::totalGlobalMem)
cudaError_t device_total_mem(int dev, size_t* out) {
  cudaDeviceProp prop;
  const cudaError_t e = cudaGetDeviceProperties(&prop, dev);
  if (e == cudaSuccess) *out = prop.totalGlobalMem;
  return e;
}
// the cache holds at most this share of the device's memory; a block released
// beyond it goes back to the driver at once
constexpr double kMaxShare = 0.4;
PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
PFN_cuCtxGetId_v12000 get_id = nullptr;
PFN_cuMemGetAddressRange_v3020 get_range = nullptr;
bool resolved = false;

// the driver functions, through the runtime's entry-point query (no link-time
// dependency on the driver library); called with mu held
bool resolve() {
  if (resolved) return get_current && get_id && get_range;
  resolved = true;
  void* f[3] = {nullptr, nullptr, nullptr};
  cudaDriverEntryPointQueryResult q[3];
  if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f[0], 4000, cudaEnableDefault, &q[0]) != cudaSuccess ||
      cudaGetDriverEntryPointByVersion("cuCtxGetId", &f[1], 12000, cudaEnableDefault, &q[1]) != cudaSuccess ||
      cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &f[2], 3020, cudaEnableDefault, &q[2]) !=
          cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  for (int k = 0; k < 3; ++k)
    if (q[k] != cudaDriverEntryPointSuccess || !f[k]) return false;
  get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f[0]);
  get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(f[1]);
  get_range = reinterpret_cast<PFN_cuMemGetAddressRange_v3020>(f[2]);
  return true;
}

// unique id of the calling thread's current context (0: unknown, no caching)
unsigned long long context_id() {
  std::lock_guard<std::mutex> lk(mu);
  if (!resolve()) return 0;
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Block sizes come in classes, four per octave (256 B granularity below
// 4 KiB): requests of slightly different sizes (a contact list that grows
// between rebuilds) share blocks, less than 25% above the request.
size_t size_class(size_t bytes) {
  if (bytes <= 4096) return (bytes + 255) & ~(size_t)255;
  int e = 63 - __builtin_clzll((unsigned long long)(bytes - 1));   // 2^e < bytes <= 2^(e+1)
  const size_t step = (size_t)1 << (e - 2);                        // quarter of the octave
  return (bytes + step - 1) / step * step;
}

void* take(unsigned long long ctx, size_t bytes, size_t* got) {
  if (!ctx) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  auto it = blocks.lower_bound({ctx, bytes});
  while (it != blocks.end() && it->first.first == ctx && it->first.second == bytes) {
    void* p = it->second;
    const size_t b = it->first.second;
    it = blocks.erase(it);
    cached_bytes -= b;
    CUdeviceptr base = 0;
    size_t size = 0;
    if (get_range(&base, &size, (CUdeviceptr)p) == CUDA_SUCCESS && base == (CUdeviceptr)p && size >= b) {
      *got = b;
      return p;
    }
  }
  return nullptr;
}

void give(unsigned long long ctx, int dev, void* p, size_t bytes) {
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != dev) cudaSetDevice(dev);
  const bool idle = cudaDeviceSynchronize() == cudaSuccess;
  if (cur != dev && cur >= 0) cudaSetDevice(cur);
  {
    std::lock_guard<std::mutex> lk(mu);
    // the device's memory size, asked once per device (the query costs far
    // more than a release)
    auto tm = total_mem.find(dev);
    if (tm == total_mem.end()) {
      size_t t = 0;
      if (device_total_mem(dev, &t) != cudaSuccess) t = 0;
      tm = total_mem.emplace(dev, t).first;
    }
    if (idle && ctx && cached_bytes + bytes <= (size_t)(kMaxShare * (double)tm->second)) {
      blocks.emplace(std::make_pair(ctx, bytes), p);
      cached_bytes += bytes;
      return;
    }
  }
  // a device in an error state, no context id, or a full cache: back to the driver
  cudaFree(p);
}

// returns the cached blocks of context ctx (every context for ctx == 0) to the driver
void trim(unsigned long long ctx) {
  std::vector<void*> out;
  {
    std::lock_guard<std::mutex> lk(mu);
    for (auto it = blocks.begin(); it != blocks.end();) {
      if (!ctx || it->first.first == ctx) {
        out.push_back(it->second);
        cached_bytes -= it->first.second;
        it = blocks.erase(it);
      } else {
        ++it;
      }
    }
  }
  for (void* p : out) cudaFree(p);
}
}  // namespace blockcache

int release_cached_memory() {
  blockcache::trim(0);
  cudaGetLastError();   // a block of a context that no longer exists fails to free; nothing to report
  return DEM_OK;
}

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  size_t cap = 0;   // bytes of the block held (at least n * sizeof(T))
  int dev = 0;
  unsigned long long ctx = 0;   // unique id of the CUDA context the block belongs to
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  // exchanges the blocks of two buffers (each keeps its block's capacity)
  void swap(DBuf& o) {
    std::swap(p, o.p);
    std::swap(n, o.n);
    std::swap(cap, o.cap);
    std::swap(dev, o.dev);
    std::swap(ctx, o.ctx);
  }
  void release() {
    if (p) {
      const uint64_t t0 = now_ns();
      blockcache::give(ctx, dev, p, cap);
      g_free_ns += now_ns() - t0;
    }
    p = nullptr;
    n = 0;
    cap = 0;
  }
  cudaError_t alloc(size_t cnt) {
    release();
    n = cnt;
    if (cnt == 0) return cudaSuccess;
    const uint64_t t0 = now_ns();
    struct Acc {
      uint64_t t0;
      ~Acc() {
        g_alloc_ns += now_ns() - t0;
        ++g_alloc_calls;
      }
    } acc{t0};
    cudaGetDevice(&dev);
    ctx = blockcache::context_id();
    const size_t bytes = blockcache::size_class(cnt * sizeof(T));
    size_t got = 0;
    p = (T*)blockcache::take(ctx, bytes, &got);
    cudaError_t e = cudaSuccess;
    if (p) {
      cap = got;
    } else {
      e = cudaMalloc((void**)&p, bytes);
      if (e == cudaErrorMemoryAllocation) {   // the cache's blocks back to the driver, then once more
        cudaGetLastError();
        blockcache::trim(ctx);
        e = cudaMalloc((void**)&p, bytes);
      }
      cap = bytes;
    }
    if (e != cudaSuccess) {
      p = nullptr;
      n = 0;
      cap = 0;
      return e;
    }
    // zero-filled before returning: the fill runs on the legacy default
    // stream, which is not ordered with the engine's non-blocking stream
    e = cudaMemsetAsync(p, 0, cnt * sizeof(T), 0);
    return e != cudaSuccess ? e : cudaStreamSynchronize(0);
  }
  cudaError_t upload(const T* h, size_t cnt) { return cudaMemcpy(p, h, cnt * sizeof(T), cudaMemcpyHostToDevice); }
  cudaError_t download(T* h, size_t cnt) const { return cudaMemcpy(h, p, cnt * sizeof(T), cudaMemcpyDeviceToHost); }
};

static uint32_t ceil_div(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

// Host worker threads for the set-up loops, started once per process and
// reused (starting threads for every loop cost milliseconds per set-up).
// run(T, fn) calls fn(0) ... fn(T - 1), the calling thread taking its share,
// and returns when all are done; one run at a time (callers on other host
// threads wait their turn).
class HostPool {
 public:
  static HostPool& get() {
    static HostPool pool;
    return pool;
  }
  uint32_t width() const { return (uint32_t)workers_.size() + 1; }
  void run(uint32_t T, const std::function<void(uint32_t)>& fn) {
    // (a process forked from this one has no workers: it runs serially)
    if (T <= 1 || workers_.empty() || getpid() != pid_) {
      for (uint32_t t = 0; t < T; ++t) fn(t);
      return;
    }
    std::lock_guard<std::mutex> one(run_mu_);
    {
      std::lock_guard<std::mutex> lk(mu_);
      job_ = &fn;
      njobs_ = T;
      next_.store(0);
      left_ = T;
      ++gen_;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return left_ == 0; });
    job_ = nullptr;
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
      ++gen_;
    }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
  }

 private:
  HostPool() : pid_(getpid()) {
    const uint32_t hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    for (uint32_t t = 1; t < hw; ++t) workers_.emplace_back([this] { loop(); });
  }
  // take job indices until none is left
  void work() {
    for (;;) {
      const uint32_t t = next_.fetch_add(1);
      if (t >= njobs_) return;
      (*job_)(t);
      std::lock_guard<std::mutex> lk(mu_);
      if (--left_ == 0) done_cv_.notify_all();
    }
  }
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      work();
    }
  }
  std::vector<std::thread> workers_;
  std::mutex mu_, run_mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(uint32_t)>* job_ = nullptr;
  uint32_t njobs_ = 0, left_ = 0;
  std::atomic<uint32_t> next_{0};
  uint64_t gen_ = 0;
  bool stop_ = false;
  pid_t pid_;
};

// the chunk count parallel_chunks uses for n items: one per 32,768 items, at
// most one per host worker
static uint32_t chunk_count(uint32_t n) {
  return std::max(1u, std::min(HostPool::get().width(), n / 32768u));
}

// fn(t, k0, k1) for the T contiguous chunks of [0, n) on the host workers
// (the same boundaries for the same n and T); fn must not throw
template <class Fn>
static void parallel_chunks(uint32_t n, uint32_t T, Fn fn) {
  if (T <= 1) {
    fn(0u, 0u, n);
    return;
  }
  HostPool::get().run(T, [&](uint32_t t) {
    fn(t, (uint32_t)((uint64_t)n * t / T), (uint32_t)((uint64_t)n * (t + 1) / T));
  });
}

// fn(begin, end) over [0, n) split into contiguous ranges on the host
// workers (set-up loops over hundreds of thousands of particles); fn must not
// throw and its ranges must write disjoint data.
template <class Fn>
static void parallel_ranges(uint32_t n, Fn fn) {
  parallel_chunks(n, chunk_count(n), [&](uint32_t, uint32_t k0, uint32_t k1) { fn(k0, k1); });
}

struct SampleHost {
  dem_material mat{};
  dem_loading load{};
  uint32_t n = 0;
  std::vector<float> xyz, rad;     // caller order
  std::vector<uint32_t> perm;      // storage position k -> caller index
  std::vector<uint32_t> inv;       // caller index -> storage position
  uint32_t p_begin = 0;
  double rmin = 0, rmax = 0, rmean = 0;
  Potential pot{};
  double dt = 0;
  double E_b = 0, G_b = 0, hm_E = 0, hm_G = 0;
  int32_t bonds_initial = 0;
  uint32_t lat_count = 0;   // lateral surface particles (uniaxial specimens)
  double lat_rho0 = 0;      // their mean radial distance at set-up
};

template <class Real>
class Engine final : public EngineBase {
 public:
  using V4 = typename RT<Real>::V4;

  explicit Engine(const dem_options& o) : opt_(o) {}
  ~Engine() override {
    invalidate_graph();
    if (stream_) cudaStreamDestroy(stream_);
  }

  int precision() const override { return DualK<Real>::K ? 2 : (sizeof(Real) == 8 ? 1 : 0); }

  int init() {
    CK(cudaSetDevice(opt_.device));
    CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    int dev = opt_.device;
    CK(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev));
    // the pair kernel: one bond tile per block and pass, as many blocks as fit
    // on the GPU; register budget for pair_min_blocks blocks per SM: 1..4 of
    // 256 threads, and for FP32 also 5..8 of 128 threads (102, 85, 72 and 64
    // registers).  0 = 7 for FP32 (128 threads, 72 registers, no spills: 28
    // warps per SM, measured 3% faster than 3 x 256 threads at 80 registers
    // and than 64 registers with spills), 2 for FP64, 1 for the sensitivity
    // build.
    // deterministic force accumulation: fixed point (FP32: separate 64-bit
    // accumulators; FP64 and the sensitivity build: in place of the doubles)
    det_ = opt_.deterministic != 0;
    user_grid_ = opt_.pair_grid != 0;
    RC(set_pair_config(opt_.pair_min_blocks));
    if (!opt_.particle_block) opt_.particle_block = 256;
    if (!opt_.graph_steps) opt_.graph_steps = 100;
    skin_user_ = opt_.skin_factor > 0;
    if (!skin_user_) opt_.skin_factor = 0.1;
    return DEM_OK;
  }

  int add_sample(const dem_material* mat, const dem_loading* load, const float* xyz, const float* radii, uint32_t n,
                 int32_t* id) override {
    if (setup_done_) return DEM_ERR_STATE;
    if (!mat || !load || !xyz || n == 0) return DEM_ERR_ARG;
    for (size_t k = 0; k < 3 * (size_t)n; ++k)
      if (!std::isfinite(xyz[k])) return DEM_ERR_ARG;
    SampleHost s;
    s.mat = *mat;
    s.load = *load;
    s.n = n;
    s.xyz.assign(xyz, xyz + 3 * (size_t)n);
    if (radii)
      s.rad.assign(radii, radii + n);
    else
      s.rad.assign(n, (float)mat->p_r);
    for (float r : s.rad)
      if (!(r > 0) || !std::isfinite(r)) return DEM_ERR_ARG;
    samples_.push_back(std::move(s));
    if (id) *id = (int32_t)samples_.size() - 1;
    return DEM_OK;
  }

  // ---------------------------------------------------------------- set-up
  // DEM_TRACE=1 in the environment: set-up phase times on stderr (the
  // stream is drained at each mark, so the device work of a phase counts in it)
  struct PhaseTrace {
    bool on = std::getenv("DEM_TRACE") != nullptr;
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    std::string line;
    void mark(const char* what, cudaStream_t st) {
      if (!on) return;
      cudaStreamSynchronize(st);
      const auto now = std::chrono::steady_clock::now();
      char b[96];
      std::snprintf(b, sizeof b, " %s %.2f ms", what, std::chrono::duration<double, std::milli>(now - t).count());
      line += b;
      t = now;
    }
    uint64_t a0 = g_alloc_ns.load(), f0 = g_free_ns.load(), c0 = g_alloc_calls.load();
    void flush(const char* head) {
      if (on)
        std::fprintf(stderr, "dem trace: %s%s (device allocations %llu: %.2f ms, releases %.2f ms)\n", head,
                     line.c_str(), (unsigned long long)(g_alloc_calls.load() - c0),
                     1e-6 * (double)(g_alloc_ns.load() - a0), 1e-6 * (double)(g_free_ns.load() - f0));
    }
  };

  int setup() override {
    if (setup_done_) return DEM_ERR_STATE;
    if (samples_.empty()) return DEM_ERR_STATE;
    CK(cudaSetDevice(opt_.device));
    PhaseTrace tr;
    const uint32_t S = (uint32_t)samples_.size();
    np_ = 0;
    for (auto& s : samples_) {
      s.p_begin = np_;
      np_ += s.n;
      derive(s);
    }
    // Morton order of each sample (keys from its positions quantised by r_min,
    // a stable sort): on the device, unless the sample index and the keys
    // need more than 64 bits, then on the host (the same order either way)
    std::vector<MortonFrame> frames(S);
    int mbits = 0;
    for (uint32_t si = 0; si < S; ++si) mbits = std::max(mbits, morton_frame(samples_[si], frames[si]));
    int sbits = 0;
    while (sbits < 32 && ((uint64_t)(S - 1) >> sbits) != 0) ++sbits;
    const bool dev_order = mbits + sbits <= 64;
    if (!dev_order)
      for (auto& s : samples_) morton_order(s);
    tr.mark("order", stream_);
    // per-particle state, built on the device from the caller's arrays (one
    // upload of positions, radii and the storage order per sample)
    CK(pos_.alloc(np_));
    CK(vel_.alloc(np_));
    CK(omg_.alloc(np_));
    CK(frc_.alloc(np_));
    CK(mom_.alloc(np_));
    if (det_ && sizeof(Real) == 4) {
      CK(frcq_.alloc(4 * (size_t)np_));   // zero-filled
      CK(momq_.alloc(4 * (size_t)np_));
    }
    CK(wallO_.alloc(np_));
    CK(wflag_.alloc(np_));
    CK(pos_ref_.alloc(np_));
    CK(mass_.alloc(np_));
    CK(sid_.alloc(np_));
    CK(orig_.alloc(np_));
    {
      DBuf<float> stage;
      DBuf<InitSample> tab;
      CK(stage.alloc(5 * (size_t)np_));
      std::vector<InitSample> ht(S);
      for (uint32_t si = 0; si < S; ++si) {
        const SampleHost& s = samples_[si];
        ht[si] = InitSample{s.p_begin, s.n, s.pot.m_ro, s.dt};
        for (int d = 0; d < 4; ++d) {
          const float* src = d < 3 ? s.xyz.data() + (size_t)d * s.n : s.rad.data();
          CK(cudaMemcpyAsync(stage.p + (size_t)d * np_ + s.p_begin, src, s.n * sizeof(float), cudaMemcpyHostToDevice,
                             stream_));
        }
        if (!dev_order)
          CK(cudaMemcpyAsync(stage.p + 4 * (size_t)np_ + s.p_begin, s.perm.data(), s.n * sizeof(uint32_t),
                             cudaMemcpyHostToDevice, stream_));
      }
      if (dev_order) RC(device_morton(stage.p, frames, mbits, mbits + sbits));
      CK(tab.alloc(S));
      CK(cudaMemcpyAsync(tab.p, ht.data(), S * sizeof(InitSample), cudaMemcpyHostToDevice, stream_));
      k_init_particles<Real><<<grid1(np_), 256, 0, stream_>>>(stage.p, np_, tab.p, S, pos_.p, vel_.p, omg_.p, mass_.p,
                                                             sid_.p, orig_.p);
      CK(cudaGetLastError());
      CK(cudaStreamSynchronize(stream_));   // the stage and the host table are released here
    }
    tr.mark("upload", stream_);
    RC(mark_lateral());
    tr.mark("lateral", stream_);
    // per-sample constants and controllers
    RC(upload_params());
    tr.mark("params", stream_);
    // contact grids
    RC(make_grids());
    tr.mark("grids", stream_);
    // bonds
    RC(build_bonds());
    tr.mark("bonds", stream_);
    // contact list
    RC(build_contacts(true));
    tr.mark("contacts", stream_);
    RC(init_controllers());
    CK(blocks_done_.alloc(1));
    if (DualK<Real>::K) CK(sfl_tan_.alloc((size_t)S * (4 * DualK<Real>::K + 2)));
    CK(stat_.alloc(2));
    min_skin_ = 1e300;
    max_dt_ = 0;
    for (auto& s : samples_) {
      min_skin_ = std::min(min_skin_, opt_.skin_factor * s.rmin);
      max_dt_ = std::max(max_dt_, s.dt);
    }
    CK(cudaDeviceSynchronize());
    setup_done_ = true;
    // the step graphs are captured and instantiated here, so that no later
    // call pays for an instantiation inside its own time (they are captured
    // again only after a change that invalidates them)
    tr.mark("rest", stream_);
    RC(capture_all());
    tr.mark("graphs", stream_);
    tr.flush("setup");
    return DEM_OK;
  }

  // Uniaxial specimens: mark the particles of the lateral surface near
  // mid-height (outer shell one mean diameter thick, |z - z_c| <= H/4), whose
  // mean radial distance gives the lateral strain for the Poisson ratio.
  int mark_lateral() {
    std::vector<uint8_t> h(np_, 0);
    bool any = false;
    for (auto& s : samples_) {
      s.lat_count = 0;
      const dem_loading& L = s.load;
      if (L.test != DEM_TEST_UNIAXIAL) continue;
      const double cx = L.center_real[0], cy = L.center_real[1], cz = L.center_real[2];
      const double hz = 0.25 * L.size_real[2];
      double outer = 0;
      for (uint32_t q = 0; q < s.n; ++q)
        outer = std::max(outer, std::hypot(s.xyz[q] - cx, s.xyz[s.n + q] - cy) + s.rad[q]);
      for (uint32_t k = 0; k < s.n; ++k) {
        const uint32_t q = s.perm[k];
        const double rho = std::hypot(s.xyz[q] - cx, s.xyz[s.n + q] - cy);
        if (rho + s.rad[q] >= outer - 2.0 * s.rmean && std::fabs(s.xyz[2 * s.n + q] - cz) <= hz) {
          h[s.p_begin + k] = 1;
          ++s.lat_count;
          s.lat_rho0 += rho;
        }
      }
      if (s.lat_count) s.lat_rho0 /= s.lat_count;
      any = any || s.lat_count > 0;
    }
    hlat_ = h;
    if (!any) return DEM_OK;
    CK(lat_.alloc(np_));
    CK(lat_.upload(h.data(), np_));
    return DEM_OK;
  }

  // Secant modulus and secant Poisson ratio of a uniaxial specimen at the last
  // completed step: stress from that step's platen force sums, lateral strain
  // from the mean radial distance of the marked surface particles against
  // set-up.  The sensitivity build (dual numbers) adds their derivatives;
  // other builds report zeros there.
  int sensitivities(int32_t si, dem_sensitivity* out) override {
    if (si < 0 || (size_t)si >= samples_.size() || !out) return DEM_ERR_ARG;
    if (!setup_done_) return DEM_ERR_STATE;
    constexpr int K = DualK<Real>::K;
    const SampleHost& sh = samples_[si];
    SampleCtl C;
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(&C, ctl_.p + si, sizeof(C), cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof(*out));
    const double eps = -C.Strain;
    out->strain = eps;
    out->stress = C.Stress;
    out->E_secant = std::nan("");
    out->nu_secant = std::nan("");
    if constexpr (K > 0) {
      static_assert(K == DEM_SENS_COUNT, "derivative slots");
      std::vector<double> t(4 * K + 2);
      CK(cudaMemcpy(t.data(), sfl_tan_.p + (size_t)si * (4 * K + 2), t.size() * sizeof(double),
                    cudaMemcpyDeviceToHost));
      const double g0 = t[4 * K] < 0 ? -1.0 : 1.0, g1 = t[4 * K + 1] < 0 ? -1.0 : 1.0;
      for (int k = 0; k < K; ++k) out->dstress[k] = 0.5 * (g0 * t[2 * K + k] + g1 * t[3 * K + k]) * C.inv_Area;
    }
    if (!(eps != 0)) return DEM_OK;
    out->E_secant = out->stress / eps;
    for (int k = 0; k < K; ++k) out->dE[k] = out->dstress[k] / eps;
    if (!sh.lat_count || !(sh.lat_rho0 > 0)) return DEM_OK;
    std::vector<V4> h(sh.n);
    CK(cudaMemcpy(h.data(), pos_.p + sh.p_begin, sh.n * sizeof(V4), cudaMemcpyDeviceToHost));
    const double cx = sh.load.center_real[0], cy = sh.load.center_real[1];
    double rho = 0, drho[K > 0 ? K : 1] = {};
    for (uint32_t k = 0; k < sh.n; ++k) {
      if (!hlat_[sh.p_begin + k]) continue;
      const double ex = (double)h[k].x - cx, ey = (double)h[k].y - cy, r = std::sqrt(ex * ex + ey * ey);
      rho += r;
      if constexpr (K > 0)
        for (int q = 0; q < K; ++q) drho[q] += (ex * h[k].x.d[q] + ey * h[k].y.d[q]) / r;
    }
    rho /= sh.lat_count;
    out->nu_secant = (rho - sh.lat_rho0) / sh.lat_rho0 / eps;
    for (int q = 0; q < K; ++q) out->dnu[q] = drho[q] / sh.lat_count / sh.lat_rho0 / eps;
    return DEM_OK;
  }

  void derive(SampleHost& s) {
    const dem_material& m = s.mat;
    s.rmin = 1e300;
    s.rmax = 0;
    double sum = 0;
    for (float r : s.rad) {
      s.rmin = std::min(s.rmin, (double)r);
      s.rmax = std::max(s.rmax, (double)r);
      sum += r;
    }
    s.rmean = sum / s.n;
    Potential& P = s.pot;
    P.m_E = m.E;
    P.m_nu = m.nu;
    P.m_Ec = m.Ec;
    P.m_Gc = m.Gc;
    P.b_r = m.b_r > 0 ? m.b_r : m.bond_radius_factor * s.rmin;
    // monodisperse specimens use the reference's p_r; polydisperse ones the
    // smallest radius, which bounds the stable time step
    P.p_r = (s.rmin == s.rmax) ? (double)s.rmin : s.rmin;
    if (m.p_r > 0 && s.rmin == s.rmax && (float)m.p_r == (float)s.rmin) P.p_r = m.p_r;
    P.b_d = 2.0 * P.p_r + m.gap;
    P.m_ro = m.rho;
    P.p_e = m.p_e;
    P.p_mu = m.mu;
    P.p_mur = m.mur;
    P.a_farcut = m.farcut * (m.p_r > 0 ? m.p_r : s.rmean);
    P.calculate();
    s.E_b = m.E_bond > 0 ? m.E_bond : m.E;
    s.G_b = m.kn_ks > 0 ? s.E_b / m.kn_ks : 0.5 * s.E_b / (1.0 + m.nu);
    s.dt = P.dt;
    if (m.dt_rayleigh_factor > 0) {
      // the reference's rule (0.05 min(T_Rayleigh, T_bond), potential_data::
      // CalculateParameters) with the caller's factor, for the smallest sphere
      // and the stiffest bond it can carry: T_bond = 2 sqrt(m / k), k the bond
      // stiffness max(E_b, G_b) pi b^2 / (2 r) of a bond of that sphere
      const double r = s.rmin;
      const double b = m.b_r > 0 ? P.b_r : m.bond_radius_factor * r;
      const double k = std::max(s.E_b, s.G_b) * kPiD * b * b / (2.0 * r);
      const double mass = m.rho * 4.0 * (1.0 / 3.0) * kPiD * r * r * r;
      double T = rayleigh_time(r, m.rho, m.E, m.nu);
      if (k > 0) T = std::min(T, 2.0 * std::sqrt(mass / k));
      s.dt = m.dt_rayleigh_factor * T;
    }
    if (m.dt > 0) s.dt = m.dt;
    s.hm_E = P.hm_E;
    s.hm_G = P.hm_G;
  }

  // Quantisation frame of a sample's Morton keys (lower corner of its
  // particles, 1/r_min); returns the bits a key may need (3 x the bit length
  // of the largest cell coordinate).
  int morton_frame(const SampleHost& s, MortonFrame& F) {
    const uint32_t n = s.n;
    const uint32_t T = chunk_count(n);
    F.inv_q = 1.0 / std::max(s.rmin, 1e-6);
    F.p_begin = s.p_begin;
    F.n = n;
    // lower and upper corner of the particles (per-chunk extrema, then combined)
    std::vector<double> clo(3 * (size_t)T, 1e300), chi(3 * (size_t)T, -1e300);
    parallel_chunks(n, T, [&](uint32_t t, uint32_t k0, uint32_t k1) {
      for (int d = 0; d < 3; ++d) {
        double m = 1e300, M = -1e300;
        for (uint32_t i = k0; i < k1; ++i) {
          const double v = (double)s.xyz[d * n + i];
          m = std::min(m, v);
          M = std::max(M, v);
        }
        clo[3 * t + d] = m;
        chi[3 * t + d] = M;
      }
    });
    double hi[3] = {-1e300, -1e300, -1e300};
    for (int d = 0; d < 3; ++d) F.lo[d] = 1e300;
    for (uint32_t t = 0; t < T; ++t)
      for (int d = 0; d < 3; ++d) {
        F.lo[d] = std::min(F.lo[d], clo[3 * t + d]);
        hi[d] = std::max(hi[d], chi[3 * t + d]);
      }
    int bits = 0;
    for (int d = 0; d < 3; ++d) {
      const uint32_t c = (uint32_t)std::min(std::max((hi[d] - F.lo[d]) * F.inv_q, 0.0), 2097151.0);
      int b = 0;
      while (b < 32 && (c >> b) != 0) ++b;
      bits = std::max(bits, 3 * b);
    }
    return bits;
  }

  // Morton order on the device: keys of every sample's particles (the sample
  // index above mbits), a stable LSD radix sort over `bits` bits, and the
  // storage order written into the stage's order slot (and to the host).
  int device_morton(float* stage, const std::vector<MortonFrame>& frames, int mbits, int bits) {
    const uint32_t S = (uint32_t)frames.size();
    DBuf<MortonFrame> fr;
    DBuf<uint64_t> ka, kb;
    DBuf<uint32_t> va, vb, hist, offs;
    CK(fr.alloc(S));
    CK(cudaMemcpyAsync(fr.p, frames.data(), S * sizeof(MortonFrame), cudaMemcpyHostToDevice, stream_));
    const uint32_t nblk = ceil_div(np_, kSortItems);
    CK(ka.alloc(np_));
    CK(kb.alloc(np_));
    CK(va.alloc(np_));
    CK(vb.alloc(np_));
    CK(hist.alloc(256 * (size_t)nblk));
    CK(offs.alloc(256 * (size_t)nblk + 1));
    k_morton_keys<<<grid1(np_), 256, 0, stream_>>>(stage, np_, fr.p, S, mbits, ka.p, va.p);
    for (int shift = 0; shift < bits; shift += 8) {
      k_radix_hist<<<nblk, 256, 0, stream_>>>(ka.p, np_, shift, hist.p);
      RC(scan(hist.p, offs.p, 256 * nblk));
      k_radix_scatter<<<nblk, 256, 0, stream_>>>(ka.p, va.p, np_, shift, offs.p, kb.p, vb.p);
      ka.swap(kb);
      va.swap(vb);
    }
    uint32_t* perm = reinterpret_cast<uint32_t*>(stage + 4 * (size_t)np_);
    k_morton_perm<<<grid1(np_), 256, 0, stream_>>>(va.p, np_, fr.p, S, perm);
    CK(cudaGetLastError());
    for (auto& s : samples_) {
      s.perm.resize(s.n);
      CK(cudaMemcpyAsync(s.perm.data(), perm + s.p_begin, s.n * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
      s.inv.clear();   // built when first needed (inverse())
    }
    CK(cudaStreamSynchronize(stream_));   // before the sort's buffers are released
    return DEM_OK;
  }

  void morton_order(SampleHost& s) {
    const uint32_t n = s.n;
    const uint32_t T = chunk_count(n);
    MortonFrame F;
    morton_frame(s, F);
    const double inv_q = F.inv_q;
    const double* lo = F.lo;
    // keys, and their largest value (only the digits below its top bit vary)
    // (left uninitialised: every entry is written before it is read)
    std::unique_ptr<uint64_t[]> ka(new uint64_t[n]), kb(new uint64_t[n]);
    std::unique_ptr<uint32_t[]> pa(new uint32_t[n]), pb(new uint32_t[n]);
    std::vector<uint64_t> kmax(T, 0);
    parallel_chunks(n, T, [&](uint32_t t, uint32_t i0, uint32_t i1) {
      uint64_t m = 0;
      for (uint32_t i = i0; i < i1; ++i) {
        uint32_t c[3];
        for (int d = 0; d < 3; ++d) {
          double v = ((double)s.xyz[d * n + i] - lo[d]) * inv_q;
          c[d] = (uint32_t)std::min(std::max(v, 0.0), 2097151.0);
        }
        ka[i] = morton3(c[0], c[1], c[2]);
        pa[i] = i;
        m = std::max(m, ka[i]);
      }
      kmax[t] = m;
    });
    uint64_t km = 0;
    for (uint64_t m : kmax) km = std::max(km, m);
    int bits = 0;
    while (bits < 64 && (km >> bits) != 0) ++bits;
    // stable LSD radix sort of (key, index) pairs, 8-bit digits, each pass in
    // parallel: per-chunk digit counts, offsets bucket by bucket and chunk by
    // chunk, then every chunk scatters its items in order, so equal keys keep
    // ascending index order
    std::vector<uint32_t> hist(256 * (size_t)T);
    for (int shift = 0; shift < bits; shift += 8) {
      parallel_chunks(n, T, [&](uint32_t t, uint32_t k0, uint32_t k1) {
        uint32_t* h = &hist[256 * (size_t)t];
        std::fill(h, h + 256, 0u);
        for (uint32_t k = k0; k < k1; ++k) ++h[(ka[k] >> shift) & 255];
      });
      uint32_t run = 0;
      for (uint32_t d = 0; d < 256; ++d)
        for (uint32_t t = 0; t < T; ++t) {
          const uint32_t c = hist[256 * (size_t)t + d];
          hist[256 * (size_t)t + d] = run;
          run += c;
        }
      parallel_chunks(n, T, [&](uint32_t t, uint32_t k0, uint32_t k1) {
        uint32_t* h = &hist[256 * (size_t)t];
        for (uint32_t k = k0; k < k1; ++k) {
          const uint32_t o = h[(ka[k] >> shift) & 255]++;
          kb[o] = ka[k];
          pb[o] = pa[k];
        }
      });
      ka.swap(kb);
      pa.swap(pb);
    }
    s.perm.resize(n);
    parallel_ranges(n, [&](uint32_t k0, uint32_t k1) { std::copy(pa.get() + k0, pa.get() + k1, s.perm.data() + k0); });
    s.inv.clear();   // built when first needed (inverse())
  }

  // caller index -> storage position of a sample
  const std::vector<uint32_t>& inverse(SampleHost& s) {
    if (s.inv.size() != s.n) {
      s.inv.resize(s.n);
      for (uint32_t k = 0; k < s.n; ++k) s.inv[s.perm[k]] = k;
    }
    return s.inv;
  }

  static V4 make4(Real a, Real b, Real c, Real d) {
    V4 v;
    v.x = a;
    v.y = b;
    v.z = c;
    v.w = d;
    return v;
  }

  int upload_params() {
    const uint32_t S = (uint32_t)samples_.size();
    std::vector<SampleParams<Real>> hp(S);
    std::vector<BondLaw<Real>> hl(S);
    std::vector<double> hgap(S), hskin(S);
    for (uint32_t si = 0; si < S; ++si) {
      const SampleHost& s = samples_[si];
      const dem_material& m = s.mat;
      const dem_loading& L = s.load;
      SampleParams<Real>& p = hp[si];
      p.dt = (Real)s.dt;
      p.E = (Real)s.E_b;
      p.G = (Real)s.G_b;
      p.hmE = (Real)s.hm_E;
      p.hmG = (Real)s.hm_G;
      const bool brazil = L.test == DEM_TEST_BRAZIL;
      p.wallE = brazil ? (Real)s.hm_E : (Real)(2.0 * s.hm_E);
      p.wallG = brazil ? (Real)s.hm_G : (Real)(2.0 * s.hm_G);
      // sensitivity build: bond moduli against E_bond and kn/ks, contact and
      // platen moduli against the particle E (all proportional to it)
      {
        const int kE = m.E_bond > 0 ? kSensEBond : kSensE;
        set_d(p.E, kE, 1.0);
        if (m.kn_ks > 0) {
          set_d(p.G, kE, 1.0 / m.kn_ks);
          set_d(p.G, kSensKnKs, -s.E_b / (m.kn_ks * m.kn_ks));
        } else {
          set_d(p.G, kE, s.G_b / s.E_b);
        }
        set_d(p.hmE, kSensE, s.hm_E / m.E);
        set_d(p.hmG, kSensE, s.hm_G / m.E);
        set_d(p.wallE, kSensE, (double)p.wallE / m.E);
        set_d(p.wallG, kSensE, (double)p.wallG / m.E);
      }
      p.pA = (Real)s.pot.p_A;
      p.mu = (Real)m.mu;
      set_d(p.mu, kSensMu, 1.0);   // sensitivity build: sliding friction (pairs and platens)
      p.mur = (Real)m.mur;
      p.aa_far = (Real)s.pot.aa_farcut;
      const double skin = opt_.skin_factor * s.rmin;
      p.skin_half2 = (Real)(0.25 * skin * skin);
      for (int d = 0; d < 3; ++d) {
        p.space_c[d] = (Real)(float)L.space_center[d];
        p.space_h[d] = (Real)(float)L.space_half[d];
        p.hide[d] = (Real)(float)L.hidden_point[d];
        p.wall_c[d] = (float)L.center_real[d];
      }
      p.axis = L.test == DEM_TEST_UNIAXIAL ? 2 : (brazil ? 1 : -1);
      p.zcut = (float)L.zcut;
      // lateral radius of the platen zone (compression_data::Calculate{U,B}Parameters)
      const float sx2 = (float)(0.5 * L.size_real[0]), sz2 = (float)(0.5 * L.size_real[2]);
      float Rw = brazil ? ((sx2 > sz2) ? sx2 : (float)(1.05 * sz2)) : (float)(1.5 * sx2);
      p.wall_RR = Rw * Rw;
      p.nobreak = m.nobreak;
      p.p_begin = s.p_begin;
      p.p_end = s.p_begin + s.n;
      BondLaw<Real>& l = hl[si];
      l.br_abs = m.b_r > 0 ? (Real)s.pot.b_r : Real(0);
      l.br_factor = (Real)m.bond_radius_factor;
      if (m.b_r > 0)
        set_d(l.br_abs, kSensBondRadius, 1.0);
      else
        set_d(l.br_factor, kSensBondRadius, 1.0);
      l.sn_mean = (Real)m.Ec;
      l.sn_sd = (Real)m.Ec_sd;
      l.st_mean = (Real)m.Gc;
      l.st_sd = (Real)m.Gc_sd;
      l.seed = m.seed;
      hgap[si] = m.gap;
      hskin[si] = skin;
    }
    CK(sp_.alloc(S));
    CK(sp_.upload(hp.data(), S));
    CK(law_.alloc(S));
    CK(law_.upload(hl.data(), S));
    CK(gap_.alloc(S));
    CK(gap_.upload(hgap.data(), S));
    CK(skin_.alloc(S));
    CK(skin_.upload(hskin.data(), S));
    hparams_ = hp;
    return DEM_OK;
  }

  int make_grids() {
    const uint32_t S = (uint32_t)samples_.size();
    std::vector<Grid<Real>> hg(S);
    uint32_t off = 0;
    for (uint32_t si = 0; si < S; ++si) {
      const SampleHost& s = samples_[si];
      const double skin = opt_.skin_factor * s.rmin;
      double a = 2.0 * s.rmax + skin;
      const double bond_reach = 2.0 * s.rmax + std::max(0.0, s.pot.b_d - 2.0 * s.pot.p_r);
      a = std::max(a, bond_reach) * 1.0001;
      Grid<Real>& g = hg[si];
      double lo[3], hi[3];
      for (int d = 0; d < 3; ++d) {
        lo[d] = s.load.space_center[d] - s.load.space_half[d];
        hi[d] = s.load.space_center[d] + s.load.space_half[d];
        if (s.load.space_half[d] <= 0) {  // no escape box: use the particle extent
          lo[d] = 1e300;
          hi[d] = -1e300;
          for (uint32_t i = 0; i < s.n; ++i) {
            lo[d] = std::min(lo[d], (double)s.xyz[d * s.n + i]);
            hi[d] = std::max(hi[d], (double)s.xyz[d * s.n + i]);
          }
        }
        lo[d] -= a;
        hi[d] += a;
      }
      g.ox = (Real)lo[0];
      g.oy = (Real)lo[1];
      g.oz = (Real)lo[2];
      g.inv_a = (Real)(1.0 / a);
      g.nx = (uint32_t)std::ceil((hi[0] - lo[0]) / a) + 1;
      g.ny = (uint32_t)std::ceil((hi[1] - lo[1]) / a) + 1;
      g.nz = (uint32_t)std::ceil((hi[2] - lo[2]) / a) + 1;
      g.off = off;
      off += g.nx * g.ny * g.nz;
      g.hx = (Real)(float)s.load.hidden_point[0];
      g.hy = (Real)(float)s.load.hidden_point[1];
      g.hz = (Real)(float)s.load.hidden_point[2];
      g.skip_hidden = (s.load.space_half[0] > 0 && s.load.space_half[1] > 0 && s.load.space_half[2] > 0) ? 1u : 0u;
    }
    ncell_ = off;
    CK(grids_.alloc(S));
    CK(grids_.upload(hg.data(), S));
    CK(cell_of_.alloc(np_));
    CK(cell_count_.alloc(ncell_ + 1));
    CK(cell_start_.alloc(ncell_ + 1));
    CK(cell_cursor_.alloc(ncell_ + 1));
    CK(cell_list_.alloc(np_));
    CK(cnt_.alloc(np_ + 1));
    CK(offs_.alloc(np_ + 1));
    CK(ovf_.alloc(1));
    return DEM_OK;
  }

  // exclusive scan of n values into out[0..n], out[n] = total
  int scan(const uint32_t* in, uint32_t* out, uint32_t n) {
    const uint32_t nb = ceil_div(n, kScanBlock);
    std::vector<std::pair<uint32_t*, uint32_t>> levels;
    if (scan_tmp_.n < 2 * (size_t)nb + 2048) CK(scan_tmp_.alloc(2 * (size_t)nb + 2048));
    uint32_t* sums = scan_tmp_.p;
    uint32_t* sums_scan = scan_tmp_.p + nb + 1024;
    k_scan_block<<<std::max(nb, 1u), kScanBlock, 0, stream_>>>(in, out, n, sums);
    if (nb > 1) {
      if (nb > kScanBlock) {
        // second level recursively (rare: more than ~1M elements)
        DBuf<uint32_t> s2;
        CK(s2.alloc(nb + 1));
        RC(scan(sums, s2.p, nb));
        CK(cudaMemcpyAsync(sums_scan, s2.p, nb * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream_));
        CK(cudaStreamSynchronize(stream_));
      } else {
        k_scan_block<<<1, kScanBlock, 0, stream_>>>(sums, sums_scan, nb, nullptr);
      }
      k_scan_add<<<nb, kScanBlock, 0, stream_>>>(out, n, sums_scan);
    }
    k_scan_total<<<1, 1, 0, stream_>>>(in, out, n);
    CK(cudaGetLastError());
    return DEM_OK;
  }

  int bin_cells() {
    const uint32_t g = grid1(np_);
    CK(cudaMemsetAsync(cell_count_.p, 0, (ncell_ + 1) * sizeof(uint32_t), stream_));
    k_cell_index<Real><<<g, 256, 0, stream_>>>(pos_.p, sid_.p, np_, grids_.p, cell_of_.p, cell_count_.p);
    RC(scan(cell_count_.p, cell_start_.p, ncell_));
    CK(cudaMemcpyAsync(cell_cursor_.p, cell_start_.p, (ncell_ + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                       stream_));
    k_scatter_cells<<<g, 256, 0, stream_>>>(cell_of_.p, np_, cell_cursor_.p, cell_list_.p);
    k_sort_cells<<<grid1(ncell_), 256, 0, stream_>>>(cell_start_.p, ncell_, cell_list_.p);
    CK(cudaGetLastError());
    return DEM_OK;
  }

  uint32_t grid1(uint64_t n) const {
    return std::max(1u, std::min(ceil_div(n, 256), (uint32_t)num_sms_ * 16));
  }

  PairSearch<Real> search_args(int mode) {
    PairSearch<Real> S{};
    S.pos = pos_.p;
    S.sid = sid_.p;
    S.np = np_;
    S.grids = grids_.p;
    S.cell_start = cell_start_.p;
    S.cell_list = cell_list_.p;
    S.mode = mode;
    S.count = cnt_.p;
    S.offset = offs_.p;
    S.cap = 48;
    S.overflow = ovf_.p;
    return S;
  }

  int build_bonds() {
    RC(bin_cells());
    PairSearch<Real> S = search_args(kModeBond);
    S.gap = gap_.p;
    CK(cudaMemsetAsync(ovf_.p, 0, sizeof(uint32_t), stream_));
    // one search pass: every sphere's count and its sorted partners in
    // kSearchStride slots of its own (the slots serve the contact-list builds
    // too), compacted below once the counts are scanned
    if (c_jstride_.n < (size_t)np_ * kSearchStride) CK(c_jstride_.alloc((size_t)np_ * kSearchStride));
    S.out_j = c_jstride_.p;
    k_pair_search<Real, 2><<<pair_search_blocks(np_), 128, 0, stream_>>>(S);
    RC(scan(cnt_.p, offs_.p, np_));
    uint32_t nb = 0, ovf = 0;
    CK(cudaMemcpyAsync(&nb, offs_.p + np_, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(&ovf, ovf_.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    if (ovf) return DEM_ERR_CAPACITY;
    nb_ = nb;
    // whole tiles: the pair kernel copies bond state tile by tile
    const size_t nb_pad = ((size_t)std::max(nb, 1u) + 255) / 256 * 256;
    CK(b_ij_.alloc(nb_pad));
    CK(b_s0_.alloc(nb_pad));
    CK(b_s1_.alloc(nb_pad));
    CK(b_s2_.alloc(nb_pad));
    CK(b_par_.alloc(nb_pad));
    CK(b_row_.alloc(np_ + 1));
    const uint32_t S_ = (uint32_t)samples_.size();
    DBuf<int32_t> counts;
    CK(counts.alloc(S_));
    k_expand_stride<<<grid1(np_), 256, 0, stream_>>>(offs_.p, np_, c_jstride_.p, b_ij_.p);
    CK(cudaMemcpyAsync(b_row_.p, offs_.p, (np_ + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream_));
    if (nb)
      k_bond_init<Real><<<grid1(nb), 256, 0, stream_>>>(b_ij_.p, nb, pos_.p, sid_.p, orig_.p, law_.p, b_s0_.p,
                                                       b_s1_.p, b_s2_.p, b_par_.p, counts.p);
    // bond range of every sample (bonds are stored in particle order, and the
    // particles of a sample are contiguous): the bond row at each sample's
    // first particle, and at the end, gathered on the device
    std::vector<uint32_t> hidx(S_ + 1), hrow(S_ + 1);
    for (uint32_t si = 0; si < S_; ++si) hidx[si] = samples_[si].p_begin;
    hidx[S_] = np_;
    DBuf<uint32_t> ridx, rval;
    CK(ridx.alloc(S_ + 1));
    CK(rval.alloc(S_ + 1));
    CK(cudaMemcpyAsync(ridx.p, hidx.data(), (S_ + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_));
    k_gather_u32<<<ceil_div(S_ + 1, 256), 256, 0, stream_>>>(b_row_.p, ridx.p, S_ + 1, rval.p);
    CK(cudaGetLastError());
    std::vector<int32_t> hc(S_);
    CK(cudaMemcpyAsync(hc.data(), counts.p, S_ * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(hrow.data(), rval.p, (S_ + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    for (uint32_t si = 0; si < S_; ++si) samples_[si].bonds_initial = hc[si];
    sb_begin_.assign(S_, 0);
    sb_end_.assign(S_, 0);
    for (uint32_t si = 0; si < S_; ++si) {
      sb_begin_[si] = hrow[si];
      sb_end_[si] = hrow[si + 1];
    }
    tiles_.release();
    ntiles_.release();
    tiles_on_ = false;
    ndone_seen_ = 0;
    return tile_samples();
  }

  // Sample of every bond tile of the current pair-kernel block size (~0u for
  // a tile spanning two samples).
  int tile_samples() {
    tile_s_.release();
    const uint32_t S = (uint32_t)sb_begin_.size();
    if (nb_ == 0 || S == 0) return DEM_OK;
    const uint32_t tile = opt_.pair_block, T = (nb_ + tile - 1) / tile;
    std::vector<uint32_t> h(T, ~0u);
    uint32_t si = 0;
    for (uint32_t t = 0; t < T; ++t) {
      const uint32_t b0 = t * tile, b1 = std::min(nb_, b0 + tile) - 1;
      while (si < S && sb_end_[si] <= b0) ++si;
      if (si < S && sb_begin_[si] <= b0 && b1 < sb_end_[si]) h[t] = si;
    }
    CK(tile_s_.alloc(T));
    CK(tile_s_.upload(h.data(), T));
    return DEM_OK;
  }

  // Batched runs: finished samples stop costing work.  Their contacts are left
  // out of the next contact-list builds, and once their bonds make up an
  // eighth of all bonds the pair kernel visits only the bond tiles that hold a
  // bond of an unfinished sample (a tile list read through one indirection;
  // the graph is captured again with it).  A finished sample's state no longer
  // changes either way (its pairs and particles are skipped), so results are
  // unchanged.  Called after read_flags, with the stream idle.
  int update_tiles() {
    const uint32_t S = (uint32_t)samples_.size();
    uint32_t nd = 0;
    size_t done_bonds = 0;
    for (uint32_t si = 0; si < S; ++si)
      if (hctl_[si].done) {
        ++nd;
        if (si < sb_end_.size()) done_bonds += sb_end_[si] - sb_begin_[si];
      }
    if (nd == ndone_seen_) return DEM_OK;
    ndone_seen_ = nd;
    if (!sdone_.p) CK(sdone_.alloc(S));
    std::vector<uint32_t> hd(S);
    for (uint32_t si = 0; si < S; ++si) hd[si] = hctl_[si].done ? 1u : 0u;
    CK(cudaMemcpy(sdone_.p, hd.data(), S * sizeof(uint32_t), cudaMemcpyHostToDevice));
    if (nb_ == 0 || 8 * done_bonds < (size_t)nb_) return DEM_OK;
    const uint32_t tile = opt_.pair_block, T = (nb_ + tile - 1) / tile;
    std::vector<uint8_t> act(T, 0);
    for (uint32_t si = 0; si < S; ++si)
      if (!hd[si] && sb_end_[si] > sb_begin_[si])
        for (uint32_t t = sb_begin_[si] / tile; t <= (sb_end_[si] - 1) / tile; ++t) act[t] = 1;
    std::vector<uint32_t> list;
    list.reserve(T);
    for (uint32_t t = 0; t < T; ++t)
      if (act[t]) list.push_back(t);
    if (!tiles_.p) {
      CK(tiles_.alloc(T));
      CK(ntiles_.alloc(1));
    }
    const uint32_t cnt = (uint32_t)list.size();
    if (cnt) CK(cudaMemcpy(tiles_.p, list.data(), cnt * sizeof(uint32_t), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ntiles_.p, &cnt, sizeof(uint32_t), cudaMemcpyHostToDevice));
    if (!tiles_on_) {
      tiles_on_ = true;
      invalidate_graph();
    }
    return DEM_OK;
  }

  // Rebuilds the contact list from the current positions; pairs that existed
  // keep their tangential history.
  int build_contacts(bool first) {
    RC(bin_cells());
    PairSearch<Real> S = search_args(kModeContact);
    S.gap = skin_.p;
    S.done = sdone_.p;
    S.b_row = b_row_.p;
    S.b_ij = b_ij_.p;
    CK(cudaMemsetAsync(ovf_.p, 0, sizeof(uint32_t), stream_));
    // one search pass (the counts and every particle's partners, sorted, in
    // kSearchStride slots of its own, compacted below once the counts are
    // scanned)
    if (c_jstride_.n < (size_t)np_ * kSearchStride) CK(c_jstride_.alloc((size_t)np_ * kSearchStride));
    S.out_j = c_jstride_.p;
    k_pair_search<Real, 2><<<pair_search_blocks(np_), 128, 0, stream_>>>(S);
    RC(scan(cnt_.p, offs_.p, np_));
    uint32_t nc = 0, ovf = 0;
    CK(cudaMemcpyAsync(&nc, offs_.p + np_, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(&ovf, ovf_.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    if (ovf) return DEM_ERR_CAPACITY;
    const size_t need = std::max<size_t>(nc, 1);
    if (first || need > c_ij_.n) {
      const size_t cap = std::max<size_t>(need + need / 2, (size_t)np_ * 2 + 1024);
      // keep the old list for the carry-over
      DBuf<uint2> old_ij;
      DBuf<V4> old_o;
      DBuf<uint32_t> old_row;
      const uint32_t old_nc = nc_host_;
      if (!first) {
        CK(old_ij.alloc(std::max<size_t>(old_nc, 1)));
        CK(old_o.alloc(std::max<size_t>(old_nc, 1)));
        CK(old_row.alloc(np_ + 1));
        CK(cudaMemcpyAsync(old_ij.p, c_ij_.p, old_nc * sizeof(uint2), cudaMemcpyDeviceToDevice, stream_));
        CK(cudaMemcpyAsync(old_o.p, c_o_.p, old_nc * sizeof(V4), cudaMemcpyDeviceToDevice, stream_));
        CK(cudaMemcpyAsync(old_row.p, c_row_.p, (np_ + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream_));
      }
      CK(cudaStreamSynchronize(stream_));
      CK(c_ij_.alloc(cap));
      CK(c_o_.alloc(cap));
      CK(c_ij_new_.alloc(cap));
      CK(c_o_new_.alloc(cap));
      CK(c_row_.alloc(np_ + 1));
      CK(nc_dev_.alloc(1));
      invalidate_graph();
      if (!first) {
        CK(cudaMemcpyAsync(c_ij_.p, old_ij.p, old_nc * sizeof(uint2), cudaMemcpyDeviceToDevice, stream_));
        CK(cudaMemcpyAsync(c_o_.p, old_o.p, old_nc * sizeof(V4), cudaMemcpyDeviceToDevice, stream_));
        CK(cudaMemcpyAsync(c_row_.p, old_row.p, (np_ + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream_));
        CK(cudaStreamSynchronize(stream_));
      }
    }
    k_expand_stride<<<grid1(np_), 256, 0, stream_>>>(offs_.p, np_, c_jstride_.p, c_ij_new_.p);
    if (nc) {
      if (first)
        CK(cudaMemsetAsync(c_row_.p, 0, (np_ + 1) * sizeof(uint32_t), stream_));
      k_contact_carry<Real><<<grid1(nc), 256, 0, stream_>>>(c_ij_new_.p, nc, c_o_new_.p, c_ij_.p, c_o_.p, c_row_.p);
      CK(cudaMemcpyAsync(c_ij_.p, c_ij_new_.p, nc * sizeof(uint2), cudaMemcpyDeviceToDevice, stream_));
      CK(cudaMemcpyAsync(c_o_.p, c_o_new_.p, nc * sizeof(V4), cudaMemcpyDeviceToDevice, stream_));
    }
    CK(cudaMemcpyAsync(c_row_.p, offs_.p, (np_ + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream_));
    CK(cudaMemcpyAsync(nc_dev_.p, &nc, sizeof(uint32_t), cudaMemcpyHostToDevice, stream_));
    k_copy_pos<Real><<<grid1(np_), 256, 0, stream_>>>(pos_.p, pos_ref_.p, np_);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
    nc_host_ = nc;
    ++rebuilds_;
    return DEM_OK;
  }

  int init_controllers() {
    const uint32_t S = (uint32_t)samples_.size();
    std::vector<SampleCtl> hc(S);
    rec_.resize(S);
    rec_bonds_.resize(S);
    rec_lat_.resize(S);
    for (uint32_t si = 0; si < S; ++si) {
      const SampleHost& s = samples_[si];
      const dem_loading& L = s.load;
      SampleCtl& C = hc[si];
      std::memset(&C, 0, sizeof(C));
      const bool brazil = L.test == DEM_TEST_BRAZIL;
      const int ax = brazil ? 1 : 2;
      C.brazil = brazil ? 1 : 0;
      for (int d = 0; d < 3; ++d) C.size_d[d] = L.size_real[d];
      const double pr = L.p_r_platen > 0 ? L.p_r_platen : (s.mat.p_r > 0 ? s.mat.p_r : s.rmean);
      C.p_r = pr;
      C.Size0 = C.size_d[ax];
      C.Bottom = L.center_real[ax] - 0.5 * C.size_d[ax];
      C.Top = L.center_real[ax] + 0.5 * C.size_d[ax];
      const float sx2 = (float)(0.5 * C.size_d[0]);
      const float sizez = (float)C.size_d[2];
      float area;
      if (!brazil) {
        area = (float)(kPiD * (sx2 + pr) * (sx2 + pr));
        C.ZeroStress = 0.33 * L.min_stress;
      } else {
        area = (float)(0.5 * 2 * kPiD * (sx2) * (sizez));
        C.ZeroStress = 0.5 * L.min_stress;
      }
      C.inv_Area = (float)(1.0 / area);
      C.sz0 = (double)(float)C.size_d[ax];
      C.MinStress = L.min_stress;
      C.MaxStrain = L.test == DEM_TEST_NONE ? 1e300 : L.max_strain;
      C.ConditionFracture = L.cond_fracture;
      C.VLoad = L.velocity;
      C.V = 0;
      C.dt = s.dt;
      C.max_steps = L.max_steps ? L.max_steps : ~0ull;
      C.stop_at = ~0ull;
      C.bonds = s.bonds_initial;
      C.dNsave = L.dNsave;
      uint64_t nsave = 16;
      if (L.test != DEM_TEST_NONE && L.dNsave && std::fabs(L.velocity) > 0) {
        double v = 1.5 * L.max_strain * C.size_d[ax] / (std::fabs(L.velocity) * s.dt * L.dNsave);
        nsave = (uint64_t)std::min(v, 4.0e7);
      }
      if (L.max_steps && L.dNsave) nsave = std::min<uint64_t>(nsave, L.max_steps / L.dNsave + 2);
      C.Nsave = (uint32_t)std::max<uint64_t>(nsave, 4);
      RC(alloc_rec(si, C.Nsave));
      C.rec = rec_[si]->p;
      C.rec_bonds = rec_bonds_[si]->p;
      C.rec_lat = rec_lat_[si]->p;
      C.lat_count = s.lat_count;
    }
    CK(ctl_.alloc(S));
    CK(ctl_.upload(hc.data(), S));
    return DEM_OK;
  }

  int alloc_rec(uint32_t si, uint32_t nsave) {
    rec_[si].reset(new DBuf<double>());
    rec_bonds_[si].reset(new DBuf<uint32_t>());
    rec_lat_[si].reset(new DBuf<double>());
    CK(rec_[si]->alloc(3 * ((size_t)nsave + 2)));
    CK(rec_bonds_[si]->alloc((size_t)nsave + 2));
    CK(rec_lat_[si]->alloc((size_t)nsave + 2));
    return DEM_OK;
  }

  // ---------------------------------------------------------------- stepping
  StepArgs<Real> args() {
    StepArgs<Real> A{};
    A.pos = pos_.p;
    A.vel = vel_.p;
    A.omg = omg_.p;
    A.frc = frc_.p;
    A.mom = mom_.p;
    A.wallO = wallO_.p;
    A.wflag = wflag_.p;
    A.pos_ref = pos_ref_.p;
    A.mass = mass_.p;
    A.sid = sid_.p;
    A.np = np_;
    A.b_ij = b_ij_.p;
    A.b_s0 = b_s0_.p;
    A.b_s1 = b_s1_.p;
    A.b_s2 = b_s2_.p;
    A.b_par = b_par_.p;
    A.nb = nb_;
    A.c_ij = c_ij_.p;
    A.c_o = c_o_.p;
    A.nc = nc_dev_.p;
    A.sp = sp_.p;
    A.ctl = ctl_.p;
    A.nsamples = (uint32_t)samples_.size();
    A.blocks_done = blocks_done_.p;
    A.keep_forces = 0;
    A.touching = nullptr;
    A.stat = stat_.p;
    A.lat = lat_.p;
    A.sfl_tan = sfl_tan_.p;
    A.frcq = frcq_.p;
    A.momq = momq_.p;
    A.det = det_ ? 1 : 0;
    A.tiles = tiles_on_ ? tiles_.p : nullptr;
    A.ntiles = tiles_on_ ? ntiles_.p : nullptr;
    A.tile_s = tile_s_.p;
    return A;
  }

  // Pair-kernel variant (register budget and block size) and its grid: all
  // co-resident blocks unless the caller fixed the grid.  Changing it drops
  // the captured graph and the bond-tile list (tiles are blocks).
  int set_pair_config(uint32_t min_blocks) {
    constexpr bool kSmallBlocks = sizeof(Real) == 4 && !DualK<Real>::K;
    if (min_blocks == 0 || min_blocks > (kSmallBlocks ? 8u : 4u))
      min_blocks = DualK<Real>::K ? 1 : (sizeof(Real) == 4 ? 7 : 2);
    opt_.pair_min_blocks = min_blocks;
    opt_.pair_block = min_blocks > 4 ? 128 : 256;
    pair_kernel_ = pair_kernel_ptr(min_blocks, det_);
    if (!user_grid_) {
      int per_sm = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pair_kernel_, (int)opt_.pair_block, 0));
      opt_.pair_grid = (uint32_t)num_sms_ * (uint32_t)std::max(per_sm, 1);
    }
    invalidate_graph();
    tiles_on_ = false;
    ndone_seen_ = 0;
    return setup_done_ ? tile_samples() : DEM_OK;
  }

  // Launch-schedule autotuner: advances the run by `steps` steps per candidate
  // (real steps of the simulation: the state moves on exactly as under a plain
  // run), timing each candidate's steps with CUDA events, and keeps the
  // fastest.  Candidates: the pair kernel's register budgets (FP32: 3 x 256
  // threads, 7, 6, 5 x 128 threads and 4 x 256 threads; FP64: 2, 1, 3) crossed
  // with particle-kernel blocks of 128 and 256 threads.
  int autotune(uint32_t steps, dem_tune_report* rep) override {
    if (!setup_done_ || steps == 0 || !rep) return DEM_ERR_ARG;
    std::vector<uint32_t> pairs;
    if (DualK<Real>::K)
      pairs = {1, 2};
    else if (sizeof(Real) == 4)
      pairs = {7, 3, 6, 5, 4};
    else
      pairs = {2, 1, 3};
    const uint32_t parts[2] = {256, 128};
    std::memset(rep, 0, sizeof(*rep));
    double best = 1e300;
    uint32_t bp = opt_.pair_min_blocks, bq = opt_.particle_block;
    int k = 0;
    for (uint32_t pm : pairs)
      for (uint32_t pb : parts) {
        RC(set_pair_config(pm));
        opt_.particle_block = pb;
        double ms = 0.0;
        RC(run_timed(std::min<uint64_t>(steps, opt_.graph_steps), &ms));   // warm-up and capture
        RC(run_timed(steps, &ms));
        if (k < DEM_TUNE_MAX) {
          rep->pair_min_blocks[k] = pm;
          rep->particle_block[k] = pb;
          rep->ms_per_step[k] = ms / steps;
        }
        ++k;
        if (ms < best) {
          best = ms;
          bp = pm;
          bq = pb;
        }
      }
    rep->candidates = std::min(k, (int)DEM_TUNE_MAX);
    rep->chosen_pair_min_blocks = bp;
    rep->chosen_particle_block = bq;
    rep->chosen_ms_per_step = best / steps;
    opt_.particle_block = bq;
    RC(set_pair_config(bp));
    rep->chosen_skin_factor = opt_.skin_factor;
    if (skin_user_) return DEM_OK;
    // Contact-list skin.  A thin skin lists fewer separated pairs but must be
    // rebuilt sooner (once a sphere has moved a quarter of it).  Each
    // candidate runs 4 x `steps` steps with its rebuilds included, in two
    // passes of 2 x `steps` (thin to thick, then thick to thin, so that a
    // drift of the run's speed over the tuning charges all candidates alike);
    // the list is rebuilt at the candidate's skin before each pass (that
    // rebuild timed on its own and reported).
    static constexpr double kSkins[4] = {0.1, 0.2, 0.3, 0.4};
    double tot[4] = {0, 0, 0, 0};
    for (int pass = 0; pass < 2; ++pass)
      for (int q = 0; q < 4; ++q) {
        const int c = pass ? 3 - q : q;
        float t_reb = 0.f;
        RC(set_skin(kSkins[c], &t_reb));
        if (pass == 0) rep->skin_rebuild_ms[c] = t_reb;
        double ms = 0.0;
        RC(run_timed(2 * (uint64_t)steps, &ms));
        tot[c] += ms;
      }
    int bs = 0;
    for (int c = 0; c < 4; ++c) {
      rep->skin_factor[c] = kSkins[c];
      rep->skin_ms_per_step[c] = tot[c] / (4.0 * steps);
      if (tot[c] < tot[bs]) bs = c;
    }
    rep->skin_candidates = 4;
    rep->chosen_skin_factor = kSkins[bs];
    return set_skin(kSkins[bs], nullptr);
  }

  // Contact-list skin after set-up: new cell grids (their edge grows with the
  // skin), per-sample skin parameters, and a list rebuild at the new skin
  // (tangential histories carried over as in any rebuild).
  int set_skin(double factor, float* rebuild_ms) {
    if (!setup_done_ || !(factor > 0)) return DEM_ERR_ARG;
    opt_.skin_factor = factor;
    RC(make_grids());
    RC(upload_params());
    min_skin_ = 1e300;
    for (auto& s : samples_) min_skin_ = std::min(min_skin_, factor * s.rmin);
    invalidate_graph();
    Flags f{};
    RC(read_flags(f));
    cudaEvent_t ea, eb;
    CK(cudaEventCreate(&ea));
    CK(cudaEventCreate(&eb));
    CK(cudaEventRecord(ea, stream_));
    const int rc = build_contacts(false);
    CK(cudaEventRecord(eb, stream_));
    CK(cudaEventSynchronize(eb));
    if (rebuild_ms) CK(cudaEventElapsedTime(rebuild_ms, ea, eb));
    cudaEventDestroy(ea);
    cudaEventDestroy(eb);
    RC(rc);
    return clear_rebuild_flags();
  }

  // Pair kernel variant for a register budget; deterministic FP32 contexts
  // and FP64 contexts get the variants with the warp-summed j side.
  static const void* pair_kernel_ptr(uint32_t min_blocks, bool det) {
    if constexpr (sizeof(Real) == 4 && !DualK<Real>::K) {
      if (det) {
        switch (min_blocks) {
          case 1: return (const void*)k_pairs<Real, 1, 256, true>;
          case 2: return (const void*)k_pairs<Real, 2, 256, true>;
          case 3: return (const void*)k_pairs<Real, 3, 256, true>;
          case 5: return (const void*)k_pairs<Real, 5, 128, true>;
          case 6: return (const void*)k_pairs<Real, 6, 128, true>;
          case 7: return (const void*)k_pairs<Real, 7, 128, true>;
          case 8: return (const void*)k_pairs<Real, 8, 128, true>;
          default: return (const void*)k_pairs<Real, 4, 256, true>;
        }
      }
      switch (min_blocks) {
        case 5: return (const void*)k_pairs<Real, 5, 128>;
        case 6: return (const void*)k_pairs<Real, 6, 128>;
        case 7: return (const void*)k_pairs<Real, 7, 128>;
        case 8: return (const void*)k_pairs<Real, 8, 128>;
        default: break;
      }
    }
    if constexpr (sizeof(Real) == 8) {
      switch (min_blocks) {
        case 1: return (const void*)k_pairs<Real, 1, 256, true>;
        case 2: return (const void*)k_pairs<Real, 2, 256, true>;
        case 3: return (const void*)k_pairs<Real, 3, 256, true>;
        default: return (const void*)k_pairs<Real, 4, 256, true>;
      }
    }
    switch (min_blocks) {
      case 1: return (const void*)k_pairs<Real, 1>;
      case 2: return (const void*)k_pairs<Real, 2>;
      case 3: return (const void*)k_pairs<Real, 3>;
      default: return (const void*)k_pairs<Real, 4>;
    }
  }

  void launch_pairs(const StepArgs<Real>& A) {
    const dim3 g(opt_.pair_grid), b(opt_.pair_block);
    StepArgs<Real> a = A;
    void* params[] = {&a};
    cudaLaunchKernel(pair_kernel_, g, b, params, 0, stream_);
  }

  // Particle kernel grid: the blocks that are resident at once (a grid-stride
  // loop covers the rest), at most 8 per SM.
  uint32_t particle_grid() {
    if (part_occ_block_ != opt_.particle_block) {
      int occ = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_particles<Real>, (int)opt_.particle_block, 0) !=
          cudaSuccess)
        occ = 8;
      part_occ_ = (uint32_t)std::min(std::max(occ, 1), 8);
      part_occ_block_ = opt_.particle_block;
    }
    return std::max(1u, std::min(ceil_div(np_, opt_.particle_block), (uint32_t)num_sms_ * part_occ_));
  }

  void launch_step(const StepArgs<Real>& A, int stages) {
    if (stages & 1) launch_pairs(A);
    if (stages & 2) {
      const uint32_t g = particle_grid();
      k_particles<Real><<<g, opt_.particle_block, 0, stream_>>>(A);
    }
  }

  void invalidate_graph() {
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    graph_exec_ = nullptr;
    for (auto& g : small_graphs_) {
      if (g) cudaGraphExecDestroy(g);
      g = nullptr;
    }
  }

  int capture_steps(uint32_t steps, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    StepArgs<Real> A = args();
    (void)particle_grid();   // occupancy query outside the capture
    CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    for (uint32_t k = 0; k < steps; ++k) launch_step(A, 3);
    cudaError_t e = cudaStreamEndCapture(stream_, &g);
    if (e != cudaSuccess) {
      last_cuda_ = e;
      return DEM_ERR_CUDA;
    }
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      last_cuda_ = e;
      *out = nullptr;
      return DEM_ERR_CUDA;
    }
    return DEM_OK;
  }

  // A chunk shorter than graph_steps (fast particles or a thin skin shorten
  // them) runs as graphs of 64, 16 and 4 steps and single steps, instead of
  // two kernel launches per step.
  static constexpr uint32_t kSizes[3] = {64, 16, 4};

  // Captures every step graph that is missing (the graph_steps graph and the
  // short-chunk graphs).
  int capture_all() {
    if (!graph_exec_) RC(capture_steps(opt_.graph_steps, &graph_exec_));
    for (int k = 0; k < 3; ++k)
      if (kSizes[k] < opt_.graph_steps && !small_graphs_[k]) RC(capture_steps(kSizes[k], &small_graphs_[k]));
    return DEM_OK;
  }

  int run_short_chunk(uint64_t chunk) {
    for (int k = 0; k < 3; ++k) {
      while (chunk >= kSizes[k] && kSizes[k] < opt_.graph_steps) {
        if (!small_graphs_[k]) RC(capture_steps(kSizes[k], &small_graphs_[k]));
        CK(cudaGraphLaunch(small_graphs_[k], stream_));
        chunk -= kSizes[k];
      }
    }
    StepArgs<Real> A = args();
    for (uint64_t s = 0; s < chunk; ++s) launch_step(A, 3);
    return DEM_OK;
  }

  struct Flags {
    uint32_t done, rebuild, stale, numeric;
    float v2max, d2max;
    uint32_t active;       // samples neither done nor at their stop
    uint64_t remaining;    // largest number of steps an active sample still has to go
  };

  int read_flags(Flags& f) {
    const uint32_t S = (uint32_t)samples_.size();
    hctl_.resize(S);
    float st[2] = {0.f, 0.f};
    CK(cudaMemcpyAsync(hctl_.data(), ctl_.p, S * sizeof(SampleCtl), cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(st, stat_.p, 2 * sizeof(float), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    f = {1, 0, 0, 0, st[0], st[1], 0, 0};
    for (auto& c : hctl_) {
      f.done &= c.done ? 1u : 0u;
      f.rebuild |= c.rebuild;
      f.stale |= c.stale;
      f.numeric |= c.numeric;
      if (!c.done && c.step < c.stop_at) {
        ++f.active;
        f.remaining = std::max<uint64_t>(f.remaining, c.stop_at - c.step);
      }
    }
    return DEM_OK;
  }

  // Every sample stops at its current step + n (n = ~0: runs on until done);
  // the hold flags follow.
  int set_stop(uint64_t n) {
    const uint32_t S = (uint32_t)samples_.size();
    k_set_hold<<<ceil_div(S, 128), 128, 0, stream_>>>(ctl_.p, S, n, 0);
    CK(cudaGetLastError());
    return DEM_OK;
  }

  // after a rebuild: clear the per-sample rebuild/stale flags and the
  // displacement maximum (positions are the new reference)
  int clear_rebuild_flags() {
    // rebuild and stale flags cleared, hold flags refreshed (a sample held on a
    // stale list runs again), in one launch
    const uint32_t S = (uint32_t)samples_.size();
    k_set_hold<<<ceil_div(S, 128), 128, 0, stream_>>>(ctl_.p, S, 0ull, 1);
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(stat_.p + 1, 0, sizeof(float), stream_));
    CK(cudaStreamSynchronize(stream_));
    return DEM_OK;
  }

  // Largest number of steps the next chunk may take: a particle may not move
  // more than half the skin between list builds; with the speed of the last
  // chunk and a safety factor on it (2, doubled after every stale event).
  uint64_t chunk_steps(const Flags& f) const {
    const double budget = 0.5 * min_skin_ - std::sqrt((double)f.d2max);
    const double v = std::sqrt((double)f.v2max);
    // no speed seen yet (the first chunk after set-up): a short chunk measures it
    if (!(v > 0)) return std::min<uint64_t>(opt_.graph_steps, 16);
    const double k = budget / (speed_margin_ * v * max_dt_);
    if (!(k >= 1.0)) return 1;
    return (uint64_t)std::min<double>(k, opt_.graph_steps);
  }

  int prepare() {
    if (!setup_done_) return DEM_ERR_STATE;
    if (forces_dirty_) {
      CK(cudaMemsetAsync(frc_.p, 0, np_ * sizeof(V4), stream_));
      CK(cudaMemsetAsync(mom_.p, 0, np_ * sizeof(V4), stream_));
      if (det_ && frcq_.p) {
        CK(cudaMemsetAsync(frcq_.p, 0, 4 * (size_t)np_ * sizeof(long long), stream_));
        CK(cudaMemsetAsync(momq_.p, 0, 4 * (size_t)np_ * sizeof(long long), stream_));
      }
      forces_dirty_ = false;
    }
    if (contacts_dirty_) {
      RC(build_contacts(false));
      contacts_dirty_ = false;
    }
    return DEM_OK;
  }

  // A sample whose state turned non-finite is stopped by the controller; the
  // others run on, and the call then returns DEM_ERR_NUMERIC.
  // ev (optional, two events): ev[0] is recorded once the state of the last
  // call has been read (before any contact-list rebuild of this call), ev[1]
  // after the launches of each chunk, so that [ev[0], ev[1]] spans the device
  // work of these steps and the host work between their chunks, and not the
  // bookkeeping at either end of the call.
  // Every sample advances max_steps steps (fewer if it finishes): the step
  // kernels hold a sample at its stop while the others catch up, and hold a
  // sample whose contact list went stale inside a chunk (a particle past half
  // the skin) until the list is rebuilt, so that no step runs on a list that
  // may miss a contact; the held steps are run again after the rebuild.
  // done_steps: the largest number of steps a sample advanced.
  int run(uint64_t max_steps, uint64_t* done_steps, bool stop_when_done, cudaEvent_t* ev = nullptr) {
    (void)stop_when_done;   // the loop ends once no sample is active either way
    RC(prepare());
    if (max_steps) RC(set_stop(max_steps));
    Flags f{};
    RC(read_flags(f));
    std::vector<uint64_t> step0(hctl_.size());
    for (size_t k = 0; k < hctl_.size(); ++k) step0[k] = hctl_[k].step;
    const uint32_t numeric_before = f.numeric;
    RC(update_tiles());
    if (ev) {
      CK(cudaEventRecord(ev[0], stream_));
      CK(cudaEventRecord(ev[1], stream_));
    }
    while (true) {
      if (f.stale) {
        // a particle outran the speed margin (violent fracture): chunks are
        // sized with twice the margin from now on (at most 16 x the speed)
        ++stale_events_;
        speed_margin_ = std::min(2.0 * speed_margin_, 16.0);
      }
      if (f.rebuild || f.stale || (double)f.d2max > 0.0625 * min_skin_ * min_skin_) {
        RC(build_contacts(false));
        RC(clear_rebuild_flags());
        f.d2max = 0.f;
      }
      if (!max_steps || !f.active) break;
      const uint64_t chunk = std::min(f.remaining, chunk_steps(f));
      CK(cudaMemsetAsync(stat_.p, 0, sizeof(float), stream_));  // speed maximum of this chunk
      if (chunk == opt_.graph_steps) {
        if (!graph_exec_) RC(capture_steps(opt_.graph_steps, &graph_exec_));
        CK(cudaGraphLaunch(graph_exec_, stream_));
      } else {
        RC(run_short_chunk(chunk));
      }
      if (ev) CK(cudaEventRecord(ev[1], stream_));
      CK(cudaGetLastError());
      RC(read_flags(f));
      RC(update_tiles());
    }
    uint64_t steps = 0;
    for (size_t k = 0; k < hctl_.size(); ++k) steps = std::max<uint64_t>(steps, hctl_[k].step - step0[k]);
    total_steps_ += steps;
    if (done_steps) *done_steps = steps;
    return (f.numeric && !numeric_before) ? DEM_ERR_NUMERIC : DEM_OK;
  }

  int run_until_done(uint64_t max_steps, uint64_t* done) override { return run(max_steps, done, true); }
  int step(uint32_t n) override { return run(n, nullptr, false); }

  int step_stages(int stages) override {
    RC(prepare());
    // the contact list is rebuilt by the rule of run(): once a particle has
    // moved a quarter of the skin since the last build (or past half of it)
    Flags f{};
    RC(read_flags(f));
    if (f.rebuild || f.stale || (double)f.d2max > 0.0625 * min_skin_ * min_skin_) {
      if (f.stale) ++stale_events_;
      RC(build_contacts(false));
      RC(clear_rebuild_flags());
    }
    RC(set_stop(1));
    StepArgs<Real> A = args();
    A.keep_forces = (stages & 4) ? 1 : 0;
    launch_step(A, stages & 3);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
    if (stages & 4) forces_dirty_ = true;
    if ((stages & 1) && !(stages & 2)) forces_dirty_ = true;
    return DEM_OK;
  }

  int sync() override {
    CK(cudaStreamSynchronize(stream_));
    return DEM_OK;
  }

  // ---------------------------------------------------------------- queries
  int counts(uint32_t* p, uint32_t* b, uint32_t* c, uint32_t* s) override {
    if (p) *p = np_;
    if (b) *b = nb_;
    if (c) *c = nc_host_;
    if (s) *s = (uint32_t)samples_.size();
    return DEM_OK;
  }

  int result(int32_t si, dem_result* out) override {
    if (si < 0 || (size_t)si >= samples_.size() || !out) return DEM_ERR_ARG;
    if (!setup_done_) return DEM_ERR_STATE;
    SampleCtl C;
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(&C, ctl_.p + si, sizeof(C), cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof(*out));
    out->FractureStress = C.FractureStress;
    out->FractureStrain = C.FractureStrain;
    out->Strain = C.Strain;
    out->Stress = C.Stress;
    out->dt = C.dt;
    out->platen_top = C.Top;
    out->platen_bottom = C.Bottom;
    out->platen_velocity = C.V;
    out->steps = C.step;
    out->stepsave = C.stepsave;
    out->bonds_initial = (uint32_t)samples_[si].bonds_initial;
    out->bonds_now = (uint32_t)std::max(C.bonds, 0);
    out->fracture = (int)C.Fracture;
    out->done = (int)C.done;
    out->numeric = (int)C.numeric;
    out->stale = (int)stale_events_;
    out->rebuilds = (int)std::min<uint64_t>(rebuilds_, INT32_MAX);
    // host post-processing of the record (CalculateLinearityDeviation, CalculateDestruction)
    std::vector<double> rec;
    std::vector<uint32_t> rb;
    RC(record(si, rec, rb));
    const uint32_t ns = C.stepsave;
    if (ns > 0 && rb.size() >= ns && rb[0] > 0) out->Destruction = rb[ns - 1] / (double)rb[0];
    if (!C.brazil && ns > 0 && C.FractureStrain != 0 && C.FractureStress != 0)
      out->LinearityDeviation = linearity_deviation(rec, ns, C.FractureStress, C.FractureStrain);
    std::vector<double> lat;
    if (C.lat_count) {
      lat.resize(rec_lat_[si]->n);
      CK(rec_lat_[si]->download(lat.data(), lat.size()));
    }
    chord_moduli(rec, lat, ns, out);
    return DEM_OK;
  }

  // Young's modulus as the chord slope of stress over axial strain between 10%
  // and 50% of the peak stress on the rising branch of the record, and the
  // Poisson ratio as lateral over axial strain increment between the same two
  // points (lateral strain from the mean radial distance of the marked
  // surface particles).  The reference computes neither.
  static void chord_moduli(const std::vector<double>& rec, const std::vector<double>& lat, uint32_t ns,
                           dem_result* out) {
    out->E_chord = std::nan("");
    out->nu = std::nan("");
    if (ns < 3) return;
    auto sig = [&](uint32_t k) { return 0.5 * (std::fabs(rec[3 * k + 1]) + std::fabs(rec[3 * k + 2])); };
    auto eps = [&](uint32_t k) { return -rec[3 * k]; };
    uint32_t kp = 0;
    for (uint32_t k = 1; k < ns; ++k)
      if (sig(k) > sig(kp)) kp = k;
    const double sp = sig(kp);
    if (!(sp > 0)) return;
    // first crossing of level*sp at or before the peak, linearly interpolated
    auto cross = [&](double level, double& e, double& l) -> bool {
      const double t = level * sp;
      for (uint32_t k = 1; k <= kp; ++k) {
        if (sig(k) >= t && sig(k - 1) < t) {
          const double w = (t - sig(k - 1)) / (sig(k) - sig(k - 1));
          e = eps(k - 1) + w * (eps(k) - eps(k - 1));
          l = lat.empty() ? 0.0 : lat[k - 1] + w * (lat[k] - lat[k - 1]);
          return true;
        }
      }
      return false;
    };
    double e1, l1, e5, l5;
    if (!cross(0.1, e1, l1) || !cross(0.5, e5, l5) || !(e5 > e1)) return;
    out->E_chord = 0.4 * sp / (e5 - e1);
    if (!lat.empty() && lat[0] > 0) out->nu = ((l5 - l1) / lat[0]) / (e5 - e1);
  }

  // md_results.cu:147-166 (the record holds two extra zero entries so the
  // look-ahead stays inside it)
  static double linearity_deviation(const std::vector<double>& h, uint32_t stepsave, double FS, double Fe) {
    double l_eps = 0, l_deps = 0, l_A = FS / Fe, l_dS = 0, LD = 0;
    uint32_t i = 0;
    do {
      LD += l_deps * l_dS * l_dS;
      ++i;
      if (3 * (size_t)(i + 1) + 2 >= h.size()) break;
      l_eps = -h[3 * i];
      l_deps = -0.5 * (h[3 * (i + 1)] - h[3 * (i - 1)]);
      l_dS = (l_A * l_eps - 0.5 * (h[3 * i + 2] - h[3 * i + 1]));
    } while (l_eps < Fe - 2 * l_deps && i < stepsave);
    LD /= (Fe * FS * FS);
    return LD + 1.0;
  }

  int record(int32_t si, std::vector<double>& rec, std::vector<uint32_t>& rb) {
    const size_t n = rec_[si]->n / 3;
    rec.resize(3 * n);
    rb.resize(rec_bonds_[si]->n);
    CK(rec_[si]->download(rec.data(), 3 * n));
    CK(rec_bonds_[si]->download(rb.data(), rb.size()));
    return DEM_OK;
  }

  int get_lateral_record(int32_t si, double* out, uint32_t cap, uint32_t* n) override {
    if (si < 0 || (size_t)si >= samples_.size()) return DEM_ERR_ARG;
    if (!setup_done_) return DEM_ERR_STATE;
    SampleCtl C;
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(&C, ctl_.p + si, sizeof(C), cudaMemcpyDeviceToHost));
    const uint32_t m = std::min<uint32_t>(C.stepsave, cap);
    if (out && m) CK(cudaMemcpy(out, rec_lat_[si]->p, m * sizeof(double), cudaMemcpyDeviceToHost));
    if (n) *n = C.lat_count ? C.stepsave : 0;
    return DEM_OK;
  }

  int get_record(int32_t si, double* rec, uint32_t* bonds, uint32_t cap, uint32_t* n) override {
    if (si < 0 || (size_t)si >= samples_.size()) return DEM_ERR_ARG;
    SampleCtl C;
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(&C, ctl_.p + si, sizeof(C), cudaMemcpyDeviceToHost));
    std::vector<double> r;
    std::vector<uint32_t> b;
    RC(record(si, r, b));
    const uint32_t m = std::min<uint32_t>(C.stepsave, cap);
    if (rec) std::memcpy(rec, r.data(), 3 * (size_t)m * sizeof(double));
    if (bonds) std::memcpy(bonds, b.data(), (size_t)m * sizeof(uint32_t));
    if (n) *n = C.stepsave;
    return DEM_OK;
  }

  template <class Out>
  int get_particles_t(int32_t si, Out* R, Out* V, Out* W, Out* F, Out* M, Out* O) {
    if (si < 0 || (size_t)si >= samples_.size()) return DEM_ERR_ARG;
    const SampleHost& s = samples_[si];
    CK(cudaStreamSynchronize(stream_));
    std::vector<V4> h(s.n);
    auto fetch = [&](DBuf<V4>& b, Out* dst) -> int {
      if (!dst) return DEM_OK;
      CK(cudaMemcpy(h.data(), b.p + s.p_begin, s.n * sizeof(V4), cudaMemcpyDeviceToHost));
      for (uint32_t k = 0; k < s.n; ++k) {
        const uint32_t q = s.perm[k];
        dst[q] = (Out)h[k].x;
        dst[s.n + q] = (Out)h[k].y;
        dst[2 * s.n + q] = (Out)h[k].z;
      }
      return DEM_OK;
    };
    RC(fetch(pos_, R));
    RC(fetch(vel_, V));
    RC(fetch(omg_, W));
    RC(fetch(frc_, F));
    RC(fetch(mom_, M));
    RC(fetch(wallO_, O));
    return DEM_OK;
  }
  int get_particles(int32_t si, float* R, float* V, float* W, float* F, float* M, float* O) override {
    return get_particles_t<float>(si, R, V, W, F, M, O);
  }
  int get_particles_d(int32_t si, double* R, double* V, double* W, double* F, double* M, double* O) override {
    return get_particles_t<double>(si, R, V, W, F, M, O);
  }

  int set_particles(int32_t si, const float* R, const float* V, const float* W, const float* O) override {
    if (si < 0 || (size_t)si >= samples_.size() || !setup_done_) return DEM_ERR_ARG;
    const SampleHost& s = samples_[si];
    CK(cudaStreamSynchronize(stream_));
    std::vector<V4> h(s.n);
    auto put = [&](DBuf<V4>& b, const float* src) -> int {
      if (!src) return DEM_OK;
      CK(cudaMemcpy(h.data(), b.p + s.p_begin, s.n * sizeof(V4), cudaMemcpyDeviceToHost));
      for (uint32_t k = 0; k < s.n; ++k) {
        const uint32_t q = s.perm[k];
        h[k].x = (Real)src[q];
        h[k].y = (Real)src[s.n + q];
        h[k].z = (Real)src[2 * s.n + q];
      }
      CK(cudaMemcpy(b.p + s.p_begin, h.data(), s.n * sizeof(V4), cudaMemcpyHostToDevice));
      return DEM_OK;
    };
    RC(put(pos_, R));
    RC(put(vel_, V));
    RC(put(omg_, W));
    RC(put(wallO_, O));
    if (O) {
      // platen-history flags of the sample: set where the uploaded history is non-zero
      std::vector<uint8_t> fl(s.n);
      for (uint32_t k = 0; k < s.n; ++k)
        fl[k] = (O[s.perm[k]] != 0.f || O[s.n + s.perm[k]] != 0.f || O[2 * s.n + s.perm[k]] != 0.f) ? 1 : 0;
      CK(cudaMemcpy(wflag_.p + s.p_begin, fl.data(), s.n, cudaMemcpyHostToDevice));
    }
    if (R) contacts_dirty_ = true;
    return DEM_OK;
  }

  // pair record: 16 values (1/L0, prev-dir xyz, Ot xyz, Mn xyz, Mt xyz, sigma_c, tau_c, b_r)
  // SaveLammpsDATASimple (md_savelammpsdata.cpp:9-75): LAMMPS data file of
  // one specimen in SI units - atoms, per-atom kinetic energies (translational,
  // rotational, total; zeros unless with_energy) and every intact bond once
  // per direction, as the reference lists its bonded slots (type 2).  The box
  // is the escape box (the reference's S.A, S.B); masses and inertias are per
  // sphere (the reference's single p_m, p_I for equal radii).
  int save_lammps(int32_t si, const char* path, int with_energy) override {
    if (si < 0 || (size_t)si >= samples_.size() || !path) return DEM_ERR_ARG;
    if (!setup_done_) return DEM_ERR_STATE;
    const SampleHost& s = samples_[si];
    const uint32_t n = s.n;
    std::vector<double> R(3 * (size_t)n), V(3 * (size_t)n), W(3 * (size_t)n);
    RC(get_particles_t<double>(si, R.data(), V.data(), W.data(), nullptr, nullptr, nullptr));
    uint32_t np = 0;
    RC(get_pairs(si, 0, nullptr, nullptr, nullptr, nullptr, &np));
    std::vector<uint32_t> pi(np), pj(np), pk(np);
    RC(get_pairs(si, np, pi.data(), pj.data(), pk.data(), nullptr, &np));
    std::vector<std::vector<uint32_t>> nb(n);
    size_t nbond = 0;
    for (uint32_t k = 0; k < np; ++k)
      if (pk[k] == 1) {
        nb[pi[k]].push_back(pj[k]);
        nb[pj[k]].push_back(pi[k]);
        nbond += 2;
      }
    const double length_const = 1e-3, mass_const = 1e-6, time_const = 1e-6;
    const double energy_const = mass_const * length_const / (time_const * time_const) * length_const;
    FILE* f = std::fopen(path, "w");
    if (!f) return DEM_ERR_IO;
    const dem_loading& L = s.load;
    std::fprintf(f, "LAMMPS Description T0=%g  (1st line of file)\n\n", s.dt);
    std::fprintf(f, "%u atoms\n%zu bonds\n0 angles\n0 dihedrals\n0 impropers\n1 atom types\n2 bond types\n", n,
                 nbond);
    const char* ax[3] = {"x", "y", "z"};
    for (int d = 0; d < 3; ++d)
      std::fprintf(f, "%g %g %slo %shi\n", (L.space_center[d] - L.space_half[d]) * length_const,
                   (L.space_center[d] + L.space_half[d]) * length_const, ax[d], ax[d]);
    std::fprintf(f, "Masses\n\n1 1\nBond Coeffs\n\n2 1 2\n\nAtoms\n\n");
    for (uint32_t i = 0; i < n; ++i)
      std::fprintf(f, "%u 1 %g %g %g\n", i + 1, R[i] * length_const, R[n + i] * length_const,
                   R[2 * (size_t)n + i] * length_const);
    std::fprintf(f, "Velocities\n\n");
    for (uint32_t i = 0; i < n; ++i) {
      double Et = 0, Er = 0;
      if (with_energy) {
        double m, dtm, dtI;
        particle_constants(s.rad[i], s.mat.rho, s.dt, m, dtm, dtI);
        const double I = 0.4 * m * (double)s.rad[i] * s.rad[i];
        const double v2 = V[i] * V[i] + V[n + i] * V[n + i] + V[2 * (size_t)n + i] * V[2 * (size_t)n + i];
        const double w2 = W[i] * W[i] + W[n + i] * W[n + i] + W[2 * (size_t)n + i] * W[2 * (size_t)n + i];
        Et = 0.5 * m * v2 * energy_const;
        Er = 0.5 * I * w2 * energy_const;
      }
      std::fprintf(f, "%u %g %g %g\n", i + 1, Et, Er, Et + Er);
    }
    std::fprintf(f, "\nBonds\n\n");
    size_t k = 1;
    for (uint32_t i = 0; i < n; ++i) {
      std::sort(nb[i].begin(), nb[i].end());
      for (uint32_t j : nb[i]) std::fprintf(f, "%zu 2 %u %u\n", k++, i + 1, j + 1);
    }
    const bool ok = std::fclose(f) == 0;
    return ok ? DEM_OK : DEM_ERR_IO;
  }

  int get_pairs(int32_t si, uint32_t cap, uint32_t* oi, uint32_t* oj, uint32_t* kind, float* st, uint32_t* n) override {
    return get_pairs_t<float>(si, cap, oi, oj, kind, st, n);
  }
  int get_pairs_d(int32_t si, uint32_t cap, uint32_t* oi, uint32_t* oj, uint32_t* kind, double* st,
                  uint32_t* n) override {
    return get_pairs_t<double>(si, cap, oi, oj, kind, st, n);
  }

  template <class Out>
  int get_pairs_t(int32_t si, uint32_t cap, uint32_t* oi, uint32_t* oj, uint32_t* kind, Out* st, uint32_t* n) {
    if (si < 0 || (size_t)si >= samples_.size() || !setup_done_) return DEM_ERR_ARG;
    RC(prepare());
    const SampleHost& s = samples_[si];
    CK(cudaStreamSynchronize(stream_));
    std::vector<uint2> bij(nb_), cij(nc_host_);
    std::vector<V4> s0(nb_), s1(nb_), s2(nb_), par(nb_), co(nc_host_);
    if (nb_) {
      CK(b_ij_.download(bij.data(), nb_));
      CK(b_s0_.download(s0.data(), nb_));
      CK(b_s1_.download(s1.data(), nb_));
      CK(b_s2_.download(s2.data(), nb_));
      CK(b_par_.download(par.data(), nb_));
    }
    if (nc_host_) {
      CK(c_ij_.download(cij.data(), nc_host_));
      CK(c_o_.download(co.data(), nc_host_));
    }
    uint32_t m = 0;
    const uint32_t lo = s.p_begin, hi = s.p_begin + s.n;
    auto emit = [&](uint32_t a, uint32_t b, uint32_t k, const Out v[16]) {
      if (m < cap) {
        uint32_t ia = s.perm[a - lo], ib = s.perm[b - lo];
        Out w[16];
        std::memcpy(w, v, sizeof(w));
        if (ia > ib) {  // express in the direction i -> j with i < j: mirror the vectors
          std::swap(ia, ib);
          for (int d = 1; d < 13; ++d) w[d] = -w[d];
        }
        if (oi) oi[m] = ia;
        if (oj) oj[m] = ib;
        if (kind) kind[m] = k;
        if (st) std::memcpy(st + 16 * (size_t)m, w, sizeof(w));
      }
      ++m;
    };
    for (uint32_t b = 0; b < nb_; ++b) {
      if (bij[b].x < lo || bij[b].x >= hi) continue;
      const bool intact = par[b].x > 0;
      const Out v[16] = {(Out)(intact ? par[b].x : -par[b].x),
                         (Out)s0[b].x, (Out)s0[b].y, (Out)s0[b].z,
                         (Out)s0[b].w, (Out)s1[b].x, (Out)s1[b].y,
                         (Out)s1[b].z, (Out)s1[b].w, (Out)s2[b].x,
                         (Out)s2[b].y, (Out)s2[b].z, (Out)s2[b].w,
                         (Out)par[b].y, (Out)par[b].z, (Out)par[b].w};
      emit(bij[b].x, bij[b].y, intact ? 1u : 2u, v);
    }
    for (uint32_t c = 0; c < nc_host_; ++c) {
      if (cij[c].x < lo || cij[c].x >= hi) continue;
      const Out v[16] = {0, 0, 0, 0, (Out)co[c].x, (Out)co[c].y, (Out)co[c].z, 0, 0, 0, 0, 0, 0, 0, 0, 0};
      emit(cij[c].x, cij[c].y & 0x7FFFFFFFu, 3u, v);
    }
    if (n) *n = m;
    return DEM_OK;
  }

  int set_pairs(int32_t si, uint32_t cnt, const uint32_t* ii, const uint32_t* jj, const uint32_t* kind,
                const float* st) override {
    if (si < 0 || (size_t)si >= samples_.size() || !setup_done_) return DEM_ERR_ARG;
    RC(prepare());
    SampleHost& s = samples_[si];
    const std::vector<uint32_t>& inv = inverse(s);
    CK(cudaStreamSynchronize(stream_));
    std::vector<uint2> bij(nb_), cij(nc_host_);
    std::vector<V4> s0(nb_), s1(nb_), s2(nb_), par(nb_), co(nc_host_);
    if (nb_) {
      CK(b_ij_.download(bij.data(), nb_));
      CK(b_s0_.download(s0.data(), nb_));
      CK(b_s1_.download(s1.data(), nb_));
      CK(b_s2_.download(s2.data(), nb_));
      CK(b_par_.download(par.data(), nb_));
    }
    if (nc_host_) {
      CK(c_ij_.download(cij.data(), nc_host_));
      CK(c_o_.download(co.data(), nc_host_));
    }
    std::vector<int32_t> delta(samples_.size(), 0);
    for (uint32_t k = 0; k < cnt; ++k) {
      uint32_t a = inv[ii[k]] + s.p_begin, b = inv[jj[k]] + s.p_begin;
      float v[13];
      std::memcpy(v, st + 13 * (size_t)k, sizeof(v));  // set_pairs takes the 13-value state
      if (a > b) {
        std::swap(a, b);
        for (int d = 1; d < 13; ++d) v[d] = -v[d];
      }
      // bonds: search the row of a
      bool found = false;
      auto it = std::lower_bound(bij.begin(), bij.end(), make_uint2(a, b),
                                 [](const uint2& x, const uint2& y) { return x.x < y.x || (x.x == y.x && x.y < y.y); });
      if (it != bij.end() && it->x == a && it->y == b) {
        const size_t q = it - bij.begin();
        const bool was = par[q].x > 0;
        const bool now = kind[k] == 1;
        const Real il = std::fabs(v[0]) > 0 ? (Real)std::fabs(v[0]) : (par[q].x < 0 ? -par[q].x : par[q].x);
        par[q].x = now ? il : -il;
        if (was != now) delta[si] += now ? 1 : -1;
        s0[q] = make4(v[1], v[2], v[3], v[4]);
        s1[q] = make4(v[5], v[6], v[7], v[8]);
        s2[q] = make4(v[9], v[10], v[11], v[12]);
        found = true;
      }
      if (!found) {
        for (uint32_t c = 0; c < nc_host_; ++c) {
          if (cij[c].x == a && (cij[c].y & 0x7FFFFFFFu) == b) {
            co[c] = make4(v[4], v[5], v[6], Real(0));
            const bool nz = v[4] != 0 || v[5] != 0 || v[6] != 0;
            cij[c].y = b | (nz ? 0x80000000u : 0u);
            found = true;
            break;
          }
        }
      }
      if (!found) return DEM_ERR_ARG;
    }
    if (nb_) {
      CK(b_s0_.upload(s0.data(), nb_));
      CK(b_s1_.upload(s1.data(), nb_));
      CK(b_s2_.upload(s2.data(), nb_));
      CK(b_par_.upload(par.data(), nb_));
    }
    if (nc_host_) {
      CK(c_ij_.upload(cij.data(), nc_host_));
      CK(c_o_.upload(co.data(), nc_host_));
    }
    if (delta[si]) {
      int32_t cur;
      CK(cudaMemcpy(&cur, &ctl_.p[si].bonds, sizeof(int32_t), cudaMemcpyDeviceToHost));
      cur += delta[si];
      CK(cudaMemcpy(&ctl_.p[si].bonds, &cur, sizeof(int32_t), cudaMemcpyHostToDevice));
    }
    return DEM_OK;
  }

  int set_platens(int32_t si, double top, double bottom, double v) override {
    if (si < 0 || (size_t)si >= samples_.size() || !setup_done_) return DEM_ERR_ARG;
    CK(cudaStreamSynchronize(stream_));
    SampleCtl C;
    CK(cudaMemcpy(&C, ctl_.p + si, sizeof(C), cudaMemcpyDeviceToHost));
    C.Top = top;
    C.Bottom = bottom;
    C.V = v;
    CK(cudaMemcpy(ctl_.p + si, &C, sizeof(C), cudaMemcpyHostToDevice));
    return DEM_OK;
  }

  int rebuild_contacts() override {
    if (!setup_done_) return DEM_ERR_STATE;
    return build_contacts(false);
  }

  cudaError_t last_cuda() const override { return last_cuda_; }
  uint64_t rebuilds() const override { return rebuilds_; }
  uint32_t num_sms() const override { return (uint32_t)num_sms_; }

  // device pointers of the step kernel for external timing
  void launch_raw(int stages) override {
    if (set_stop(1) != DEM_OK) return;
    StepArgs<Real> A = args();
    launch_step(A, stages);
  }
  void* stream() override { return (void*)stream_; }

  // Device time of nsteps steps: from the first step's launch (after the
  // call has read the state the last call left) to the end of the last step
  // (the flag read-back after it is not included); rebuilds and host checks
  // between chunks are.
  int run_timed(uint64_t nsteps, double* ms) override {
    RC(prepare());
    cudaEvent_t ev[2];
    CK(cudaEventCreate(&ev[0]));
    CK(cudaEventCreate(&ev[1]));
    uint64_t done = 0;
    int rc = run(nsteps, &done, false, ev);
    CK(cudaEventSynchronize(ev[1]));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, ev[0], ev[1]));
    cudaEvent_t a = ev[0], b = ev[1];
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (ms) *ms = t;
    return rc;
  }

  // Per-kernel device time of nsteps steps run the way the timed steps run:
  // captured graphs of the steps, with an event record node before the pair
  // kernel, between the two kernels and after the particle kernel of every
  // step; each graph is replayed once and the event pairs give each launch's
  // duration.  The steps go in chunks sized and separated by contact-list
  // rebuilds as in run(); a chunk in which a list went stale (its sample then
  // holds, skipping work) is run but not counted.  Also counts the touching
  // contacts (algorithmic-byte accounting).
  int profile(uint32_t nsteps, double* pair_ms, double* particle_ms, double* touching) override {
    RC(prepare());
    if (nsteps == 0) return DEM_ERR_ARG;
    DBuf<unsigned long long> cnt;
    CK(cnt.alloc(1));
    const uint32_t g = particle_grid();
    double sp = 0, sq = 0, tc_sum = 0;
    uint32_t counted = 0, attempts = 0;
    Flags f{};
    RC(read_flags(f));
    while (counted < nsteps && attempts < 4 * nsteps) {
      if (f.rebuild || f.stale || (double)f.d2max > 0.0625 * min_skin_ * min_skin_) {
        if (f.stale) ++stale_events_;
        RC(build_contacts(false));
        RC(clear_rebuild_flags());
        f.d2max = 0.f;
      }
      const uint32_t chunk = (uint32_t)std::min<uint64_t>(nsteps - counted, chunk_steps(f));
      RC(set_stop(chunk));
      CK(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long), stream_));
      CK(cudaMemsetAsync(stat_.p, 0, sizeof(float), stream_));
      StepArgs<Real> A = args();
      A.touching = cnt.p;
      std::vector<cudaEvent_t> ev(3 * (size_t)chunk);
      for (auto& e : ev) CK(cudaEventCreate(&e));
      cudaGraph_t graph = nullptr;
      cudaGraphExec_t exec = nullptr;
      // an event recorded during capture becomes an event record node only
      // with cudaEventRecordExternal (a plain record is a capture-internal
      // dependency and is never recorded when the graph runs)
      CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
      cudaError_t ce = cudaSuccess;
      for (uint32_t k = 0; k < chunk && ce == cudaSuccess; ++k) {
        ce = cudaEventRecordWithFlags(ev[3 * k], stream_, cudaEventRecordExternal);
        launch_pairs(A);
        if (ce == cudaSuccess) ce = cudaEventRecordWithFlags(ev[3 * k + 1], stream_, cudaEventRecordExternal);
        k_particles<Real><<<g, opt_.particle_block, 0, stream_>>>(A);
        if (ce == cudaSuccess) ce = cudaEventRecordWithFlags(ev[3 * k + 2], stream_, cudaEventRecordExternal);
      }
      cudaError_t e = cudaStreamEndCapture(stream_, &graph);
      if (e == cudaSuccess && ce != cudaSuccess) e = ce;
      if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
      if (graph) cudaGraphDestroy(graph);
      if (e == cudaSuccess) e = cudaGraphLaunch(exec, stream_);
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
      if (exec) cudaGraphExecDestroy(exec);
      if (e != cudaSuccess) {
        for (auto& x : ev) cudaEventDestroy(x);
        last_cuda_ = e;
        note_cuda_error(e, __FILE__, __LINE__);
        return DEM_ERR_CUDA;
      }
      attempts += chunk;
      total_steps_ += chunk;
      RC(read_flags(f));
      if (!f.stale) {
        for (uint32_t k = 0; k < chunk; ++k) {
          float t1 = 0, t2 = 0;
          CK(cudaEventElapsedTime(&t1, ev[3 * k], ev[3 * k + 1]));
          CK(cudaEventElapsedTime(&t2, ev[3 * k + 1], ev[3 * k + 2]));
          sp += t1;
          sq += t2;
        }
        unsigned long long tc = 0;
        CK(cnt.download(&tc, 1));
        tc_sum += (double)tc;
        counted += chunk;
      }
      for (auto& x : ev) cudaEventDestroy(x);
    }
    if (f.rebuild || f.stale) {
      if (f.stale) ++stale_events_;
      RC(build_contacts(false));
      RC(clear_rebuild_flags());
    }
    if (!counted) return DEM_ERR_STATE;
    if (pair_ms) *pair_ms = sp / counted;
    if (particle_ms) *particle_ms = sq / counted;
    if (touching) *touching = tc_sum / counted;
    return DEM_OK;
  }

 private:
  dem_options opt_;
  cudaStream_t stream_ = nullptr;
  cudaGraphExec_t graph_exec_ = nullptr;
  cudaGraphExec_t small_graphs_[3] = {nullptr, nullptr, nullptr};   // 64, 16 and 4 steps
  int num_sms_ = 148;
  const void* pair_kernel_ = nullptr;
  bool setup_done_ = false, forces_dirty_ = false, contacts_dirty_ = false, stale_ = false;
  cudaError_t last_cuda_ = cudaSuccess;
  uint64_t total_steps_ = 0, rebuilds_ = 0, stale_events_ = 0;
  double min_skin_ = 0, max_dt_ = 0;
  double speed_margin_ = 2.0;   // chunk sizing: the fastest particle may speed up this much within a chunk

  std::vector<SampleHost> samples_;
  std::vector<SampleParams<Real>> hparams_;
  std::vector<SampleCtl> hctl_;
  uint32_t np_ = 0, nb_ = 0, nc_host_ = 0, ncell_ = 0;

  DBuf<V4> pos_, vel_, omg_, frc_, mom_, wallO_, pos_ref_;
  DBuf<uint8_t> wflag_;
  DBuf<long long> frcq_, momq_;   // deterministic mode: fixed-point accumulators
  std::vector<uint32_t> sb_begin_, sb_end_;   // per sample: bond range
  DBuf<uint32_t> tiles_, ntiles_, sdone_;     // active bond tiles; per-sample finished flags
  DBuf<uint32_t> tile_s_;                     // per bond tile: its sample (~0u: two samples)
  bool tiles_on_ = false;
  uint32_t ndone_seen_ = 0;
  bool user_grid_ = false;
  bool skin_user_ = false;  // skin_factor given at creation: the autotuner keeps it
  uint32_t part_occ_ = 8, part_occ_block_ = 0;
  bool det_ = false;
  DBuf<Real> mass_;
  DBuf<uint32_t> sid_, orig_;
  DBuf<uint2> b_ij_;
  DBuf<V4> b_s0_, b_s1_, b_s2_, b_par_;
  DBuf<uint32_t> b_row_;
  DBuf<uint2> c_ij_, c_ij_new_;
  DBuf<V4> c_o_, c_o_new_;
  DBuf<uint32_t> c_jstride_, c_row_, nc_dev_;
  DBuf<SampleParams<Real>> sp_;
  DBuf<BondLaw<Real>> law_;
  DBuf<double> gap_, skin_;
  DBuf<SampleCtl> ctl_;
  DBuf<Grid<Real>> grids_;
  DBuf<uint32_t> cell_of_, cell_count_, cell_start_, cell_cursor_, cell_list_, cnt_, offs_, ovf_, scan_tmp_;
  DBuf<unsigned int> blocks_done_;
  DBuf<float> stat_;
  std::vector<std::unique_ptr<DBuf<double>>> rec_;
  std::vector<std::unique_ptr<DBuf<uint32_t>>> rec_bonds_;
  std::vector<std::unique_ptr<DBuf<double>>> rec_lat_;
  DBuf<uint8_t> lat_;
  std::vector<uint8_t> hlat_;
  DBuf<double> sfl_tan_;
};

EngineBase* make_engine(const dem_options& o, int* err) {
  EngineBase* e = nullptr;
  int rc = DEM_OK;
  if (o.precision == 1) {
    auto* x = new Engine<double>(o);
    rc = x->init();
    e = x;
  } else if (o.precision == 2) {
    auto* x = new Engine<Dual<kSensCount>>(o);
    rc = x->init();
    e = x;
  } else {
    auto* x = new Engine<float>(o);
    rc = x->init();
    e = x;
  }
  if (rc != DEM_OK) {
    delete e;
    e = nullptr;
  }
  if (err) *err = rc;
  return e;
}

// ------------------------------------------------------------------ reference-layout parity exports
namespace {
int ref_grid_bin(const float* xyz, uint32_t n, float a, uint32_t nx, uint32_t ny, uint32_t nz, DBuf<float4>& pos,
                 DBuf<uint32_t>& sid, DBuf<Grid<float>>& grid, DBuf<uint32_t>& cell_of, DBuf<uint32_t>& cstart,
                 DBuf<uint32_t>& clist, uint32_t& ncell) {
  std::vector<float4> h(n);
  for (uint32_t i = 0; i < n; ++i) h[i] = make_float4(xyz[i], xyz[n + i], xyz[2 * n + i], 0.f);
  ncell = nx * ny * nz;
  Grid<float> g{0.f, 0.f, 0.f, (float)(1.0 / (double)a), nx, ny, nz, 0, 0.f, 0.f, 0.f, 0u};
  if (pos.alloc(n) || sid.alloc(n) || grid.alloc(1) || cell_of.alloc(n) || cstart.alloc(ncell + 1) || clist.alloc(n))
    return DEM_ERR_CUDA;
  if (pos.upload(h.data(), n) || grid.upload(&g, 1)) return DEM_ERR_CUDA;
  DBuf<uint32_t> count, cursor, tmp1, tmp2;
  if (count.alloc(ncell + 1) || cursor.alloc(ncell + 1)) return DEM_ERR_CUDA;
  const uint32_t gb = std::max(1u, ceil_div(n, 256));
  k_cell_index<float><<<gb, 256>>>(pos.p, sid.p, n, grid.p, cell_of.p, count.p);
  // scan (host-side simple three-level, sizes here are small)
  const uint32_t nb = ceil_div(ncell, kScanBlock);
  if (tmp1.alloc(nb + 1) || tmp2.alloc(nb + 1)) return DEM_ERR_CUDA;
  k_scan_block<<<nb, kScanBlock>>>(count.p, cstart.p, ncell, tmp1.p);
  if (nb > 1) {
    if (nb > kScanBlock) return DEM_ERR_CAPACITY;
    k_scan_block<<<1, kScanBlock>>>(tmp1.p, tmp2.p, nb, nullptr);
    k_scan_add<<<nb, kScanBlock>>>(cstart.p, ncell, tmp2.p);
  }
  k_scan_total<<<1, 1>>>(count.p, cstart.p, ncell);
  if (cudaMemcpy(cursor.p, cstart.p, (ncell + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice)) return DEM_ERR_CUDA;
  k_scatter_cells<<<gb, 256>>>(cell_of.p, n, cursor.p, clist.p);
  k_sort_cells<<<std::max(1u, ceil_div(ncell, 256)), 256>>>(cstart.p, ncell, clist.p);
  if (cudaDeviceSynchronize()) return DEM_ERR_CUDA;
  return DEM_OK;
}
}  // namespace

int ref_cells(const float* xyz, uint32_t n, float a, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t* CI,
              uint32_t* CIs, uint32_t* pnC) {
  DBuf<float4> pos;
  DBuf<uint32_t> sid, cell_of, cstart, clist;
  DBuf<Grid<float>> grid;
  uint32_t ncell = 0;
  int rc = ref_grid_bin(xyz, n, a, nx, ny, nz, pos, sid, grid, cell_of, cstart, clist, ncell);
  if (rc) return rc;
  std::vector<uint32_t> co(n), cs(ncell + 1), cl(n);
  if (cell_of.download(co.data(), n) || cstart.download(cs.data(), ncell + 1) || clist.download(cl.data(), n))
    return DEM_ERR_CUDA;
  if (CI) std::memcpy(CI, co.data(), n * sizeof(uint32_t));
  if (CIs)
    for (uint32_t k = 0; k < n; ++k) {
      CIs[k] = co[cl[k]];
      CIs[n + k] = cl[k];
    }
  if (pnC) {
    std::memset(pnC, 0, 2 * (size_t)ncell * sizeof(uint32_t));
    for (uint32_t c = 0; c < ncell; ++c)
      if (cs[c + 1] > cs[c]) {
        pnC[c] = cs[c];
        pnC[ncell + c] = cs[c + 1] - cs[c];
      }
  }
  return DEM_OK;
}

int ref_neighbor_sets(const float* xyz, uint32_t n, float a, uint32_t nx, uint32_t ny, uint32_t nz, float add_thr,
                      float del_thr, uint32_t cap, uint32_t* sets, uint32_t* overflow) {
  DBuf<float4> pos;
  DBuf<uint32_t> sid, cell_of, cstart, clist;
  DBuf<Grid<float>> grid;
  uint32_t ncell = 0;
  int rc = ref_grid_bin(xyz, n, a, nx, ny, nz, pos, sid, grid, cell_of, cstart, clist, ncell);
  if (rc) return rc;
  DBuf<uint32_t> out, cnt, ovf;
  if (out.alloc((size_t)n * cap) || cnt.alloc(n) || ovf.alloc(1)) return DEM_ERR_CUDA;
  PairSearch<float> S{};
  S.pos = pos.p;
  S.sid = sid.p;
  S.np = n;
  S.grids = grid.p;
  S.cell_start = cstart.p;
  S.cell_list = clist.p;
  S.mode = kModeRefSet;
  S.add_thr = add_thr;
  S.del_thr = del_thr;
  S.count = cnt.p;
  S.out_j = out.p;
  S.cap = cap;
  S.overflow = ovf.p;
  const uint32_t gb = pair_search_blocks(n);
  k_pair_search<float, false><<<gb, 128>>>(S);
  k_pair_search<float, true><<<gb, 128>>>(S);
  if (cudaDeviceSynchronize()) return DEM_ERR_CUDA;
  if (out.download(sets, (size_t)n * cap)) return DEM_ERR_CUDA;
  uint32_t o = 0;
  if (ovf.download(&o, 1)) return DEM_ERR_CUDA;
  if (overflow) *overflow = o;
  return DEM_OK;
}

}  // namespace dem
