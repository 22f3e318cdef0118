// Host runtime and C ABI of the B200 HIT_Solver backend (see include/hitb200.h).
//
// A plan owns one device arena holding every scratch buffer of its solve,
// the per-solve descriptor (SolveDev) and the CTA work lists of each kernel.
// Launch sequences mirror the reference's loop body; every scalar the
// reference pulls to the host (dt, Lax-Friedrichs speeds, sensor rms, Mach,
// forcing power) stays in the device scalar block.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/hitb200.h"
#include "common.cuh"
#include "kernels_fft.cuh"
#include "kernels_init.cuh"
#include "kernels_npnoise.cuh"
#include "kernels_reduce.cuh"
#include "kernels_spectra.cuh"
#include "kernels_stencil.cuh"
#include "sensor_step.cuh"
#include "stage_persist.cuh"

using namespace hitb200;

static_assert(ST_NONFINITE == HITB200_ST_NONFINITE && ST_NONPOS_RHO == HITB200_ST_NONPOS_RHO &&
                  ST_NONPOS_P == HITB200_ST_NONPOS_P && ST_BARRIER == HITB200_ST_BARRIER &&
                  ST_NOISE == HITB200_ST_NOISE,
              "status bits of the device code and of the C ABI must agree");

namespace {

thread_local std::string g_last_error;

int cuda_fail(cudaError_t e, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? HITB200_ERR_OOM : HITB200_ERR_CUDA;
}
#define HB_CUDA(call)                                  \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)
#define HB_LAUNCHED(name)                                    \
  do {                                                       \
    cudaError_t e_ = cudaGetLastError();                     \
    if (e_ != cudaSuccess) return cuda_fail(e_, name);       \
  } while (0)

int invalid(const std::string& msg) {
  g_last_error = msg;
  return HITB200_ERR_INVALID;
}

// Streams and fork / join events of one graph capture, released on every
// exit path.
struct CaptureRes {
  cudaStream_t st[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  ~CaptureRes() {
    for (cudaStream_t s : st)
      if (s) cudaStreamDestroy(s);
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
  }
};

// Captures `launch(streams)` into an executable graph on private streams:
// one, or two forked from the first and joined back (`branches` = 2), so
// that the graph holds two independent chains of kernels.  Every stream and
// event is created before the capture begins and released after it ends.
template <class F>
int capture_graph(int branches, F&& launch, cudaGraphExec_t* out) {
  *out = nullptr;
  CaptureRes c;
  for (int i = 0; i < branches; ++i) HB_CUDA(cudaStreamCreateWithFlags(&c.st[i], cudaStreamNonBlocking));
  if (branches > 1)
    for (cudaEvent_t& e : c.ev) HB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  HB_CUDA(cudaStreamBeginCapture(c.st[0], cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaSuccess;
  if (branches > 1) {
    e = cudaEventRecord(c.ev[0], c.st[0]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c.st[1], c.ev[0], 0);
  }
  const int r = e == cudaSuccess ? launch(c.st) : HITB200_OK;
  if (e == cudaSuccess && branches > 1) {
    e = cudaEventRecord(c.ev[1], c.st[1]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c.st[0], c.ev[1], 0);
  }
  cudaGraph_t gr = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(c.st[0], &gr);
  if (e != cudaSuccess || r != HITB200_OK || ee != cudaSuccess) {
    if (gr) cudaGraphDestroy(gr);
    if (r != HITB200_OK) return r;
    return cuda_fail(e != cudaSuccess ? e : ee, "graph capture");
  }
  e = cudaGraphInstantiate(out, gr, 0);
  cudaGraphDestroy(gr);
  if (e != cudaSuccess) {
    *out = nullptr;
    return cuda_fail(e, "cudaGraphInstantiate");
  }
  return HITB200_OK;
}

bool is_none(double v) { return std::isnan(v); }

// ---- device block cache -----------------------------------------------------------
// Plan arenas and batch tables are device blocks in 2 MiB granules.  A
// destroyed plan or batch returns its block here instead of to cudaFree:
// on the B200 a cudaFree of a plan arena or of a batch table took 10 ms to
// 0.7 s even on an idle device, and a cudaMalloc 10-40 ms, which stalled a
// serving loop that retires and admits solves every few rounds.  A request
// takes the smallest cached block of its device that fits, if that wastes
// at most half of it.  The cache holds at most kBlockCacheMax bytes;
// hitb200_release_cached_blocks() frees them, and an allocation that fails
// frees this device's blocks and retries.
struct DevBlock {
  void* ptr = nullptr;
  size_t bytes = 0;
  int dev = 0;
};
constexpr size_t kBlockGranule = size_t(2) << 20;
constexpr size_t kBlockCacheMax = size_t(8) << 30;
std::mutex g_blocks_mu;
std::multimap<std::pair<int, size_t>, void*> g_blocks;  // (device, bytes) -> block
size_t g_blocks_bytes = 0;

// Frees the cached blocks of device `dev` (every device for dev < 0); the
// caller holds g_blocks_mu.
void release_blocks_locked(int dev) {
  if (g_blocks.empty()) return;
  int cur = 0, set = -1;
  cudaGetDevice(&cur);
  for (auto it = g_blocks.begin(); it != g_blocks.end();) {
    if (dev >= 0 && it->first.first != dev) {
      ++it;
      continue;
    }
    if (it->first.first != (set < 0 ? cur : set)) {
      set = it->first.first;
      cudaSetDevice(set);
    }
    cudaFree(it->second);
    g_blocks_bytes -= it->first.second;
    it = g_blocks.erase(it);
  }
  if (set >= 0 && set != cur) cudaSetDevice(cur);
}

cudaError_t block_alloc(size_t bytes, DevBlock* out) {
  const size_t want = (bytes + kBlockGranule - 1) / kBlockGranule * kBlockGranule;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> lk(g_blocks_mu);
    auto it = g_blocks.lower_bound({dev, want});
    if (it != g_blocks.end() && it->first.first == dev && it->first.second <= 2 * want) {
      *out = {it->second, it->first.second, dev};
      g_blocks_bytes -= it->first.second;
      g_blocks.erase(it);
      return cudaSuccess;
    }
  }
  void* ptr = nullptr;
  e = cudaMalloc(&ptr, want);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    {
      std::lock_guard<std::mutex> lk(g_blocks_mu);
      release_blocks_locked(dev);
    }
    e = cudaMalloc(&ptr, want);
  }
  if (e != cudaSuccess) return e;
  *out = {ptr, want, dev};
  return cudaSuccess;
}

// Waits for every queued launch of the block's device (whichever device is
// current).
cudaError_t sync_block_device(const DevBlock& b) {
  int cur = 0;
  cudaError_t e = cudaGetDevice(&cur);
  if (e != cudaSuccess) return e;
  if (cur != b.dev) cudaSetDevice(b.dev);
  e = cudaDeviceSynchronize();
  if (cur != b.dev) cudaSetDevice(cur);
  return e;
}

// Returns a block to the cache (or to cudaFree when the cache is full).  No
// queued work may use it any more: the caller synchronised its device.
void block_free(DevBlock& b) {
  if (!b.ptr) return;
  std::lock_guard<std::mutex> lk(g_blocks_mu);
  if (g_blocks_bytes + b.bytes <= kBlockCacheMax) {
    g_blocks.insert({{b.dev, b.bytes}, b.ptr});
    g_blocks_bytes += b.bytes;
  } else {
    int cur = 0;
    cudaGetDevice(&cur);
    if (b.dev != cur) cudaSetDevice(b.dev);
    cudaFree(b.ptr);
    if (b.dev != cur) cudaSetDevice(cur);
  }
  b = DevBlock{};
}

// numpy.fft.fftfreq integer bins of an n-point transform.
int fft_bin(int j, int n) {
  const int half = (n - 1) / 2 + 1;
  return j < half ? j : j - n;
}
// 2 pi fftfreq(n, d)[j] evaluated the way numpy does (bin * (1 / (n d))).
double wavenumber(int m, int n, double d) { return 2.0 * M_PI * ((double)m * (1.0 / ((double)n * d))); }

struct Arena {
  size_t off = 0;
  size_t take(size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) & ~(size_t)255;
    return o;
  }
};

struct ModeTables {
  std::vector<int2> drag, force;
  std::vector<double2> kvec;
  std::vector<int> partner;
};

ModeTables build_modes(const hitb200_desc& d) {
  ModeTables t;
  const double dx = (d.x_max - d.x_min) / d.nx, dy = (d.y_max - d.y_min) / d.ny;
  for (int jy = 0; jy < d.ny; ++jy)
    for (int jx = 0; jx < d.nx; ++jx) {
      const int mx = fft_bin(jx, d.nx), my = fft_bin(jy, d.ny);
      const double kx = wavenumber(mx, d.nx, dx), ky = wavenumber(my, d.ny, dy);
      const double k2 = kx * kx + ky * ky;
      const double mag = std::sqrt(k2);
      if (d.periodic && d.drag_coefficient > 0.0 && d.drag_kmax > 0.0 && mag >= 0.0 && k2 > 0.0 &&
          mag <= d.drag_kmax)
        t.drag.push_back(make_int2(mx, my));
      if (d.periodic && d.forcing_on && mag >= d.forcing_kmin && mag <= d.forcing_kmax && mag > 0.0) {
        t.force.push_back(make_int2(mx, my));
        t.kvec.push_back(make_double2(kx, ky));
      }
    }
  t.partner.assign(kMaxForce, 0);
  for (size_t i = 0; i < t.force.size(); ++i) {
    const int px = fft_bin(((-t.force[i].x) % d.nx + d.nx) % d.nx, d.nx);
    const int py = fft_bin(((-t.force[i].y) % d.ny + d.ny) % d.ny, d.ny);
    int p = (int)i;
    for (size_t k = 0; k < t.force.size(); ++k)
      if (t.force[k].x == px && t.force[k].y == py) p = (int)k;
    t.partner[i] = p;
  }
  return t;
}

constexpr size_t kSweepSmemMax = 227 * 1024;  // opt-in shared memory per CTA on sm_100

int lines_per_cta(int n, int nlines, int elem) {
  // R = 2 when its shared memory lets two CTAs share an SM and the grid still
  // has at least two CTAs per SM worth of lines; otherwise 1.
  int best = 1;
  for (int R : {2, 1}) {
    const size_t b = elem == 4 ? SweepLayout<float>(n, R).bytes() : SweepLayout<double>(n, R).bytes();
    if (b > 110 * 1024) continue;
    if ((nlines + R - 1) / R < 2 * 148 && R > 1) continue;
    best = R;
    break;
  }
  return best;
}

int guard_blocks_for(const hitb200_desc& d) {
  if (d.periodic || d.guard_cells <= 0) return 1;
  const long band = 2L * d.guard_cells * (d.nx + d.ny);
  return (int)std::max(1L, std::min(64L, (band + 255) / 256));
}

// Sweep nodes per thread (128 threads per line).
int mch_for(int n) {
  return n <= 128 ? 1 : n <= 256 ? 2 : n <= 512 ? 4 : 8;
}

// Default kernel variants from the launch sizes: the throughput variants
// (more resident CTAs, fewer registers) once a launch has several waves of
// CTAs per SM, the latency variants below that.
void default_tuning(int n_x, int n_y, int n_tiles32, int* t) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  t[HITB200_TUNE_SWEEP_X] = n_x >= 6 * sms;
  t[HITB200_TUNE_SWEEP_Y] = n_y >= 4 * sms;
  t[HITB200_TUNE_PREPASS] = n_tiles32 >= 4 * sms;
  t[HITB200_TUNE_FUSED_SENSOR] = 0;  // measured slower at 512^2; the autotuner decides
  t[HITB200_TUNE_Y_PANEL] = 0;
  t[HITB200_TUNE_PERSISTENT] = 0;  // the autotuner decides (batches only)
}

}  // namespace

struct hitb200_plan {
  hitb200_desc desc{};
  SolveDev hs{};            // host copy of the device descriptor
  SolveDev* d_solve = nullptr;
  unsigned char* arena = nullptr;
  size_t arena_bytes = 0;
  DevBlock arena_block;     // the arena's cached device block
  Work* d_tiles = nullptr;
  Work* d_tiles32 = nullptr;
  Work* d_xlines = nullptr;
  Work* d_ylines = nullptr;
  Work* d_srows = nullptr;  // forcing-synthesis row blocks
  int* d_partner = nullptr;
  int n_tiles = 0, n_tiles32 = 0, n_x = 0, n_y = 0, Rx = 1, Ry = 1, n_srows = 0;
  int elem = 8;
  size_t smem_x = 0, smem_y = 0, smem_sensor = 0;
  // the other y-panel width (tuning knob HITB200_TUNE_Y_PANEL; Ry2 == Ry
  // when there is none) and its line list
  int Ry2 = 1, n_y2 = 0;
  size_t smem_y2 = 0;
  Work* d_ylines2 = nullptr;
  // graph replay of hitb200_step
  cudaGraphExec_t graph = nullptr;
  cudaStream_t graph_stream = nullptr;
  const double* graph_q = nullptr;
  bool in_batch = false;
  SolveDev* own_solve = nullptr;  // the arena's descriptor (d_solve points into a batch table while batched)
  int tuning[HITB200_TUNE_COUNT] = {};  // kernel variants (tuning knobs)
  bool fuse_ok = false;  // all of the fused sensor's CTAs fit on the GPU at once
  int sensor_w = -1;          // width of the step sensor instantiation (-1: generic sensor)
  size_t smem_sensor_step = 0;
  bool has_gen = false;       // the reference's noise stream generated on the device (noise_mode 2)
  NoiseBufs gen{};
};

struct hitb200_batch {
  std::vector<hitb200_plan*> plans;
  bool owns_plans = true;  // false for hitb200_batch_from_plans
  int tuning[HITB200_TUNE_COUNT] = {};
  SolveDev* d_solves = nullptr;  // start of the tables' device block
  DevBlock tables;
  Work *d_tiles = nullptr, *d_tiles32 = nullptr, *d_xlines = nullptr, *d_ylines = nullptr;
  Work* d_srows = nullptr;
  int* d_partner = nullptr;
  int n_tiles = 0, n_tiles32 = 0, n_x = 0, n_y = 0, elem = 8, mch_x = 1, mch_y = 1, guard_blocks = 1;
  int n_srows = 0;
  // first item of each member in each work list (n + 1 entries): the lists
  // hold the members' items in member order
  std::vector<int> off_tiles, off_tiles32, off_xl, off_yl, off_srows;
  int rx_max = 1, ry_max = 1;
  size_t smem_x = 0, smem_y = 0, smem_sensor = 0;
  // the other y-panel width's line list (tuning knob HITB200_TUNE_Y_PANEL;
  // has_y2 false when there is none)
  bool has_y2 = false;
  Work* d_ylines2 = nullptr;
  int n_y2 = 0, ry_max2 = 1;
  size_t smem_y2 = 0;
  std::vector<int> off_yl2;
  int sensor_w = -1;  // shared width of the members' step sensor (-1: generic sensor)
  size_t smem_sensor_step = 0;
  // Sweep work by launch group (0 all members, 1 and 2 the halves of
  // hitb200_batch_run's graph branches), list (0 x lines, 1 y panels, 2 y
  // panels of the other width) and nodes-per-thread class (1, 2, 4, 8 nodes
  // per sweep thread): each member's lines run in a launch of its own class,
  // as when it runs alone (the line solves' order of operations depends on
  // the class).
  struct SegRec {
    int off = 0, n = 0;
    size_t smem = 0;
  };
  Work* d_segs = nullptr;
  SegRec segs[3][3][4];
  // Persistent stage launches (tuning knob HITB200_TUNE_PERSISTENT).  Launch
  // groups: 0 all members (hitb200_batch_step), 1 and 2 the two halves of
  // hitb200_batch_run's graph branches ([0, cut) and [cut, n)).
  bool can_persist = false;
  int cut = 1;
  Work *d_xl4 = nullptr, *d_yl4 = nullptr;  // 4-row x groups and 4-column y panels
  QItem* d_qitems = nullptr;
  QCtl* d_qctl = nullptr;     // one queue per group
  unsigned* d_qdep = nullptr;  // [members][4] phase counters
  int q_off[4] = {};           // items of group g: [q_off[g], q_off[g + 1])
  int q_npre[3] = {};          // prepass items at the start of group g
  size_t smem_stage = 0, stage_sh_off = 0, stage_xstride = 0;  // dynamic shared memory layout
  int stage_grid = 0;          // CTAs of a stage launch (all resident at once)
  int any_outflow = 0, any_forcing = 0, any_hv = 0, any_noise_upload = 0;
  cudaGraphExec_t graph = nullptr;
  cudaStream_t graph_stream = nullptr;
};

namespace {

// ---- launch helpers shared by plans and batches ----------------------------------
struct LaunchSet {
  const SolveDev* solves;
  int nsolves;
  const Work *tiles, *tiles32, *xl, *yl, *srows;
  const int* partner;
  int n_tiles, n_tiles32, n_x, n_y, elem, mch_x, mch_y, guard_blocks, n_srows;
  int thr_x, thr_y;  // sweep CTA sizes: kLineThreads per line of the widest work item
  int occ_x, occ_y, occ_pre;  // kernel variants: 0 latency, 1 throughput (tuning knobs)
  int fused;                  // prepass fused into the sensor (single solves, tuning knob)
  size_t smem_x, smem_y, smem_sensor;
  int sensor_w;             // step sensor instantiation shared by the solves (-1: generic)
  size_t smem_sensor_step;
  const NoiseBufs* gen = nullptr;  // single plans of noise_mode 2: the noise stream's buffers
  double* gen_out = nullptr;       // ... and the noise field they fill
  cudaStream_t st;
  // cells of all solves, and of the solves carrying viscous / forcing terms
  double cells = 0, cells_visc = 0, cells_force = 0;
  int pdl = 0;  // launch the step's kernels with programmatic dependent launch
  int solve0 = 0;  // first member of a part of a batch (noise_rng's member 0)
  // persistent stage launches (batches): the launch group's items and queue
  int persist = 0;
  const QItem* qitems = nullptr;
  int nq = 0, nq_pre = 0, stage_grid = 0;
  // sweep launches: one per nodes-per-thread class present (single plans
  // have one; a batch runs each member with its own class, as alone)
  struct SweepSeg {
    const Work* w;
    int n, mch;
    size_t smem;
  };
  SweepSeg sx[4] = {}, sy[4] = {};
  int nsx = 0, nsy = 0;
  // batches: the hyperviscosity chain as grid-stride loops over a few CTAs
  // per SM (hv_sms: the SM count; 0 for single plans, one CTA per tile)
  int hv_sms = 0;
  QCtl* qctl = nullptr;
  unsigned* qdep = nullptr;
  const Work *qtiles = nullptr, *xl4 = nullptr, *yl4 = nullptr;  // whole-batch lists
  size_t smem_stage = 0, stage_sh_off = 0, stage_xstride = 0;
};

// A kernel launch on L's stream; with L.pdl the launch allows programmatic
// dependent launch, so that the kernel's CTAs may start their prologue while
// the previous kernel finishes (the kernel waits in pdl_wait before it reads
// anything the previous kernel wrote).
template <typename... KP, typename... A>
void launch_k(void (*k)(KP...), dim3 grid, dim3 block, size_t smem, const LaunchSet& L, A... args) {
  if (!L.pdl) {
    k<<<grid, block, smem, L.st>>>(args...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = L.st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k, args...);
}

// Optional per-launch event recorder for hitb200_step_profile.  bytes are the
// algorithmic DRAM bytes of the launch: unique inputs read once plus outputs
// written once, at their stored precision.
struct Prof {
  cudaStream_t st;
  std::vector<cudaEvent_t> ev;
  std::vector<const char*> names;
  std::vector<double> bytes;
  void mark(const char* n, double b) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, st);
    ev.push_back(e);
    names.push_back(n);
    bytes.push_back(b);
  }
  void end() {
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, st);
    ev.push_back(e);
  }
  ~Prof() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
  }
};
#define PMARK(name, b) \
  if (prof) prof->mark(name, b)

// Dynamic shared-memory opt-ins are per device; each kernel remembers the
// largest size it was granted on each device.
constexpr int kMaxAttrDevices = 64;
std::mutex g_attr_mu;

inline int attr_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxAttrDevices) dev = 0;
  return dev;
}

template <typename T, int AXIS, int MCH, int OCC>
void set_sweep_attr(size_t bytes) {
  static size_t done[kMaxAttrDevices] = {};
  const int dev = attr_device();
  std::lock_guard<std::mutex> lock(g_attr_mu);
  if (bytes > done[dev]) {
    cudaFuncSetAttribute(sweep_kernel<T, AXIS, MCH, OCC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)bytes);
    done[dev] = bytes;
  }
}

template <typename T>
void set_sensor_attr(size_t bytes) {
  static size_t done[kMaxAttrDevices] = {};
  const int dev = attr_device();
  std::lock_guard<std::mutex> lock(g_attr_mu);
  if (bytes > done[dev]) {
    cudaFuncSetAttribute(sensor_kernel<T, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    cudaFuncSetAttribute(sensor_kernel<T, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    cudaFuncSetAttribute(sensor_kernel<T, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    done[dev] = bytes;
  }
}

// Widths with a step-sensor instantiation (sensor_step_kernel); others use
// the generic sensor_kernel.
inline int step_sensor_width(int w) { return (w == 3 || w == 4) ? w : -1; }
inline size_t step_sensor_bytes(int w, int elem, bool visc) {
  return w == 3 ? step_sensor_smem_bytes<3>(elem, visc) : w == 4 ? step_sensor_smem_bytes<4>(elem, visc) : 0;
}
template <typename T, int W>
void set_step_sensor_attr(size_t bytes) {
  static size_t done[kMaxAttrDevices] = {};
  const int dev = attr_device();
  std::lock_guard<std::mutex> lock(g_attr_mu);
  if (bytes > done[dev]) {
    cudaFuncSetAttribute(sensor_step_kernel<T, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    cudaFuncSetAttribute(hv_sensor_loop_kernel<T, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    done[dev] = bytes;
  }
}

// The persistent stage kernel's opt-in (per instantiation, by nodes per sweep
// thread, and device).
void set_stage_attr(const void* fn, int mch, size_t bytes) {
  static size_t done[3][kMaxAttrDevices] = {};
  const int dev = attr_device();
  std::lock_guard<std::mutex> lock(g_attr_mu);
  size_t& d = done[mch == 1 ? 0 : mch == 2 ? 1 : 2][dev];
  if (bytes > d) {
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    d = bytes;
  }
}

template <typename T, int AXIS>
void launch_sweep_seg(const LaunchSet& L, const LaunchSet::SweepSeg& g, int stage, int mode, const Bind& b) {
  const int mch = g.mch;
  const int nb = g.n;
  const size_t sm = g.smem;
  const Work* w = g.w;
  const int thr = AXIS == 0 ? L.thr_x : L.thr_y;
  const int occ = AXIS == 0 ? L.occ_x : L.occ_y;
#define HB_SWEEP(M)                                                                        \
  case M:                                                                                  \
    if (occ) {                                                                             \
      set_sweep_attr<T, AXIS, M, 1>(sm);                                                   \
      launch_k(sweep_kernel<T, AXIS, M, 1>, nb, thr, sm, L, L.solves, w, stage, mode, b);  \
    } else {                                                                               \
      set_sweep_attr<T, AXIS, M, 0>(sm);                                                   \
      launch_k(sweep_kernel<T, AXIS, M, 0>, nb, thr, sm, L, L.solves, w, stage, mode, b);  \
    }                                                                                      \
    break;
  switch (mch) {
    HB_SWEEP(1)
    HB_SWEEP(2)
    HB_SWEEP(4)
    HB_SWEEP(8)
  }
#undef HB_SWEEP
}

template <typename T, int AXIS>
void launch_sweep_t(const LaunchSet& L, int stage, int mode, const Bind& b) {
  const int ns = AXIS == 0 ? L.nsx : L.nsy;
  for (int i = 0; i < ns; ++i) launch_sweep_seg<T, AXIS>(L, AXIS == 0 ? L.sx[i] : L.sy[i], stage, mode, b);
}

void launch_sweep(const LaunchSet& L, int axis, int stage, int mode, const Bind& b) {
  if (L.elem == 4)
    axis == 0 ? launch_sweep_t<float, 0>(L, stage, mode, b) : launch_sweep_t<float, 1>(L, stage, mode, b);
  else
    axis == 0 ? launch_sweep_t<double, 0>(L, stage, mode, b) : launch_sweep_t<double, 1>(L, stage, mode, b);
}

template <typename T>
void launch_sensor_t(const LaunchSet& L, int sel, int enf, int visc, const Bind& b, uint8_t* mo) {
  if (b.use)
    launch_k(sensor_kernel<T, true, false>, L.n_tiles32, kSensorThreads, L.smem_sensor, L, L.solves,
             L.tiles32, sel, enf, visc, b, mo);
  else if (L.sensor_w == 4)
    launch_k(sensor_step_kernel<T, 4>, L.n_tiles32, kSensorThreads, L.smem_sensor_step, L, L.solves,
             L.tiles32, sel, enf, visc);
  else if (L.sensor_w == 3)
    launch_k(sensor_step_kernel<T, 3>, L.n_tiles32, kSensorThreads, L.smem_sensor_step, L, L.solves,
             L.tiles32, sel, enf, visc);
  else
    launch_k(sensor_kernel<T, false, false>, L.n_tiles32, kSensorThreads, L.smem_sensor, L, L.solves,
             L.tiles32, sel, enf, visc, b, mo);
}
void launch_sensor(const LaunchSet& L, int sel, int enf, int visc, const Bind& b, uint8_t* mo) {
  if (L.elem == 4) launch_sensor_t<float>(L, sel, enf, visc, b, mo);
  else launch_sensor_t<double>(L, sel, enf, visc, b, mo);
}
// The prepass of `sel`'s state fused with its sensor: one cooperative launch
// of the FUSED sensor (single solves whose tiles are all resident at once).
template <typename T>
void launch_presensor_t(const LaunchSet& L, int sel) {
  Bind nb{};
  uint8_t* mo = nullptr;
  int enf = sel == 3 ? 0 : 1, visc = sel == 3 ? 0 : 1;
  void* args[] = {(void*)&L.solves, (void*)&L.tiles32, (void*)&sel, (void*)&enf, (void*)&visc,
                  (void*)&nb, (void*)&mo};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(L.n_tiles32);
  cfg.blockDim = dim3(kSensorThreads);
  cfg.dynamicSmemBytes = L.smem_sensor;
  cfg.stream = L.st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelExC(&cfg, (const void*)sensor_kernel<T, false, true>, args);
}
void launch_presensor(const LaunchSet& L, int sel) {
  if (L.elem == 4) launch_presensor_t<float>(L, sel);
  else launch_presensor_t<double>(L, sel);
}

// One SSP-RK3 stage of a batch's launch group in one persistent launch
// (stage_persist.cuh); the first stage's list skips the prepass items.
void launch_stage(const LaunchSet& L, int stage) {
  const int skip = stage == 0 ? L.nq_pre : 0;
  const int n = L.nq - skip;
  const int grid = std::max(1, std::min(L.stage_grid, n));
  const QItem* it = L.qitems + skip;
  const int s0 = L.solve0, s1 = L.solve0 + L.nsolves;
  // the sweeps' nodes per thread are the batch's (the line solves' order of
  // operations depends on them)
  void (*k)(const SolveDev*, const Work*, const Work*, const Work*, const QItem*, int, QCtl*, unsigned*, int,
            int, int, unsigned, unsigned) = L.mch_x == 1   ? stage_kernel<float, 4, 1>
                                  : L.mch_x == 2 ? stage_kernel<float, 4, 2>
                                                 : stage_kernel<float, 4, 4>;
  k<<<grid, kStageThreads, L.smem_stage, L.st>>>(L.solves, L.qtiles, L.yl4, L.xl4, it, n, L.qctl, L.qdep, s0,
                                                  s1, stage, (unsigned)L.stage_sh_off, (unsigned)L.stage_xstride);
}

// The stage kernel of a batch (nodes per sweep thread mch on both axes).
const void* stage_fn(int mch) {
  return mch == 1 ? (const void*)stage_kernel<float, 4, 1>
                  : mch == 2 ? (const void*)stage_kernel<float, 4, 2> : (const void*)stage_kernel<float, 4, 4>;
}

void launch_hv(const LaunchSet& L, const Bind& b) {
  const int grid = L.hv_sms > 0 ? std::max(1, std::min(L.n_tiles, 4 * L.hv_sms)) : L.n_tiles;
  if (L.elem == 4) launch_k(hv_kernel<float>, grid, kStencilThreads, 0, L, L.solves, L.tiles, L.n_tiles, b);
  else launch_k(hv_kernel<double>, grid, kStencilThreads, 0, L, L.solves, L.tiles, L.n_tiles, b);
}

// The hyperviscosity prepass and sensor of a batch as grid-stride loops
// (hv_prepass_loop_kernel, hv_sensor_loop_kernel).
void launch_hv_prepass_loop(const LaunchSet& L) {
  const int grid = std::max(1, std::min(L.n_tiles32, 4 * L.hv_sms));
  if (L.elem == 4) hv_prepass_loop_kernel<float><<<grid, kPreThreads, 0, L.st>>>(L.solves, L.tiles32, L.n_tiles32);
  else hv_prepass_loop_kernel<double><<<grid, kPreThreads, 0, L.st>>>(L.solves, L.tiles32, L.n_tiles32);
}
void launch_hv_sensor_loop(const LaunchSet& L) {
  const int grid = std::max(1, std::min(L.n_tiles32, 2 * L.hv_sms));
  const size_t sm = L.smem_sensor_step;
  if (L.elem == 4) {
    if (L.sensor_w == 4) hv_sensor_loop_kernel<float, 4><<<grid, kSensorThreads, sm, L.st>>>(L.solves, L.tiles32, L.n_tiles32);
    else hv_sensor_loop_kernel<float, 3><<<grid, kSensorThreads, sm, L.st>>>(L.solves, L.tiles32, L.n_tiles32);
  } else {
    if (L.sensor_w == 4) hv_sensor_loop_kernel<double, 4><<<grid, kSensorThreads, sm, L.st>>>(L.solves, L.tiles32, L.n_tiles32);
    else hv_sensor_loop_kernel<double, 3><<<grid, kSensorThreads, sm, L.st>>>(L.solves, L.tiles32, L.n_tiles32);
  }
}
void launch_prepass(const LaunchSet& L, int buf, int mode, int enf, const Bind& b) {
#define HB_PRE(TT, O) \
  launch_k(prepass_kernel<TT, O>, L.n_tiles32, kPreThreads, 0, L, L.solves, L.tiles32, buf, mode, enf, b)
  if (L.elem == 4) {
    if (L.occ_pre) HB_PRE(float, 1);
    else HB_PRE(float, 0);
  } else {
    if (L.occ_pre) HB_PRE(double, 1);
    else HB_PRE(double, 0);
  }
#undef HB_PRE
}

// The reference's forcing-noise field of the step from its PCG64 stream
// (kernels_npnoise.cuh), into the solve's noise buffer.
void launch_noise_gen(const LaunchSet& L) {
  const NoiseBufs& b = *L.gen;
  const int per = kNoiseThreads * kNoiseChunk;
  const int nblk = (int)((b.P + per - 1) / per);
  npnoise_classify_kernel<<<nblk, kNoiseThreads, 0, L.st>>>(L.solves, b, S_PCG);
  npnoise_scan_kernel<<<1, 1024, 0, L.st>>>(L.solves, b, nblk);
  npnoise_compact_kernel<<<nblk, kNoiseThreads, 0, L.st>>>(L.solves, b);
  npnoise_resolve_kernel<<<1, kNoiseResolveThreads, 0, L.st>>>(L.solves, b);
  npnoise_scatter_kernel<<<nblk, kNoiseThreads, 0, L.st>>>(L.solves, b, L.gen_out, (long long)L.cells,
                                                           S_PCG);
}

// The reference's loop body (OOP/hit2d.py:828-879; riemann_config3.py:728-740).
int launch_step_sequence(const LaunchSet& L, int any_forcing, int noise_upload, int any_outflow,
                         int any_hv, Prof* prof = nullptr) {
  Bind nb{};
  const double N = L.cells, e = L.elem;
  if (L.fused) {
    PMARK("presensor", 65 * N + 3 * e * L.cells_visc);
    launch_presensor(L, 0);  // the step's prepass and the first stage's sensor
  } else {
    PMARK("prepass", 32 * N);
    launch_prepass(L, 0, PRE_STEP, 1, nb);
  }
  if (any_forcing) {
    if (L.gen) {
      PMARK("noise_gen", 8 * L.cells_force);
      launch_noise_gen(L);
    }
    if (noise_upload || L.gen) {
      PMARK("noise_dft", 8 * L.cells_force);
      noise_dft_kernel<<<L.n_tiles32, kRedThreads, 0, L.st>>>(L.solves, L.tiles32, nb);
    } else {
      PMARK("noise_rng", 0.0);
      noise_rng_kernel<<<L.nsolves, 128, 0, L.st>>>(L.solves + L.solve0, L.nsolves,
                                                     L.partner + (size_t)L.solve0 * kMaxForce);
    }
    PMARK("force_synth", 48 * L.cells_force);
    force_synth_kernel<<<L.n_srows, kRedThreads, 0, L.st>>>(L.solves, L.srows, nb);
  }
  for (int stage = 0; stage < 3; ++stage) {
    if (L.persist) {
      PMARK("stage", (stage == 0 ? 0 : 32 * N) + 33 * N + 3 * e * L.cells_visc + 33 * N + 4 * e * N +
                         (stage == 0 ? 65 : 97) * N + 4 * e * N + 3 * e * L.cells_visc + 16 * L.cells_force);
      launch_stage(L, stage);
      continue;
    }
    if (L.fused) {
      if (stage > 0) {
        PMARK("presensor", 65 * N + 3 * e * L.cells_visc);
        launch_presensor(L, stage);
      }
    } else {
      if (stage > 0) {
        PMARK("prepass", 32 * N);
        launch_prepass(L, stage, PRE_STAGE, 1, nb);
      }
      PMARK("sensor", 33 * N + 3 * e * L.cells_visc);
      launch_sensor(L, stage, 1, 1, nb, nullptr);
    }
    // y sweep: q, mask -> -dG/dy; x sweep: q, mask, -dG/dy, sources (, q) -> stage state
    PMARK("sweep_y", 33 * N + 4 * e * N);
    launch_sweep(L, 1, stage, SW_STAGE, nb);
    PMARK("sweep_x", (stage == 0 ? 65 : 97) * N + 4 * e * N + 3 * e * L.cells_visc + 16 * L.cells_force);
    launch_sweep(L, 0, stage, SW_STAGE, nb);
  }
  if (any_hv) {
    if (L.fused) {
      PMARK("hv_presensor", 65 * N);
      launch_presensor(L, 3);
    } else if (L.hv_sms > 0 && (L.sensor_w == 3 || L.sensor_w == 4)) {
      PMARK("hv_prepass", 32 * N);
      launch_hv_prepass_loop(L);
      PMARK("hv_sensor", 33 * N);
      launch_hv_sensor_loop(L);
    } else {
      PMARK("hv_prepass", 32 * N);
      launch_prepass(L, 1, PRE_SENSOR, 0, nb);
      PMARK("hv_sensor", 33 * N);
      launch_sensor(L, 3, 0, 0, nb, nullptr);
    }
    PMARK("hv", 65 * N);
    launch_hv(L, nb);  // applies the outflow guard of outflow solves too
  }
  if (prof) prof->end();
  HB_LAUNCHED("step kernels");
  return HITB200_OK;
}

int finish_profile(Prof& pr, float* ms, double* bytes, int32_t cap, int32_t* count, char* names,
                   size_t names_size) {
  HB_CUDA(cudaStreamSynchronize(pr.st));
  const int n = (int)pr.names.size();
  if (count) *count = n;
  std::string all;
  for (int i = 0; i < n; ++i) {
    float t = 0.f;
    HB_CUDA(cudaEventElapsedTime(&t, pr.ev[i], pr.ev[i + 1]));
    if (i < cap) {
      if (ms) ms[i] = t;
      if (bytes) bytes[i] = pr.bytes[i];
    }
    all += pr.names[i];
    all += '\n';
  }
  if (names && names_size > 0) {
    std::strncpy(names, all.c_str(), names_size - 1);
    names[names_size - 1] = 0;
  }
  return HITB200_OK;
}

LaunchSet plan_launch_set(hitb200_plan* p, cudaStream_t st) {
  LaunchSet L;
  L.solves = p->d_solve;
  L.nsolves = 1;
  L.tiles = p->d_tiles;
  L.tiles32 = p->d_tiles32;
  L.n_tiles32 = p->n_tiles32;
  L.srows = p->d_srows;
  L.n_srows = p->n_srows;
  L.guard_blocks = guard_blocks_for(p->desc);
  L.xl = p->d_xlines;
  L.yl = p->d_ylines;
  L.partner = p->d_partner;
  L.n_tiles = p->n_tiles;
  L.n_x = p->n_x;
  L.n_y = p->n_y;
  L.elem = p->elem;
  L.mch_x = mch_for(p->desc.nx);
  L.mch_y = mch_for(p->desc.ny);
  L.thr_x = kLineThreads * p->Rx;
  L.thr_y = kLineThreads * p->Ry;
  if (p->tuning[HITB200_TUNE_Y_PANEL] && p->Ry2 != p->Ry) {
    L.yl = p->d_ylines2;
    L.n_y = p->n_y2;
    L.thr_y = kLineThreads * p->Ry2;
  }
  L.occ_x = p->tuning[HITB200_TUNE_SWEEP_X];
  L.occ_y = p->tuning[HITB200_TUNE_SWEEP_Y];
  L.occ_pre = p->tuning[HITB200_TUNE_PREPASS];
  L.fused = p->tuning[HITB200_TUNE_FUSED_SENSOR] && p->fuse_ok;
  L.smem_x = p->smem_x;
  L.smem_y = p->tuning[HITB200_TUNE_Y_PANEL] && p->Ry2 != p->Ry ? p->smem_y2 : p->smem_y;
  L.sx[0] = {L.xl, L.n_x, L.mch_x, L.smem_x};
  L.sy[0] = {L.yl, L.n_y, L.mch_y, L.smem_y};
  L.nsx = L.nsy = 1;
  L.smem_sensor = p->smem_sensor;
  L.gen = p->has_gen ? &p->gen : nullptr;
  L.gen_out = p->has_gen ? const_cast<double*>(p->hs.noise) : nullptr;
  L.sensor_w = p->sensor_w;
  L.smem_sensor_step = p->smem_sensor_step;
  L.st = st;
  L.cells = (double)p->desc.nx * p->desc.ny;
  // programmatic dependent launch only in the step sequence (set by its
  // callers), whose kernel order makes each kernel's early loads safe
  L.pdl = 0;
  L.cells_visc = p->desc.viscosity > 0.0 ? L.cells : 0.0;
  L.cells_force = p->desc.forcing_on ? L.cells : 0.0;
  return L;
}

// Shared-memory opt-in of every kernel a launch set may use; called at plan /
// batch creation so that no attribute call happens during graph capture.
void prime_attributes(int elem, int mch_x, int mch_y, size_t smem_x, size_t smem_y,
                      size_t smem_sensor, int sensor_w, size_t smem_sensor_step) {
  auto sweep = [&](auto tag, int axis, int mch, size_t bytes) {
    using T = decltype(tag);
#define HB_ATTR(M)                                                    \
  if (mch == M) {                                                     \
    if (axis == 0) {                                                  \
      set_sweep_attr<T, 0, M, 0>(bytes);                              \
      set_sweep_attr<T, 0, M, 1>(bytes);                              \
    } else {                                                          \
      set_sweep_attr<T, 1, M, 0>(bytes);                              \
      set_sweep_attr<T, 1, M, 1>(bytes);                              \
    }                                                                 \
  }
    HB_ATTR(1) HB_ATTR(2) HB_ATTR(4) HB_ATTR(8)
#undef HB_ATTR
  };
  if (elem == 4) {
    sweep(float{}, 0, mch_x, smem_x);
    sweep(float{}, 1, mch_y, smem_y);
    set_sensor_attr<float>(smem_sensor);
    if (sensor_w == 4) set_step_sensor_attr<float, 4>(smem_sensor_step);
    if (sensor_w == 3) set_step_sensor_attr<float, 3>(smem_sensor_step);
  } else {
    sweep(double{}, 0, mch_x, smem_x);
    sweep(double{}, 1, mch_y, smem_y);
    set_sensor_attr<double>(smem_sensor);
    if (sensor_w == 4) set_step_sensor_attr<double, 4>(smem_sensor_step);
    if (sensor_w == 3) set_step_sensor_attr<double, 3>(smem_sensor_step);
  }
}

// Shared-memory opt-in of one sweep instantiation family (both variants).
void prime_sweep_attr(int elem, int axis, int mch, size_t bytes) {
#define HB_ATTR1(TT, M)                          \
  if (mch == M) {                                \
    if (axis == 0) {                             \
      set_sweep_attr<TT, 0, M, 0>(bytes);        \
      set_sweep_attr<TT, 0, M, 1>(bytes);        \
    } else {                                     \
      set_sweep_attr<TT, 1, M, 0>(bytes);        \
      set_sweep_attr<TT, 1, M, 1>(bytes);        \
    }                                            \
  }
  if (elem == 4) {
    HB_ATTR1(float, 1) HB_ATTR1(float, 2) HB_ATTR1(float, 4) HB_ATTR1(float, 8)
  } else {
    HB_ATTR1(double, 1) HB_ATTR1(double, 2) HB_ATTR1(double, 4) HB_ATTR1(double, 8)
  }
#undef HB_ATTR1
}

int validate_desc(const hitb200_desc* d) {
  if (!d) return invalid("descriptor is NULL");
  if (d->nx <= 0 || d->ny <= 0) return invalid("nx and ny must be positive");
  if (d->nx > kMaxLine || d->ny > kMaxLine)
    return (g_last_error = "grid lines longer than 1024 nodes are not supported", HITB200_ERR_UNSUPPORTED);
  if (!(d->x_max > d->x_min) || !(d->y_max > d->y_min)) return invalid("domain extent must be positive");
  if (d->precision != 0 && d->precision != 1) return invalid("precision must be 0 (fp64) or 1 (fp32 bulk)");
  if (d->scheme != 0 && d->scheme != 1) return invalid("scheme must be 'hybrid' or 'weno'");
  if (d->sensor_width < 0 || d->sensor_width > kMaxWidth)
    return (g_last_error = "sensor width must be in [0, 8]", HITB200_ERR_UNSUPPORTED);
  if (d->hv_interval < 0) return invalid("hyperviscosity_interval must be >= 0");
  if (d->noise_mode < 0 || d->noise_mode > 2) return invalid("noise_mode must be 0, 1 or 2");
  if (!d->periodic && (d->guard_cells < 0)) return invalid("guard_cells must be >= 0");
  if (!d->periodic && d->guard_cells > 0 && (d->nx <= 2 * d->guard_cells || d->ny <= 2 * d->guard_cells))
    return invalid("state is too small for the requested guard cells");
  if (d->forcing_on) {
    if (!d->periodic) return invalid("forcing needs a periodic grid");
    if (d->forcing_kmin < 0.0 || d->forcing_kmax <= 0.0 || d->forcing_kmin > d->forcing_kmax)
      return invalid("forcing shell must satisfy 0 <= k_min <= k_max");
    if (d->forcing_correlation_time <= 0.0) return invalid("forcing correlation time must be positive");
    if (!(d->alpha_memory >= 0.0 && d->alpha_memory < 1.0)) return invalid("alpha_memory must be in [0, 1)");
  }
  if (d->mach_control && !is_none(d->target_power)) {
    if (d->mach_target <= 0.0) return invalid("Mach control requires a positive target Mach number");
    if (!(d->mach_memory >= 0.0 && d->mach_memory < 1.0)) return invalid("mach_control_memory must be in [0, 1)");
    if (d->mach_exponent <= 0.0) return invalid("mach_control_exponent must be positive");
  }
  return HITB200_OK;
}

}  // namespace

// =================================================================================
extern "C" {

const char* hitb200_version(void) { return "hitb200 sm_100a 1.0"; }

size_t hitb200_desc_size(void) { return sizeof(hitb200_desc); }

const char* hitb200_status_string(int status) {
  switch (status) {
    case HITB200_OK: return "ok";
    case HITB200_ERR_NONFINITE: return "state contains NaN or Inf values";
    case HITB200_ERR_NONPOSITIVE: return "state contains non-positive density or pressure";
    default: return g_last_error.empty() ? "error" : g_last_error.c_str();
  }
}

int hitb200_desc_init(hitb200_desc* d) {
  if (!d) return invalid("descriptor is NULL");
  std::memset(d, 0, sizeof(*d));
  const double nan = std::nan("");
  d->nx = d->ny = 128;
  d->x_min = d->y_min = 0.0;
  d->x_max = d->y_max = 2.0 * M_PI;
  d->periodic = 1;
  d->precision = 0;
  d->scheme = 0;
  d->gamma = 1.4;
  d->sensor_width = 4;
  d->boundary_guard = 0;
  d->compression_threshold = 2.5;
  d->jump_threshold = 0.04;
  d->shear_threshold = nan;
  d->viscosity = 1.0e-3;
  d->prandtl = 0.72;
  d->gas_constant = 1.0;
  d->hv_mn = 0.002;
  d->hv_weight[0] = 0.25;
  d->hv_weight[1] = 1.0;
  d->hv_weight[2] = 1.0;
  d->hv_weight[3] = 0.25;
  d->hv_interval = 5;
  d->guard_cells = 0;
  d->drag_coefficient = 0.0;
  d->drag_kmax = 2.0;
  d->cooling_time = nan;
  d->cooling_target_pressure = nan;
  d->forcing_on = 1;
  d->forcing_kmin = 0.0;
  d->forcing_kmax = 3.0;
  d->forcing_correlation_time = 1.0;
  d->forcing_rms = 1.0;
  d->target_power = 1.0e-3;
  d->min_power = 1.0e-6;
  d->max_rescale = 20.0;
  d->alpha_memory = 0.2;
  d->mach_control = 0;
  d->mach_target = 0.1;
  d->mach_memory = 0.995;
  d->mach_exponent = 2.0;
  d->mach_min_power = nan;
  d->mach_max_power = nan;
  d->cfl = 0.05;
  d->tfinal = 1.0;
  d->fixed_dt = 0;
  d->noise_mode = 0;
  d->seed = 1234;
  return HITB200_OK;
}

int hitb200_release_cached_blocks(void) {
  std::lock_guard<std::mutex> lk(g_blocks_mu);
  release_blocks_locked(-1);
  return HITB200_OK;
}

size_t hitb200_cached_block_bytes(void) {
  std::lock_guard<std::mutex> lk(g_blocks_mu);
  return g_blocks_bytes;
}

}  // extern "C"

namespace {
// Buffers of the device noise stream for N normals (kernels_npnoise.cuh).
long long noise_gen_positions(size_t N) { return (long long)N + (long long)N / 8 + 4096; }
size_t noise_gen_bytes(size_t N) {
  const size_t P = (size_t)noise_gen_positions(N);
  const size_t nblk = (P + kNoiseThreads * kNoiseChunk - 1) / (kNoiseThreads * kNoiseChunk);
  // val, deficit (8 B), slow, reach (4 B), cons, outf, visited (1 B), counts, offsets
  return 8 * P * 2 + 4 * P * 2 + 3 * P + 4 * (2 * nblk + 1) + 4 + 64 * 8;
}
NoiseBufs noise_gen_layout(unsigned char* base, size_t N) {
  NoiseBufs b{};
  const size_t P = (size_t)noise_gen_positions(N);
  const size_t nblk = (P + kNoiseThreads * kNoiseChunk - 1) / (kNoiseThreads * kNoiseChunk);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    unsigned char* q = base + off;
    off = (off + bytes + 7) & ~(size_t)7;
    return q;
  };
  b.val = reinterpret_cast<double*>(take(8 * P));
  b.deficit = reinterpret_cast<long long*>(take(8 * P));
  b.slow = reinterpret_cast<unsigned*>(take(4 * P));
  b.reach = reinterpret_cast<unsigned*>(take(4 * P));
  b.cons = take(P);
  b.outf = take(P);
  b.visited = take(P);
  b.cta_count = reinterpret_cast<unsigned*>(take(4 * nblk));
  b.cta_off = reinterpret_cast<unsigned*>(take(4 * (nblk + 1)));
  b.nslow = reinterpret_cast<unsigned*>(take(4));
  b.P = (long long)P;
  return b;
}

// The ziggurat table of the device noise stream, once per device.
cudaError_t upload_zig_tables() {
  static bool done[kMaxAttrDevices] = {};
  const int dev = attr_device();
  std::lock_guard<std::mutex> lock(g_attr_mu);
  if (done[dev]) return cudaSuccess;
  cudaError_t e = cudaMemcpyToSymbol(g_zig_w, zig::kZigW, sizeof(zig::kZigW));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_zig_k, zig::kZigK, sizeof(zig::kZigK));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_zig_f, zig::kZigF, sizeof(zig::kZigF));
  if (e == cudaSuccess) done[dev] = true;
  return e;
}
}  // namespace

extern "C" {

size_t hitb200_plan_device_bytes(const hitb200_desc* d) {
  if (validate_desc(d) != HITB200_OK) return 0;
  const size_t N = (size_t)d->nx * d->ny;
  const int elem = d->precision == 1 ? 4 : 8;
  const int ntx = (d->nx + kHvTX - 1) / kHvTX, nty = (d->ny + kHvTY - 1) / kHvTY;
  const size_t ntile = (size_t)ntx * nty;
  ModeTables mt = build_modes(*d);
  Arena a;
  a.take(sizeof(SolveDev));
  a.take(2 * 4 * N * sizeof(double));                        // q1, q2
  a.take(4 * N * elem);                                      // rx
  if (d->viscosity > 0.0) a.take(3 * N * elem);              // vis
  a.take(N);                                                 // mask
  if (d->forcing_on) a.take(2 * N * sizeof(double));         // fx, fy
  if (d->forcing_on && d->noise_mode != 1) a.take(N * sizeof(double));
  if (d->forcing_on && d->noise_mode == 2) a.take(noise_gen_bytes(N));
  a.take((d->nx + d->ny) * sizeof(double2));
  a.take((mt.drag.size() + mt.force.size() + 1) * sizeof(int2));
  a.take((mt.force.size() + 1) * sizeof(double2));
  a.take(kMaxForce * sizeof(int));
  a.take(SCAL_SIZE * sizeof(double));
  a.take(ntile * (R_FIXED + 4 * mt.drag.size()) * sizeof(double));
  a.take(ntile * (2 * mt.force.size() + 1) * sizeof(double));
  a.take(std::max(ntile, (size_t)d->ny) * 4 * sizeof(double));  // synthesis partials
  a.take(ntile * NDIAG * sizeof(double));
  a.take(8 * sizeof(unsigned) + sizeof(int) + NDIAG * sizeof(double));
  a.take(ntile * sizeof(Work));
  a.take((size_t)((d->nx + kSenTX - 1) / kSenTX) * ((d->ny + kSenTY - 1) / kSenTY) * sizeof(Work));
  a.take((size_t)(d->ny + d->nx) * sizeof(Work));
  a.take((size_t)d->nx * sizeof(Work));  // the other y-panel width's lines
  a.take((size_t)d->ny * sizeof(Work));  // synthesis row blocks (at most one per row)
  return a.off;
}

int hitb200_plan_create(const hitb200_desc* d, hitb200_plan** out) {
  if (!out) return invalid("plan pointer is NULL");
  *out = nullptr;
  int st = validate_desc(d);
  if (st != HITB200_OK) return st;
  ModeTables mt = build_modes(*d);
  if ((int)mt.drag.size() > kMaxDrag)
    return (g_last_error = "drag band holds more than 32 modes", HITB200_ERR_UNSUPPORTED);
  if ((int)mt.force.size() > kMaxForce)
    return (g_last_error = "forcing shell holds more than 128 modes", HITB200_ERR_UNSUPPORTED);
  if (d->forcing_on && mt.force.empty()) return invalid("forcing shell contains no Fourier modes on this grid");
  for (const std::vector<int2>* v : {&mt.drag, &mt.force})
    for (const int2& m : *v)
      if (std::abs(m.x) > kMaxKx || (v == &mt.drag && std::abs(m.y) > kMaxKyDrag))
        return (g_last_error = "drag / forcing modes beyond |kx| = 16 (drag |ky| = 4) grid bins are not supported",
                HITB200_ERR_UNSUPPORTED);

  hitb200_plan* p = new hitb200_plan();
  p->desc = *d;
  p->elem = d->precision == 1 ? 4 : 8;
  const int nx = d->nx, ny = d->ny;
  const size_t N = (size_t)nx * ny;
  const int ntx = (nx + kHvTX - 1) / kHvTX, nty = (ny + kHvTY - 1) / kHvTY;
  p->n_tiles = ntx * nty;
  p->Rx = lines_per_cta(nx, ny, p->elem);
  p->Ry = lines_per_cta(ny, nx, p->elem);
  // y panels: at least 16-byte row segments where the shared memory allows
  if (p->Ry < 2 && nx >= 2 &&
      (p->elem == 4 ? SweepLayout<float>(ny, 2).bytes() : SweepLayout<double>(ny, 2).bytes()) <= kSweepSmemMax)
    p->Ry = 2;
  p->n_x = (ny + p->Rx - 1) / p->Rx;
  p->n_y = (nx + p->Ry - 1) / p->Ry;
  default_tuning(p->n_x, p->n_y, ((nx + kSenTX - 1) / kSenTX) * ((ny + kSenTY - 1) / kSenTY), p->tuning);
  p->smem_x = p->elem == 4 ? SweepLayout<float>(nx, p->Rx).bytes() : SweepLayout<double>(nx, p->Rx).bytes();
  p->smem_y = p->elem == 4 ? SweepLayout<float>(ny, p->Ry).bytes() : SweepLayout<double>(ny, p->Ry).bytes();
  {
    const int alt = p->Ry == 4 ? 2 : 4;
    const size_t b2 = p->elem == 4 ? SweepLayout<float>(ny, alt).bytes() : SweepLayout<double>(ny, alt).bytes();
    p->Ry2 = (nx >= alt && b2 <= 110 * 1024) ? alt : p->Ry;
    p->n_y2 = (nx + p->Ry2 - 1) / p->Ry2;
    p->smem_y2 = p->elem == 4 ? SweepLayout<float>(ny, p->Ry2).bytes() : SweepLayout<double>(ny, p->Ry2).bytes();
  }
  p->smem_sensor = sensor_smem_bytes(d->sensor_width, p->elem, d->viscosity > 0.0);
  p->sensor_w = step_sensor_width(d->sensor_width);
  p->smem_sensor_step = step_sensor_bytes(p->sensor_w, p->elem, d->viscosity > 0.0);
  if (p->smem_x > kSweepSmemMax || p->smem_y > kSweepSmemMax) {
    delete p;
    return (g_last_error = "grid lines too long for the sweep's shared memory", HITB200_ERR_UNSUPPORTED);
  }

  // ---- arena layout ----
  Arena a;
  const size_t o_solve = a.take(sizeof(SolveDev));
  const size_t o_q1 = a.take(4 * N * sizeof(double));
  const size_t o_q2 = a.take(4 * N * sizeof(double));
  const size_t o_rx = a.take(4 * N * p->elem);
  const size_t o_vis = d->viscosity > 0.0 ? a.take(3 * N * p->elem) : 0;
  const size_t o_mask = a.take(N);
  const size_t o_fx = d->forcing_on ? a.take(N * p->elem) : 0;
  const size_t o_fy = d->forcing_on ? a.take(N * p->elem) : 0;
  const size_t o_noise = (d->forcing_on && d->noise_mode != 1) ? a.take(N * sizeof(double)) : 0;
  const size_t o_gen = (d->forcing_on && d->noise_mode == 2) ? a.take(noise_gen_bytes(N)) : 0;
  const size_t o_tw = a.take((nx + ny) * sizeof(double2));
  const size_t o_modes = a.take((mt.drag.size() + mt.force.size() + 1) * sizeof(int2));
  const size_t o_kvec = a.take((mt.force.size() + 1) * sizeof(double2));
  const size_t o_partner = a.take(kMaxForce * sizeof(int));
  const size_t o_scal = a.take(SCAL_SIZE * sizeof(double));
  const size_t nred = R_FIXED + 4 * mt.drag.size();
  const size_t o_ppre = a.take(p->n_tiles * nred * sizeof(double));
  const size_t o_pnoise = a.take(p->n_tiles * (2 * mt.force.size() + 1) * sizeof(double));
  const int srows = synth_rows(nx);
  p->n_srows = (ny + srows - 1) / srows;
  const size_t o_psynth = a.take((size_t)std::max(p->n_tiles, p->n_srows) * 4 * sizeof(double));
  const size_t o_pdiag = a.take(p->n_tiles * NDIAG * sizeof(double));
  const size_t o_cnt = a.take(8 * sizeof(unsigned) + sizeof(int) + NDIAG * sizeof(double));
  const size_t o_tiles = a.take(p->n_tiles * sizeof(Work));
  const int ntx32 = (nx + kSenTX - 1) / kSenTX, nty32 = (ny + kSenTY - 1) / kSenTY;
  p->n_tiles32 = ntx32 * nty32;
  const size_t o_tiles32 = a.take(p->n_tiles32 * sizeof(Work));
  const size_t o_xl = a.take(p->n_x * sizeof(Work));
  const size_t o_yl = a.take(p->n_y * sizeof(Work));
  const size_t o_yl2 = a.take(p->n_y2 * sizeof(Work));
  const size_t o_sr = a.take(p->n_srows * sizeof(Work));
  p->arena_bytes = a.off;
  cudaError_t e = block_alloc(a.off, &p->arena_block);
  if (e != cudaSuccess) {
    delete p;
    return cuda_fail(e, "cudaMalloc(plan arena)");
  }
  p->arena = static_cast<unsigned char*>(p->arena_block.ptr);
  unsigned char* base = p->arena;
  SolveDev& s = p->hs;
  std::memset(&s, 0, sizeof(s));
  s.nx = nx;
  s.ny = ny;
  s.periodic = d->periodic;
  s.scheme = d->scheme;
  s.precision = d->precision;
  s.dx = (d->x_max - d->x_min) / nx;
  s.dy = (d->y_max - d->y_min) / ny;
  s.gamma = d->gamma;
  s.width = d->sensor_width;
  s.boundary_guard = d->periodic ? 0 : d->boundary_guard;
  s.comp_thr = d->compression_threshold;
  s.jump_thr = d->jump_threshold;
  // periodic: shear on when the threshold is given; outflow: when given and > 0
  s.shear_on = !is_none(d->shear_threshold) && (d->periodic || d->shear_threshold > 0.0);
  s.shear_thr = is_none(d->shear_threshold) ? 0.0 : d->shear_threshold;
  s.mu = d->viscosity;
  s.gas_r = d->gas_constant;
  s.kappa = d->viscosity * (d->gamma * d->gas_constant / (d->gamma - 1.0)) / d->prandtl;
  const double h = std::min(s.dx, s.dy);
  for (int c = 0; c < 4; ++c) s.hv_coef[c] = d->hv_mn * d->hv_weight[c] * std::pow(h, 4.0);
  const bool hv_on = d->hv_mn > 0.0 && d->hv_interval > 0 && d->scheme == 0;
  s.hv_interval = hv_on ? d->hv_interval : 0;
  s.guard = d->periodic ? 0 : d->guard_cells;
  s.n_drag = (int)mt.drag.size();
  s.drag_on = s.n_drag > 0;
  s.drag_coef = d->drag_coefficient;
  s.cooling_on = !is_none(d->cooling_time) && d->cooling_time > 0.0 && d->periodic;
  s.cooling_tau = s.cooling_on ? d->cooling_time : 1.0;
  s.cooling_pref = is_none(d->cooling_target_pressure) ? 1.0 / d->gamma : d->cooling_target_pressure;
  s.forcing_on = d->forcing_on;
  s.n_force = (int)mt.force.size();
  s.kx_drag = s.kx_force = 0;
  for (const int2& m : mt.drag) s.kx_drag = std::max(s.kx_drag, std::abs(m.x));
  s.ky_drag = 0;
  for (const int2& m : mt.drag) s.ky_drag = std::max(s.ky_drag, std::abs(m.y));
  for (const int2& m : mt.force) s.kx_force = std::max(s.kx_force, std::abs(m.x));
  {
    int pos = 0;
    for (int k = 0; k <= kMaxKx + 1; ++k) {
      s.f_kofs[k] = (short)pos;
      for (size_t m = 0; m < mt.force.size(); ++m)
        if (std::abs(mt.force[m].x) == k) s.f_order[pos++] = (unsigned char)m;
    }
  }
  s.f_tau = d->forcing_correlation_time;
  s.f_rms = d->forcing_rms;
  s.f_has_target = !is_none(d->target_power);
  s.f_target = d->target_power;
  s.f_min_power = d->min_power;
  s.f_has_max_rescale = !is_none(d->max_rescale);
  s.f_max_rescale = d->max_rescale;
  s.f_alpha_memory = d->alpha_memory;
  s.mach_control = d->mach_control;
  s.mach_target = d->mach_target;
  s.mach_memory = d->mach_memory;
  s.mach_exponent = d->mach_exponent;
  s.has_mach_min = !is_none(d->mach_min_power);
  s.mach_min_power = d->mach_min_power;
  s.has_mach_max = !is_none(d->mach_max_power);
  s.mach_max_power = d->mach_max_power;
  s.cfl = d->cfl;
  s.tfinal = d->tfinal;
  s.fixed_dt = d->fixed_dt;
  s.noise_mode = d->noise_mode;
  s.seed = d->seed;
  s.nblk_pre = s.nblk_noise = s.nblk_diag = p->n_tiles32;
  s.nblk_synth = p->n_srows;
  s.nred = (int)nred;
  s.q = nullptr;
  s.q1 = reinterpret_cast<double*>(base + o_q1);
  s.q2 = reinterpret_cast<double*>(base + o_q2);
  s.rx = base + o_rx;
  s.vis = d->viscosity > 0.0 ? (void*)(base + o_vis) : nullptr;
  s.mask = base + o_mask;
  s.fx = d->forcing_on ? reinterpret_cast<void*>(base + o_fx) : nullptr;
  s.fy = d->forcing_on ? reinterpret_cast<void*>(base + o_fy) : nullptr;
  s.noise = o_noise ? reinterpret_cast<double*>(base + o_noise) : nullptr;
  if (o_gen) {
    p->has_gen = true;
    p->gen = noise_gen_layout(base + o_gen, N);
    const cudaError_t ze = upload_zig_tables();
    if (ze != cudaSuccess) {
      block_free(p->arena_block);
      delete p;
      return cuda_fail(ze, "cudaMemcpyToSymbol(ziggurat tables)");
    }
  }
  s.twx = reinterpret_cast<double2*>(base + o_tw);
  s.twy = s.twx + nx;
  s.modes = reinterpret_cast<int2*>(base + o_modes);
  s.kvec = reinterpret_cast<double2*>(base + o_kvec);
  s.scal = reinterpret_cast<double*>(base + o_scal);
  s.part_pre = reinterpret_cast<double*>(base + o_ppre);
  s.part_noise = reinterpret_cast<double*>(base + o_pnoise);
  s.part_synth = reinterpret_cast<double*>(base + o_psynth);
  s.part_diag = reinterpret_cast<double*>(base + o_pdiag);
  s.counters = reinterpret_cast<unsigned*>(base + o_cnt);
  s.near_count = reinterpret_cast<int*>(s.counters + 8);
  s.diag_out = reinterpret_cast<double*>(base + o_cnt + 64);
  p->d_solve = reinterpret_cast<SolveDev*>(base + o_solve);
  p->own_solve = p->d_solve;
  p->d_partner = reinterpret_cast<int*>(base + o_partner);
  p->d_tiles = reinterpret_cast<Work*>(base + o_tiles);
  p->d_tiles32 = reinterpret_cast<Work*>(base + o_tiles32);
  p->d_xlines = reinterpret_cast<Work*>(base + o_xl);
  p->d_ylines = reinterpret_cast<Work*>(base + o_yl);
  p->d_ylines2 = reinterpret_cast<Work*>(base + o_yl2);
  p->d_srows = reinterpret_cast<Work*>(base + o_sr);

  // ---- host-built tables ----
  std::vector<double2> tw(nx + ny);
  for (int j = 0; j < nx; ++j) {
    const double th = 2.0 * M_PI * (double)j / (double)nx;
    tw[j] = make_double2(std::cos(th), -std::sin(th));
  }
  for (int j = 0; j < ny; ++j) {
    const double th = 2.0 * M_PI * (double)j / (double)ny;
    tw[nx + j] = make_double2(std::cos(th), -std::sin(th));
  }
  std::vector<int2> modes(mt.drag);
  modes.insert(modes.end(), mt.force.begin(), mt.force.end());
  modes.push_back(make_int2(0, 0));
  std::vector<double2> kvec(mt.kvec);
  kvec.push_back(make_double2(0, 0));
  std::vector<double> scal(SCAL_SIZE, 0.0);
  scal[S_ACTIVE] = 1.0;
  scal[S_MAX_STEPS] = -1.0;
  scal[S_POWER] = s.f_has_target ? d->target_power : std::nan("");
  scal[S_POWER_DESIRED] = scal[S_POWER];
  scal[S_F_ALPHA] = 1.0;
  scal[S_F_SCALE] = 0.0;
  scal[S_COMP_LIM] = -INFINITY;
  scal[S_SHEAR_LIM] = INFINITY;
  std::vector<Work> tiles;
  for (int ty = 0; ty < nty; ++ty)
    for (int tx = 0; tx < ntx; ++tx) tiles.push_back({0, tx * kHvTX, ty * kHvTY, (int)tiles.size()});
  std::vector<Work> tiles32;
  for (int ty = 0; ty < nty32; ++ty)
    for (int tx = 0; tx < ntx32; ++tx) tiles32.push_back({0, tx * kSenTX, ty * kSenTY, (int)tiles32.size()});
  std::vector<Work> xl, yl;
  for (int r = 0; r < ny; r += p->Rx) xl.push_back({0, r, std::min(p->Rx, ny - r), 0});
  for (int c = 0; c < nx; c += p->Ry) yl.push_back({0, c, std::min(p->Ry, nx - c), 0});
  std::vector<Work> yl2;
  for (int c = 0; c < nx; c += p->Ry2) yl2.push_back({0, c, std::min(p->Ry2, nx - c), 0});
  std::vector<Work> sr;
  for (int r = 0; r < ny; r += srows) sr.push_back({0, 0, r, (int)sr.size()});

#define HB_PUT(dst, src, bytes)                                                  \
  do {                                                                           \
    e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);                     \
    if (e != cudaSuccess) {                                                      \
      block_free(p->arena_block);                                                \
      delete p;                                                                  \
      return cuda_fail(e, "cudaMemcpy(plan tables)");                            \
    }                                                                            \
  } while (0)
  HB_PUT(s.twx, tw.data(), tw.size() * sizeof(double2));
  HB_PUT(s.modes, modes.data(), modes.size() * sizeof(int2));
  HB_PUT(s.kvec, kvec.data(), kvec.size() * sizeof(double2));
  HB_PUT(p->d_partner, mt.partner.data(), kMaxForce * sizeof(int));
  HB_PUT(s.scal, scal.data(), SCAL_SIZE * sizeof(double));
  HB_PUT(p->d_tiles, tiles.data(), tiles.size() * sizeof(Work));
  HB_PUT(p->d_tiles32, tiles32.data(), tiles32.size() * sizeof(Work));
  HB_PUT(p->d_xlines, xl.data(), xl.size() * sizeof(Work));
  HB_PUT(p->d_ylines, yl.data(), yl.size() * sizeof(Work));
  HB_PUT(p->d_ylines2, yl2.data(), yl2.size() * sizeof(Work));
  HB_PUT(p->d_srows, sr.data(), sr.size() * sizeof(Work));
  HB_PUT(p->d_solve, &s, sizeof(SolveDev));
#undef HB_PUT
  e = cudaMemset(s.counters, 0, 8 * sizeof(unsigned) + sizeof(int));
  if (e != cudaSuccess) {
    block_free(p->arena_block);
    delete p;
    return cuda_fail(e, "cudaMemset(counters)");
  }
  prime_attributes(p->elem, mch_for(nx), mch_for(ny), p->smem_x, std::max(p->smem_y, p->smem_y2), p->smem_sensor, p->sensor_w,
                   p->smem_sensor_step);
  {
    // the fused sensor needs every tile's CTA resident at once (grid barrier)
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t oe = p->elem == 4
        ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sensor_kernel<float, false, true>,
                                                        kSensorThreads, p->smem_sensor)
        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sensor_kernel<double, false, true>,
                                                        kSensorThreads, p->smem_sensor);
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    p->fuse_ok = oe == cudaSuccess && coop && (long)per_sm * sms >= p->n_tiles32;
    cudaGetLastError();
  }
  {
    // powers of the compact-solve root for the non-periodic end corrections
    double tab[kPowTab];
    for (int k = 0; k < kPowTab; ++k) tab[k] = std::pow(kRhoSolve, (double)k);
    const cudaError_t e = cudaMemcpyToSymbol(g_rho_pow, tab, sizeof(tab));
    if (e != cudaSuccess) {
      hitb200_plan_destroy(p);
      return cuda_fail(e, "cudaMemcpyToSymbol(rho powers)");
    }
  }
  *out = p;
  return HITB200_OK;
}

int hitb200_plan_destroy(hitb200_plan* p) {
  if (!p) return HITB200_OK;
  if (p->graph) cudaGraphExecDestroy(p->graph);
  if (p->arena_block.ptr) {
    // queued launches of this plan may still use the arena
    sync_block_device(p->arena_block);
    block_free(p->arena_block);
  }
  delete p;
  return HITB200_OK;
}

// ---- bind the caller's state pointer into the device descriptor ------------------
static int bind_state(hitb200_plan* p, double* q, cudaStream_t st) {
  if (p->hs.q == q) return HITB200_OK;
  p->hs.q = q;
  HB_CUDA(cudaMemcpyAsync(&p->d_solve->q, &p->hs.q, sizeof(double*), cudaMemcpyHostToDevice, st));
  HB_CUDA(cudaStreamSynchronize(st));
  return HITB200_OK;
}

int hitb200_enforce(hitb200_plan* p, const double* q, double* out, void* stream) {
  if (!p || !q || !out) return invalid("NULL argument");
  const size_t plane = (size_t)p->desc.nx * p->desc.ny;
  enforce_kernel<<<(int)std::min<size_t>((plane + 255) / 256, 4096), 256, 0, (cudaStream_t)stream>>>(
      q, out, plane, p->desc.gamma);
  HB_LAUNCHED("enforce_kernel");
  return HITB200_OK;
}

int hitb200_enforce_state(const double* q, double* out, int64_t ncells, double gamma, void* stream) {
  if (!q || !out) return invalid("NULL argument");
  if (ncells <= 0) return invalid("ncells must be positive");
  enforce_kernel<<<(int)std::min<int64_t>((ncells + 255) / 256, 4096), 256, 0, (cudaStream_t)stream>>>(
      q, out, (size_t)ncells, gamma);
  HB_LAUNCHED("enforce_kernel");
  return HITB200_OK;
}

int hitb200_sensor(hitb200_plan* p, const double* q, uint8_t* mask, int enforce_first, void* stream) {
  if (!p || !q || !mask) return invalid("NULL argument");
  LaunchSet L = plan_launch_set(p, (cudaStream_t)stream);
  Bind b{};
  b.use = 1;
  b.qin = q;
  launch_prepass(L, 0, PRE_SENSOR, enforce_first, b);
  launch_sensor(L, 0, enforce_first, 0, b, mask);
  HB_LAUNCHED("sensor");
  return HITB200_OK;
}

int hitb200_axis_derivative(hitb200_plan* p, const double* q, const uint8_t* mask, int axis,
                            double* out, void* stream) {
  if (!p || !q || !mask || !out) return invalid("NULL argument");
  if (axis != 0 && axis != 1) return invalid("axis must be 0 (x) or 1 (y)");
  LaunchSet L = plan_launch_set(p, (cudaStream_t)stream);
  Bind b{};
  b.use = 1;
  b.qin = q;
  b.mask = mask;
  b.out = out;
  launch_prepass(L, 0, PRE_STAGE, 1, b);
  launch_sweep(L, axis, 0, SW_DERIV, b);
  HB_LAUNCHED("axis_derivative");
  return HITB200_OK;
}

int hitb200_rhs(hitb200_plan* p, const double* q, int terms, const double* fx, const double* fy,
                double* out, void* stream) {
  if (!p || !q || !out) return invalid("NULL argument");
  if ((terms & HITB200_TERM_FORCING) && (!fx || !fy)) return invalid("forcing term needs fx and fy");
  if ((terms & ~HITB200_TERM_ALL) != 0) return invalid("unknown rhs term bits");
  if ((terms & HITB200_TERM_VISCOUS) && p->desc.viscosity > 0.0 && !p->hs.vis)
    return invalid("plan has no viscous buffer");
  LaunchSet L = plan_launch_set(p, (cudaStream_t)stream);
  Bind b{};
  b.use = 1;
  b.qin = q;
  b.mask = p->hs.mask;
  b.out = out;
  b.fx = fx;
  b.fy = fy;
  b.terms = terms;
  launch_prepass(L, 0, PRE_STAGE, 1, b);
  launch_sensor(L, 0, 1, (terms & HITB200_TERM_VISCOUS) ? 1 : 0, b, p->hs.mask);
  launch_sweep(L, 1, 0, SW_RHS, b);
  launch_sweep(L, 0, 0, SW_RHS, b);
  HB_LAUNCHED("rhs");
  return HITB200_OK;
}

int hitb200_viscous_rhs(hitb200_plan* p, const double* q, double* out, void* stream) {
  if (!p || !q || !out) return invalid("NULL argument");
  const size_t plane = (size_t)p->desc.nx * p->desc.ny;
  if (p->desc.viscosity == 0.0) {
    HB_CUDA(cudaMemsetAsync(out, 0, 4 * plane * sizeof(double), (cudaStream_t)stream));
    return HITB200_OK;
  }
  LaunchSet L = plan_launch_set(p, (cudaStream_t)stream);
  Bind b{};
  b.use = 1;
  b.qin = q;
  launch_prepass(L, 0, PRE_SENSOR, 0, b);
  launch_sensor(L, 0, 0, 1, b, p->hs.mask);
  const int nb = (int)std::min<size_t>((plane + 255) / 256, 4096);
  if (p->elem == 4)
    vis_copy_kernel<float><<<nb, 256, 0, (cudaStream_t)stream>>>((const float*)p->hs.vis, out, plane);
  else
    vis_copy_kernel<double><<<nb, 256, 0, (cudaStream_t)stream>>>((const double*)p->hs.vis, out, plane);
  HB_LAUNCHED("viscous_rhs");
  return HITB200_OK;
}

int hitb200_hyperviscosity(hitb200_plan* p, const double* q, const uint8_t* active, double* out,
                           void* stream) {
  if (!p || !q || !out) return invalid("NULL argument");
  if (!active) return invalid("active_mask is required: hyperviscosity may only be applied on compact-FD nodes");
  if (q == out) return invalid("hyperviscosity output must not alias its input");
  LaunchSet L = plan_launch_set(p, (cudaStream_t)stream);
  Bind b{};
  b.use = 1;
  b.qin = q;
  b.qout = out;
  b.mask = active;
  b.invert_mask = 0;
  launch_hv(L, b);
  HB_LAUNCHED("hyperviscosity");
  return HITB200_OK;
}

int hitb200_outflow_guard(hitb200_plan* p, double* q, void* stream) {
  if (!p || !q) return invalid("NULL argument");
  Bind b{};
  b.use = 1;
  b.qout = q;
  guard_kernel<<<dim3(guard_blocks_for(p->desc), 1), 256, 0, (cudaStream_t)stream>>>(p->d_solve, 1, 0, b);
  HB_LAUNCHED("guard_kernel");
  return HITB200_OK;
}

int hitb200_stable_time_step(hitb200_plan* p, const double* q, double cfl, double remaining,
                             double* dt_out) {
  if (!p || !q || !dt_out) return invalid("NULL argument");
  LaunchSet L = plan_launch_set(p, 0);
  Bind b{};
  b.use = 1;
  b.qin = q;
  launch_prepass(L, 0, PRE_CHECK, 0, b);
  HB_LAUNCHED("prepass");
  double sr = 0.0;
  HB_CUDA(cudaMemcpy(&sr, p->hs.scal + S_DT, sizeof(double), cudaMemcpyDeviceToHost));
  double dt = cfl / sr;
  if (!std::isnan(remaining)) dt = std::min(dt, remaining);
  *dt_out = dt;
  return HITB200_OK;
}

int hitb200_validate(hitb200_plan* p, const double* q) {
  if (!p || !q) return invalid("NULL argument");
  LaunchSet L = plan_launch_set(p, 0);
  Bind b{};
  b.use = 1;
  b.qin = q;
  double zero = 0.0;
  HB_CUDA(cudaMemcpy(p->hs.scal + S_STATUS, &zero, sizeof(double), cudaMemcpyHostToDevice));
  launch_prepass(L, 0, PRE_CHECK, 0, b);
  HB_LAUNCHED("prepass");
  double stv = 0.0;
  HB_CUDA(cudaMemcpy(&stv, p->hs.scal + S_STATUS, sizeof(double), cudaMemcpyDeviceToHost));
  const int bits = (int)stv;
  if (bits & ST_NONFINITE) return HITB200_ERR_NONFINITE;
  if (bits & (ST_NONPOS_RHO | ST_NONPOS_P)) return HITB200_ERR_NONPOSITIVE;
  return HITB200_OK;
}

int hitb200_forcing_update(hitb200_plan* p, const double* q, const double* noise, double dt,
                           double target_power, double* fx, double* fy, void* stream) {
  if (!p || !q || !fx || !fy) return invalid("NULL argument");
  if (!p->desc.forcing_on) return invalid("plan has no forcing");
  if (!(dt > 0.0)) return invalid("forcing update requires dt > 0");
  if (!noise && p->desc.noise_mode == 0) return invalid("noise field required (noise_mode 0)");
  cudaStream_t st = (cudaStream_t)stream;
  const double decay = std::exp(-dt / p->desc.forcing_correlation_time);
  const double vals[3] = {decay, std::sqrt(std::max(1.0 - decay * decay, 0.0)), target_power};
  HB_CUDA(cudaMemcpyAsync(p->hs.scal + S_F_DECAY, &vals[0], sizeof(double), cudaMemcpyHostToDevice, st));
  HB_CUDA(cudaMemcpyAsync(p->hs.scal + S_XI_SCALE, &vals[1], sizeof(double), cudaMemcpyHostToDevice, st));
  HB_CUDA(cudaMemcpyAsync(p->hs.scal + S_POWER, &vals[2], sizeof(double), cudaMemcpyHostToDevice, st));
  LaunchSet L = plan_launch_set(p, st);
  Bind b{};
  b.use = 1;
  if (noise) {
    b.qin = noise;
    noise_dft_kernel<<<L.n_tiles32, kRedThreads, 0, st>>>(L.solves, L.tiles32, b);
  } else {
    noise_rng_kernel<<<1, 128, 0, st>>>(L.solves, 1, L.partner);
  }
  Bind b2{};
  b2.use = 1;
  b2.qin = q;
  force_synth_kernel<<<L.n_srows, kRedThreads, 0, st>>>(L.solves, L.srows, b2);
  const size_t plane = (size_t)p->desc.nx * p->desc.ny;
  const int nb = (int)std::min<size_t>((plane + 255) / 256, 4096);
  if (p->elem == 4) {
    scale_copy_kernel<<<nb, 256, 0, st>>>((const float*)p->hs.fx, fx, p->hs.scal, S_F_SCALE, plane);
    scale_copy_kernel<<<nb, 256, 0, st>>>((const float*)p->hs.fy, fy, p->hs.scal, S_F_SCALE, plane);
  } else {
    scale_copy_kernel<<<nb, 256, 0, st>>>((const double*)p->hs.fx, fx, p->hs.scal, S_F_SCALE, plane);
    scale_copy_kernel<<<nb, 256, 0, st>>>((const double*)p->hs.fy, fy, p->hs.scal, S_F_SCALE, plane);
  }
  HB_LAUNCHED("forcing_update");
  HB_CUDA(cudaStreamSynchronize(st));  // host-side scalars above live on this stack frame
  return HITB200_OK;
}

int hitb200_step(hitb200_plan* p, double* q, const double* noise, void* stream) {
  if (!p || !q) return invalid("NULL argument");
  if (p->in_batch) return invalid("plan belongs to a batch; use hitb200_batch_step");
  cudaStream_t st = (cudaStream_t)stream;
  const int upload = p->desc.forcing_on && p->desc.noise_mode == 0;
  if (upload && !noise) return invalid("noise field required (noise_mode 0)");
  int r = bind_state(p, q, st);
  if (r != HITB200_OK) return r;
  if (upload)
    HB_CUDA(cudaMemcpyAsync((void*)p->hs.noise, noise, (size_t)p->desc.nx * p->desc.ny * sizeof(double),
                            cudaMemcpyDefault, st));
  LaunchSet L = plan_launch_set(p, st);
  L.pdl = 1;  // one solve's launches are single waves: the next kernel's CTAs
              // stage their inputs while the previous kernel finishes
  return launch_step_sequence(L, p->desc.forcing_on, upload, !p->desc.periodic, p->hs.hv_interval > 0);
}

int hitb200_run(hitb200_plan* p, double* q, int32_t nsteps, void* stream) {
  if (!p || !q) return invalid("NULL argument");
  if (p->in_batch) return invalid("plan belongs to a batch; use hitb200_batch_run");
  if (nsteps < 0) return invalid("nsteps must be >= 0");
  if (p->desc.forcing_on && p->desc.noise_mode == 0)
    return invalid("hitb200_run needs noise_mode 1 or 2 (device noise) when forcing is on");
  cudaStream_t st = (cudaStream_t)stream;
  int r = bind_state(p, q, st);
  if (r != HITB200_OK) return r;
  if (!p->graph || p->graph_stream != st) {
    if (p->graph) cudaGraphExecDestroy(p->graph);
    p->graph = nullptr;
    LaunchSet L = plan_launch_set(p, nullptr);
    L.pdl = 1;  // one solve's launches are single waves: the next kernel's CTAs
                // stage their inputs while the previous kernel finishes
    r = capture_graph(1, [&](cudaStream_t* cs) {
      L.st = cs[0];
      return launch_step_sequence(L, p->desc.forcing_on, 0, !p->desc.periodic, p->hs.hv_interval > 0);
    }, &p->graph);
    if (r != HITB200_OK) return r;
    p->graph_stream = st;
  }
  for (int i = 0; i < nsteps; ++i) HB_CUDA(cudaGraphLaunch(p->graph, st));
  return HITB200_OK;
}

int hitb200_set_time(hitb200_plan* p, double time, int64_t step, double dt, int64_t max_steps) {
  if (!p) return invalid("NULL argument");
  double v[4] = {dt, time, (double)step, 1.0};
  double ms = max_steps < 0 ? -1.0 : (double)max_steps;
  HB_CUDA(cudaMemcpy(p->hs.scal + S_DT, v, 4 * sizeof(double), cudaMemcpyHostToDevice));
  HB_CUDA(cudaMemcpy(p->hs.scal + S_MAX_STEPS, &ms, sizeof(double), cudaMemcpyHostToDevice));
  return HITB200_OK;
}

int hitb200_read_scalars(hitb200_plan* p, double* out, int32_t n) {
  if (!p || !out) return invalid("NULL argument");
  if (n < 0 || n > HITB200_S_COUNT) return invalid("n out of range");
  HB_CUDA(cudaDeviceSynchronize());
  HB_CUDA(cudaMemcpy(out, p->hs.scal, n * sizeof(double), cudaMemcpyDeviceToHost));
  int near = 0;
  HB_CUDA(cudaMemcpy(&near, p->hs.near_count, sizeof(int), cudaMemcpyDeviceToHost));
  if (n > HITB200_S_NEAR_THRESHOLD) out[HITB200_S_NEAR_THRESHOLD] = near;
  return HITB200_OK;
}

int hitb200_copy_scalars_async(hitb200_plan* p, double* dst, int32_t n, void* stream) {
  if (!p || !dst) return invalid("NULL argument");
  if (n < 0 || n > HITB200_S_COUNT) return invalid("n out of range");
  HB_CUDA(cudaMemcpyAsync(dst, p->hs.scal, n * sizeof(double), cudaMemcpyDefault, (cudaStream_t)stream));
  return HITB200_OK;
}

size_t hitb200_state_block_size(void) { return (size_t)SCAL_SIZE; }

int hitb200_set_noise_stream(hitb200_plan* p, const uint64_t* stream_state) {
  if (!p || !stream_state) return invalid("NULL argument");
  if (!p->has_gen) return invalid("the plan has no device noise stream (noise_mode 2 with forcing)");
  double v[4];
  static_assert(sizeof(double) == sizeof(uint64_t), "64-bit slots");
  std::memcpy(v, stream_state, sizeof(v));
  HB_CUDA(cudaDeviceSynchronize());
  HB_CUDA(cudaMemcpy(p->hs.scal + S_PCG, v, sizeof(v), cudaMemcpyHostToDevice));
  return HITB200_OK;
}

int hitb200_noise_field(hitb200_plan* p, double* out, void* stream) {
  if (!p || !out) return invalid("NULL argument");
  if (!p->has_gen) return invalid("the plan has no device noise stream (noise_mode 2 with forcing)");
  if (p->in_batch) return invalid("plan belongs to a batch");
  LaunchSet L = plan_launch_set(p, (cudaStream_t)stream);
  L.gen_out = out;
  launch_noise_gen(L);
  HB_LAUNCHED("noise stream");
  return HITB200_OK;
}

int hitb200_get_noise_stream(hitb200_plan* p, uint64_t* stream_state) {
  if (!p || !stream_state) return invalid("NULL argument");
  if (!p->has_gen) return invalid("the plan has no device noise stream (noise_mode 2 with forcing)");
  double v[4];
  HB_CUDA(cudaDeviceSynchronize());
  HB_CUDA(cudaMemcpy(v, p->hs.scal + S_PCG, sizeof(v), cudaMemcpyDeviceToHost));
  std::memcpy(stream_state, v, sizeof(v));
  return HITB200_OK;
}

int hitb200_save_state_block(hitb200_plan* p, double* out, size_t n) {
  if (!p || !out) return invalid("NULL argument");
  if (n != (size_t)SCAL_SIZE) return invalid("the state block holds hitb200_state_block_size() doubles");
  HB_CUDA(cudaDeviceSynchronize());
  HB_CUDA(cudaMemcpy(out, p->hs.scal, n * sizeof(double), cudaMemcpyDeviceToHost));
  return HITB200_OK;
}

int hitb200_load_state_block(hitb200_plan* p, const double* in, size_t n) {
  if (!p || !in) return invalid("NULL argument");
  if (n != (size_t)SCAL_SIZE) return invalid("the state block holds hitb200_state_block_size() doubles");
  HB_CUDA(cudaDeviceSynchronize());
  HB_CUDA(cudaMemcpy(p->hs.scal, in, n * sizeof(double), cudaMemcpyHostToDevice));
  return HITB200_OK;
}

int hitb200_set_barrier_test(int32_t extra_arrivals, double limit_seconds) {
  if (extra_arrivals < 0 || extra_arrivals > 1) return invalid("extra_arrivals must be 0 or 1");
  if (!(limit_seconds > 0.0) || limit_seconds > 10.0) return invalid("limit_seconds must be in (0, 10]");
  const unsigned extra = (unsigned)extra_arrivals;
  const unsigned long long ns = (unsigned long long)(limit_seconds * 1e9);
  HB_CUDA(cudaDeviceSynchronize());
  HB_CUDA(cudaMemcpyToSymbol(g_barrier_extra, &extra, sizeof(extra)));
  HB_CUDA(cudaMemcpyToSymbol(g_barrier_limit_ns, &ns, sizeof(ns)));
  return HITB200_OK;
}

int hitb200_diagnostics(hitb200_plan* p, const double* q, double* out, int32_t n) {
  if (!p || !q || !out) return invalid("NULL argument");
  LaunchSet L = plan_launch_set(p, 0);
  Bind b{};
  b.use = 1;
  b.qin = q;
  diag_kernel<<<L.n_tiles32, kRedThreads, 0, 0>>>(L.solves, L.tiles32, b);
  HB_LAUNCHED("diag_kernel");
  double raw[NDIAG];
  HB_CUDA(cudaMemcpy(raw, p->hs.diag_out, sizeof(raw), cudaMemcpyDeviceToHost));
  const double N = (double)p->desc.nx * p->desc.ny;
  const double area = (p->desc.x_max - p->desc.x_min) * (p->desc.y_max - p->desc.y_min);
  const double mr = raw[D_RHO] / N, mu = raw[D_U] / N, mv = raw[D_V] / N;
  // fluctuation moments mean(rho (u - <u>)^2) etc. from raw sums
  const double uu = raw[D_RUU] / N - 2.0 * mu * raw[D_RU] / N + mu * mu * mr;
  const double vv = raw[D_RVV] / N - 2.0 * mv * raw[D_RV] / N + mv * mv * mr;
  const double uv = raw[D_RUV] / N - mu * raw[D_RV] / N - mv * raw[D_RU] / N + mu * mv * mr;
  const double sum = uu + vv, cov = std::sqrt(std::max(uu * vv, 0.0));
  const double vals[17] = {0.5 * sum,
                           0.5 * uu,
                           0.5 * vv,
                           sum > 0.0 ? std::fabs(uu - vv) / sum : 0.0,
                           cov > 0.0 ? uv / cov : 0.0,
                           std::sqrt(raw[D_VEL2] / N),
                           std::sqrt(raw[D_VEL2] / N) / (raw[D_C] / N),
                           mr,
                           raw[D_P] / N,
                           mr * area,
                           raw[D_Q1] / N * area,
                           raw[D_Q2] / N * area,
                           raw[D_Q3] / N * area,
                           raw[D_RHOMIN],
                           raw[D_RHOMAX],
                           raw[D_PMIN],
                           raw[D_PMAX]};
  for (int i = 0; i < n && i < 17; ++i) out[i] = vals[i];
  return HITB200_OK;
}

// ---- batched form ---------------------------------------------------------------------
// Work lists, descriptor table and launch shape of a batch over b->plans.
static int batch_build(hitb200_batch* b) {
  std::vector<SolveDev> hs;
  std::vector<Work> tiles, tiles32, xl, yl, sr;
  std::vector<int> partner;
  const int n = (int)b->plans.size();
  // y panels of 4 columns (full 32-byte row segments of the FP64 state)
  // when the batch has enough columns for several waves of such CTAs and
  // every member's panel fits in shared memory; else each plan's own width
  int ry4 = 1;
  {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long cols = 0;
    for (hitb200_plan* p : b->plans) {
      cols += (p->desc.nx + 3) / 4;
      const size_t by = p->elem == 4 ? SweepLayout<float>(p->desc.ny, 4).bytes()
                                     : SweepLayout<double>(p->desc.ny, 4).bytes();
      if (by > 110 * 1024 || p->desc.nx < 4) ry4 = 0;
    }
    if (cols < 4L * sms) ry4 = 0;
  }
  // the other panel width: each plan's own where the default is 4, else 4
  // where every member's 4-column panel fits
  bool has_y2 = true;
  if (!ry4)
    for (hitb200_plan* p : b->plans) {
      const size_t by = p->elem == 4 ? SweepLayout<float>(p->desc.ny, 4).bytes()
                                     : SweepLayout<double>(p->desc.ny, 4).bytes();
      if (by > 110 * 1024 || p->desc.nx < 4) has_y2 = false;
    }
  // row chunks of the forcing synthesis per CTA: enough CTAs for about four
  // per SM, at most 8 chunks each (a chunk alone is a short CTA whose fixed
  // costs, barriers and the ticket, dominate)
  int synth_group = 1;
  {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long chunks = 0;
    for (hitb200_plan* p : b->plans) chunks += (p->desc.ny + synth_rows(p->desc.nx) - 1) / synth_rows(p->desc.nx);
    synth_group = (int)std::max(1L, std::min(8L, chunks / (4L * sms)));
  }
  std::vector<Work> yl2;
  b->off_yl2.clear();
  b->ry_max2 = 1;
  b->smem_y2 = 0;
  auto mark = [&]() {
    b->off_tiles.push_back((int)tiles.size());
    b->off_tiles32.push_back((int)tiles32.size());
    b->off_xl.push_back((int)xl.size());
    b->off_yl.push_back((int)yl.size());
    b->off_srows.push_back((int)sr.size());
  };
  b->off_tiles.clear(); b->off_tiles32.clear(); b->off_xl.clear(); b->off_yl.clear(); b->off_srows.clear();
  for (int i = 0; i < n; ++i) {
    mark();
    hitb200_plan* p = b->plans[i];
    hs.push_back(p->hs);
    const int ntx = (p->desc.nx + kHvTX - 1) / kHvTX, nty = (p->desc.ny + kHvTY - 1) / kHvTY;
    int k = 0;
    for (int ty = 0; ty < nty; ++ty)
      for (int tx = 0; tx < ntx; ++tx) tiles.push_back({i, tx * kHvTX, ty * kHvTY, k++});
    const int ntx32 = (p->desc.nx + kSenTX - 1) / kSenTX, nty32 = (p->desc.ny + kSenTY - 1) / kSenTY;
    int k32 = 0;
    for (int ty = 0; ty < nty32; ++ty)
      for (int tx = 0; tx < ntx32; ++tx) tiles32.push_back({i, tx * kSenTX, ty * kSenTY, k32++});
    b->guard_blocks = std::max(b->guard_blocks, guard_blocks_for(p->desc));
    for (int r0 = 0; r0 < p->desc.ny; r0 += p->Rx) xl.push_back({i, r0, std::min(p->Rx, p->desc.ny - r0), 0});
    const int ry = ry4 ? 4 : p->Ry;
    for (int c0 = 0; c0 < p->desc.nx; c0 += ry) yl.push_back({i, c0, std::min(ry, p->desc.nx - c0), 0});
    b->off_yl2.push_back((int)yl2.size());
    if (has_y2) {
      const int ry2 = ry4 ? p->Ry : 4;
      for (int c0 = 0; c0 < p->desc.nx; c0 += ry2) yl2.push_back({i, c0, std::min(ry2, p->desc.nx - c0), 0});
      b->ry_max2 = std::max(b->ry_max2, ry2);
      b->smem_y2 = std::max(b->smem_y2, p->elem == 4 ? SweepLayout<float>(p->desc.ny, ry2).bytes()
                                                       : SweepLayout<double>(p->desc.ny, ry2).bytes());
    }
    // forcing synthesis: synth_group consecutive row chunks per CTA (each
    // with its own partial row, so the grouping changes no result)
    const int srows = synth_rows(p->desc.nx);
    const int nchk = (p->desc.ny + srows - 1) / srows;
    for (int k0 = 0; k0 < nchk; k0 += synth_group)
      sr.push_back({i, std::min(synth_group, nchk - k0), k0 * srows, k0});
    ModeTables mt = build_modes(p->desc);
    partner.insert(partner.end(), mt.partner.begin(), mt.partner.end());
    b->elem = p->elem;
    b->mch_x = std::max(b->mch_x, mch_for(p->desc.nx));
    b->mch_y = std::max(b->mch_y, mch_for(p->desc.ny));
    b->rx_max = std::max(b->rx_max, p->Rx);
    b->ry_max = std::max(b->ry_max, ry);
    b->smem_x = std::max(b->smem_x, p->smem_x);
    b->smem_y = std::max(b->smem_y, ry4 ? (p->elem == 4 ? SweepLayout<float>(p->desc.ny, 4).bytes()
                                                         : SweepLayout<double>(p->desc.ny, 4).bytes())
                                         : p->smem_y);
    b->smem_sensor = std::max(b->smem_sensor, p->smem_sensor);
    b->sensor_w = i == 0 ? p->sensor_w : (b->sensor_w == p->sensor_w ? b->sensor_w : -1);
    b->smem_sensor_step = std::max(b->smem_sensor_step, p->smem_sensor_step);
    b->any_outflow |= !p->desc.periodic;
    b->any_forcing |= p->desc.forcing_on;
    b->any_hv |= p->hs.hv_interval > 0;
    b->any_noise_upload |= (p->desc.forcing_on && p->desc.noise_mode != 1);
  }
  mark();
  b->off_yl2.push_back((int)yl2.size());
  // The members in two groups (contiguous, balanced by cells) for the two
  // branches of hitb200_batch_run's graph.
  b->cut = n;
  if (n > 1) {
    double tot = 0.0, acc = 0.0;
    for (hitb200_plan* p : b->plans) tot += (double)p->desc.nx * p->desc.ny;
    for (b->cut = 1; b->cut < n - 1; ++b->cut) {
      acc += (double)b->plans[b->cut - 1]->desc.nx * b->plans[b->cut - 1]->desc.ny;
      if (acc >= 0.5 * tot) break;
    }
  }
  // Persistent stage launches: FP32-bulk members with a shared step-sensor
  // width and lines of at most 512 nodes (4 nodes per sweep thread).  Their
  // sweep items are 4-row x groups and 4-column y panels of 512 threads;
  // each launch group's queue holds its members' prepass tile pairs, sensor
  // tiles, y panels and x groups, phase after phase.
  std::vector<Work> xl4, yl4;
  std::vector<QItem> qi;
  {
    int maxn = 0;
    for (hitb200_plan* p : b->plans) maxn = std::max(maxn, std::max(p->desc.nx, p->desc.ny));
    b->can_persist = b->elem == 4 && b->sensor_w == 4 && maxn <= 512 && b->mch_x == b->mch_y;
    // one nodes-per-thread class: the stage kernel's sweeps run with one
    for (hitb200_plan* p : b->plans)
      if (mch_for(p->desc.nx) != b->mch_x || mch_for(p->desc.ny) != b->mch_y) b->can_persist = false;
  }
  if (b->can_persist) {
    std::vector<int> ox{0}, oy{0};
    size_t sm = std::max(stage_pre_smem_bytes<float>(), (size_t)(kPreThreads + R_FIXED + 4 * kMaxDrag) * 8);
    size_t xs = 0;
    for (int i = 0; i < n; ++i) {
      const hitb200_desc& d = b->plans[i]->desc;
      for (int r0 = 0; r0 < d.ny; r0 += kStageLines) xl4.push_back({i, r0, std::min(kStageLines, d.ny - r0), 0});
      for (int c0 = 0; c0 < d.nx; c0 += kStageLines) yl4.push_back({i, c0, std::min(kStageLines, d.nx - c0), 0});
      ox.push_back((int)xl4.size());
      oy.push_back((int)yl4.size());
      xs = std::max(xs, SweepLayout<float>(d.nx, 1).bytes());
      sm = std::max(sm, SweepLayout<float>(d.ny, kStageLines).bytes());
    }
    b->stage_xstride = (xs + 15) & ~(size_t)15;
    sm = std::max(sm, kStageLines * b->stage_xstride);
    b->stage_sh_off = (std::max(sm, b->smem_sensor_step) + 15) & ~(size_t)15;
    b->smem_stage = b->stage_sh_off + kStageLines * sizeof(StageSweepShared<float>);
    auto group = [&](int g, int g0, int g1) {
      b->q_off[g] = (int)qi.size();
      for (int i = g0; i < g1; ++i) {
        const int t0 = b->off_tiles32[i], nt = b->off_tiles32[i + 1] - t0;
        for (int k = 0; k < nt; k += 2) qi.push_back({Q_PRE, t0 + k, std::min(2, nt - k), 0, 0});
      }
      b->q_npre[g] = (int)qi.size() - b->q_off[g];
      for (int i = g0; i < g1; ++i) {
        const int t0 = b->off_tiles32[i], nt = b->off_tiles32[i + 1] - t0;
        for (int k = 0; k < nt; ++k) qi.push_back({Q_SEN, t0 + k, 1, 1, 0});
      }
      for (int i = g0; i < g1; ++i) {
        const int nt = b->off_tiles32[i + 1] - b->off_tiles32[i];
        for (int k = oy[i]; k < oy[i + 1]; ++k) qi.push_back({Q_SWY, k, 1, nt, 0});
      }
      for (int i = g0; i < g1; ++i) {
        const int nt = b->off_tiles32[i + 1] - b->off_tiles32[i];
        for (int k = ox[i]; k < ox[i + 1]; ++k) qi.push_back({Q_SWX, k, 1, oy[i + 1] - oy[i], nt});
      }
    };
    group(0, 0, n);
    group(1, 0, b->cut);
    group(2, b->cut, n);
    b->q_off[3] = (int)qi.size();
  }
  b->has_y2 = has_y2;
  std::vector<Work> sw;  // the sweep lists in segments
  for (int g = 0; g < 3; ++g) {
    const int g0 = g == 2 ? b->cut : 0, g1 = g == 1 ? b->cut : n;
    for (int li = 0; li < 3; ++li) {
      const std::vector<Work>& src = li == 0 ? xl : (li == 1 ? yl : yl2);
      const std::vector<int>& off = li == 0 ? b->off_xl : (li == 1 ? b->off_yl : b->off_yl2);
      for (int c = 0; c < 4; ++c) {
        hitb200_batch::SegRec& r = b->segs[g][li][c];
        r.off = (int)sw.size();
        r.smem = 0;
        if (li < 2 || has_y2)
          for (int i = g0; i < g1; ++i) {
            const hitb200_plan* p = b->plans[i];
            if (mch_for(li == 0 ? p->desc.nx : p->desc.ny) != (1 << c)) continue;
            sw.insert(sw.end(), src.begin() + off[i], src.begin() + off[i + 1]);
            size_t by = p->smem_x;
            if (li > 0) {
              const int ry = li == 1 ? (ry4 ? 4 : p->Ry) : (ry4 ? p->Ry : 4);
              by = p->elem == 4 ? SweepLayout<float>(p->desc.ny, ry).bytes()
                                : SweepLayout<double>(p->desc.ny, ry).bytes();
            }
            r.smem = std::max(r.smem, by);
          }
        r.n = (int)sw.size() - r.off;
      }
    }
  }
  b->n_y2 = (int)yl2.size();
  if (b->any_noise_upload) return invalid("batched solves draw forcing noise with the device RNG (noise_mode 1)");
  b->n_tiles = (int)tiles.size();
  b->n_tiles32 = (int)tiles32.size();
  b->n_x = (int)xl.size();
  b->n_y = (int)yl.size();
  b->n_srows = (int)sr.size();
  default_tuning(b->n_x, b->n_y, b->n_tiles32, b->tuning);
  const std::vector<QCtl> qctl0(3, QCtl{0u, 0u, 0u, 0u});
  const std::vector<unsigned> qdep0(b->can_persist ? 4 * (size_t)n : 0, 0u);
  size_t bytes = hs.size() * sizeof(SolveDev) +
                 (tiles.size() + tiles32.size() + xl.size() + yl.size() + yl2.size() + sr.size() + xl4.size() +
                  yl4.size()) * sizeof(Work) +
                 partner.size() * sizeof(int) + qi.size() * sizeof(QItem) + qctl0.size() * sizeof(QCtl) +
                 qdep0.size() * sizeof(unsigned) + sw.size() * sizeof(Work) + 1024 + 14 * 256;
  cudaError_t e = block_alloc(bytes, &b->tables);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(batch tables)");
  unsigned char* buf = static_cast<unsigned char*>(b->tables.ptr);
  size_t off = 0;
  cudaError_t ce = cudaSuccess;
  auto put = [&](const void* src, size_t nbytes) -> unsigned char* {
    unsigned char* d = buf + off;
    off += (nbytes + 255) & ~(size_t)255;
    if (nbytes > 0 && ce == cudaSuccess) ce = cudaMemcpy(d, src, nbytes, cudaMemcpyHostToDevice);
    return d;
  };
  b->d_solves = reinterpret_cast<SolveDev*>(put(hs.data(), hs.size() * sizeof(SolveDev)));
  b->d_tiles = reinterpret_cast<Work*>(put(tiles.data(), tiles.size() * sizeof(Work)));
  b->d_tiles32 = reinterpret_cast<Work*>(put(tiles32.data(), tiles32.size() * sizeof(Work)));
  b->d_xlines = reinterpret_cast<Work*>(put(xl.data(), xl.size() * sizeof(Work)));
  b->d_ylines = reinterpret_cast<Work*>(put(yl.data(), yl.size() * sizeof(Work)));
  b->d_ylines2 = yl2.empty() ? nullptr : reinterpret_cast<Work*>(put(yl2.data(), yl2.size() * sizeof(Work)));
  b->d_srows = reinterpret_cast<Work*>(put(sr.data(), sr.size() * sizeof(Work)));
  b->d_partner = reinterpret_cast<int*>(put(partner.data(), partner.size() * sizeof(int)));
  b->d_segs = reinterpret_cast<Work*>(put(sw.data(), sw.size() * sizeof(Work)));
  if (b->can_persist) {
    b->d_xl4 = reinterpret_cast<Work*>(put(xl4.data(), xl4.size() * sizeof(Work)));
    b->d_yl4 = reinterpret_cast<Work*>(put(yl4.data(), yl4.size() * sizeof(Work)));
    b->d_qitems = reinterpret_cast<QItem*>(put(qi.data(), qi.size() * sizeof(QItem)));
    b->d_qctl = reinterpret_cast<QCtl*>(put(qctl0.data(), qctl0.size() * sizeof(QCtl)));
    b->d_qdep = reinterpret_cast<unsigned*>(put(qdep0.data(), qdep0.size() * sizeof(unsigned)));
  }
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaMemcpy(batch tables)");
  if (b->sensor_w < 0) b->smem_sensor_step = 0;
  prime_attributes(b->elem, b->mch_x, b->mch_y, b->smem_x, std::max(b->smem_y, b->smem_y2), b->smem_sensor, b->sensor_w,
                   b->smem_sensor_step);
  for (int li = 0; li < 3; ++li)
    for (int c = 0; c < 4; ++c)
      if (b->segs[0][li][c].n > 0) prime_sweep_attr(b->elem, li == 0 ? 0 : 1, 1 << c, b->segs[0][li][c].smem);
  if (b->can_persist) {
    // CTAs of a stage launch: as many as are resident at once
    int dev = 0, sms = 148, nb = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const void* fn = stage_fn(b->mch_x);
    set_stage_attr(fn, b->mch_x, b->smem_stage);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kStageThreads, b->smem_stage) != cudaSuccess || nb < 1) {
      cudaGetLastError();
      b->can_persist = false;
    } else {
      b->stage_grid = nb * sms;
    }
  }
  // member plans use the batch's copy of their descriptor while batched
  for (int i = 0; i < n; ++i) {
    b->plans[i]->d_solve = b->d_solves + i;
    b->plans[i]->in_batch = true;
  }
  return HITB200_OK;
}

int hitb200_batch_create(const hitb200_desc* descs, int32_t n, hitb200_batch** out) {
  if (!descs || !out || n <= 0) return invalid("batch needs at least one descriptor");
  *out = nullptr;
  for (int i = 1; i < n; ++i)
    if (descs[i].precision != descs[0].precision) return invalid("batch members must share precision");
  hitb200_batch* b = new hitb200_batch();
  for (int i = 0; i < n; ++i) {
    hitb200_plan* p = nullptr;
    int r = hitb200_plan_create(&descs[i], &p);
    if (r != HITB200_OK) {
      hitb200_batch_destroy(b);
      return r;
    }
    b->plans.push_back(p);
  }
  const int r = batch_build(b);
  if (r != HITB200_OK) {
    hitb200_batch_destroy(b);
    return r;
  }
  *out = b;
  return HITB200_OK;
}

int hitb200_batch_from_plans(hitb200_plan* const* plans, int32_t n, hitb200_batch** out) {
  if (!plans || !out || n <= 0) return invalid("batch needs at least one plan");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (!plans[i]) return invalid("NULL plan");
    if (plans[i]->in_batch) return invalid("plan already belongs to a batch");
    if (plans[i]->desc.precision != plans[0]->desc.precision)
      return invalid("batch members must share precision");
    for (int j = 0; j < i; ++j)
      if (plans[j] == plans[i]) return invalid("plan listed twice");
  }
  hitb200_batch* b = new hitb200_batch();
  b->owns_plans = false;
  b->plans.assign(plans, plans + n);
  const int r = batch_build(b);
  if (r != HITB200_OK) {
    hitb200_batch_destroy(b);
    return r;
  }
  *out = b;
  return HITB200_OK;
}

int hitb200_batch_destroy(hitb200_batch* b) {
  if (!b) return HITB200_OK;
  int status = HITB200_OK;
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->tables.ptr) {
    // the tables may still be read by queued launches of this batch
    const cudaError_t e = sync_block_device(b->tables);
    if (e != cudaSuccess) status = cuda_fail(e, "cudaDeviceSynchronize(batch destroy)");
    block_free(b->tables);
  }
  for (hitb200_plan* p : b->plans) {
    if (b->owns_plans) {
      p->d_solve = nullptr;
      hitb200_plan_destroy(p);
    } else if (p->d_solve != p->own_solve) {
      // hand the plan back with its own descriptor, carrying the state bound meanwhile
      p->d_solve = p->own_solve;
      p->in_batch = false;
      const cudaError_t e = cudaMemcpy(&p->own_solve->q, &p->hs.q, sizeof(double*), cudaMemcpyHostToDevice);
      if (e != cudaSuccess && status == HITB200_OK) status = cuda_fail(e, "cudaMemcpy(plan state)");
    } else {
      p->in_batch = false;
    }
  }
  delete b;
  return status;
}

hitb200_plan* hitb200_batch_plan(hitb200_batch* b, int32_t i) {
  if (!b || i < 0 || i >= (int)b->plans.size()) return nullptr;
  return b->plans[i];
}

int hitb200_batch_bind(hitb200_batch* b, double* const* q) {
  if (!b || !q) return invalid("NULL argument");
  for (size_t i = 0; i < b->plans.size(); ++i) {
    if (!q[i]) return invalid("NULL state pointer");
    b->plans[i]->hs.q = q[i];
    HB_CUDA(cudaMemcpy(&b->d_solves[i].q, &q[i], sizeof(double*), cudaMemcpyHostToDevice));
  }
  return HITB200_OK;
}

static LaunchSet batch_launch_set(hitb200_batch* b, cudaStream_t st);

int hitb200_step_profile(hitb200_plan* p, double* q, const double* noise, float* ms, double* bytes,
                         int32_t cap, int32_t* count, char* names, size_t names_size, void* stream) {
  if (!p || !q) return invalid("NULL argument");
  if (p->in_batch) return invalid("plan belongs to a batch; use hitb200_batch_step_profile");
  cudaStream_t st = (cudaStream_t)stream;
  const int upload = p->desc.forcing_on && p->desc.noise_mode == 0;
  if (upload && !noise) return invalid("noise field required (noise_mode 0)");
  int r = bind_state(p, q, st);
  if (r != HITB200_OK) return r;
  if (upload)
    HB_CUDA(cudaMemcpyAsync((void*)p->hs.noise, noise, (size_t)p->desc.nx * p->desc.ny * sizeof(double),
                            cudaMemcpyDefault, st));
  Prof pr;
  pr.st = st;
  LaunchSet L = plan_launch_set(p, st);
  L.pdl = 1;  // one solve's launches are single waves: the next kernel's CTAs
              // stage their inputs while the previous kernel finishes
  r = launch_step_sequence(L, p->desc.forcing_on, upload, !p->desc.periodic, p->hs.hv_interval > 0, &pr);
  if (r != HITB200_OK) return r;
  return finish_profile(pr, ms, bytes, cap, count, names, names_size);
}

int hitb200_batch_step_profile(hitb200_batch* b, float* ms, double* bytes, int32_t cap,
                               int32_t* count, char* names, size_t names_size, void* stream) {
  if (!b) return invalid("NULL argument");
  for (hitb200_plan* p : b->plans)
    if (!p->hs.q) return invalid("batch state not bound");
  Prof pr;
  pr.st = (cudaStream_t)stream;
  LaunchSet L = batch_launch_set(b, pr.st);
  int r = launch_step_sequence(L, b->any_forcing, 0, b->any_outflow, b->any_hv, &pr);
  if (r != HITB200_OK) return r;
  return finish_profile(pr, ms, bytes, cap, count, names, names_size);
}

// The sweep segments of launch group g (see hitb200_batch::segs).
static void batch_segs(LaunchSet& L, const hitb200_batch* b, int g) {
  const bool y2 = b->tuning[HITB200_TUNE_Y_PANEL] && b->has_y2;
  L.nsx = L.nsy = 0;
  for (int c = 0; c < 4; ++c) {
    const hitb200_batch::SegRec& rx = b->segs[g][0][c];
    if (rx.n > 0) L.sx[L.nsx++] = {b->d_segs + rx.off, rx.n, 1 << c, rx.smem};
    const hitb200_batch::SegRec& ry = b->segs[g][y2 ? 2 : 1][c];
    if (ry.n > 0) L.sy[L.nsy++] = {b->d_segs + ry.off, ry.n, 1 << c, ry.smem};
  }
}

static LaunchSet batch_launch_set(hitb200_batch* b, cudaStream_t st) {
  LaunchSet L;
  L.solves = b->d_solves;
  L.nsolves = (int)b->plans.size();
  L.tiles = b->d_tiles;
  L.tiles32 = b->d_tiles32;
  L.n_tiles32 = b->n_tiles32;
  L.srows = b->d_srows;
  L.n_srows = b->n_srows;
  L.guard_blocks = b->guard_blocks;
  L.xl = b->d_xlines;
  L.yl = b->d_ylines;
  L.partner = b->d_partner;
  L.n_tiles = b->n_tiles;
  L.n_x = b->n_x;
  L.n_y = b->n_y;
  L.elem = b->elem;
  L.mch_x = b->mch_x;
  L.mch_y = b->mch_y;
  L.thr_x = kLineThreads * b->rx_max;
  L.thr_y = kLineThreads * b->ry_max;
  const bool y2 = b->tuning[HITB200_TUNE_Y_PANEL] && b->has_y2;
  if (y2) {
    L.yl = b->d_ylines2;
    L.n_y = b->n_y2;
    L.thr_y = kLineThreads * b->ry_max2;
  }
  L.occ_x = b->tuning[HITB200_TUNE_SWEEP_X];
  L.occ_y = b->tuning[HITB200_TUNE_SWEEP_Y];
  L.occ_pre = b->tuning[HITB200_TUNE_PREPASS];
  L.fused = 0;  // the fused sensor's grid barrier spans one solve
  L.pdl = 0;    // many waves per launch: early CTAs of the next kernel would hold slots
                // the current one still needs (8 x 512^2 HIT step 1.352 -> 1.364 ms with it)
  L.smem_x = b->smem_x;
  L.smem_y = y2 ? b->smem_y2 : b->smem_y;
  L.smem_sensor = b->smem_sensor;
  L.sensor_w = b->sensor_w;
  L.smem_sensor_step = b->smem_sensor_step;
  L.st = st;
  batch_segs(L, b, 0);
  {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    L.hv_sms = sms;
  }
  L.persist = b->tuning[HITB200_TUNE_PERSISTENT] && b->can_persist;
  if (b->can_persist) {
    L.qitems = b->d_qitems + b->q_off[0];
    L.nq = b->q_off[1] - b->q_off[0];
    L.nq_pre = b->q_npre[0];
    L.qctl = b->d_qctl;
    L.qdep = b->d_qdep;
    L.qtiles = b->d_tiles32;
    L.xl4 = b->d_xl4;
    L.yl4 = b->d_yl4;
    L.smem_stage = b->smem_stage;
    L.stage_sh_off = b->stage_sh_off;
    L.stage_xstride = b->stage_xstride;
    L.stage_grid = b->stage_grid;
  }
  for (hitb200_plan* p : b->plans) {
    const double n = (double)p->desc.nx * p->desc.ny;
    L.cells += n;
    if (p->desc.viscosity > 0.0) L.cells_visc += n;
    if (p->desc.forcing_on) L.cells_force += n;
  }
  return L;
}

int hitb200_batch_step(hitb200_batch* b, void* stream) {
  if (!b) return invalid("NULL argument");
  for (hitb200_plan* p : b->plans)
    if (!p->hs.q) return invalid("batch state not bound");
  LaunchSet L = batch_launch_set(b, (cudaStream_t)stream);
  return launch_step_sequence(L, b->any_forcing, 0, b->any_outflow, b->any_hv);
}

// The launch set of members [s0, s1) of batch b: the same tables, the
// members' contiguous ranges of every work list.
static LaunchSet batch_sub_set(hitb200_batch* b, cudaStream_t st, int s0, int s1) {
  LaunchSet L = batch_launch_set(b, st);
  L.tiles = b->d_tiles + b->off_tiles[s0];
  L.n_tiles = b->off_tiles[s1] - b->off_tiles[s0];
  L.tiles32 = b->d_tiles32 + b->off_tiles32[s0];
  L.n_tiles32 = b->off_tiles32[s1] - b->off_tiles32[s0];
  L.xl = b->d_xlines + b->off_xl[s0];
  L.n_x = b->off_xl[s1] - b->off_xl[s0];
  if (b->tuning[HITB200_TUNE_Y_PANEL] && b->has_y2) {
    L.yl = b->d_ylines2 + b->off_yl2[s0];
    L.n_y = b->off_yl2[s1] - b->off_yl2[s0];
  } else {
    L.yl = b->d_ylines + b->off_yl[s0];
    L.n_y = b->off_yl[s1] - b->off_yl[s0];
  }
  L.srows = b->d_srows + b->off_srows[s0];
  L.n_srows = b->off_srows[s1] - b->off_srows[s0];
  // work items name members by their index in the whole batch (L.solves stays
  // the whole table); noise_rng takes the members from solve0 by CTA
  L.solve0 = s0;
  L.nsolves = s1 - s0;
  batch_segs(L, b, (s0 == 0 && s1 == (int)b->plans.size()) ? 0 : (s0 == 0 ? 1 : 2));
  if (b->can_persist) {
    const int g = (s0 == 0 && s1 == (int)b->plans.size()) ? 0 : (s0 == 0 ? 1 : 2);
    L.qitems = b->d_qitems + b->q_off[g];
    L.nq = b->q_off[g + 1] - b->q_off[g];
    L.nq_pre = b->q_npre[g];
    L.qctl = b->d_qctl + g;
  }
  L.cells = L.cells_visc = L.cells_force = 0.0;
  for (int i = s0; i < s1; ++i) {
    const hitb200_desc& d = b->plans[i]->desc;
    const double c = (double)d.nx * d.ny;
    L.cells += c;
    if (d.viscosity > 0.0) L.cells_visc += c;
    if (d.forcing_on) L.cells_force += c;
  }
  return L;
}

int hitb200_batch_run(hitb200_batch* b, int32_t nsteps, void* stream) {
  if (!b) return invalid("NULL argument");
  for (hitb200_plan* p : b->plans)
    if (!p->hs.q) return invalid("batch state not bound");
  cudaStream_t st = (cudaStream_t)stream;
  if (!b->graph || b->graph_stream != st) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    // The members in two groups (contiguous, balanced by cells), one branch
    // of the graph each, so that one group's kernels fill the other's tails:
    // 8 x 512^2 HIT step 1.300 -> 1.173 ms, 64-solve ensemble 5.31 -> 5.21 ms
    // (3, 4 and 8 groups measured no better).  Results do not depend on it:
    // every kernel works on one member at a time.
    const int n = (int)b->plans.size();
    const int cut = b->cut;
    // (persistent stage launches keep the two branches too: one branch for
    // the whole batch measured 1.38 against 1.25 ms per 8 x 512^2 HIT step)
    const int r = capture_graph(n > 1 ? 2 : 1, [&](cudaStream_t* cs) {
      if (n == 1) {
        LaunchSet L = batch_launch_set(b, cs[0]);
        return launch_step_sequence(L, b->any_forcing, 0, b->any_outflow, b->any_hv);
      }
      int rr = HITB200_OK;
      for (int g = 0; g < 2; ++g) {
        LaunchSet Lg = g == 0 ? batch_sub_set(b, cs[0], 0, cut) : batch_sub_set(b, cs[1], cut, n);
        const int rg = launch_step_sequence(Lg, b->any_forcing, 0, b->any_outflow, b->any_hv);
        if (rr == HITB200_OK) rr = rg;
      }
      return rr;
    }, &b->graph);
    if (r != HITB200_OK) return r;
    b->graph_stream = st;
  }
  for (int i = 0; i < nsteps; ++i) HB_CUDA(cudaGraphLaunch(b->graph, st));
  return HITB200_OK;
}

}  // extern "C"

// ---- kernel variants (autotuner knobs) -------------------------------------------
static int tuning_set(int* dst, const int32_t* knobs, int32_t n, int n_x, int n_y, int n_tiles32) {
  if (!knobs || n <= 0 || n > HITB200_TUNE_COUNT) return invalid("tuning knobs: 1..HITB200_TUNE_COUNT values");
  int def[HITB200_TUNE_COUNT];
  default_tuning(n_x, n_y, n_tiles32, def);
  for (int i = 0; i < n; ++i) {
    if (knobs[i] < -1 || knobs[i] > 1) return invalid("tuning knob must be -1 (default), 0 or 1");
    dst[i] = knobs[i] < 0 ? def[i] : knobs[i];
  }
  return HITB200_OK;
}

extern "C" int hitb200_plan_set_tuning(hitb200_plan* p, const int32_t* knobs, int32_t n) {
  if (!p) return invalid("NULL argument");
  if (p->in_batch) return invalid("plan belongs to a batch; tune the batch");
  const int r = tuning_set(p->tuning, knobs, n, p->n_x, p->n_y, p->n_tiles32);
  p->tuning[HITB200_TUNE_PERSISTENT] = 0;  // a batch form
  if (r == HITB200_OK && p->graph) {
    cudaGraphExecDestroy(p->graph);
    p->graph = nullptr;
  }
  return r;
}

extern "C" int hitb200_plan_get_tuning(const hitb200_plan* p, int32_t* knobs, int32_t n) {
  if (!p || !knobs) return invalid("NULL argument");
  if (n <= 0 || n > HITB200_TUNE_COUNT) return invalid("tuning knobs: 1..HITB200_TUNE_COUNT values");
  for (int i = 0; i < n; ++i) knobs[i] = p->tuning[i];
  return HITB200_OK;
}

extern "C" int hitb200_batch_set_tuning(hitb200_batch* b, const int32_t* knobs, int32_t n) {
  if (!b) return invalid("NULL argument");
  const int r = tuning_set(b->tuning, knobs, n, b->n_x, b->n_y, b->n_tiles32);
  if (!b->can_persist) b->tuning[HITB200_TUNE_PERSISTENT] = 0;
  if (r == HITB200_OK && b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return r;
}

extern "C" int hitb200_batch_get_tuning(const hitb200_batch* b, int32_t* knobs, int32_t n) {
  if (!b || !knobs) return invalid("NULL argument");
  if (n <= 0 || n > HITB200_TUNE_COUNT) return invalid("tuning knobs: 1..HITB200_TUNE_COUNT values");
  for (int i = 0; i < n; ++i) knobs[i] = b->tuning[i];
  return HITB200_OK;
}

// =============================================================================
// Initial states on the device (OOP/hit2d.py:158-204,
// OOP/problems/riemann_config3.py:59-99).
// =============================================================================
namespace {

int init_grid_check(int32_t nx, int32_t ny, double dx, double dy) {
  if (nx <= 0 || ny <= 0) return invalid("initial state: nx and ny must be positive");
  if (!(dx > 0.0) || !(dy > 0.0) || !std::isfinite(dx) || !std::isfinite(dy))
    return invalid("initial state: dx and dy must be positive and finite");
  return HITB200_OK;
}

int init_blocks(long long n) {
  return (int)std::max(1LL, std::min((n + kInitThreads - 1) / kInitThreads, 8192LL));
}

}  // namespace

extern "C" int hitb200_hit_streamfunction(const double* modes, int32_t n_modes, int32_t nx,
                                          int32_t ny, double x_min, double dx, double y_min,
                                          double dy, double* psi, void* stream) {
  if (!psi || (n_modes > 0 && !modes)) return invalid("hit_streamfunction: NULL pointer");
  if (n_modes < 0) return invalid("hit_streamfunction: n_modes must be >= 0");
  const int r = init_grid_check(nx, ny, dx, dy);
  if (r != HITB200_OK) return r;
  const long long n = (long long)nx * ny;
  hit_psi_kernel<<<init_blocks(n), kInitThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      modes, n_modes, nx, ny, x_min, dx, y_min, dy, psi);
  HB_LAUNCHED("hit_psi_kernel");
  return HITB200_OK;
}

extern "C" size_t hitb200_hit_compose_workspace_bytes(void) {
  return (size_t)kInitSumBlocks * 3 * sizeof(double);
}

extern "C" int hitb200_hit_compose(const double* u, const double* v, int32_t nx, int32_t ny,
                                   double gamma, double target_mach, double c_mean, double* q,
                                   double* vrms_out, void* workspace, size_t workspace_bytes,
                                   void* stream) {
  if (!u || !v || !q || !vrms_out || !workspace) return invalid("hit_compose: NULL pointer");
  if (nx <= 0 || ny <= 0) return invalid("hit_compose: nx and ny must be positive");
  if (!(gamma > 1.0)) return invalid("hit_compose: gamma must be > 1");
  if (workspace_bytes < hitb200_hit_compose_workspace_bytes())
    return invalid("hit_compose: workspace smaller than hitb200_hit_compose_workspace_bytes");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long long n = (long long)nx * ny;
  double* part = static_cast<double*>(workspace);
  hit_ic_sum_kernel<0><<<kInitSumBlocks, kInitThreads, 0, st>>>(u, v, n, part);
  HB_LAUNCHED("hit_ic_sum_kernel<0>");
  hit_ic_sum_kernel<1><<<kInitSumBlocks, kInitThreads, 0, st>>>(u, v, n, part);
  HB_LAUNCHED("hit_ic_sum_kernel<1>");
  hit_ic_compose_kernel<<<init_blocks(n), kInitThreads, 0, st>>>(u, v, n, part, gamma, target_mach,
                                                                  c_mean, q, vrms_out);
  HB_LAUNCHED("hit_ic_compose_kernel");
  return HITB200_OK;
}

extern "C" int hitb200_riemann_initial_state(const double* states, int32_t nx, int32_t ny,
                                             double x_min, double dx, double y_min, double dy,
                                             double x_split, double y_split, double gamma,
                                             double* q, void* stream) {
  if (!states || !q) return invalid("riemann_initial_state: NULL pointer");
  const int r = init_grid_check(nx, ny, dx, dy);
  if (r != HITB200_OK) return r;
  if (!(gamma > 1.0)) return invalid("riemann_initial_state: gamma must be > 1");
  QuadStates s;
  std::memcpy(s.s, states, sizeof(s.s));
  const long long n = (long long)nx * ny;
  quadrant_kernel<<<init_blocks(n), kInitThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      s, nx, ny, x_min, dx, y_min, dy, x_split, y_split, gamma, q);
  HB_LAUNCHED("quadrant_kernel");
  return HITB200_OK;
}

// =============================================================================
// Shell spectra (HIT2DSpectra.compute, OOP/postprocess/spectra.py:48-149).
// The caller owns every buffer, the transform between the two calls and the
// workspace: [n_snap][kSpecMeanBlocks][3] mean partials, then
// [n_snap][blocks][2][ns] shell partials, ns = min(nx, ny) / 2 + 1.
// =============================================================================
namespace {

// Row blocks per snapshot of the shell kernel: about 8 CTAs per SM over the
// whole batch, at least one row per warp.
int spectra_row_blocks(int n_snap, int ny, int* rows_per_cta) {
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int target = std::max(1, (8 * sms + n_snap - 1) / n_snap);
  const int most = (ny + kSpecWarps - 1) / kSpecWarps;
  const int want = std::min(target, most);
  const int rows = (ny + want - 1) / want;
  *rows_per_cta = rows;
  return (ny + rows - 1) / rows;
}

size_t spectra_ws_bytes(int n_snap, int nx, int ny) {
  int rows = 0;
  const int nblk = spectra_row_blocks(n_snap, ny, &rows);
  const size_t ns = (size_t)std::min(nx, ny) / 2 + 1;
  return ((size_t)n_snap * kSpecMeanBlocks * 3 + (size_t)n_snap * nblk * 2 * ns) * sizeof(double);
}

int spectra_check(int32_t n_snap, int32_t nx, int32_t ny, const void* ws, size_t ws_bytes) {
  if (n_snap <= 0) return invalid("spectra: n_snap must be positive");
  if (nx < 2 || ny < 2) return invalid("spectra: nx and ny must be at least 2");
  if ((size_t)std::min(nx, ny) / 2 + 1 > (size_t)kSpecMaxShells) {
    g_last_error = "spectra: min(nx, ny) / 2 + 1 shells above the supported 1025 (grids up to 2048)";
    return HITB200_ERR_UNSUPPORTED;
  }
  if (!ws) return invalid("spectra: workspace is NULL");
  if (ws_bytes < spectra_ws_bytes(n_snap, nx, ny))
    return invalid("spectra: workspace smaller than hitb200_spectra_workspace_bytes");
  return HITB200_OK;
}

template <bool CONS>
int spectra_fields_t(const double* a, const double* u, const double* v, int32_t n_snap, int32_t nx,
                     int32_t ny, int32_t favre, double* out, void* ws, cudaStream_t st) {
  const long long ncell = (long long)nx * ny;
  double* part = static_cast<double*>(ws);
  spectra_mean_kernel<CONS><<<dim3(kSpecMeanBlocks, n_snap), kSpecThreads, 0, st>>>(a, u, v, ncell,
                                                                                    favre, part);
  HB_LAUNCHED("spectra_mean_kernel");
  const long long want = (ncell + 4LL * kSpecThreads - 1) / (4LL * kSpecThreads);
  const int nb = (int)std::max(1LL, std::min(want, 4096LL));
  spectra_fields_kernel<CONS><<<dim3(nb, n_snap), kSpecThreads, 0, st>>>(a, u, v, ncell, favre, part,
                                                                         kSpecMeanBlocks, out);
  HB_LAUNCHED("spectra_fields_kernel");
  return HITB200_OK;
}

}  // namespace

extern "C" size_t hitb200_spectra_workspace_bytes(int32_t n_snap, int32_t nx, int32_t ny) {
  if (n_snap <= 0 || nx < 2 || ny < 2) return 0;
  return spectra_ws_bytes(n_snap, nx, ny);
}

extern "C" int hitb200_spectra_fields(const double* rho, const double* u, const double* v,
                                      int32_t n_snap, int32_t nx, int32_t ny, int32_t favre,
                                      double* out, void* workspace, size_t workspace_bytes,
                                      void* stream) {
  if (!rho || !u || !v || !out) return invalid("spectra: NULL field pointer");
  const int r = spectra_check(n_snap, nx, ny, workspace, workspace_bytes);
  if (r != HITB200_OK) return r;
  return spectra_fields_t<false>(rho, u, v, n_snap, nx, ny, favre ? 1 : 0, out, workspace,
                                 static_cast<cudaStream_t>(stream));
}

extern "C" int hitb200_spectra_state_fields(const double* q, int32_t n_snap, int32_t nx, int32_t ny,
                                            int32_t favre, double* out, void* workspace,
                                            size_t workspace_bytes, void* stream) {
  if (!q || !out) return invalid("spectra: NULL state pointer");
  const int r = spectra_check(n_snap, nx, ny, workspace, workspace_bytes);
  if (r != HITB200_OK) return r;
  return spectra_fields_t<true>(q, nullptr, nullptr, n_snap, nx, ny, favre ? 1 : 0, out, workspace,
                                static_cast<cudaStream_t>(stream));
}

extern "C" int hitb200_spectra_shells(const void* spec, int32_t n_snap, int32_t nx, int32_t ny,
                                      double dx, double dy, double* energy, double* enstrophy,
                                      void* workspace, size_t workspace_bytes, void* stream) {
  if (!spec || !energy || !enstrophy) return invalid("spectra: NULL pointer");
  if (!(dx > 0.0) || !(dy > 0.0) || !std::isfinite(dx) || !std::isfinite(dy))
    return invalid("spectra: dx and dy must be positive and finite");
  const int r = spectra_check(n_snap, nx, ny, workspace, workspace_bytes);
  if (r != HITB200_OK) return r;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int ns = std::min(nx, ny) / 2 + 1;
  int rows = 0;
  const int nblk = spectra_row_blocks(n_snap, ny, &rows);
  // dk and 1 / (n d) as the reference's NumPy expressions round them
  const double dk = std::min(2.0 * M_PI / (nx * dx), 2.0 * M_PI / (ny * dy));
  const double inv_nxdx = 1.0 / ((double)nx * dx), inv_nydy = 1.0 / ((double)ny * dy);
  const double norm = (double)nx * (double)ny;
  const double inv_norm = 1.0 / (norm * norm);
  double* part = static_cast<double*>(workspace) + (size_t)n_snap * kSpecMeanBlocks * 3;
  const size_t smem = (size_t)kSpecWarps * 2 * ns * sizeof(double);
  {
    static size_t done[kMaxAttrDevices] = {};
    const int dev = attr_device();
    std::lock_guard<std::mutex> lock(g_attr_mu);
    if (smem > 48 * 1024 && smem > done[dev]) {
      HB_CUDA(cudaFuncSetAttribute(spectra_shell_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
      done[dev] = smem;
    }
  }
  spectra_shell_kernel<<<dim3(nblk, n_snap), kSpecThreads, smem, st>>>(
      static_cast<const double2*>(spec), nx, ny, inv_nxdx, inv_nydy, dk, inv_norm, ns, rows, part);
  HB_LAUNCHED("spectra_shell_kernel");
  spectra_final_kernel<<<dim3((2 * ns + kSpecThreads - 1) / kSpecThreads, n_snap), kSpecThreads, 0,
                         st>>>(part, nblk, ns, energy, enstrophy);
  HB_LAUNCHED("spectra_final_kernel");
  return HITB200_OK;
}

// =============================================================================
// Stable time step without a plan and without allocating.
//
// Who needs it: a caller that must not allocate device memory at the point
// where it wants the CFL time step.  Creating a plan allocates its arena with
// cudaMalloc, and destroying one calls cudaFree, which synchronises the whole
// device; a serving loop that shares the GPU with other streams, or a process
// whose device memory is already reserved by its own caching pool, cannot
// afford either.  This entry point keeps its reduction scratch in one
// fixed-size array in the library's own device memory instead.
//
// Scratch (g_dt_scratch, 256 + 8 * kDtScratchTiles bytes on every device that
// loads the library, held until the process exits):
//   bytes [0, 4)      ticket counter of the last-CTA reduction.  It MUST be
//                     zero when a call starts: it is zero when the module is
//                     loaded and every call leaves it at zero again.
//   bytes [256, ...)  one partial maximum (double) per 32 x 32-cell tile;
//                     written before it is read, needs no initial value.
// Every call on a device uses the same scratch and it keeps the last call's
// contents, so two calls whose kernels may overlap on the GPU (different
// streams, or different host threads without ordering) race and give wrong
// results; calls on one stream are ordered and safe.
// =============================================================================
namespace {

constexpr int kDtScratchTiles = 1024;  // up to 1024 tiles of 32 x 32 cells (1,048,576 cells)
constexpr int kDtScratchHead = 256;
constexpr int kMaxScratchDevices = 64;

static __device__ __align__(256) unsigned char g_dt_scratch[kDtScratchHead + 8 * kDtScratchTiles];

// Device address of g_dt_scratch on the current device.  In host code the
// name g_dt_scratch is only a host-side stand-in, so the address is looked up
// with that device current on every call (the first call on a device may
// also load the module there); it is not cached, so that a context created
// again after cudaDeviceReset gets its own module's address.
int dt_scratch_address(unsigned char** out) {
  int dev = 0;
  HB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxScratchDevices)
    return invalid("device ordinal out of range for the static time-step scratch");
  void* p = nullptr;
  HB_CUDA(cudaGetSymbolAddress(&p, g_dt_scratch));
  *out = static_cast<unsigned char*>(p);
  return HITB200_OK;
}

// Spectral-radius maximum of the raw state (the time-step reduction of the
// prepass, OOP/spatial_operator.py:369-377), one CTA per 32 x 32 tile; the
// last CTA reduces the partials and writes dt = min(cfl / max, remaining).
__global__ void __launch_bounds__(kRedThreads)
    dt_scratch_kernel(const double* __restrict__ q, int nx, int ny, double dx, double dy,
                      double g, double cfl, double remaining, unsigned char* scratch,
                      double* dt_out) {
  unsigned* ticket = reinterpret_cast<unsigned*>(scratch);
  double* part = reinterpret_cast<double*>(scratch + kDtScratchHead);
  const int ntx = (nx + kTileX - 1) / kTileX;
  const int x0 = (blockIdx.x % ntx) * kTileX, y0 = (blockIdx.x / ntx) * kTileY;
  const int tx = threadIdx.x & 31, ty0 = threadIdx.x >> 5;
  const size_t plane = (size_t)nx * ny;
  const double idx_ = 1.0 / dx, idy_ = 1.0 / dy;
  // NaN-propagating maximum, as the reference's np.max: a non-finite cell
  // makes dt NaN instead of being skipped by fmax
  auto nan_max = [](double m, double x) { return (x != x || x > m) ? x : m; };
  double sr = 0.0;
  for (int a = ty0; a < kTileY; a += kRedWarps) {
    const int gj = y0 + a, gi = x0 + tx;
    if (gj >= ny || gi >= nx) continue;
    const size_t o = (size_t)gj * nx + gi;
    const double q0 = q[o], q1 = q[o + plane], q2 = q[o + 2 * plane], q3 = q[o + 3 * plane];
    const double rho = q0 > kRhoFloor ? q0 : kRhoFloor;
    const double rinv = 1.0 / rho;
    const double ur = q1 * rinv, vr = q2 * rinv;
    const double kin = 0.5 * rho * (ur * ur + vr * vr);
    const double p_raw = (g - 1.0) * (q3 - kin);
    const double pr = p_raw > kPFloor ? p_raw : kPFloor;
    const double cr = sqrt(g * pr * rinv);
    sr = nan_max(sr, (fabs(ur) + cr) * idx_ + (fabs(vr) + cr) * idy_);
  }
  __shared__ double sm[kRedWarps];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sr = nan_max(sr, __shfl_xor_sync(0xffffffffu, sr, o));
  if (tx == 0) sm[ty0] = sr;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = sm[0];
    for (int w = 1; w < kRedWarps; ++w) m = nan_max(m, sm[w]);
    part[blockIdx.x] = m;
  }
  if (!last_block(ticket, gridDim.x)) return;
  if (threadIdx.x >= 32) return;
  double m = 0.0;
  for (int b = tx; b < (int)gridDim.x; b += 32) m = nan_max(m, __ldcg(part + b));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = nan_max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (tx == 0) {
    double dt = cfl / m;
    if (!isnan(remaining)) dt = fmin(dt, remaining);
    *dt_out = dt;
  }
}

}  // namespace

extern "C" int hitb200_stable_time_step_noalloc(const double* q, int32_t nx, int32_t ny, double dx,
                                                double dy, double gamma, double cfl,
                                                double remaining_time, double* dt_out,
                                                void* stream) {
  if (!q || !dt_out) return invalid("NULL argument");
  if (nx <= 0 || ny <= 0) return invalid("nx and ny must be positive");
  if (!(dx > 0.0) || !(dy > 0.0)) return invalid("dx and dy must be positive");
  if (!(gamma > 1.0)) return invalid("gamma must exceed 1");
  if (!(cfl > 0.0)) return invalid("cfl must be positive");
  const long long tiles = (((long long)nx + kTileX - 1) / kTileX) * (((long long)ny + kTileY - 1) / kTileY);
  if (tiles > kDtScratchTiles) {
    g_last_error = "grid of " + std::to_string(nx) + " x " + std::to_string(ny) + " cells needs " +
                   std::to_string(tiles) + " tiles of 32 x 32 cells; the static scratch of "
                   "hitb200_stable_time_step_noalloc holds at most 1024";
    return HITB200_ERR_UNSUPPORTED;
  }
  unsigned char* scratch = nullptr;
  const int st = dt_scratch_address(&scratch);
  if (st != HITB200_OK) return st;
  dt_scratch_kernel<<<(unsigned)tiles, kRedThreads, 0, (cudaStream_t)stream>>>(
      q, nx, ny, dx, dy, gamma, cfl, remaining_time, scratch, dt_out);
  HB_LAUNCHED("dt_scratch_kernel");
  return HITB200_OK;
}

// =============================================================================
// Line transforms: spectral diagnostics, the initial condition's spectral
// derivatives and the real 2-D transform of the shell spectra
// (kernels_fft.cuh).  Grid lines up to kFftMaxN points.
// =============================================================================
namespace {

// e^{-2 pi i j / n}, j in [0, n), as the plan's twiddle tables are formed.
std::vector<double2> fft_roots(int n) {
  std::vector<double2> w(n);
  for (int j = 0; j < n; ++j) {
    const double th = 2.0 * M_PI * (double)j / (double)n;
    w[j] = make_double2(std::cos(th), -std::sin(th));
  }
  return w;
}

template <bool IN_REAL, bool OUT_REAL, int C>
void fft_attr(size_t bytes) {
  static size_t done[kMaxAttrDevices] = {};
  const int dev = attr_device();
  std::lock_guard<std::mutex> lock(g_attr_mu);
  if (bytes > done[dev]) {
    cudaFuncSetAttribute(fft_lines_kernel<IN_REAL, OUT_REAL, C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)bytes);
    done[dev] = bytes;
  }
}

template <bool IN_REAL, bool OUT_REAL, bool COLS>
void fft_p2_attr(size_t bytes) {
  static size_t done[kMaxAttrDevices] = {};
  const int dev = attr_device();
  std::lock_guard<std::mutex> lock(g_attr_mu);
  if (bytes > done[dev]) {
    cudaFuncSetAttribute(fft_p2_kernel<IN_REAL, OUT_REAL, COLS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)bytes);
    done[dev] = bytes;
  }
}

// `fields` batches of `lines` lines of n points (see FftLines); C > 1:
// the lines are adjacent columns.  Power-of-two lengths take the radix-8
// register kernel, others the mixed-radix one.
template <bool IN_REAL, bool OUT_REAL, int C>
void fft_launch(const void* in, void* out, int n, int lines, int fields, FftLines li, FftLines lo,
                int out_count, int sign, const double2* W, double scale, cudaStream_t st) {
  if (fft_pow2_ok(n) && !(IN_REAL && C > 1)) {
    int logn = 0;
    while ((1 << logn) < n) ++logn;
    const int L = kFftP2Points >> logn;
    const int clines = IN_REAL ? (lines + 1) / 2 : lines;
    const size_t smem = fft_p2_smem_bytes(n);
    fft_p2_attr<IN_REAL, OUT_REAL, (C > 1)>(smem);
    const long long grid = (long long)fields * ((clines + L - 1) / L);
    fft_p2_kernel<IN_REAL, OUT_REAL, (C > 1)><<<(unsigned)grid, kFftThreads, smem, st>>>(
        in, out, n, logn, lines, li, lo, out_count, sign, W, scale);
    return;
  }
  const size_t smem = fft_smem_bytes(n, C);
  fft_attr<IN_REAL, OUT_REAL, C>(smem);
  const long long grid = (long long)fields * ((lines + C - 1) / C);
  fft_lines_kernel<IN_REAL, OUT_REAL, C><<<(unsigned)grid, kFftThreads, smem, st>>>(
      in, out, n, lines, li, lo, out_count, sign, W, fft_radices(n), scale);
}

// Column transforms (in place, complex) of `fields` arrays [ny][w] (w columns).
void fft_columns(double2* a, int ny, int w, int fields, int sign, const double2* W, double scale,
                 cudaStream_t st) {
  const FftLines l{(long long)ny * w, 1, w};
  if (fft_smem_bytes(ny, 4) <= 160 * 1024)
    fft_launch<false, false, 4>(a, a, ny, w, fields, l, l, ny, sign, W, scale, st);
  else
    fft_launch<false, false, 2>(a, a, ny, w, fields, l, l, ny, sign, W, scale, st);
}

int fft_grid_check(int32_t nx, int32_t ny) {
  if (nx <= 0 || ny <= 0) return invalid("transform: nx and ny must be positive");
  if (nx > kFftMaxN || ny > kFftMaxN)
    return (g_last_error = "transform: grid lines longer than 1024 points are not supported",
            HITB200_ERR_UNSUPPORTED);
  return HITB200_OK;
}

constexpr int kSpecReduceBlocks = 512;

// Workspace of the spectral diagnostics: rho, u, v [3][n] and the four real
// results [4][n] (doubles), then (16-byte aligned) the transforms of u, v
// [2][n] and of the four products [4][n], the reduction partials, totals and
// ticket.
size_t spectral_c1_off(size_t n) { return (7 * n * sizeof(double) + 255) & ~(size_t)255; }
size_t spectral_ws(int nx, int ny) {
  const size_t n = (size_t)nx * ny;
  return spectral_c1_off(n) + 6 * n * sizeof(double2) + kSpecReduceBlocks * 4 * sizeof(double) +
         8 * sizeof(double) + 256;
}

}  // namespace

extern "C" size_t hitb200_spectral_workspace_bytes(int32_t nx, int32_t ny) {
  if (nx <= 0 || ny <= 0) return 0;
  return spectral_ws(nx, ny);
}

extern "C" int hitb200_spectral_diagnostics(hitb200_plan* p, const double* q, double kmax, double* out,
                                            double* div, double* vort, void* workspace,
                                            size_t workspace_bytes, void* stream) {
  if (!p || !q || !out) return invalid("NULL argument");
  if (!p->desc.periodic) return invalid("spectral diagnostics need a periodic grid");
  const int nx = p->desc.nx, ny = p->desc.ny;
  int r = fft_grid_check(nx, ny);
  if (r != HITB200_OK) return r;
  if (!workspace || workspace_bytes < spectral_ws(nx, ny))
    return invalid("workspace smaller than hitb200_spectral_workspace_bytes");
  cudaStream_t st = (cudaStream_t)stream;
  const long long n = (long long)nx * ny;
  double* ruv = static_cast<double*>(workspace);  // [3][n] rho, u, v
  double* dwb = ruv + 3 * n;                       // [4][n] div, vort, u_low, v_low
  double2* c1 = reinterpret_cast<double2*>(static_cast<unsigned char*>(workspace) + spectral_c1_off(n));
  double2* c2 = c1 + 2 * n;                               // [4][n]
  double* part = reinterpret_cast<double*>(c2 + 4 * n);
  double* res = part + kSpecReduceBlocks * 4;
  unsigned* ticket = reinterpret_cast<unsigned*>(res + 4);
  HB_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned), st));
  const int blocks = (int)std::min<long long>(kSpecReduceBlocks, (n + 255) / 256);
  spec_prims_kernel<<<blocks, 256, 0, st>>>(q, ruv, n, p->desc.gamma);
  // fft2 of u and v: rows (real input), then columns
  fft_launch<true, false, 1>(ruv + n, c1, nx, ny, 2, FftLines{n, nx, 1}, FftLines{n, nx, 1}, nx, -1,
                             p->hs.twx, 1.0, st);
  fft_columns(c1, ny, nx, 2, -1, p->hs.twy, 1.0, st);
  spec_multiply_kernel<<<blocks, 256, 0, st>>>(c1, c2, nx, ny, p->hs.dx, p->hs.dy,
                                               kmax > 0.0 ? kmax : -1.0);
  // ifft2 (real parts) of the four products
  fft_columns(c2, ny, nx, 4, +1, p->hs.twy, 1.0 / ny, st);
  fft_launch<false, true, 1>(c2, dwb, nx, ny, 4, FftLines{n, nx, 1}, FftLines{n, nx, 1}, nx, +1,
                             p->hs.twx, 1.0 / nx, st);
  spec_reduce_kernel<<<blocks, 256, 0, st>>>(ruv, dwb, c1, n, part, ticket, res, div, vort);
  HB_LAUNCHED("spectral diagnostics");
  double h[4];
  HB_CUDA(cudaMemcpyAsync(h, res, sizeof(h), cudaMemcpyDeviceToHost, st));
  HB_CUDA(cudaStreamSynchronize(st));
  const double N = (double)n;
  out[0] = std::sqrt(h[0] / N);
  out[1] = std::sqrt(h[1] / N);
  // large_scale_kinetic_fraction (OOP/hit2d.py:429-449)
  const double total = h[3] / N;
  out[2] = (kmax <= 0.0 || total <= DBL_EPSILON) ? 0.0 : (h[2] / N) / total;
  return HITB200_OK;
}

extern "C" size_t hitb200_hit_velocity_workspace_bytes(int32_t nx, int32_t ny) {
  if (nx <= 0 || ny <= 0) return 0;
  return 3 * (size_t)nx * ny * sizeof(double2) + (size_t)(nx + ny) * sizeof(double2) + 256;
}

extern "C" int hitb200_hit_velocity(const double* psi, int32_t nx, int32_t ny, double dx, double dy,
                                    double* u, double* v, void* workspace, size_t workspace_bytes,
                                    void* stream) {
  if (!psi || !u || !v) return invalid("NULL argument");
  int r = fft_grid_check(nx, ny);
  if (r != HITB200_OK) return r;
  if (!(dx > 0.0) || !(dy > 0.0)) return invalid("dx and dy must be positive");
  if (!workspace || workspace_bytes < hitb200_hit_velocity_workspace_bytes(nx, ny))
    return invalid("workspace smaller than hitb200_hit_velocity_workspace_bytes");
  cudaStream_t st = (cudaStream_t)stream;
  const long long n = (long long)nx * ny;
  double2* ph = static_cast<double2*>(workspace);
  double2* uv = ph + n;
  double2* wx = uv + 2 * n;
  double2* wy = wx + nx;
  const std::vector<double2> rx = fft_roots(nx), ry = fft_roots(ny);
  HB_CUDA(cudaMemcpyAsync(wx, rx.data(), nx * sizeof(double2), cudaMemcpyHostToDevice, st));
  HB_CUDA(cudaMemcpyAsync(wy, ry.data(), ny * sizeof(double2), cudaMemcpyHostToDevice, st));
  fft_launch<true, false, 1>(psi, ph, nx, ny, 1, FftLines{n, nx, 1}, FftLines{n, nx, 1}, nx, -1, wx, 1.0,
                             st);
  fft_columns(ph, ny, nx, 1, -1, wy, 1.0, st);
  const int blocks = (int)std::min<long long>(1024, (n + 255) / 256);
  spec_velocity_kernel<<<blocks, 256, 0, st>>>(ph, uv, nx, ny, dx, dy);
  fft_columns(uv, ny, nx, 2, +1, wy, 1.0 / ny, st);
  fft_launch<false, true, 1>(uv, u, nx, ny, 1, FftLines{n, nx, 1}, FftLines{n, nx, 1}, nx, +1, wx,
                             1.0 / nx, st);
  fft_launch<false, true, 1>(uv + n, v, nx, ny, 1, FftLines{n, nx, 1}, FftLines{n, nx, 1}, nx, +1, wx,
                             1.0 / nx, st);
  HB_LAUNCHED("hit velocity transforms");
  // the host tables must outlive their (staged) copies
  HB_CUDA(cudaStreamSynchronize(st));
  return HITB200_OK;
}

extern "C" size_t hitb200_rfft2_workspace_bytes(int32_t nx, int32_t ny) {
  if (nx <= 0 || ny <= 0) return 0;
  return (size_t)(nx + ny) * sizeof(double2) + 256;
}

extern "C" int hitb200_rfft2(const double* in, int32_t n_fields, int32_t nx, int32_t ny, void* out,
                             void* workspace, size_t workspace_bytes, void* stream) {
  if (!in || !out) return invalid("NULL argument");
  if (n_fields <= 0) return invalid("n_fields must be positive");
  int r = fft_grid_check(nx, ny);
  if (r != HITB200_OK) return r;
  if (!workspace || workspace_bytes < hitb200_rfft2_workspace_bytes(nx, ny))
    return invalid("workspace smaller than hitb200_rfft2_workspace_bytes");
  cudaStream_t st = (cudaStream_t)stream;
  double2* wx = static_cast<double2*>(workspace);
  double2* wy = wx + nx;
  const std::vector<double2> rx = fft_roots(nx), ry = fft_roots(ny);
  HB_CUDA(cudaMemcpyAsync(wx, rx.data(), nx * sizeof(double2), cudaMemcpyHostToDevice, st));
  HB_CUDA(cudaMemcpyAsync(wy, ry.data(), ny * sizeof(double2), cudaMemcpyHostToDevice, st));
  const int nh = nx / 2 + 1;
  const long long n = (long long)nx * ny;
  double2* o = static_cast<double2*>(out);
  fft_launch<true, false, 1>(in, o, nx, ny, n_fields, FftLines{n, nx, 1}, FftLines{(long long)ny * nh, nh, 1},
                             nh, -1, wx, 1.0, st);
  fft_columns(o, ny, nh, n_fields, -1, wy, 1.0, st);
  HB_LAUNCHED("rfft2 transforms");
  HB_CUDA(cudaStreamSynchronize(st));
  return HITB200_OK;
}

