// Shared device-side definitions of the HIT_Solver B200 backend.
//
// Data layout in HBM (per solve):
//   state q, stage buffers q1, q2 : double [4][ny][nx]   (x fastest)
//   x-sweep partial rhs  rx        : T      [4][ny][nx]
//   viscous terms       vis        : T      [3][ny][nx]   (rows rho*u, rho*v, E)
//   sensor mask         mask       : uint8  [ny][nx]
//   forcing shape       fx, fy     : double [ny][nx]      (unit-rms, unscaled)
//   reduction partials             : double [blocks][NRED]
//   scalar block        scal       : double [SCAL_SIZE]
// T is float in the FP32-bulk form and double in the plain FP64 form.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hitb200 {

constexpr double kRhoFloor = 1e-10;
constexpr double kPFloor = 1e-10;
constexpr double kCompactA = 0.375;   // 3/8, compact scheme alpha
constexpr int kHalo = 5;              // staged halo of the sweep lines
constexpr int kMaxLine = 1024;        // longest supported grid line
constexpr int kMaxDrag = 32;          // max drag modes (|k| <= kmax band)
constexpr int kMaxForce = 128;        // max forcing shell modes
// Forcing synthesis CTAs cover whole rows: about 1024 cells each, at most
// kSynthMaxRows rows (the rows' mode table is built once per row).
constexpr int kSynthMaxRows = 32;
constexpr int kSynthTerms = 512;   // (row, mode) terms of one row-table chunk
__host__ __device__ constexpr int synth_rows(int nx) {
  return nx >= 1024 ? 1 : (1024 / nx > kSynthMaxRows ? kSynthMaxRows : 1024 / nx);
}
constexpr int kMaxWidth = 8;          // max sensor dilation width
constexpr int kMaxKx = 16;            // max |x wavenumber bin| of drag / forcing modes
constexpr int kMaxKyDrag = 4;         // max |y wavenumber bin| of drag modes

// ---- reduction slots of the per-stage prepass -------------------------------
enum Red : int {
  R_AX = 0,     // max |u| + c      (enforced state)
  R_AY,         // max |v| + c
  R_DIV2,       // sum div^2        (sensor divergence)
  R_VORT2,      // sum vort^2
  R_RHO,        // max |rho|
  R_P,          // max |p|
  R_E,          // max |e|, e = p / (rho (gamma - 1))
  R_PSUM,       // sum p            (raw state, cooling)
  R_SR,         // max (|u|+c)/dx + (|v|+c)/dy   (raw state, time step)
  R_VEL2,       // sum u^2 + v^2    (raw state, Mach)
  R_CSUM,       // sum c            (raw state, Mach)
  R_NONFINITE,  // max of 0/1 flags (raw state)
  R_NONPOS_RHO,
  R_NONPOS_P,
  R_FIXED,      // first drag slot: 4 per drag mode (Re/Im of rho*u and rho*v DFT)
};

// ---- scalar block slots ------------------------------------------------------
// 0..31 mirror enum hitb200_scalar of the public header.
enum Scal : int {
  S_ALPHA_X = 0, S_ALPHA_Y, S_DIV_RMS, S_VORT_RMS, S_DT, S_TIME, S_STEP, S_ACTIVE, S_MACH,
  S_POWER, S_POWER_DESIRED, S_F_ALPHA, S_F_ALPHA_TARGET, S_F_POWER_BEFORE, S_F_INJECTED,
  S_F_FXX, S_F_FYY, S_F_FXY, S_F_AF, S_F_DECAY, S_F_SCALE, S_MAX_STEPS, S_STATUS,
  S_NEAR, S_HV_APPLIED,
  // internal
  S_COMP_LIM = 32,   // node flagged if div < S_COMP_LIM (-inf when off)
  S_SHEAR_LIM,       // node flagged if |vort| > S_SHEAR_LIM (+inf when off)
  S_EPS_RHO, S_EPS_P, S_EPS_E,
  S_COOL,            // uniform energy source (0 when off)
  S_HV_STEP,         // 1 if the current step ends with hyperviscosity
  S_XI_SCALE,        // scale of the noise DFT (1 for caller noise)
  S_DRAG = 64,       // 4 per drag mode: c * Re/Im of the rho*u and rho*v mode sums
  S_PHI = S_DRAG + 4 * kMaxDrag,          // OU potential: 2 per forcing mode
  S_XI = S_PHI + 2 * kMaxForce,           // noise DFT of the step: 2 per mode
  // PCG64 stream of the reference's forcing noise (noise_mode 2): the bit
  // patterns of state.lo, state.hi, inc.lo, inc.hi
  S_PCG = S_XI + 2 * kMaxForce,
  SCAL_SIZE = S_PCG + 4,
};

// Status bits accumulated in S_STATUS.
enum StatusBits : int { ST_NONFINITE = 1, ST_NONPOS_RHO = 2, ST_NONPOS_P = 4, ST_BARRIER = 8, ST_NOISE = 16 };

// ---- per-solve descriptor (device resident, read-only in kernels) -------------
struct SolveDev {
  int nx, ny;
  int periodic, scheme, precision;
  double dx, dy, gamma;
  // sensor
  int width, boundary_guard, shear_on;
  double comp_thr, jump_thr, shear_thr;
  // viscous
  double mu, kappa, gas_r;
  // hyperviscosity (mn * w_c * h^4)
  double hv_coef[4];
  int hv_interval;
  int guard;
  // sources
  int drag_on, n_drag;
  int kx_drag, kx_force;  // max |x bin| of the drag / forcing modes
  int ky_drag;            // max |y bin| of the drag modes
  unsigned char f_order[kMaxForce];  // forcing modes ordered by |x bin| ...
  short f_kofs[kMaxKx + 2];          // ... with |x bin| = k at f_order[f_kofs[k] .. f_kofs[k+1])
  double drag_coef;
  int cooling_on;
  double cooling_tau, cooling_pref;
  int forcing_on, n_force;
  double f_tau, f_rms, f_target, f_min_power, f_max_rescale, f_alpha_memory;
  int f_has_target, f_has_max_rescale;
  int mach_control;
  double mach_target, mach_memory, mach_exponent, mach_min_power, mach_max_power;
  int has_mach_min, has_mach_max;
  double cfl, tfinal;
  int fixed_dt;
  int noise_mode;
  unsigned long long seed;
  // block counts of the reducing kernels (for the last-block finalize)
  int nblk_pre, nblk_noise, nblk_synth, nblk_diag;
  int nred;  // R_FIXED + 4 * n_drag
  // buffers
  double *q, *q1, *q2;
  void *rx, *vis;
  uint8_t *mask;
  void *fx, *fy;             // unit-rms forcing shape, T [ny][nx] (T = float in the FP32-bulk form)
  const double *noise;
  double2 *twx, *twy;        // e^{-2 pi i j / n}, j in [0, n)
  int2 *modes;               // n_drag drag modes, then n_force forcing modes (integer mx, my)
  double2 *kvec;             // physical (kx, ky) of the forcing modes
  double *scal;
  double *part_pre, *part_noise, *part_synth, *part_diag;
  unsigned *counters;        // [0] prepass, [1] noise, [2] synth, [3] diag, [4..6] grid barrier
  int *near_count;
  double *diag_out;          // diagnostics results (device)
};

// Work item of one CTA: solve index and two integer coordinates.
struct Work {
  int solve;
  int a;  // sweeps: first line; tiles: x0
  int b;  // sweeps: number of lines; tiles: y0
  int c;  // tiles: block index within the solve (for partials)
};

// ---- small device helpers --------------------------------------------------------
// Periodic wrap / outflow clamp of a node index within one grid length of
// the domain (larger offsets, only on tiny grids, fall back to a modulo).
__device__ __forceinline__ int fold_node(int i, int n, int periodic) {
  if (periodic) {
    if (i < 0) i += n;
    else if (i >= n) i -= n;
    if (i < 0 || i >= n) {
      i %= n;
      if (i < 0) i += n;
    }
    return i;
  }
  return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

// (m * j) mod n in [0, n) for a Fourier mode m and grid index j (32-bit: |m| <= n).
__device__ __forceinline__ int mode_index(int m, int j, int n) {
  int t = (m * j) % n;
  return t < 0 ? t + n : t;
}

template <typename T>
struct Prim {
  T rho, u, v, p;
};

// primitive_from_conservative (OOP/equations.py:136-145), in T arithmetic.
template <typename T>
__device__ __forceinline__ Prim<T> primitives(T q0, T q1, T q2, T q3, T gamma) {
  Prim<T> w;
  w.rho = q0 > T(kRhoFloor) ? q0 : T(kRhoFloor);
  w.u = q1 / w.rho;
  w.v = q2 / w.rho;
  T kin = T(0.5) * w.rho * (w.u * w.u + w.v * w.v);
  T p = (gamma - T(1)) * (q3 - kin);
  w.p = p > T(kPFloor) ? p : T(kPFloor);
  return w;
}

// enforce_physical_state (OOP/equations.py:165-181) of one node, in place.
template <typename T>
__device__ __forceinline__ void enforce_node(T& q0, T& q1, T& q2, T& q3, T gamma) {
  T rho = q0 > T(kRhoFloor) ? q0 : T(kRhoFloor);
  T u = q1 / rho, v = q2 / rho;
  T kin = T(0.5) * rho * (u * u + v * v);
  T p = (gamma - T(1)) * (q3 - kin);
  q0 = rho;
  q1 = rho * u;
  q2 = rho * v;
  q3 = p > T(kPFloor) ? q3 : T(kPFloor) / (gamma - T(1)) + kin;
}

// enforce_node with one reciprocal instead of two quotients (results within
// two ulp of the quotient form); used for the stage states the step writes.
template <typename T>
__device__ __forceinline__ void enforce_node_rcp(T& q0, T& q1, T& q2, T& q3, T gamma) {
  const T rho = q0 > T(kRhoFloor) ? q0 : T(kRhoFloor);
  const T rinv = T(1) / rho;
  const T u = q1 * rinv, v = q2 * rinv;
  const T kin = T(0.5) * rho * (u * u + v * v);
  const T p = (gamma - T(1)) * (q3 - kin);
  q0 = rho;
  q1 = rho * u;
  q2 = rho * v;
  q3 = p > T(kPFloor) ? q3 : T(kPFloor) / (gamma - T(1)) + kin;
}
// 1 / x correctly rounded: the same value as the division, in fewer
// instructions for FP32
template <typename T>
__device__ __forceinline__ T rcp_rn(T x) {
  if constexpr (sizeof(T) == 4) return __frcp_rn(x);
  else return 1.0 / x;
}

// the same with the floor energy kPFloor / (gamma - 1) computed by the caller
template <typename T>
__device__ __forceinline__ void enforce_node_rcp(T& q0, T& q1, T& q2, T& q3, T gamma, T pfl) {
  const T rho = q0 > T(kRhoFloor) ? q0 : T(kRhoFloor);
  const T rinv = T(1) / rho;
  const T u = q1 * rinv, v = q2 * rinv;
  const T kin = T(0.5) * rho * (u * u + v * v);
  const T p = (gamma - T(1)) * (q3 - kin);
  q0 = rho;
  q1 = rho * u;
  q2 = rho * v;
  q3 = p > T(kPFloor) ? q3 : pfl + kin;
}

// Programmatic dependent launch.  A kernel launched with programmatic stream
// serialization may start while the previous kernel of the stream finishes:
// pdl_wait() blocks until that kernel has completed and its writes are
// visible, so everything that reads what it wrote comes after pdl_wait().
// pdl_release() lets the next kernel start its prologue.  Both are no-ops in
// a launch without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// The wait of a work item for the phase before it, in the kernels launched
// one per phase: the programmatic-launch wait on the previous kernel.
// (early() is the wait for an earlier kernel's output read before that:
// complete at launch here.)  The work item runs on the whole CTA: tid(),
// nthreads() and sync() are the CTA's thread index, size and barrier.
struct PdlDep {
  static constexpr bool kQueued = false;
  static constexpr int kXR = 2;  // most x lines of a sweep item
  __device__ __forceinline__ void wait() const { pdl_wait(); }
  __device__ __forceinline__ void early() const {}
  __device__ __forceinline__ void release() const { pdl_release(); }
  // unsigned, as the special registers themselves: the sweeps' index
  // arithmetic measured 2.5-4.5 % slower on int copies of them
  __device__ __forceinline__ unsigned tid() const { return threadIdx.x; }
  __device__ __forceinline__ unsigned nthreads() const { return blockDim.x; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
  __device__ __forceinline__ bool sync_or(bool p) const { return __syncthreads_or(p) != 0; }
};

// Barrier of the `count` threads of group `id` (1..15; barrier 0 is the
// CTA's), optionally with the OR of a predicate over them.
__device__ __forceinline__ void group_sync(unsigned id, unsigned count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ bool group_sync_or(unsigned id, unsigned count, bool p) {
  unsigned r;
  asm volatile(
      "{\n\t.reg .pred pi, po;\n\t"
      "setp.ne.u32 pi, %1, 0;\n\t"
      "bar.red.or.pred po, %2, %3, pi;\n\t"
      "selp.u32 %0, 1, 0, po;\n\t}"
      : "=r"(r)
      : "r"((unsigned)p), "r"(id), "r"(count)
      : "memory");
  return r != 0u;
}

// Bulk asynchronous copies (the TMA unit, no tensor map, no multicast) from
// this GPU's global memory into this CTA's shared memory, completed on a
// shared-memory mbarrier.  Source, destination and size are multiples of 16
// bytes.
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  // the initialised barrier visible to the copy engine (async proxy)
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"((unsigned long long)__cvta_generic_to_global(src)), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned dynamic_smem_bytes() {
  unsigned v;
  asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(v));
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double cmul_re(double2 a, double2 b) { return a.x * b.x - a.y * b.y; }
__device__ __forceinline__ double cmul_im(double2 a, double2 b) { return a.x * b.y + a.y * b.x; }

}  // namespace hitb200
