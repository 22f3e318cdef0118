// Stencil kernels: shock sensor (+ viscous terms), the x / y line sweeps of
// the hybrid compact/WENO7 flux derivative with their fused epilogues, the
// biharmonic hyperviscosity, the outflow guard and the state clean.
#pragma once

#include "common.cuh"
#include "kernels_reduce.cuh"
#include "weno.cuh"

namespace hitb200 {

constexpr unsigned kFull = 0xffffffffu;


constexpr int kStencilThreads = 256;
constexpr int kLineThreads = 128;  // sweep threads per grid line of a CTA
// Occupancy targets of the throughput variant of the sweeps (OCC = 1): CTAs
// per SM, of 256 threads for x (up to 2 lines) and 512 for y (up to 4
// lines); they bound the registers per thread, so that many solves' lines
// share an SM.  The latency variants keep 128 registers per thread, for
// launches too small to fill the GPU twice over.
#ifndef HITB200_SWEEP_MIN_BLOCKS_X
#define HITB200_SWEEP_MIN_BLOCKS_X 4
#endif
#ifndef HITB200_SWEEP_MIN_BLOCKS_Y
#define HITB200_SWEEP_MIN_BLOCKS_Y 2
#endif
constexpr int kSweepMinBlocksX = HITB200_SWEEP_MIN_BLOCKS_X;
constexpr int kSweepMinBlocksY = HITB200_SWEEP_MIN_BLOCKS_Y;
constexpr int kSenTX = 32, kSenTY = 32;  // sensor tile
constexpr int kSensorThreads = 512;
constexpr int kHvTX = 32, kHvTY = 16;    // hyperviscosity tile

// =============================================================================
// Shock sensor (OOP/spatial_operator.py:147-176, 263-304;
// OOP/problems/riemann_config3.py:128-162, 288-326) and viscous terms
// (OOP/equations.py:232-267) on a 32 x 16 tile with a (width + 1) halo.
// Raw flags are evaluated on the tile plus a width-wide ring, then dilated
// separably: a row pass (OR over +-width in x) and a column pass.
// =============================================================================
template <typename T>
__device__ __forceinline__ T type_eps() {
  return sizeof(T) == 4 ? T(FLT_EPSILON) : T(DBL_EPSILON);
}

// Exact quotient test, out of line: reached only within ~8 ulp of a threshold.
template <typename T>
__device__ __noinline__ bool quotient_gt(T num, T den, T thr) {
  return num / den > thr;
}

// fl(num / den) > thr for den > 0, exactly as the reference's IEEE quotient
// compares, but decided by a multiplication unless the quotient lies within
// ~8 ulp of the threshold (then the quotient itself is formed).  FP64 form.
template <typename T>
__device__ __forceinline__ bool ratio_gt(T num, T den, T thr) {
  const T t = thr * den;
  const T d = num - t;
  if (fabs(d) > T(8) * type_eps<T>() * t) return d > T(0);
  return quotient_gt(num, den, thr);
}

// |num / den - thr| within tol * thr (a node "within roundoff" of the threshold)
template <typename T>
__device__ __forceinline__ bool ratio_near(T num, T den, T thr, T tol) {
  const T t = thr * den;
  return fabs(num - t) <= tol * t;
}

// FP32 form of the tests below: num / (den0 + eps) > thr is decided as
// margin = num - thr den0 (one rounding) > thr eps.  eps, a multiple of the
// quantity's global maximum from the prepass, is the same for all of one
// quantity's tests, so the step's sensor forms the margins before the
// prepass has finished.  Its masks differ from the FP64 ones only at nodes
// within FP32 roundoff of a threshold.
template <typename T>
__device__ __forceinline__ T fma_rn(T a, T b, T c) {
  if constexpr (sizeof(T) == 4) return __fmaf_rn(a, b, c);
  else return __fma_rn(a, b, c);
}
template <typename T>
__device__ __forceinline__ T pair_margin(T a, T b, T thr) {
  return fma_rn(-thr, fabs(b) + fabs(a), fabs(b - a));
}
template <typename T>
__device__ __forceinline__ T curv_margin(T am, T a, T ap, T thr) {
  return fma_rn(-thr, fabs(ap) + T(2) * fabs(a) + fabs(am), fabs(ap - T(2) * a + am));
}

// Two-point jump |b - a| / (|b| + |a| + eps) > thr of the pair (a, b): the
// reference's right jump of a and left jump of b are the same expression
// (OOP/spatial_operator.py:149-153), so it is evaluated once per edge.
template <typename T, bool NEAR>
__device__ __forceinline__ bool pair_gt(T a, T b, T eps, T thr, T tol, bool& near) {
  const T num = fabs(b - a), den = fabs(b) + fabs(a) + eps;
  if (NEAR) near = near || ratio_near(num, den, thr, tol);
  if constexpr (sizeof(T) == 4) return pair_margin(a, b, thr) > thr * eps;
  return ratio_gt(num, den, thr);
}

// Curvature |ap - 2a + am| / (|ap| + 2|a| + |am| + eps) > thr (OOP/spatial_operator.py:155-165).
template <typename T, bool NEAR>
__device__ __forceinline__ bool curv_gt(T am, T a, T ap, T eps, T thr, T tol, bool& near) {
  const T num = fabs(ap - T(2) * a + am), den = fabs(ap) + T(2) * fabs(a) + fabs(am) + eps;
  if (NEAR) near = near || ratio_near(num, den, thr, tol);
  if constexpr (sizeof(T) == 4) return curv_margin(am, a, ap, thr) > thr * eps;
  return ratio_gt(num, den, thr);
}

__host__ __device__ inline int sensor_halo(int width) { return width + 1 > 2 ? width + 1 : 2; }

// Viscous stage: stresses and energy fluxes of the tile plus a one-node ring.
constexpr int kVisX = kSenTX + 2, kVisY = kSenTY + 2;

// Shared-memory layout of the sensor: staged primitives, raw and row-dilated
// flags, then (FP32) the per-node test margins of the raw nodes.
__host__ __device__ inline size_t sensor_margin_off(int width, int elem) {
  const int hw = sensor_halo(width);
  const size_t sx = kSenTX + 2 * hw, sy = kSenTY + 2 * hw;
  const size_t prim = 5 * sx * sy * (size_t)elem;
  const size_t rx = kSenTX + 2 * width, ry = kSenTY + 2 * width;
  const size_t raw = ry * rx;
  const size_t row = ry * kSenTX;
  return (prim + raw + row + 32 + 15) & ~(size_t)15;
}
constexpr int kSenMargins = 5;  // rho, p, e margins, divergence, |vorticity|
__host__ __device__ inline size_t sensor_flag_end(int width, int elem) {
  const size_t rx = kSenTX + 2 * width, ry = kSenTY + 2 * width;
  return sensor_margin_off(width, elem) + (elem == 4 ? kSenMargins * rx * ry * 4 : 0);
}

// Dynamic shared memory of the sensor kernel; `viscous` adds the five
// stress / flux arrays of the viscous terms.
__host__ __device__ inline size_t sensor_smem_bytes(int width, int elem, bool viscous) {
  return sensor_flag_end(width, elem) + (viscous ? 5 * (size_t)kVisX * kVisY * elem : 0);
}

// Central difference quotient of the sensor.  FP64 divides by 2h exactly as
// the reference; FP32 multiplies by the reciprocal.
template <typename T>
__device__ __forceinline__ T dq(T a, T b, T h2, T ih2) {
  if constexpr (sizeof(T) == 8) return (a - b) / h2;
  else return (a - b) * ih2;
}

// Row / column of a flattened index in a table of row length `w`, with the
// float reciprocal `iw` = 1 / w (exact for the index ranges used here).
__device__ __forceinline__ int row_of(int idx, int w, float iw) {
  int r = __float2int_rd(((float)idx + 0.5f) * iw);
  if (r * w > idx) --r;
  else if ((r + 1) * w <= idx) ++r;
  return r;
}

// sel: 0 q, 1 q1, 2 q2, 3 hyperviscosity input (stage-3 output q1, runs only on
// hyperviscosity steps).  want_visc: also write the viscous terms.  NEAR:
// count nodes within roundoff of a threshold (sensor API; off in the fused
// step).
// CTAs per SM the FP32 sensor is compiled for; the FP64 one holds one CTA
// per SM anyway (its staged tile and viscous arrays take ~120 KB) and gets
// the full register budget instead.
#ifndef HITB200_SENSOR_MIN_BLOCKS
#define HITB200_SENSOR_MIN_BLOCKS 2
#endif
// FUSED (one solve, cooperative launch with every tile resident): the CTA
// first reduces its tile's prepass quantities, all CTAs meet at a grid
// barrier, each then finalises the reductions itself (the same fixed order
// as the prepass kernel, so results are bit-identical to the two-kernel
// path), CTA 0 runs the prepass scalar logic, and the sensor proceeds with
// its thresholds.  sel 0 then stands for the step's prepass (time step,
// Mach control), sel 1, 2 for the stage prepasses and sel 3 for the
// hyperviscosity sensor's.
template <typename T, bool NEAR, bool FUSED>
__global__ void __launch_bounds__(kSensorThreads, sizeof(T) == 8 ? 1 : HITB200_SENSOR_MIN_BLOCKS)
    sensor_kernel(const SolveDev* __restrict__ solves, const Work* __restrict__ work, int sel,
                  int enf, int want_visc, Bind bind, uint8_t* __restrict__ mask_out) {
  extern __shared__ __align__(16) unsigned char smem[];
  const Work wk = work[blockIdx.x];
  const SolveDev& S = solves[wk.solve];
  const double* sc = S.scal;
  // Launched after the prepass of its state, the unfused sensor stages that
  // state (written two or more kernels earlier, so complete when this CTA
  // starts: the prepass releases its dependents only after its own wait) and
  // waits for the prepass only before it reads the thresholds.  The fused
  // form computes the prepass itself and waits first.
  if constexpr (FUSED) pdl_wait();
  // the hyperviscosity flag is written by the step's first kernel
  if (!bind.use && sel == 3 && sc[S_HV_STEP] == 0.0) return;
  if constexpr (FUSED) {
    if (!bind.use && sel != 3 && sel != 0 && sc[S_ACTIVE] == 0.0) return;
  }
  const int pre_mode = sel == 0 ? PRE_STEP : (sel == 3 ? PRE_SENSOR : PRE_STAGE);
  int pre_slots = 0;
  if constexpr (FUSED) {
    __shared__ PreShared<T> pre_sh;
    pre_slots = prepass_tile<T>(S, wk, sel == 3 ? 1 : sel, pre_mode, sel == 3 ? 0 : 1, bind, true, pre_sh);
  }
  const double* q = bind.use ? bind.qin : (sel == 3 ? S.q1 : stage_in(S, sel));
  uint8_t* mask = bind.use ? mask_out : S.mask;
  const int nx = S.nx, ny = S.ny, per = S.periodic;
  const size_t plane = (size_t)nx * ny;
  const int W = S.width, HW = sensor_halo(W);
  const int SX = kSenTX + 2 * HW, SY = kSenTY + 2 * HW;
  const int x0 = wk.a, y0 = wk.b;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5, nty = blockDim.x >> 5;
  const T g = T(S.gamma);
  const T igm1 = T(1.0 / (S.gamma - 1.0));
  T* RHO = reinterpret_cast<T*>(smem);
  T* U = RHO + SX * SY;
  T* V = U + SX * SY;
  T* P = V + SX * SY;
  T* E = P + SX * SY;
  const int RX = kSenTX + 2 * W, RY = kSenTY + 2 * W;
  uint8_t* RAW = reinterpret_cast<uint8_t*>(E + SX * SY);
  uint8_t* ROW = RAW + RX * RY;
  const int off = HW - W;                 // smem offset of raw index 0

  // ---- staged primitives of the tile and its (width + 1) halo ----
  const float isx = 1.0f / (float)SX;
#pragma unroll 2
  for (int idx = threadIdx.x; idx < SX * SY; idx += blockDim.x) {
    const int a = row_of(idx, SX, isx), b = idx - a * SX;
    const int gj = fold_node(y0 - HW + a, ny, per), gi = fold_node(x0 - HW + b, nx, per);
    const size_t o = (size_t)gj * nx + gi;
    T q0 = T(__ldcg(q + o)), q1 = T(__ldcg(q + o + plane)), q2 = T(__ldcg(q + o + 2 * plane)),
      q3 = T(__ldcg(q + o + 3 * plane));
    if constexpr (sizeof(T) == 8) {
      if (enf) enforce_node(q0, q1, q2, q3, g);
      const Prim<T> p = primitives(q0, q1, q2, q3, g);
      RHO[idx] = p.rho;
      U[idx] = p.u;
      V[idx] = p.v;
      P[idx] = p.p;
      E[idx] = p.p / (p.rho * (g - T(1)));
    } else {
      const T rho = q0 > T(kRhoFloor) ? q0 : T(kRhoFloor);
      const T rinv = __frcp_rn(rho);
      T u = q1 * rinv, v = q2 * rinv;
      const T kin = T(0.5) * rho * (u * u + v * v);
      T pr = (g - T(1)) * (q3 - kin);
      if (enf) {
        q1 = rho * u;
        q2 = rho * v;
        q3 = pr > T(kPFloor) ? q3 : T(kPFloor) / (g - T(1)) + kin;
        u = q1 * rinv;
        v = q2 * rinv;
        pr = (g - T(1)) * (q3 - T(0.5) * rho * (u * u + v * v));
      }
      pr = pr > T(kPFloor) ? pr : T(kPFloor);
      RHO[idx] = rho;
      U[idx] = u;
      V[idx] = v;
      P[idx] = pr;
      E[idx] = pr * rinv * igm1;
    }
  }
  __syncthreads();
  const T thr = T(S.jump_thr);
  const T tdx = T(2.0 * S.dx), tdy = T(2.0 * S.dy), hx = T(S.dx), hy = T(S.dy);
  const T itdx = T(1.0 / (2.0 * S.dx)), itdy = T(1.0 / (2.0 * S.dy));
  const float irx = 1.0f / (float)RX;
  const int nstrip = (RY + 3) >> 2;
  // FP32 without near counting: the largest test margin (pair_margin,
  // curv_margin) per node and quantity, and the velocity gradients, are
  // formed here, before the wait for the prepass (while its last CTA
  // finishes the reductions), and compared with its thresholds after it:
  // 512^2 FP32 step 0.2376 -> 0.2163 ms.  The other forms test node by node
  // after the wait, with the same FP32 decision.
  constexpr bool kMargin = sizeof(T) == 4 && !NEAR;
  const int RXY = RX * RY;
  float* MG = reinterpret_cast<float*>(smem + sensor_margin_off(W, (int)sizeof(T)));  // [5][RY][RX]
  if constexpr (kMargin) {
    for (int t = threadIdx.x; t < RX * nstrip; t += blockDim.x) {
      const int s = row_of(t, RX, irx), br = t - s * RX;
      const int ar0 = 4 * s, nrow = min(4, RY - ar0);
      const int gi = x0 - W + br;
      const int c0 = (ar0 + off) * SX + br + off;  // staged index of raw node (ar0, br)
      auto quantity = [&](const T* A, float* out) {
        T col[6], lf[4], rt[4];
#pragma unroll
        for (int j = 0; j < 6; ++j) col[j] = j <= nrow + 1 ? A[c0 + (j - 1) * SX] : T(0);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          lf[k] = k < nrow ? A[c0 + k * SX - 1] : T(0);
          rt[k] = k < nrow ? A[c0 + k * SX + 1] : T(0);
        }
        T my[5];
#pragma unroll
        for (int j = 0; j < 5; ++j) my[j] = pair_margin(col[j], col[j + 1], thr);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          if (k >= nrow) continue;
          T m = fmax(my[k], my[k + 1]);
          m = fmax(m, pair_margin(lf[k], col[k + 1], thr));
          m = fmax(m, pair_margin(col[k + 1], rt[k], thr));
          m = fmax(m, curv_margin(lf[k], col[k + 1], rt[k], thr));
          m = fmax(m, curv_margin(col[k], col[k + 1], col[k + 2], thr));
          out[(ar0 + k) * RX + br] = m;
        }
      };
      quantity(RHO, MG);
      quantity(P, MG + RXY);
      quantity(E, MG + 2 * RXY);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (k >= nrow) continue;
        const int gj = y0 - W + ar0 + k;
        const int c = c0 + k * SX;
        const bool cx = per || (gi > 0 && gi < nx - 1), cy = per || (gj > 0 && gj < ny - 1);
        T dudx = T(0), dvdy = T(0);
        if (cx) dudx = dq(U[c + 1], U[c - 1], tdx, itdx);
        else if (nx > 1) dudx = gi == 0 ? (U[c + 1] - U[c]) / hx : (U[c] - U[c - 1]) / hx;
        if (cy) dvdy = dq(V[c + SX], V[c - SX], tdy, itdy);
        else if (ny > 1) dvdy = gj == 0 ? (V[c + SX] - V[c]) / hy : (V[c] - V[c - SX]) / hy;
        MG[3 * RXY + (ar0 + k) * RX + br] = dudx + dvdy;
        if (S.shear_on) {
          T dvdx = T(0), dudy = T(0);
          if (cx) dvdx = dq(V[c + 1], V[c - 1], tdx, itdx);
          else if (nx > 1) dvdx = gi == 0 ? (V[c + 1] - V[c]) / hx : (V[c] - V[c - 1]) / hx;
          if (cy) dudy = dq(U[c + SX], U[c - SX], tdy, itdy);
          else if (ny > 1) dudy = gj == 0 ? (U[c + SX] - U[c]) / hy : (U[c] - U[c - SX]) / hy;
          MG[4 * RXY + (ar0 + k) * RX + br] = fabs(dvdx - dudy);
        }
      }
    }
  }
  if constexpr (!FUSED) {
    pdl_wait();  // below: the prepass's thresholds and the solve's flags
    // a finished solve's launch is a no-op
    if (!bind.use && sel != 3 && sc[S_ACTIVE] == 0.0) return;
  }
  pdl_release();

  double l_eps_r, l_eps_p, l_eps_e, l_comp, l_shear;
  if constexpr (FUSED) {
    // all tiles' partials are written: finalise them here (the same fixed
    // order in every CTA), thresholds exactly as prepass_scalars forms them
    grid_barrier(&S.counters[4], &S.counters[5], gridDim.x, &S.counters[6]);
    __shared__ double fred[R_FIXED + 4 * kMaxDrag];
    __shared__ double fchunk[kPreThreads];
    prepass_finalize(S, pre_slots, fred, fchunk);
    // The last CTA past the barrier writes the scalar block (every CTA holds
    // the same reductions) and reports a wait that ran out: by then every
    // CTA that gave up has set the flag.
    if (threadIdx.x == 0) {
      __threadfence();
      if (atomicAdd(&S.counters[7], 1u) == gridDim.x - 1u) {
        S.counters[7] = 0u;
        prepass_scalars(S, fred, S.scal, pre_mode, false);
        if (atomicExch(&S.counters[6], 0u))
          S.scal[S_STATUS] = (double)((int)S.scal[S_STATUS] | ST_BARRIER);
      }
    }
    const double N = (double)nx * (double)ny;
    const double div_rms = sqrt(fred[R_DIV2] / N), vort_rms = sqrt(fred[R_VORT2] / N);
    l_comp = div_rms > 1e-12 ? -S.comp_thr * div_rms : -INFINITY;
    l_shear = (S.shear_on && vort_rms > 1e-12) ? S.shear_thr * vort_rms : INFINITY;
    l_eps_r = 1e-14 + 1e-12 * fred[R_RHO];
    l_eps_p = 1e-14 + 1e-12 * fred[R_P];
    l_eps_e = 1e-14 + 1e-12 * fred[R_E];
  } else {
    l_eps_r = sc[S_EPS_RHO];
    l_eps_p = sc[S_EPS_P];
    l_eps_e = sc[S_EPS_E];
    l_comp = sc[S_COMP_LIM];
    l_shear = sc[S_SHEAR_LIM];
  }
  const T eps_r = T(l_eps_r), eps_p = T(l_eps_p), eps_e = T(l_eps_e);
  const T comp_lim = T(l_comp), shear_lim = T(l_shear);
  const bool comp_on = isfinite(comp_lim), shear_on = isfinite(shear_lim);
  const T tol = T(32) * type_eps<T>();

  // ---- raw flags on the tile plus a width-wide ring ----
  // Thread task: a strip of up to 4 consecutive raw rows of one raw column.
  // The strip's column values (rows -1 .. +4) and its left / right
  // neighbours stay in registers; each y edge of the strip is tested once,
  // x edges and curvatures per node, with the reference's operand order.
  int near_count = 0;
  if constexpr (kMargin) {
    __syncthreads();  // the margins of every raw node
    const T lim_r = thr * eps_r, lim_p = thr * eps_p, lim_e = thr * eps_e;
    for (int idx = threadIdx.x; idx < RXY; idx += blockDim.x) {
      const int ar = row_of(idx, RX, irx), br = idx - ar * RX;
      const int gj = y0 - W + ar, gi = x0 - W + br;
      bool mk = MG[idx] > lim_r || MG[RXY + idx] > lim_p || MG[2 * RXY + idx] > lim_e;
      if (comp_on) mk = mk || MG[3 * RXY + idx] < comp_lim;
      if (shear_on) mk = mk || MG[4 * RXY + idx] > shear_lim;
      if (!per && S.boundary_guard > 0) {
        const int bg = S.boundary_guard;
        if (gj < bg || gj >= ny - bg || gi < bg || gi >= nx - bg) mk = true;
      }
      if (!per && !(gj >= 0 && gj < ny && gi >= 0 && gi < nx)) mk = false;
      RAW[idx] = mk ? 1 : 0;
    }
  }
  for (int t = threadIdx.x; !kMargin && t < RX * nstrip; t += blockDim.x) {
    const int s = row_of(t, RX, irx), br = t - s * RX;
    const int ar0 = 4 * s, nrow = min(4, RY - ar0);
    const int gi = x0 - W + br;
    const int c0 = (ar0 + off) * SX + br + off;  // staged index of raw node (ar0, br)
    bool m[4] = {false, false, false, false}, nr[4] = {false, false, false, false};
    // jumps and curvatures of one staged quantity
    auto quantity = [&](const T* A, T eps) {
      T col[6], lf[4], rt[4];
#pragma unroll
      for (int j = 0; j < 6; ++j) col[j] = j <= nrow + 1 ? A[c0 + (j - 1) * SX] : T(0);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        lf[k] = k < nrow ? A[c0 + k * SX - 1] : T(0);
        rt[k] = k < nrow ? A[c0 + k * SX + 1] : T(0);
      }
      bool ey[5];
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        bool nn = false;
        ey[j] = j <= nrow && pair_gt<T, NEAR>(col[j], col[j + 1], eps, thr, tol, nn);
        if (NEAR && j <= nrow) {
          if (j < 4) nr[j] = nr[j] || nn;
          if (j > 0) nr[j - 1] = nr[j - 1] || nn;
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (k >= nrow) continue;
        bool nn = false;
        bool f = ey[k] | ey[k + 1];
        f |= pair_gt<T, NEAR>(lf[k], col[k + 1], eps, thr, tol, nn);
        f |= pair_gt<T, NEAR>(col[k + 1], rt[k], eps, thr, tol, nn);
        f |= curv_gt<T, NEAR>(lf[k], col[k + 1], rt[k], eps, thr, tol, nn);
        f |= curv_gt<T, NEAR>(col[k], col[k + 1], col[k + 2], eps, thr, tol, nn);
        m[k] = m[k] || f;
        if (NEAR) nr[k] = nr[k] || nn;
      }
    };
    quantity(RHO, eps_r);
    quantity(P, eps_p);
    quantity(E, eps_e);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k >= nrow) continue;
      const int ar = ar0 + k, gj = y0 - W + ar;
      const bool inside = gj >= 0 && gj < ny && gi >= 0 && gi < nx;
      const int c = c0 + k * SX;
      bool mk = m[k], near = NEAR && nr[k];
      // sensor velocity gradients: central; first-order one-sided at outflow edges
      const bool cx = per || (gi > 0 && gi < nx - 1), cy = per || (gj > 0 && gj < ny - 1);
      if (comp_on) {
        T dudx = T(0), dvdy = T(0);
        if (cx) dudx = dq(U[c + 1], U[c - 1], tdx, itdx);
        else if (nx > 1) dudx = gi == 0 ? (U[c + 1] - U[c]) / hx : (U[c] - U[c - 1]) / hx;
        if (cy) dvdy = dq(V[c + SX], V[c - SX], tdy, itdy);
        else if (ny > 1) dvdy = gj == 0 ? (V[c + SX] - V[c]) / hy : (V[c] - V[c - SX]) / hy;
        const T div = dudx + dvdy;
        mk = mk || div < comp_lim;
        if (NEAR) near = near || fabs(div - comp_lim) <= tol * fabs(comp_lim);
      }
      if (shear_on) {
        T dvdx = T(0), dudy = T(0);
        if (cx) dvdx = dq(V[c + 1], V[c - 1], tdx, itdx);
        else if (nx > 1) dvdx = gi == 0 ? (V[c + 1] - V[c]) / hx : (V[c] - V[c - 1]) / hx;
        if (cy) dudy = dq(U[c + SX], U[c - SX], tdy, itdy);
        else if (ny > 1) dudy = gj == 0 ? (U[c + SX] - U[c]) / hy : (U[c] - U[c - SX]) / hy;
        const T av = fabs(dvdx - dudy);
        mk = mk || av > shear_lim;
        if (NEAR) near = near || fabs(av - shear_lim) <= tol * shear_lim;
      }
      if (!per && S.boundary_guard > 0) {
        const int bg = S.boundary_guard;
        if (gj < bg || gj >= ny - bg || gi < bg || gi >= nx - bg) mk = true;
      }
      if (!per && !inside) mk = false;
      RAW[ar * RX + br] = mk ? 1 : 0;
      // nodes of this tile whose metric sits within roundoff of a threshold
      if (NEAR && near && inside && ar >= W && ar < W + kSenTY && br >= W && br < W + kSenTX)
        ++near_count;
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < RY * kSenTX; idx += blockDim.x) {
    const int ar = idx >> 5, bx = idx & 31;
    uint8_t v = 0;
    for (int d = 0; d <= 2 * W; ++d) v |= RAW[ar * RX + bx + d];
    ROW[idx] = v;
  }
  __syncthreads();
  for (int a = ty; a < kSenTY; a += nty) {
    const int gj = y0 + a, gi = x0 + tx;
    if (gj >= ny || gi >= nx) continue;
    uint8_t v = 0;
    for (int d = 0; d <= 2 * W; ++d) v |= ROW[(a + d) * kSenTX + tx];
    mask[(size_t)gj * nx + gi] = v;
  }
  if (NEAR) {
    near_count = warp_sum(near_count);
    if (tx == 0 && near_count > 0) atomicAdd(S.near_count, near_count);
  }

  if (!want_visc || S.mu == 0.0) return;
  // viscous stress and heat-flux divergence (OOP/equations.py:232-267), as the
  // reference evaluates it: velocity / temperature gradients, then stresses
  // and energy fluxes at every node of the tile plus a one-node ring, then
  // their central differences.
  const T mu = T(S.mu), kap = T(S.kappa), rgas = T(S.gas_r);
  const T two3 = T(2.0 / 3.0);
  T* TXX = reinterpret_cast<T*>(smem + sensor_flag_end(W, (int)sizeof(T)));
  T* TYY = TXX + kVisX * kVisY;
  T* TXY = TYY + kVisX * kVisY;
  T* QX = TXY + kVisX * kVisY;
  T* QY = QX + kVisX * kVisY;
  __syncthreads();  // E (internal energy) is free: the mask is complete
  // temperature p / (rho R): FP64 divides as the reference; FP32 forms
  // (p * (1 / rho)) / R with the staging's reciprocal, as the step sensor does
  const T irg = T(1.0 / S.gas_r);
  for (int idx = threadIdx.x; idx < SX * SY; idx += blockDim.x) {
    if constexpr (sizeof(T) == 8) E[idx] = P[idx] / (RHO[idx] * rgas);
    else E[idx] = (P[idx] * __frcp_rn(RHO[idx])) * irg;
  }
  __syncthreads();
  const float ivx = 1.0f / (float)kVisX;
  for (int idx = threadIdx.x; idx < kVisX * kVisY; idx += blockDim.x) {
    const int a = row_of(idx, kVisX, ivx), b = idx - a * kVisX;
    const int c = (a + HW - 1) * SX + (b + HW - 1);
    const T ux = dq(U[c + 1], U[c - 1], tdx, itdx), vx = dq(V[c + 1], V[c - 1], tdx, itdx);
    const T uy = dq(U[c + SX], U[c - SX], tdy, itdy), vy = dq(V[c + SX], V[c - SX], tdy, itdy);
    const T dv = ux + vy;
    const T txx = T(2) * mu * ux - two3 * mu * dv;
    const T tyy = T(2) * mu * vy - two3 * mu * dv;
    const T txy = mu * (uy + vx);
    const T tx_ = dq(E[c + 1], E[c - 1], tdx, itdx), ty_ = dq(E[c + SX], E[c - SX], tdy, itdy);
    TXX[idx] = txx;
    TYY[idx] = tyy;
    TXY[idx] = txy;
    QX[idx] = U[c] * txx + V[c] * txy + kap * tx_;
    QY[idx] = U[c] * txy + V[c] * tyy + kap * ty_;
  }
  __syncthreads();
  T* visp = reinterpret_cast<T*>(S.vis);
  for (int a = ty; a < kSenTY; a += nty) {
    const int gj = y0 + a, gi = x0 + tx;
    if (gj >= ny || gi >= nx) continue;
    const int i = (a + 1) * kVisX + tx + 1;
    const T r1 = dq(TXX[i + 1], TXX[i - 1], tdx, itdx) + dq(TXY[i + kVisX], TXY[i - kVisX], tdy, itdy);
    const T r2 = dq(TXY[i + 1], TXY[i - 1], tdx, itdx) + dq(TYY[i + kVisX], TYY[i - kVisX], tdy, itdy);
    const T r3 = dq(QX[i + 1], QX[i - 1], tdx, itdx) + dq(QY[i + kVisX], QY[i - kVisX], tdy, itdy);
    const size_t o = (size_t)gj * nx + gi;
    visp[o] = r1;
    visp[plane + o] = r2;
    visp[2 * plane + o] = r3;
  }
}

// =============================================================================
// Line sweeps.  A CTA owns R whole grid lines (rows for x, columns for y) of
// one solve, 128 threads per line; thread t of a line owns the MN
// consecutive nodes [t MN, t MN + MN) and keeps them in registers from the
// face fluxes to the epilogue:
//   L  stage the flux and enforced state of every node of the lines plus a
//      halo (periodic wrap or clamped edge) in shared memory, and the mask;
//   W  the WENO7 face fluxes that a flagged face needs, compacted by warp
//      ballots over 32-face chunks;
//   H  per component, the hybrid face fluxes of the thread's MN + 1 faces
//      (6-point compact flux, or the compactised WENO7 flux on flagged
//      faces) and raw_i = (H_{i+1/2} - H_{i-1/2}) / h of its nodes;
//   S  the compact tridiagonal solve 3/8 d_{i-1} + d_i + 3/8 d_{i+1} = raw_i
//      as two first-order recurrences (factorisation below): each thread runs
//      them over its nodes, and a scan of the per-thread affine maps across
//      the line (warp shuffles, then the line's 4 warps through shared
//      memory) supplies each thread's carry-in;
//   E  the fused epilogue (y: partial rhs -dG/dy; x: full rhs, sources, RK
//      stage combine, clean filter and outflow guard).
//
// Factorisation: a s^-1 + 1 + a s = (-a/rho)(1 - rho s^-1)(1 - rho s) with
// rho = (sqrt(1 - 4 a^2) - 1) / (2 a) = (sqrt(7) - 4) / 3 for a = 3/8, so
// d = (-rho/a) (1 - rho s)^-1 (1 - rho s^-1)^-1 raw: a forward recurrence
// y_i = raw_i + rho y_{i-1} and a backward one z_i = y_i + rho z_{i+1}.
// Periodic lines close each recurrence exactly (y_{-1} = y_{n-1} gives
// y_{-1} = y~_{n-1} / (1 - rho^n)); outflow lines (identity first and last
// rows, riemann_config3.py:244-264) add the two homogeneous solutions rho^i
// and rho^(n-1-i) fitted to the end rows.
// =============================================================================
constexpr double kRhoSolve = -0.45141622964513645;  // (sqrt(7) - 4) / 3
constexpr double kSolveScale = 1.2037766123870306;  // -rho / a
constexpr int kPowTab = 128;                         // rho^k below 1e-43 beyond this

// rho^k, k in [0, kPowTab); filled once by the host (hitb200_plan_create).
// Outflow sweeps copy it to shared memory while they stage their lines: read
// from global memory at the end-row correction, every CTA of a launch asked
// for the same few lines of L2 at once.
__device__ double g_rho_pow[kPowTab];

constexpr int kSweepHalo = 8;  // staged nodes left of node 0 (WENO reads 5)
#ifndef HITB200_SWEEP_X_BULK
#define HITB200_SWEEP_X_BULK 1
#endif
// The x sweep of the FP32-bulk form stages its rows by bulk copies (the
// TMA unit) into shared memory.  Bit-identical to the load path; measured
// on a B200, 8 x 512^2 batched HIT step 1.063 -> 1.053 ms, sweep_x 66.1 ->
// 64.7 us per launch (with separate landing rows, costing two resident
// CTAs per SM: 1.067 -> 1.202 ms).
constexpr bool kSweepXBulk = HITB200_SWEEP_X_BULK != 0;
constexpr unsigned long long kBulkWaitNs = 2000000000ull;  // bound of a copy wait

// Shared memory of one sweep CTA holding R lines of n nodes:
//   FQ  [R][8][LS]  flux F_c (c < 4) and enforced state Q_c (c >= 4) of nodes
//                   -8 .. LS - 9; node i at index i + 8 so that each
//                   thread's nodes start on a 16-byte boundary.  Reused by
//                   the x-sweep epilogue for the new rows (FP64) when guard
//                   cells are written.
//   WB  [R][4][LW]  WENO face fluxes W_{f+1/2}, f in [-2, n], of needed faces
//   MK  [R][n + 2]  sensor mask of nodes -1 .. n
template <typename T>
struct SweepLayout {
  int n, LS, LW, R, LQ;
  __host__ __device__ SweepLayout(int n_, int R_) : n(n_), R(R_) {
    LS = (kSweepHalo + n + 16 + 7) & ~7;
    // a line's 8 staged rows, plus 8 elements: the lines of a y panel, which
    // a warp's lanes stage at the same node, start on different banks
    LQ = 8 * LS + 8;
    LW = (n + 3 + 3) & ~3;
  }
  // byte offsets of the regions; the kernel and the host use the same ones
  __host__ __device__ size_t off_wb() const { return (size_t)R * LQ * sizeof(T); }
  __host__ __device__ size_t off_mk() const { return off_wb() + (size_t)R * 4 * LW * sizeof(T); }
  __host__ __device__ size_t bytes() const {
    return (off_mk() + (size_t)R * (n + 2) + 15) & ~(size_t)15;
  }
};

enum SweepMode : int { SW_STAGE = 0, SW_DERIV = 1, SW_RHS = 2 };

// rhs terms of rhs_with_forcing (OOP/hit2d.py:847-867) that a solve carries:
// 1 inviscid, 2 viscous, 4 forcing, 8 drag, 16 cooling.
__device__ __forceinline__ int fused_terms(const SolveDev& S) {
  return 1 | (S.mu > 0.0 ? 2 : 0) | (S.forcing_on ? 4 : 0) | (S.drag_on ? 8 : 0) |
         (S.cooling_on ? 16 : 0);
}

constexpr double kB1C1 = 1.0 / 20.0 + (-1.0 / 480.0);
constexpr double kA1B1C1 = 25.0 / 32.0 + 1.0 / 20.0 + (-1.0 / 480.0);

// 6-point compact interface flux C_{i+1/2} (OOP/spatial_operator.py:179-189).
template <typename T>
__device__ __forceinline__ T compact_face(const T* F, int s) {
  return T(-1.0 / 480.0) * (F[s + 3] + F[s - 2]) + T(kB1C1) * (F[s + 2] + F[s - 1]) +
         T(kA1B1C1) * (F[s + 1] + F[s]);
}

// WENO7 flux W_{i+1/2} of the Lax-Friedrichs split f+- = (F +- alpha Q) / 2
// (OOP/spatial_operator.py:192-211).
template <typename T>
__device__ __forceinline__ T weno_face(const T* F, const T* Q, int s, T alpha) {
  T fp[8], fm[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const T f = F[s - 3 + k], aq = alpha * Q[s - 3 + k];
    fp[k] = T(0.5) * (f + aq);
    fm[k] = T(0.5) * (f - aq);
  }
  return weno7(fp[0], fp[1], fp[2], fp[3], fp[4], fp[5], fp[6]) +
         weno7(fm[7], fm[6], fm[5], fm[4], fm[3], fm[2], fm[1]);
}

// Position of the j-th (0-based) set bit of `mask` (j < popc(mask)).
__device__ __forceinline__ int nth_set_bit(unsigned mask, int j) {
  int pos = 0;
#pragma unroll
  for (int w = 16; w > 0; w >>= 1) {
    const unsigned lo = mask & ((1u << w) - 1u);
    const int c = __popc(lo);
    if (j >= c) {
      j -= c;
      mask >>= w;
      pos += w;
    } else {
      mask = lo;
    }
  }
  return pos;
}

// Outflow guard source index: guard cells copy cell g (n-g-1), riemann_config3.py:419-429.
__device__ __forceinline__ int guard_src(int i, int n, int g) {
  return i < g ? g : (i > n - g - 1 ? n - g - 1 : i);
}

// Affine map y -> m y + a[c] of the recurrence over a run of nodes (one
// multiplier for all four components, which share rho).
template <typename T>
struct Affine {
  T m, a[4];
};

// Loads v[j] = row[base + j], j < N, from shared memory; 16-byte vector loads
// when the start is aligned (always, for the thread layout of the sweep).
// A thread's `len` consecutive values (len <= N) stored from index 0 of dst:
// 16-byte stores when the run is whole and dst is aligned to 16 bytes (the
// sweeps' derivative rows: every thread starts at a multiple of N of an
// aligned row), so that the lanes' stores fall on different banks.
template <typename T, int N>
__device__ __forceinline__ void store_run(T* dst, const T (&v)[N], int len) {
  constexpr int PER = 16 / sizeof(T);  // values per 16-byte store
  if constexpr (N % PER == 0) {
    if (len == N) {
#pragma unroll
      for (int k = 0; k < N; k += PER) {
        if constexpr (sizeof(T) == 4)
          *reinterpret_cast<float4*>(dst + k) = make_float4(v[k], v[k + 1], v[k + 2], v[k + 3]);
        else
          *reinterpret_cast<double2*>(dst + k) = make_double2(v[k], v[k + 1]);
      }
      return;
    }
  }
#pragma unroll
  for (int k = 0; k < N; ++k)
    if (k < len) dst[k] = v[k];
}

template <typename T, int N>
__device__ __forceinline__ void load_run(const T* row, int base, T (&v)[N]) {
  constexpr int VEC = 16 / sizeof(T);
  if constexpr (N % VEC == 0) {
    if (((base * (int)sizeof(T)) & 15) == 0) {
#pragma unroll
      for (int j = 0; j < N; j += VEC) {
        if constexpr (sizeof(T) == 4) {
          const float4 f = *reinterpret_cast<const float4*>(row + base + j);
          v[j] = f.x;
          v[j + 1] = f.y;
          v[j + 2] = f.z;
          v[j + 3] = f.w;
        } else {
          const double2 f = *reinterpret_cast<const double2*>(row + base + j);
          v[j] = f.x;
          v[j + 1] = f.y;
        }
      }
      return;
    }
  }
#pragma unroll
  for (int j = 0; j < N; ++j) v[j] = row[base + j];
}

// v[j] = p[j] for j < len (0 beyond), with 16-byte vector loads through the
// read-only path when the whole run is present and aligned.
template <typename T, int N>
__device__ __forceinline__ void gload_run(const T* p, int len, T (&v)[N]) {
  constexpr int VEC = 16 / sizeof(T);
  if constexpr (N % VEC == 0) {
    if (len == N && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
#pragma unroll
      for (int j = 0; j < N; j += VEC) {
        if constexpr (sizeof(T) == 4) {
          const float4 f = __ldg(reinterpret_cast<const float4*>(p + j));
          v[j] = f.x;
          v[j + 1] = f.y;
          v[j + 2] = f.z;
          v[j + 3] = f.w;
        } else {
          const double2 f = __ldg(reinterpret_cast<const double2*>(p + j));
          v[j] = f.x;
          v[j + 1] = f.y;
        }
      }
      return;
    }
  }
#pragma unroll
  for (int j = 0; j < N; ++j) v[j] = j < len ? p[j] : T(0);
}

// One sweep of the split RHS over R whole grid lines (rows for AXIS 0, columns
// for AXIS 1), 128 threads per line, MN nodes per thread.  The y sweep runs
// first and leaves -dG/dy in the partial-rhs buffer; the x sweep runs second
// and, in mode SW_STAGE, finishes the stage:
//   stage 0: q1 = clean(q + dt L)
//   stage 1: q2 = clean(3/4 q + 1/4 (q1 + dt L))
//   stage 2:      clean(1/3 q + 2/3 (q2 + dt L))     (OOP/time_operator.py:21-26)
// with L = -dF/dx - dG/dy + viscous + forcing + drag + cooling and clean the
// enforce filter plus, on outflow grids, the guard cells.
// V consecutive elements (V = 1 or 2) in one access; V = 2 needs a pointer
// aligned to 2 elements.
template <int V>
struct VecWidth {
  static constexpr int value = V;
};
template <typename E>
struct Vec2Of;
template <>
struct Vec2Of<double> {
  using type = double2;
};
template <>
struct Vec2Of<float> {
  using type = float2;
};
template <int V, typename E>
__device__ __forceinline__ void vld(const E* p, E (&v)[V]) {
  if constexpr (V == 2) {
    const typename Vec2Of<E>::type t = *reinterpret_cast<const typename Vec2Of<E>::type*>(p);
    v[0] = t.x;
    v[1] = t.y;
  } else {
    v[0] = *p;
  }
}
template <int V, typename E>
__device__ __forceinline__ void vst(E* p, const E (&v)[V]) {
  if constexpr (V == 2) {
    typename Vec2Of<E>::type t;
    t.x = v[0];
    t.y = v[1];
    *reinterpret_cast<typename Vec2Of<E>::type*>(p) = t;
  } else {
    *p = v[0];
  }
}

// Line of a node index `idx` among consecutive runs of `len` (x lines of a
// work item: at most 2, or 4 in the persistent stage kernel).
template <int XR>
__device__ __forceinline__ int xline_of(int idx, int len) {
  if constexpr (XR <= 2) return idx >= len ? 1 : 0;
  else return (idx >= len ? 1 : 0) + (idx >= 2 * len ? 1 : 0) + (idx >= 3 * len ? 1 : 0);
}

// Statically sized shared memory of a sweep work item; XR is the most x lines
// an item holds (1 for the y sweep, which has no drag rows).
template <typename T, int XR>
struct SweepShared {
  Affine<T> scan_f[4][4], scan_b[4][4];  // per line, per warp totals
  T ends[4][4][4];                         // raw_0, raw_n-1, p_0, p_n-1
  T rpow[kPowTab];                         // rho^k for the outflow end rows
  double2 dpx[XR][kMaxKx + 1], dpy[XR][kMaxKx + 1];  // drag band rows (x sweep)
  unsigned long long tbar;                 // bulk-copy barrier (x sweep)
};

// The work of one CTA of the sweep (work item wk), or of a group of its
// threads.  Dep is the wait for the previous phase: PdlDep in the sweep
// kernels (programmatic dependent launch), the persistent stage kernel's
// counter wait otherwise (Dep::kQueued; then every value the same launch may
// have written is read through L2).  Dep also names the item's threads
// (tid, nthreads), their barrier (sync, sync_or) and the most x lines an
// item holds (kXR).
template <typename T, int AXIS, int MN, typename Dep, typename SH>
__device__ __forceinline__ void sweep_body(const SolveDev* __restrict__ solves, const Work wk, int stage,
                                           int mode, const Bind& bind, unsigned char* smem, SH& sh,
                                           const Dep& dep) {
  constexpr bool QD = Dep::kQueued;
  constexpr int XR = Dep::kXR;
  // the item's threads (the CTA, or a group of it): read where used, as the
  // special registers they are for the CTA
  const auto tid = [&]() { return dep.tid(); };
  const auto nthr = [&]() { return dep.nthreads(); };
  auto& scan_f = sh.scan_f;
  auto& scan_b = sh.scan_b;
  auto& ends = sh.ends;
  const SolveDev& S = solves[wk.solve];
  const double* sc = S.scal;
  const int nx = S.nx, ny = S.ny, per = S.periodic;
  const int n = AXIS == 0 ? nx : ny;
  const size_t plane = (size_t)nx * ny;
  const int line0 = wk.a, R = wk.b;
  // ranges the plans guarantee (lines of 1..kMaxLine nodes, items of 1..4
  // lines starting inside the grid), stated for the index arithmetic
  if constexpr (AXIS == 0) {
    __builtin_assume(nx >= 1 && nx <= kMaxLine && ny >= 1 && ny <= kMaxLine);
    __builtin_assume(R >= 1 && R <= 4 && line0 >= 0 && line0 < kMaxLine);
  }
  const int rsh = R > 2 ? 2 : (R > 1 ? 1 : 0);  // R is 1 or 2 (x lines), up to 4 (y lines)
  const int RL = 1 << rsh;
  const SweepLayout<T> L(n, RL);
  const int LS = L.LS, LW = L.LW, LQ = L.LQ;
  const T g = T(S.gamma);
  const double h = AXIS == 0 ? S.dx : S.dy;
  const double* qin = bind.use ? bind.qin : stage_in(S, stage);
  const uint8_t* mask = bind.use ? bind.mask : S.mask;
  T* FQ = reinterpret_cast<T*>(smem);
  T* WB = reinterpret_cast<T*>(smem + L.off_wb());
  uint8_t* MK = smem + L.off_mk();
  const int lane = tid() & 31, warp = tid() >> 5, nwarp = nthr() >> 5;
  auto& rpow = sh.rpow;
  auto ldsc = [&](int i) -> double {
    if constexpr (QD) return __ldcg(sc + i);
    else return sc[i];
  };
  if (!per)
    for (int t = tid(); t < kPowTab; t += nthr()) rpow[t] = T(__ldg(&g_rho_pow[t]));
  auto rho_pow = [&](int k) -> T { return (k >= 0 && k < kPowTab) ? rpow[k] : T(0); };

  // ---- L: stage flux and enforced state of the lines ---------------------------
  // x lines: consecutive threads take consecutive nodes of a row; y lines:
  // consecutive threads take the R columns of a row, then the next row.
  const int nl = AXIS == 0 ? R * LS : (LS << rsh);
  const T pfl = T(kPFloor) / (g - T(1));  // floor energy of enforce_physical_state
  // one node: enforce_physical_state, then primitive_from_conservative of the
  // result, and the node's flux and enforced state into FQ
  auto stage_node = [&](int r, int p, T a0, T a1, T a2, T a3) {
    const T rho = a0 > T(kRhoFloor) ? a0 : T(kRhoFloor);
    const T rinv = rcp_rn(rho);
    T u = a1 * rinv, v = a2 * rinv;
    const T kin = T(0.5) * rho * (u * u + v * v);
    T pr = (g - T(1)) * (a3 - kin);
    a1 = rho * u;
    a2 = rho * v;
    a3 = pr > T(kPFloor) ? a3 : pfl + kin;
    u = a1 * rinv;
    v = a2 * rinv;
    pr = (g - T(1)) * (a3 - T(0.5) * rho * (u * u + v * v));
    pr = pr > T(kPFloor) ? pr : T(kPFloor);
    const T un = AXIS == 0 ? u : v;
    T* f = FQ + r * LQ + p;
    f[0 * LS] = AXIS == 0 ? a1 : a2;
    f[1 * LS] = a1 * un + (AXIS == 0 ? pr : T(0));
    f[2 * LS] = a2 * un + (AXIS == 0 ? T(0) : pr);
    f[3 * LS] = (a3 + pr) * un;
    f[4 * LS] = rho;
    f[5 * LS] = a1;
    f[6 * LS] = a2;
    f[7 * LS] = a3;
  };
  bool bulk = false;
  if constexpr (AXIS == 0 && sizeof(T) == 4 && kSweepXBulk && !QD) {
    // x lines by bulk copies: the R rows' n interior nodes of each of the four
    // planes land as FP64 in shared memory through the copy engine; the
    // threads fetch the few halo nodes meanwhile
    bulk = !bind.use && (nx & 1) == 0 && (reinterpret_cast<uintptr_t>(qin) & 15) == 0;
  }
  if (bulk) {
    auto& tbar = sh.tbar;
    // The FP64 landing rows [R][4][LS] take the place of FQ ([R][8][LS] of
    // T): each thread moves its nodes' values into registers before the
    // flux staging overwrites them.
    double* SQ = reinterpret_cast<double*>(smem);
    if (tid() == 0) mbar_init(&tbar, 1);
    dep.sync();
    if (tid() == 0) {
      mbar_expect_tx(&tbar, (unsigned)(R * 4 * n * sizeof(double)));
      for (int rr = 0; rr < R; ++rr)
        for (int c = 0; c < 4; ++c)
          bulk_g2s(SQ + (rr * 4 + c) * LS + kSweepHalo, qin + c * plane + (size_t)(line0 + rr) * nx,
                   (unsigned)(n * sizeof(double)), &tbar);
    }
    const int nh = LS - n;  // halo slots of a line: p < kSweepHalo or p >= kSweepHalo + n
    for (int idx = tid(); idx < R * 4 * nh; idx += nthr()) {
      const int rc = idx / nh, h = idx - rc * nh;
      const int pp = h < kSweepHalo ? h : h + n;
      const int gp = fold_node(pp - kSweepHalo, n, per);
      SQ[rc * LS + pp] = __ldcg(qin + (rc & 3) * plane + (size_t)(line0 + (rc >> 2)) * nx + gp);
    }
    // bounded wait for the copies; a CTA whose copies do not land in time
    // reports it (ST_BARRIER at the next prepass) and skips its lines
    const unsigned long long t0 = global_ns();
    unsigned it = 0;
    bool done = mbar_try_wait(&tbar, 0);
    while (!done) {
      if ((++it & 63) == 0 && global_ns() - t0 > kBulkWaitNs) break;
      done = mbar_try_wait(&tbar, 0);
    }
    if (dep.sync_or(!done)) {
      if (tid() == 0) atomicOr(&S.counters[6], 1u);
      const unsigned long long t1 = global_ns();
      while (!mbar_try_wait(&tbar, 0) && global_ns() - t1 < kBulkWaitNs) {
      }
      return;
    }
    // a line's LS nodes over its 128 threads: at most MN + 1 nodes a thread
    T held[4][MN + 1];
#pragma unroll
    for (int j = 0; j <= MN; ++j) {
      const int idx = tid() + j * nthr();
      if (idx < nl) {
        const int r = idx >= LS ? 1 : 0, pp = idx - r * LS;
        const double* sq = SQ + r * 4 * LS + pp;
#pragma unroll
        for (int c = 0; c < 4; ++c) held[c][j] = T(sq[c * LS]);
      }
    }
    dep.sync();
#pragma unroll
    for (int j = 0; j <= MN; ++j) {
      const int idx = tid() + j * nthr();
      if (idx < nl) {
        const int r = idx >= LS ? 1 : 0, pp = idx - r * LS;
        stage_node(r, pp, held[0][j], held[1][j], held[2][j], held[3][j]);
      }
    }
  } else {
#pragma unroll 4
    for (int idx = tid(); idx < nl; idx += nthr()) {
      int r, p;
      if (AXIS == 0) {
        r = xline_of<XR>(idx, LS);
        p = idx - r * LS;
      } else {
        r = idx & (RL - 1);
        p = idx >> rsh;
        if (r >= R) continue;
      }
      const int gp = fold_node(p - kSweepHalo, n, per);
      const size_t o = AXIS == 0 ? (size_t)(line0 + r) * nx + gp : (size_t)gp * nx + line0 + r;
      stage_node(r, p, T(__ldcg(qin + o)), T(__ldcg(qin + o + plane)), T(__ldcg(qin + o + 2 * plane)),
                 T(__ldcg(qin + o + 3 * plane)));
    }
  }
  // The stage input was written two or more kernels earlier (complete when
  // this CTA starts: the previous kernel releases its dependents only after
  // its own wait).  The y sweep reads the mask of the sensor just before it,
  // so it waits here, and then releases the x sweep at once: the x sweep
  // reads the previous kernel's output (the partial rhs) only in its
  // epilogue and waits there, so its CTAs run their line solves in the y
  // sweep's tail (512^2 FP32 step 0.2436 -> 0.2378 ms).  Everything the x
  // sweep reads before its wait (mask, Lax-Friedrichs speed, flags) was
  // written two or more kernels earlier and is read from L2.
  if constexpr (AXIS == 1) {
    dep.wait();
    dep.release();
  } else {
    dep.early();  // below: the mask and the Lax-Friedrichs speed
  }
  // a finished solve's launch is a no-op; its flag is tested once the staging
  // loads are in flight, so that they do not wait for the scalar block
  const bool active = bind.use || ((AXIS == 0 || QD) ? __ldcg(&sc[S_ACTIVE]) : sc[S_ACTIVE]) != 0.0;
  const T alpha = T(AXIS == 0 ? __ldcg(&sc[S_ALPHA_X]) : ldsc(S_ALPHA_Y));
  const int weno_all = S.scheme == 1;
  const int nm = AXIS == 0 ? R * (n + 2) : ((n + 2) << rsh);
  unsigned anyf = 0;  // a flagged node among this thread's
#pragma unroll 4
  for (int idx = tid(); idx < nm; idx += nthr()) {
    int r, p;
    if (AXIS == 0) {
      r = xline_of<XR>(idx, n + 2);
      p = idx - r * (n + 2);
    } else {
      r = idx & (RL - 1);
      p = idx >> rsh;
      if (r >= R) continue;
    }
    const int gp = fold_node(p - 1, n, per);
    const size_t o = AXIS == 0 ? (size_t)(line0 + r) * nx + gp : (size_t)gp * nx + line0 + r;
    const uint8_t mv = weno_all ? 1 : ((AXIS == 0 || QD) ? __ldcg(&mask[o]) : mask[o]);
    MK[r * (n + 2) + p] = mv;
    anyf |= mv;
  }
  // lines without a flagged node (most of a low-Mach HIT solve's) skip the
  // WENO phase and the face flags
  const bool anyflag = dep.sync_or(anyf) != 0;
  if (!active) {
    if constexpr (AXIS == 0) dep.wait();  // keeps the chain of waits unbroken
    return;
  }

  // face il + 1/2 (il in [-1, n-1]) is flagged when node il or il + 1 is
  auto flagged = [&](const uint8_t* mk, int f) -> bool {
    return f >= -1 && f <= n - 1 && (mk[f] | mk[f + 1]);
  };

  // ---- W: WENO fluxes where a flagged face needs them ----------------------------
  // Warp task = 32 consecutive faces of one line; the faces that need W (a
  // flagged face among itself and its neighbours) are found by ballot and
  // their (face, component) pairs are spread over the warp's lanes.
  const int nch = (n + 3 + 31) >> 5;
  for (int task = warp; anyflag && task < R * nch; task += nwarp) {
    int r = 0, ch = task;
    while (ch >= nch) {
      ch -= nch;
      ++r;
    }
    const uint8_t* mk = MK + r * (n + 2) + 1;  // mk[i] = node i, i in [-1, n]
    const int il0 = ch * 32 - 2;
    // Face il needs W when a flagged face lies among il - 1 .. il + 1, that
    // is when one of the nodes il - 1 .. il + 2 is flagged (nodes outside
    // [-1, n] count as unflagged; faces run over [-1, n - 1]).  Bit t of
    // the 35-bit word nb is node il0 - 1 + t; bit `lane` of the OR of its
    // four shifts is face il0 + lane's need.
    const int j0 = il0 - 1 + lane, j1 = il0 + 31 + lane;
    const unsigned b0 = __ballot_sync(kFull, j0 >= -1 && j0 <= n && mk[j0]);
    const unsigned b1 = __ballot_sync(kFull, lane < 3 && j1 <= n && mk[j1]);
    const unsigned long long nb = (unsigned long long)b0 | ((unsigned long long)b1 << 32);
    const int nvalid = n - il0 + 1;  // faces il0 .. n
    const unsigned valid = nvalid >= 32 ? kFull : (nvalid <= 0 ? 0u : (1u << nvalid) - 1u);
    const unsigned bal = (unsigned)(nb | (nb >> 1) | (nb >> 2) | (nb >> 3)) & valid;
    const int items = 4 * __popc(bal);
    for (int k = lane; k < items; k += 32) {
      const int c = k & 3, f = il0 + nth_set_bit(bal, k >> 2);
      const T* F = FQ + r * LQ + c * LS + kSweepHalo;
      const T* Q = FQ + r * LQ + (4 + c) * LS + kSweepHalo;
      const int fe = per ? f : min(max(f, -1), n - 1);
      WB[(size_t)(r * 4 + c) * LW + f + 2] = weno_face<T>(F, Q, fe, alpha);
    }
  }
  dep.sync();

  // ---- H: this thread's faces and raw differences, in registers ------------------
  const int r = tid() >> 7;         // line of the CTA
  const int tl = tid() & 127;       // thread within the line
  const int lw = tl >> 5;                 // warp within the line
  const int i0 = tl * MN;                 // first node
  const int len = r < R ? max(0, min(MN, n - i0)) : 0;
  const T inv_h = T(1.0 / h);
  const T rho = T(kRhoSolve);
  T x[4][MN];
  bool fl[MN + 1];
  {
    const uint8_t* mk = MK + min(r, R - 1) * (n + 2) + 1;
#pragma unroll
    for (int j = 0; j <= MN; ++j) {
      const int f = i0 - 1 + j;  // face f + 1/2
      fl[j] = anyflag && len > 0 && f <= n - 1 && flagged(mk, f);
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    T H[MN + 1];
    if (len > 0) {
      T fv[MN + 8];  // F_c of nodes i0 - 4 .. i0 + MN + 3
      load_run<T, MN + 8>(FQ + r * LQ + c * LS, kSweepHalo + i0 - 4, fv);
      const T* Wc = WB + (size_t)(r * 4 + c) * LW + 2;
#pragma unroll
      for (int j = 0; j <= MN; ++j) {
        if (fl[j]) {
          const int f = i0 - 1 + j;
          T hf = T(kCompactA) * Wc[f + 1] + Wc[f];
          H[j] = hf + T(kCompactA) * Wc[f - 1];
        } else {
          // 6-point compact flux of face i0 - 1 + j (OOP/spatial_operator.py:179-189)
          H[j] = T(-1.0 / 480.0) * (fv[j + 6] + fv[j + 1]) + T(kB1C1) * (fv[j + 5] + fv[j + 2]) +
                 T(kA1B1C1) * (fv[j + 4] + fv[j + 3]);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < MN; ++k) x[c][k] = (k < len) ? (H[k + 1] - H[k]) * inv_h : T(0);
  }

  // ---- S: forward recurrence y_i = raw_i + rho y_{i-1} ------------------------------
  T raw0[4], rawl[4];
  const int owner_last = (n - 1) / MN, k_last = (n - 1) - owner_last * MN;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    raw0[c] = x[c][0];
    T v = T(0);
#pragma unroll
    for (int k = 0; k < MN; ++k)
      if (k == k_last) v = x[c][k];
    rawl[c] = v;
  }
  Affine<T> fw;
  fw.m = T(1);
#pragma unroll
  for (int c = 0; c < 4; ++c) fw.a[c] = T(0);
#pragma unroll
  for (int k = 0; k < MN; ++k)
    if (k < len) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        fw.a[c] = x[c][k] + rho * fw.a[c];
        x[c][k] = fw.a[c];
      }
      fw.m *= rho;
    }
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const T mo = __shfl_up_sync(kFull, fw.m, off);
    T ao[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) ao[c] = __shfl_up_sync(kFull, fw.a[c], off);
    if (lane >= off) {
#pragma unroll
      for (int c = 0; c < 4; ++c) fw.a[c] = fw.m * ao[c] + fw.a[c];
      fw.m *= mo;
    }
  }
  if (lane == 31 && r < 4) scan_f[r][lw] = fw;
  // exclusive prefix within the warp
  Affine<T> fe;
  fe.m = __shfl_up_sync(kFull, fw.m, 1);
#pragma unroll
  for (int c = 0; c < 4; ++c) fe.a[c] = __shfl_up_sync(kFull, fw.a[c], 1);
  if (lane == 0) {
    fe.m = T(1);
#pragma unroll
    for (int c = 0; c < 4; ++c) fe.a[c] = T(0);
  }
  dep.sync();
  {
    const int rr = min(r, 3);
    Affine<T> pre, tot;  // maps of the warps before this one, and of the whole line
    pre.m = tot.m = T(1);
#pragma unroll
    for (int c = 0; c < 4; ++c) pre.a[c] = tot.a[c] = T(0);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const Affine<T> wj = scan_f[rr][j];
      if (j < lw) {
#pragma unroll
        for (int c = 0; c < 4; ++c) pre.a[c] = wj.m * pre.a[c] + wj.a[c];
        pre.m *= wj.m;
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) tot.a[c] = wj.m * tot.a[c] + wj.a[c];
      tot.m *= wj.m;
    }
    // periodic: y_{-1} = y_{n-1} closes the cycle exactly
    const T icyc = per ? T(1) / (T(1) - tot.m) : T(0);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const T ybnd = per ? tot.a[c] * icyc : T(0);
      const T yin = fe.m * (pre.m * ybnd + pre.a[c]) + fe.a[c];
      T pw = rho;
#pragma unroll
      for (int k = 0; k < MN; ++k)
        if (k < len) {
          x[c][k] += pw * yin;
          pw *= rho;
        }
    }
  }

  // ---- S: backward recurrence z_i = y_i + rho z_{i+1} -------------------------------
  Affine<T> bw;
  bw.m = T(1);
#pragma unroll
  for (int c = 0; c < 4; ++c) bw.a[c] = T(0);
#pragma unroll
  for (int k = MN - 1; k >= 0; --k)
    if (k < len) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        bw.a[c] = x[c][k] + rho * bw.a[c];
        x[c][k] = bw.a[c];
      }
      bw.m *= rho;
    }
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const T mo = __shfl_down_sync(kFull, bw.m, off);
    T ao[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) ao[c] = __shfl_down_sync(kFull, bw.a[c], off);
    if (lane + off < 32) {
#pragma unroll
      for (int c = 0; c < 4; ++c) bw.a[c] = bw.m * ao[c] + bw.a[c];
      bw.m *= mo;
    }
  }
  if (lane == 0 && r < 4) scan_b[r][lw] = bw;
  Affine<T> be;
  be.m = __shfl_down_sync(kFull, bw.m, 1);
#pragma unroll
  for (int c = 0; c < 4; ++c) be.a[c] = __shfl_down_sync(kFull, bw.a[c], 1);
  if (lane == 31) {
    be.m = T(1);
#pragma unroll
    for (int c = 0; c < 4; ++c) be.a[c] = T(0);
  }
  dep.sync();
  {
    const int rr = min(r, 3);
    Affine<T> post, tot;  // maps of the warps after this one (innermost last), whole line
    post.m = tot.m = T(1);
#pragma unroll
    for (int c = 0; c < 4; ++c) post.a[c] = tot.a[c] = T(0);
#pragma unroll
    for (int j = 3; j >= 0; --j) {
      const Affine<T> wj = scan_b[rr][j];
      if (j > lw) {
#pragma unroll
        for (int c = 0; c < 4; ++c) post.a[c] = wj.m * post.a[c] + wj.a[c];
        post.m *= wj.m;
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) tot.a[c] = wj.m * tot.a[c] + wj.a[c];
      tot.m *= wj.m;
    }
    const T icyc = per ? T(1) / (T(1) - tot.m) : T(0);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const T zbnd = per ? tot.a[c] * icyc : T(0);
      const T zin = be.m * (post.m * zbnd + post.a[c]) + be.a[c];
      T pw = rho;
#pragma unroll
      for (int k = MN - 1; k >= 0; --k)
        if (k < len) {
          x[c][k] = T(kSolveScale) * (x[c][k] + pw * zin);
          pw *= rho;
        }
    }
  }

  if (!per) {
    // identity end rows (riemann_config3.py:244-264): d = p + A rho^i + B rho^(n-1-i)
    if (len > 0 && tl == 0) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        ends[r][c][0] = raw0[c];
        ends[r][c][2] = x[c][0];
      }
    }
    if (len > 0 && tl == owner_last) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        T pl = T(0);
#pragma unroll
        for (int k = 0; k < MN; ++k)
          if (k == k_last) pl = x[c][k];
        ends[r][c][1] = rawl[c];
        ends[r][c][3] = pl;
      }
    }
    dep.sync();
    // the homogeneous terms are below roundoff beyond ~80 nodes from an end
    if (len > 0 && (i0 < 96 || i0 + len > n - 96)) {
      if (n == 1) {
        x[0][0] = ends[r][0][0];
        x[1][0] = ends[r][1][0];
        x[2][0] = ends[r][2][0];
        x[3][0] = ends[r][3][0];
      } else {
        const T e = rho_pow(n - 1);
        const T den = T(1) - e * e;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const T r0 = ends[r][c][0] - ends[r][c][2], r1 = ends[r][c][1] - ends[r][c][3];
          const T ca = (r0 - e * r1) / den, cb = (r1 - e * r0) / den;
#pragma unroll
          for (int k = 0; k < MN; ++k)
            if (k < len) x[c][k] += ca * rho_pow(i0 + k) + cb * rho_pow(n - 1 - i0 - k);
        }
      }
    }
  }

  // ---- E: epilogue ----------------------------------------------------------------------
  if constexpr (AXIS == 0) {
    dep.wait();  // below: the y sweep's partial rhs
    dep.release();
  }
  const int terms = bind.use ? bind.terms : fused_terms(S);
  if (AXIS == 1) {
    // y sweep: partial rhs -dG/dy (or the bare derivative for the API),
    // staged in shared memory and written with consecutive threads on the
    // R columns of a row, then the next row
    T* XS = WB;  // [R][4][LW]
#pragma unroll
    for (int c = 0; c < 4; ++c) store_run<T, MN>(XS + (r * 4 + c) * LW + i0, x[c], len);
    dep.sync();
    T* rx = reinterpret_cast<T*>(S.rx);
    for (int idx = tid(); idx < (n << rsh); idx += nthr()) {
      const int rr = idx & (RL - 1), p = idx >> rsh;
      if (rr >= R) continue;
      const size_t o = (size_t)p * nx + line0 + rr;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const T d = XS[(rr * 4 + c) * LW + p];
        if (mode == SW_DERIV) bind.out[c * plane + o] = double(d);
        else rx[c * plane + o] = (terms & 1) ? -d : T(0);
      }
    }
    return;
  }
  if (mode == SW_DERIV) {
    // x derivative for the API
    T* rx = reinterpret_cast<T*>(S.rx);
#pragma unroll
    for (int k = 0; k < MN; ++k) {
      if (k >= len) continue;
      const int p = i0 + k;
      const int row = AXIS == 0 ? line0 + r : p, col = AXIS == 0 ? p : line0 + r;
      const size_t o = (size_t)row * nx + col;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (mode == SW_DERIV) bind.out[c * plane + o] = double(x[c][k]);
        else rx[c * plane + o] = (terms & 1) ? -x[c][k] : T(0);
      }
    }
    return;
  }
  // x sweep: full rhs, then the stage combine and the clean filter
  const double fs = ldsc(S_F_SCALE);
  const double dt = ldsc(S_DT);
  const double* q0 = bind.use ? bind.q0 : S.q;
  double* qo = bind.use ? bind.qout : stage_out(S, stage);
  const T* ry = reinterpret_cast<const T*>(S.rx);
  const int gc = (mode == SW_STAGE && !per) ? S.guard : 0;
  // drag band S = -c lowpass(m) (OOP/hit2d.py:352-399) of the CTA's rows:
  // P_k(y) = sum over modes with |kx| = k of C_m e^{i ky y} (conjugated for
  // kx < 0), C_m the mode's scaled transform from the prepass
  auto& dpx = sh.dpx;
  auto& dpy = sh.dpy;
  const bool drag = (terms & 8) && S.drag_on;
  if (drag) {
    const int K = S.kx_drag;
    for (int t = tid(); t < R * (K + 1); t += nthr()) {
      const int rr = t / (K + 1), k = t - rr * (K + 1);
      const int row = line0 + rr;
      double2 sx = make_double2(0.0, 0.0), sy = make_double2(0.0, 0.0);
      for (int md = 0; md < S.n_drag; ++md) {
        const int2 km = S.modes[md];
        if (abs(km.x) != k) continue;
        const double2 e = S.twy[mode_index(km.y, row, ny)];
        const double er = e.x, ei = -e.y;  // e^{+i ky y}
        const double* cf = sc + S_DRAG + 4 * md;
        double ar, ai, br, bi;
        if constexpr (QD) {
          const double c0 = __ldcg(cf), c1 = __ldcg(cf + 1), c2 = __ldcg(cf + 2), c3 = __ldcg(cf + 3);
          ar = c0 * er - c1 * ei;
          ai = c0 * ei + c1 * er;
          br = c2 * er - c3 * ei;
          bi = c2 * ei + c3 * er;
        } else {
          ar = cf[0] * er - cf[1] * ei;
          ai = cf[0] * ei + cf[1] * er;
          br = cf[2] * er - cf[3] * ei;
          bi = cf[2] * ei + cf[3] * er;
        }
        if (km.x < 0) {
          ai = -ai;
          bi = -bi;
        }
        sx.x += ar;
        sx.y += ai;
        sy.x += br;
        sy.y += bi;
      }
      dpx[rr][k] = sx;
      dpy[rr][k] = sy;
    }
  }
  // The derivatives go to shared memory (the WENO buffer is free once the
  // faces are formed) and the epilogue walks the rows with consecutive
  // threads on consecutive nodes, so that every global access is coalesced.
  T* XS = WB;  // [R][4][LW]
#pragma unroll
  for (int c = 0; c < 4; ++c) store_run<T, MN>(XS + (r * 4 + c) * LW + i0, x[c], len);
  dep.sync();  // derivatives and drag table ready; FQ free for the guard staging
  double* ST = reinterpret_cast<double*>(smem);  // new rows (guard staging), reuses FQ
  // Solve fields in registers and read-only inputs behind restrict-qualified
  // pointers: the stores to the stage output below cannot force reloads.
  const double gam = S.gamma, cool = (terms & 16) ? ldsc(S_COOL) : 0.0;
  const bool visc = (terms & 2) && S.mu > 0.0;
  const int kxd = S.kx_drag;
  const T* __restrict__ visp = reinterpret_cast<const T*>(S.vis);
  // caller's FP64 accelerations (API) or the solve's scaled unit-rms shape (T)
  const double* __restrict__ bfx = bind.fx;
  const double* __restrict__ bfy = bind.fy;
  const T* __restrict__ sfx = static_cast<const T*>(S.fx);
  const T* __restrict__ sfy = static_cast<const T*>(S.fy);
  const double2* __restrict__ twx = S.twx;
  const double* __restrict__ qinr = qin;
  const T* __restrict__ ryr = ry;
  // Two consecutive nodes per thread with 16-byte (FP64) and 8-byte (FP32)
  // vector accesses when the row length is even and every caller pointer is
  // 16-byte aligned (arena buffers always are): half the load instructions
  // and twice the bytes in flight per load.
  const uintptr_t al = (uintptr_t)qinr | (uintptr_t)q0 | (uintptr_t)qo |
                       (bind.use ? ((uintptr_t)bfx | (uintptr_t)bfy | (uintptr_t)bind.out) : 0);
  const bool vec = (nx & 1) == 0 && (al & 15) == 0;
  const double pfl64 = kPFloor / (gam - 1.0);
  // The rhs terms are summed in the bulk type T (in the FP32-bulk form the
  // sum is FP32, as every term is); FP64 takes over in the stage combine.
  auto epilogue = [&](auto vt) {
    constexpr int V = decltype(vt)::value;
    const int pl = (int)plane;
    // pass 1: the full rhs of every node in T, back into XS (the same thread
    // reads it in pass 2); the FP64 stage combine runs as a separate pass so
    // that neither pass holds the other's inputs in registers
    for (int idx = tid() * V; idx < R * n; idx += nthr() * V) {
      const int rr = xline_of<XR>(idx, n), col = idx - rr * n;
      const int o = (line0 + rr) * nx + col;
      T acc[4][V];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        vld<V>(ryr + c * pl + o, acc[c]);
        if (terms & 1) {
          T xs[V];
          vld<V>(XS + (rr * 4 + c) * LW + col, xs);
#pragma unroll
          for (int v = 0; v < V; ++v) acc[c][v] -= xs[v];
        }
      }
      if (visc) {
#pragma unroll
        for (int c = 1; c < 4; ++c) {
          T vs[V];
          vld<V>(visp + (c - 1) * pl + o, vs);
#pragma unroll
          for (int v = 0; v < V; ++v) acc[c][v] += vs[v];
        }
      }
      if (terms & (4 | 8)) {
        double q3[3][V];
#pragma unroll
        for (int c = 0; c < 3; ++c) vld<V>(qinr + c * pl + o, q3[c]);
        T tfx[V], tfy[V];
        if (terms & 4) {
          if (bind.use) {
            double fx2[V], fy2[V];
            vld<V>(bfx + o, fx2);
            vld<V>(bfy + o, fy2);
#pragma unroll
            for (int v = 0; v < V; ++v) {
              tfx[v] = T(fx2[v]);
              tfy[v] = T(fy2[v]);
            }
          } else {
            vld<V>(sfx + o, tfx);
            vld<V>(sfy + o, tfy);
#pragma unroll
            for (int v = 0; v < V; ++v) {
              if constexpr (sizeof(T) == 4) {
                tfx[v] = float(fs) * tfx[v];
                tfy[v] = float(fs) * tfy[v];
              } else {
                tfx[v] = fs * tfx[v];
                tfy[v] = fs * tfy[v];
              }
            }
          }
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
          // rho, u, v of primitive_from_conservative (one reciprocal)
          T prho, pu, pv;
          if constexpr (sizeof(T) == 4) {
            prho = fmaxf(float(q3[0][v]), float(kRhoFloor));
            const float prinv = __frcp_rn(prho);
            pu = float(q3[1][v]) * prinv;
            pv = float(q3[2][v]) * prinv;
          } else {
            prho = q3[0][v] > kRhoFloor ? q3[0][v] : kRhoFloor;
            const double prinv = 1.0 / prho;
            pu = q3[1][v] * prinv;
            pv = q3[2][v] * prinv;
          }
          if (terms & 4) {
            acc[1][v] += prho * tfx[v];
            acc[2][v] += prho * tfy[v];
            acc[3][v] += prho * (pu * tfx[v] + pv * tfy[v]);
          }
          if (drag) {
            // Re sum_k P_k(row) e^{i k x}: the drag band synthesised per row
            T lx = T(dpx[rr][0].x), ly = T(dpy[rr][0].x);
            int ix = 0;
            for (int kk = 1; kk <= kxd; ++kk) {
              ix += col + v;
              if (ix >= nx) ix -= nx;  // (k x) mod nx
              const double2 e = twx[ix];
              const T er = T(e.x), ei = -T(e.y);  // e^{+i k x}
              lx += T(dpx[rr][kk].x) * er - T(dpx[rr][kk].y) * ei;
              ly += T(dpy[rr][kk].x) * er - T(dpy[rr][kk].y) * ei;
            }
            acc[1][v] += lx;
            acc[2][v] += ly;
            acc[3][v] += pu * lx + pv * ly;
          }
        }
      }
      if (terms & 16) {
#pragma unroll
        for (int v = 0; v < V; ++v) acc[3][v] += T(cool);
      }
      if (mode == SW_RHS) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          double r[V];
#pragma unroll
          for (int v = 0; v < V; ++v) r[v] = double(acc[c][v]);
          vst<V>(bind.out + c * pl + o, r);
        }
      } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) vst<V>(XS + (rr * 4 + c) * LW + col, acc[c]);
      }
    }
    if (mode == SW_RHS) return;
    // pass 2: stage combine in FP64 and the clean filter
    for (int idx = tid() * V; idx < R * n; idx += nthr() * V) {
      const int rr = xline_of<XR>(idx, n), col = idx - rr * n;
      const int o = (line0 + rr) * nx + col;
      double sv[4][V];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        double qa[V];
        T r[V];
        vld<V>(qinr + c * pl + o, qa);
        vld<V>(XS + (rr * 4 + c) * LW + col, r);
#pragma unroll
        for (int v = 0; v < V; ++v) sv[c][v] = __fma_rn(dt, double(r[v]), qa[v]);
      }
      if (stage != 0) {
        const double wa = stage == 1 ? 0.75 : 1.0 / 3.0, wb = stage == 1 ? 0.25 : 2.0 / 3.0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          double b[V];
          vld<V>(q0 + c * pl + o, b);
#pragma unroll
          for (int v = 0; v < V; ++v) sv[c][v] = __fma_rn(wa, b[v], __dmul_rn(wb, sv[c][v]));
        }
      }
#pragma unroll
      for (int v = 0; v < V; ++v) enforce_node_rcp(sv[0][v], sv[1][v], sv[2][v], sv[3][v], gam, pfl64);
      if (gc == 0) {
#pragma unroll
        for (int c = 0; c < 4; ++c) vst<V>(qo + c * pl + o, sv[c]);
      } else {
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
          for (int v = 0; v < V; ++v) ST[(rr * 4 + c) * n + col + v] = sv[c][v];
      }
    }
  };
#ifndef HITB200_NO_VEC_EPILOGUE
  if (vec) epilogue(VecWidth<2>{});
#else
  if (false) epilogue(VecWidth<2>{});
#endif
  else epilogue(VecWidth<1>{});
  if (gc == 0 || mode != SW_STAGE) return;
  // Outflow guard fused: every row j takes row J(j) = clamp(j, g, ny-g-1) and
  // every column i column I(i); the CTA owning row J(j) writes row j.
  dep.sync();
  for (int rr = 0; rr < R; ++rr) {
    const int j0 = line0 + rr;
    if (j0 != guard_src(j0, ny, gc)) continue;  // a guard row: written by its source
    const int jlo = j0 == gc ? 0 : j0, jhi = j0 == ny - gc - 1 ? ny - 1 : j0;
    const int cnt = (jhi - jlo + 1) * nx;
    for (int idx = tid(); idx < cnt; idx += nthr()) {
      const int jj = idx / nx, i = idx - jj * nx;
      const size_t o = (size_t)(jlo + jj) * nx + i;
      const int si = guard_src(i, nx, gc);
#pragma unroll
      for (int c = 0; c < 4; ++c) qo[c * plane + o] = ST[(size_t)(rr * 4 + c) * n + si];
    }
  }
}

template <typename T, int AXIS, int MN, int OCC>
__global__ void __launch_bounds__(AXIS == 0 ? 256 : 512,
                                  AXIS == 0 ? (OCC ? kSweepMinBlocksX : 2) : (OCC ? kSweepMinBlocksY : 1))
    sweep_kernel(const SolveDev* __restrict__ solves, const Work* __restrict__ work, int stage,
                 int mode, Bind bind) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ SweepShared<T, AXIS == 0 ? 2 : 1> sh;
  sweep_body<T, AXIS, MN>(solves, work[blockIdx.x], stage, mode, bind, smem, sh, PdlDep{});
}

// =============================================================================
// Biharmonic hyperviscosity q - mn w h^4 active lap(lap q), then enforce
// (OOP/spatial_operator.py:394-435 periodic; riemann_config3.py:390-416 with
// an edge-padded Laplacian, applied to the padded Laplacian again).
// =============================================================================
// The CTAs take the tiles work[0 .. nwork) in a grid-stride loop: single
// plans launch one CTA per tile; batches launch a few CTAs per SM, so that
// the steps without hyperviscosity, whose tiles are all no-ops, cost a small
// fraction of one CTA per tile.
template <typename T>
__global__ void __launch_bounds__(kStencilThreads)
    hv_kernel(const SolveDev* __restrict__ solves, const Work* __restrict__ work, int nwork, Bind bind) {
  constexpr int QX = kHvTX + 4, QY = kHvTY + 4, LX = kHvTX + 2, LY = kHvTY + 2;
  __shared__ T Qs[4][QY][QX];
  __shared__ T Ls[4][LY][LX];
  for (int item = blockIdx.x; item < nwork; item += gridDim.x) {
  if (item > (int)blockIdx.x) __syncthreads();  // shared memory of the previous tile
  const Work wk = work[item];
  const SolveDev& S = solves[wk.solve];
  // the hyperviscosity flag is written by the step's first kernel
  if (!bind.use && S.scal[S_HV_STEP] == 0.0) continue;
  const double* q = bind.use ? bind.qin : S.q1;
  double* out = bind.use ? bind.qout : S.q;
  const uint8_t* mask = bind.use ? bind.mask : S.mask;
  const int inv = bind.use ? bind.invert_mask : 1;
  const int nx = S.nx, ny = S.ny, per = S.periodic;
  const size_t plane = (size_t)nx * ny;
  const int x0 = wk.a, y0 = wk.b;
  for (int idx = threadIdx.x; idx < QX * QY; idx += blockDim.x) {
    const int a = idx / QX, b = idx % QX;
    const int gj = fold_node(y0 - 2 + a, ny, per), gi = fold_node(x0 - 2 + b, nx, per);
    const size_t o = (size_t)gj * nx + gi;
#pragma unroll
    for (int c = 0; c < 4; ++c) Qs[c][a][b] = T(__ldcg(q + c * plane + o));
  }
  // the input state was written two or more kernels earlier (complete when
  // this CTA starts); the mask comes from the sensor just before and is
  // read only by the final update, so the first Laplacian precedes the wait
  __syncthreads();
  const T dx2 = T(S.dx * S.dx), dy2 = T(S.dy * S.dy);
  const T idx2 = T(1.0 / (S.dx * S.dx)), idy2 = T(1.0 / (S.dy * S.dy));
  // second differences: FP64 divides by h^2 as the reference; FP32 multiplies
  auto d2 = [&](T a, T b, T c, T h2, T ih2) -> T {
    if constexpr (sizeof(T) == 8) return (a - T(2) * b + c) / h2;
    else return (a - T(2) * b + c) * ih2;
  };
  for (int idx = threadIdx.x; idx < LX * LY; idx += blockDim.x) {
    int a = idx / LX, b = idx % LX;
    // outflow: the Laplacian is itself edge-padded before the second pass
    int gj = y0 - 1 + a, gi = x0 - 1 + b;
    if (!per) {
      const int cj = gj < 0 ? 0 : (gj >= ny ? ny - 1 : gj);
      const int ci = gi < 0 ? 0 : (gi >= nx ? nx - 1 : gi);
      a += cj - gj;
      b += ci - gi;
    }
    const int qa = a + 1, qb = b + 1;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const T lx = d2(Qs[c][qa][qb + 1], Qs[c][qa][qb], Qs[c][qa][qb - 1], dx2, idx2);
      const T ly = d2(Qs[c][qa + 1][qb], Qs[c][qa][qb], Qs[c][qa - 1][qb], dy2, idy2);
      Ls[c][idx / LX][idx % LX] = lx + ly;
    }
  }
  __syncthreads();
  pdl_wait();  // below: the sensor's mask
  pdl_release();
  // solve fields in registers: the stores below cannot force reloads
  const double gam = S.gamma;
  const int gcell = (!bind.use && !per) ? S.guard : 0;  // fused outflow guard of the step
  const double hc[4] = {S.hv_coef[0], S.hv_coef[1], S.hv_coef[2], S.hv_coef[3]};
  for (int idx = threadIdx.x; idx < kHvTX * kHvTY; idx += blockDim.x) {
    const int ty = idx / kHvTX, tx = idx % kHvTX;
    const int gj = y0 + ty, gi = x0 + tx;
    if (gj >= ny || gi >= nx) continue;
    const size_t o = (size_t)gj * nx + gi;
    const bool active = inv ? (mask[o] == 0) : (mask[o] != 0);
    const int a = ty + 1, b = tx + 1;
    double s[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const T bx = d2(Ls[c][a][b + 1], Ls[c][a][b], Ls[c][a][b - 1], dx2, idx2);
      const T by = d2(Ls[c][a + 1][b], Ls[c][a][b], Ls[c][a - 1][b], dy2, idy2);
      const double bih = double(bx + by);
      s[c] = q[c * plane + o] - (active ? hc[c] : 0.0) * bih;
    }
    enforce_node_rcp(s[0], s[1], s[2], s[3], gam);
    if (gcell == 0) {
#pragma unroll
      for (int c = 0; c < 4; ++c) out[c * plane + o] = s[c];
      continue;
    }
    // Outflow guard fused (riemann_config3.py:419-429): guard cells are not
    // written by their own threads; the thread of each source cell writes
    // its value to itself and to the guard cells that copy it.
    const bool guard_cell = gj < gcell || gj >= ny - gcell || gi < gcell || gi >= nx - gcell;
    if (guard_cell) continue;
    const int jlo = gj == gcell ? 0 : gj, jhi = gj == ny - gcell - 1 ? ny - 1 : gj;
    const int ilo = gi == gcell ? 0 : gi, ihi = gi == nx - gcell - 1 ? nx - 1 : gi;
    for (int jj = jlo; jj <= jhi; ++jj)
      for (int ii = ilo; ii <= ihi; ++ii) {
        const size_t od = (size_t)jj * nx + ii;
#pragma unroll
        for (int c = 0; c < 4; ++c) out[c * plane + od] = s[c];
      }
  }
  }
}

// Outflow guard: every guard cell takes the value of the nearest interior
// cell column/row g or n-g-1 (x first, then y: the corner takes (g, g)).
// sel: 0 q, 1 q1, 2 q2, 3 stage-3 output; one CTA per solve.
__global__ void guard_kernel(const SolveDev* __restrict__ solves, int nsolves, int sel, Bind bind) {
  const int s = blockIdx.y;
  if (s >= nsolves) return;
  const SolveDev& S = solves[s];
  if (S.periodic || S.guard <= 0) return;
  if (!bind.use && S.scal[S_ACTIVE] == 0.0 && sel != 0) return;
  double* q = bind.use ? bind.qout : (sel == 0 ? S.q : sel == 1 ? S.q1 : sel == 2 ? S.q2 : stage_out(S, 2));
  const int nx = S.nx, ny = S.ny, gc = S.guard;
  const size_t plane = (size_t)nx * ny;
  const int top = 2 * gc * nx;                 // full rows
  const int side = 2 * gc * (ny - 2 * gc);     // side columns of interior rows
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < top + side; t += gridDim.x * blockDim.x) {
    int j, i;
    if (t < top) {
      const int rr = t / nx;
      i = t % nx;
      j = rr < gc ? rr : ny - 2 * gc + rr;
    } else {
      const int u = t - top, cc = u % (2 * gc);
      j = gc + u / (2 * gc);
      i = cc < gc ? cc : nx - 2 * gc + cc;
    }
    const int J = j < gc ? gc : (j > ny - gc - 1 ? ny - gc - 1 : j);
    const int I = i < gc ? gc : (i > nx - gc - 1 ? nx - gc - 1 : i);
    if (J == j && I == i) continue;
    const size_t dst = (size_t)j * nx + i, src = (size_t)J * nx + I;
#pragma unroll
    for (int c = 0; c < 4; ++c) q[c * plane + dst] = q[c * plane + src];
  }
}

__global__ void enforce_kernel(const double* __restrict__ q, double* __restrict__ out, size_t plane,
                               double gamma) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < plane;
       i += (size_t)gridDim.x * blockDim.x) {
    double s0 = q[i], s1 = q[plane + i], s2 = q[2 * plane + i], s3 = q[3 * plane + i];
    enforce_node(s0, s1, s2, s3, gamma);
    out[i] = s0;
    out[plane + i] = s1;
    out[2 * plane + i] = s2;
    out[3 * plane + i] = s3;
  }
}

// out[c] = scale * a  (forcing accelerations for the API, viscous copy)
template <typename A>
__global__ void scale_copy_kernel(const A* __restrict__ a, double* __restrict__ out,
                                  const double* __restrict__ scal, int slot, size_t n) {
  const double s = slot >= 0 ? scal[slot] : 1.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = s * double(a[i]);
}

template <typename T>
__global__ void vis_copy_kernel(const T* __restrict__ vis, double* __restrict__ out, size_t plane) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < plane;
       i += (size_t)gridDim.x * blockDim.x) {
    out[i] = 0.0;
    out[plane + i] = double(vis[i]);
    out[2 * plane + i] = double(vis[plane + i]);
    out[3 * plane + i] = double(vis[2 * plane + i]);
  }
}

}  // namespace hitb200
