// Shock sensor of the time step with a compile-time dilation width
// (OOP/spatial_operator.py:147-176, 263-304; OOP/problems/riemann_config3.py:
// 128-162, 288-326) and the viscous terms (OOP/equations.py:232-267).
//
// The tests and their arithmetic are those of sensor_kernel, so the masks are
// the same; what differs is the data flow around them:
//   * the staged tile and its (W + 1)-halo are read with a row-per-warp
//     mapping and, for tiles away from the grid edges, without index folding;
//   * the temperature of the viscous terms is staged with the primitives, and
//     the viscous terms are formed right after staging (they do not depend on
//     the thresholds), before the wait for the step's previous kernel;
//   * every raw node's tests are decided by the thread of its (4-row strip,
//     column) task, which keeps its margins (FP32) in registers across the
//     wait, and the 4 flag bits of each task are gathered by warp ballots into
//     one 64-bit word per raw row;
//   * the (2W + 1)^2 box dilation is then W-independent word arithmetic: a
//     row pass of 2W + 1 shifts and ORs per raw row, a column pass of 2W + 1
//     ORs per tile row, and the mask is written 4 bytes at a time.
// W is a template parameter so that every loop bound is a constant; widths
// without an instantiation use sensor_kernel.
#pragma once

#include "kernels_stencil.cuh"

namespace hitb200 {

template <int W>
struct StepSensorShape {
  static constexpr int HW = W + 1 > 2 ? W + 1 : 2;
  static constexpr int SX = kSenTX + 2 * HW, SY = kSenTY + 2 * HW;
  static constexpr int RX = kSenTX + 2 * W, RY = kSenTY + 2 * W;
  static constexpr int NSTRIP = (RY + 3) / 4;
  static constexpr int NTASK = RX * NSTRIP;
  static constexpr int OFF = HW - W;  // staged index of raw index 0
  static_assert(RX <= 64, "a raw row must fit one 64-bit word");
  static_assert(NTASK <= kSensorThreads, "one strip task per thread");
};

// Byte offsets of the shared-memory regions: six staged arrays (rho, u, v, p,
// e, temperature), the raw-row words, the row-dilated words, then the five
// viscous stress / flux arrays.
template <int W>
__host__ __device__ inline size_t step_sensor_bits_off(int elem) {
  using Sh = StepSensorShape<W>;
  return ((size_t)6 * Sh::SX * Sh::SY * elem + 15) & ~(size_t)15;
}
template <int W>
__host__ __device__ inline size_t step_sensor_visc_off(int elem) {
  using Sh = StepSensorShape<W>;
  return (step_sensor_bits_off<W>(elem) + (size_t)Sh::RY * 8 + (size_t)Sh::RY * 4 + 15) & ~(size_t)15;
}
template <int W>
__host__ __device__ inline size_t step_sensor_smem_bytes(int elem, bool viscous) {
  return step_sensor_visc_off<W>(elem) + (viscous ? 5 * (size_t)kVisX * kVisY * elem : 0);
}

// One tile (work item wk) of the step sensor, with dynamic shared memory smem.
// sel: 0 q, 1 q1, 2 q2 (stage inputs, enforced first, viscous terms written
// when the solve is viscous), 3 the hyperviscosity input (q1 on hyperviscosity
// steps, not enforced, no viscous terms).  Dep is the wait for the prepass
// (PdlDep in sensor_step_kernel; the persistent stage kernel's counter wait,
// after which the scalars are read through L2).
template <typename T, int W, typename Dep>
__device__ __forceinline__ void sensor_step_body(const SolveDev* __restrict__ solves, const Work wk, int sel,
                                                 int enf, int want_visc, unsigned char* smem,
                                                 const Dep& dep) {
  using Sh = StepSensorShape<W>;
  constexpr int HW = Sh::HW, SX = Sh::SX, SY = Sh::SY, RX = Sh::RX, RY = Sh::RY;
  constexpr int OFF = Sh::OFF, NTASK = Sh::NTASK;
  const SolveDev& S = solves[wk.solve];
  const double* sc = S.scal;
  auto ldsc = [&](int i) -> double {
    if constexpr (Dep::kQueued) return __ldcg(sc + i);
    else return sc[i];
  };
  // the hyperviscosity flag is written by the step's first kernel
  if (sel == 3 && sc[S_HV_STEP] == 0.0) return;
  const double* __restrict__ q = sel == 3 ? S.q1 : stage_in(S, sel);
  const int nx = S.nx, ny = S.ny, per = S.periodic;
  const size_t plane = (size_t)nx * ny;
  const int x0 = wk.a, y0 = wk.b;
  // ranges the plans guarantee, stated for the index arithmetic
  __builtin_assume(nx >= 1 && nx <= kMaxLine && ny >= 1 && ny <= kMaxLine);
  __builtin_assume(x0 >= 0 && x0 < kMaxLine && y0 >= 0 && y0 < kMaxLine);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NWARP = kSensorThreads / 32;
  const bool visc = want_visc && S.mu != 0.0;
  T* RHO = reinterpret_cast<T*>(smem);
  T* U = RHO + SX * SY;
  T* V = U + SX * SY;
  T* P = V + SX * SY;
  T* E = P + SX * SY;
  T* TT = E + SX * SY;
  unsigned long long* RB = reinterpret_cast<unsigned long long*>(smem + step_sensor_bits_off<W>(sizeof(T)));
  unsigned* DR = reinterpret_cast<unsigned*>(RB + RY);
  const T g = T(S.gamma);
  const T gm1 = g - T(1);
  const T pfl = T(kPFloor) / gm1;  // the quotient every enforced node forms
  const T igm1 = T(1.0 / (S.gamma - 1.0));
  const T rgas = T(S.gas_r);
  const T irg = T(1.0 / S.gas_r);
  for (int t = threadIdx.x; t < RY; t += blockDim.x) RB[t] = 0ull;

  // ---- staged primitives of the tile and its halo: warp = row, lane = column ----
  const bool inner = x0 - HW >= 0 && x0 + kSenTX + HW <= nx && y0 - HW >= 0 && y0 + kSenTY + HW <= ny;
#pragma unroll 1
  for (int a = warp; a < SY; a += NWARP) {
    const int gj = inner ? y0 - HW + a : fold_node(y0 - HW + a, ny, per);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int b = lane + 32 * h;
      if (b >= SX) continue;
      const int gi = inner ? x0 - HW + b : fold_node(x0 - HW + b, nx, per);
      const size_t o = (size_t)gj * nx + gi;
      const double d0 = __ldcg(q + o), d1 = __ldcg(q + o + plane), d2 = __ldcg(q + o + 2 * plane),
                   d3 = __ldcg(q + o + 3 * plane);
      const int idx = a * SX + b;
      if constexpr (sizeof(T) == 8) {
        double q0 = d0, q1 = d1, q2 = d2, q3 = d3;
        if (enf) {
          // enforce_physical_state (OOP/equations.py:165-181)
          const double rho = q0 > kRhoFloor ? q0 : kRhoFloor;
          const double u = q1 / rho, v = q2 / rho;
          const double kin = 0.5 * rho * (u * u + v * v);
          const double pr = gm1 * (q3 - kin);
          q0 = rho;
          q1 = rho * u;
          q2 = rho * v;
          q3 = pr > kPFloor ? q3 : pfl + kin;
        }
        const Prim<double> p = primitives(q0, q1, q2, q3, (double)g);
        RHO[idx] = p.rho;
        U[idx] = p.u;
        V[idx] = p.v;
        P[idx] = p.p;
        E[idx] = p.p / (p.rho * gm1);
        if (visc) TT[idx] = p.p / (p.rho * rgas);
      } else {
        T q0 = T(d0), q1 = T(d1), q2 = T(d2), q3 = T(d3);
        const T rho = q0 > T(kRhoFloor) ? q0 : T(kRhoFloor);
        const T rinv = __frcp_rn(rho);
        T u = q1 * rinv, v = q2 * rinv;
        const T kin = T(0.5) * rho * (u * u + v * v);
        T pr = gm1 * (q3 - kin);
        if (enf) {
          q1 = rho * u;
          q2 = rho * v;
          q3 = pr > T(kPFloor) ? q3 : pfl + kin;
          u = q1 * rinv;
          v = q2 * rinv;
          pr = gm1 * (q3 - T(0.5) * rho * (u * u + v * v));
        }
        pr = pr > T(kPFloor) ? pr : T(kPFloor);
        RHO[idx] = rho;
        U[idx] = u;
        V[idx] = v;
        P[idx] = pr;
        const T pr_r = pr * rinv;
        E[idx] = pr_r * igm1;
        if (visc) TT[idx] = pr_r * irg;
      }
    }
  }
  __syncthreads();
  const T tdx = T(2.0 * S.dx), tdy = T(2.0 * S.dy), hx = T(S.dx), hy = T(S.dy);
  const T itdx = T(1.0 / (2.0 * S.dx)), itdy = T(1.0 / (2.0 * S.dy));

  // ---- viscous stress and heat-flux divergence (OOP/equations.py:232-267) ----
  // They need only the staged primitives, so they are formed before the wait.
  if (visc) {
    const T mu = T(S.mu), kap = T(S.kappa);
    const T two3 = T(2.0 / 3.0);
    T* TXX = reinterpret_cast<T*>(smem + step_sensor_visc_off<W>(sizeof(T)));
    T* TYY = TXX + kVisX * kVisY;
    T* TXY = TYY + kVisX * kVisY;
    T* QX = TXY + kVisX * kVisY;
    T* QY = QX + kVisX * kVisY;
#pragma unroll 1
    for (int a = warp; a < kVisY; a += NWARP) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int b = lane + 32 * h;
        if (b >= kVisX) continue;
        const int c = (a + HW - 1) * SX + (b + HW - 1);
        const T ux = dq(U[c + 1], U[c - 1], tdx, itdx), vx = dq(V[c + 1], V[c - 1], tdx, itdx);
        const T uy = dq(U[c + SX], U[c - SX], tdy, itdy), vy = dq(V[c + SX], V[c - SX], tdy, itdy);
        const T dv = ux + vy;
        const T txx = T(2) * mu * ux - two3 * mu * dv;
        const T tyy = T(2) * mu * vy - two3 * mu * dv;
        const T txy = mu * (uy + vx);
        const T tx_ = dq(TT[c + 1], TT[c - 1], tdx, itdx), ty_ = dq(TT[c + SX], TT[c - SX], tdy, itdy);
        const int i = a * kVisX + b;
        TXX[i] = txx;
        TYY[i] = tyy;
        TXY[i] = txy;
        QX[i] = U[c] * txx + V[c] * txy + kap * tx_;
        QY[i] = U[c] * txy + V[c] * tyy + kap * ty_;
      }
    }
    __syncthreads();
    T* visp = reinterpret_cast<T*>(S.vis);
#pragma unroll 1
    for (int a = warp; a < kSenTY; a += NWARP) {
      const int gj = y0 + a, gi = x0 + lane;
      if (gj >= ny || gi >= nx) continue;
      const int i = (a + 1) * kVisX + lane + 1;
      const T r1 = dq(TXX[i + 1], TXX[i - 1], tdx, itdx) + dq(TXY[i + kVisX], TXY[i - kVisX], tdy, itdy);
      const T r2 = dq(TXY[i + 1], TXY[i - 1], tdx, itdx) + dq(TYY[i + kVisX], TYY[i - kVisX], tdy, itdy);
      const T r3 = dq(QX[i + 1], QX[i - 1], tdx, itdx) + dq(QY[i + kVisX], QY[i - kVisX], tdy, itdy);
      const size_t o = (size_t)gj * nx + gi;
      visp[o] = r1;
      visp[plane + o] = r2;
      visp[2 * plane + o] = r3;
    }
  }

  // ---- raw tests: one (4-row strip, raw column) task per thread ----------------
  const T thr = T(S.jump_thr);
  const int t = threadIdx.x;
  const bool has_task = t < NTASK;
  const int s = t / RX, br = t - s * RX;
  const int ar0 = 4 * s;
  const int nrow = (RY % 4 == 0) ? 4 : min(4, RY - ar0);
  const int c0 = (ar0 + OFF) * SX + br + OFF;  // staged index of raw node (ar0, br)
  const int gi = x0 - W + br;
  const bool shear_req = S.shear_on;
  // velocity gradients of the sensor: central; first-order one-sided at outflow edges
  T dvg[4] = {T(0), T(0), T(0), T(0)}, vor[4] = {T(0), T(0), T(0), T(0)};
  if (has_task) {
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
      dvg[k] = dudx + dvdy;
      if (shear_req) {
        T dvdx = T(0), dudy = T(0);
        if (cx) dvdx = dq(V[c + 1], V[c - 1], tdx, itdx);
        else if (nx > 1) dvdx = gi == 0 ? (V[c + 1] - V[c]) / hx : (V[c] - V[c - 1]) / hx;
        if (cy) dudy = dq(U[c + SX], U[c - SX], tdy, itdy);
        else if (ny > 1) dudy = gj == 0 ? (U[c + SX] - U[c]) / hy : (U[c] - U[c - SX]) / hy;
        vor[k] = fabs(dvdx - dudy);
      }
    }
  }
  // FP32: the largest test margin of each node and quantity (pair_margin,
  // curv_margin), formed before the wait and compared after it
  T mg[3][4];
  auto column = [&](const T* A, T (&col)[6], T (&lf)[4], T (&rt)[4]) {
#pragma unroll
    for (int j = 0; j < 6; ++j) col[j] = j <= nrow + 1 ? A[c0 + (j - 1) * SX] : T(0);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      lf[k] = k < nrow ? A[c0 + k * SX - 1] : T(0);
      rt[k] = k < nrow ? A[c0 + k * SX + 1] : T(0);
    }
  };
  if constexpr (sizeof(T) == 4) {
    if (has_task) {
      const T* QA[3] = {RHO, P, E};
#pragma unroll
      for (int qi = 0; qi < 3; ++qi) {
        T col[6], lf[4], rt[4];
        column(QA[qi], col, lf, rt);
        T my[5];
#pragma unroll
        for (int j = 0; j < 5; ++j) my[j] = pair_margin(col[j], col[j + 1], thr);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          T m = fmax(my[k], my[k + 1]);
          m = fmax(m, pair_margin(lf[k], col[k + 1], thr));
          m = fmax(m, pair_margin(col[k + 1], rt[k], thr));
          m = fmax(m, curv_margin(lf[k], col[k + 1], rt[k], thr));
          m = fmax(m, curv_margin(col[k], col[k + 1], col[k + 2], thr));
          mg[qi][k] = m;
        }
      }
    }
  }

  dep.wait();  // below: the prepass's thresholds and the solve's flags
  // a finished solve's launch is a no-op
  if (sel != 3 && ldsc(S_ACTIVE) == 0.0) return;
  dep.release();
  const double l_comp = ldsc(S_COMP_LIM), l_shear = ldsc(S_SHEAR_LIM);
  const T eps_q[3] = {T(ldsc(S_EPS_RHO)), T(ldsc(S_EPS_P)), T(ldsc(S_EPS_E))};
  const T comp_lim = T(l_comp), shear_lim = T(l_shear);
  const bool comp_on = isfinite(comp_lim), shear_on = isfinite(shear_lim);

  unsigned bits = 0;  // bit k: raw row ar0 + k of this column flagged
  if (has_task) {
    bool m[4] = {false, false, false, false};
    if constexpr (sizeof(T) == 4) {
#pragma unroll
      for (int qi = 0; qi < 3; ++qi) {
        const T lim = thr * eps_q[qi];
#pragma unroll
        for (int k = 0; k < 4; ++k) m[k] = m[k] || mg[qi][k] > lim;
      }
    } else {
      // FP64: the reference's quotients, decided exactly (ratio_gt)
      const T* QA[3] = {RHO, P, E};
#pragma unroll
      for (int qi = 0; qi < 3; ++qi) {
        T col[6], lf[4], rt[4];
        column(QA[qi], col, lf, rt);
        const T eps = eps_q[qi];
        bool nn = false;
        bool ey[5];
#pragma unroll
        for (int j = 0; j < 5; ++j) ey[j] = j <= nrow && pair_gt<T, false>(col[j], col[j + 1], eps, thr, T(0), nn);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          if (k >= nrow) continue;
          bool f = ey[k] | ey[k + 1];
          f |= pair_gt<T, false>(lf[k], col[k + 1], eps, thr, T(0), nn);
          f |= pair_gt<T, false>(col[k + 1], rt[k], eps, thr, T(0), nn);
          f |= curv_gt<T, false>(lf[k], col[k + 1], rt[k], eps, thr, T(0), nn);
          f |= curv_gt<T, false>(col[k], col[k + 1], col[k + 2], eps, thr, T(0), nn);
          m[k] = m[k] || f;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k >= nrow) continue;
      const int gj = y0 - W + ar0 + k;
      bool mk = m[k];
      if (comp_on) mk = mk || dvg[k] < comp_lim;
      if (shear_on) mk = mk || vor[k] > shear_lim;
      if (!per) {
        const int bg = S.boundary_guard;
        if (bg > 0 && (gj < bg || gj >= ny - bg || gi < bg || gi >= nx - bg)) mk = true;
        if (!(gj >= 0 && gj < ny && gi >= 0 && gi < nx)) mk = false;
      }
      bits |= (mk ? 1u : 0u) << k;
    }
  }
  // ---- flag bits into one 64-bit word per raw row (warp ballots) ----------------
  // Warp w holds tasks 32 w .. 32 w + 31: lanes [0, L) are columns b0 .. of
  // strip s0, the rest columns 0 .. of strip s0 + 1 (RX >= 32).
  if (32 * warp < NTASK) {
    const int tw0 = 32 * warp;
    const int s0 = tw0 / RX, b0 = tw0 - s0 * RX;
    const int L = min(32, RX - b0);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const unsigned bal = __ballot_sync(kFull, (bits >> k) & 1u);
      if (lane == 0) {
        const unsigned lo = L == 32 ? bal : (bal & ((1u << L) - 1u));
        if (lo) atomicOr(&RB[4 * s0 + k], (unsigned long long)lo << b0);
        if (L < 32) {
          const unsigned hi = bal >> L;
          if (hi) atomicOr(&RB[4 * (s0 + 1) + k], (unsigned long long)hi);
        }
      }
    }
  }
  __syncthreads();
  // ---- (2W + 1)^2 dilation: rows by shifts, columns by ORs of rows ---------------
  // bit i of DR[r] = raw row r has a flagged node among raw columns i .. i + 2W,
  // i.e. within W columns of tile column i
  for (int r = threadIdx.x; r < RY; r += blockDim.x) {
    const unsigned long long wv = RB[r];
    unsigned long long acc = 0ull;
#pragma unroll
    for (int d = 0; d <= 2 * W; ++d) acc |= wv >> d;
    DR[r] = (unsigned)acc;
  }
  __syncthreads();
  uint8_t* mask = S.mask;
  if (threadIdx.x < kSenTY * 8) {
    const int a = threadIdx.x >> 3, c = (threadIdx.x & 7) * 4;
    unsigned mrow = 0;
#pragma unroll
    for (int d = 0; d <= 2 * W; ++d) mrow |= DR[a + d];
    const int gj = y0 + a, gx = x0 + c;
    if (gj < ny && gx < nx) {
      const unsigned b4 = (mrow >> c) & 0xFu;
      uint8_t* dst = mask + (size_t)gj * nx + gx;
      if (gx + 3 < nx && ((reinterpret_cast<uintptr_t>(dst) & 3) == 0)) {
        *reinterpret_cast<uchar4*>(dst) =
            make_uchar4(b4 & 1u, (b4 >> 1) & 1u, (b4 >> 2) & 1u, (b4 >> 3) & 1u);
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (gx + j < nx) dst[j] = (b4 >> j) & 1u;
      }
    }
  }
}

template <typename T, int W>
__global__ void __launch_bounds__(kSensorThreads, sizeof(T) == 8 ? 1 : HITB200_SENSOR_MIN_BLOCKS)
    sensor_step_kernel(const SolveDev* __restrict__ solves, const Work* __restrict__ work, int sel,
                       int enf, int want_visc) {
  extern __shared__ __align__(16) unsigned char smem[];
  sensor_step_body<T, W>(solves, work[blockIdx.x], sel, enf, want_visc, smem, PdlDep{});
}

// The hyperviscosity sensor of a batch (sel 3) as a grid-stride loop over its
// tiles (see hv_prepass_loop_kernel): the same tiles and results as
// sensor_step_kernel's.
template <typename T, int W>
__global__ void __launch_bounds__(kSensorThreads, sizeof(T) == 8 ? 1 : HITB200_SENSOR_MIN_BLOCKS)
    hv_sensor_loop_kernel(const SolveDev* __restrict__ solves, const Work* __restrict__ work, int nwork) {
  extern __shared__ __align__(16) unsigned char smem[];
  for (int item = blockIdx.x; item < nwork; item += gridDim.x) {
    sensor_step_body<T, W>(solves, work[item], 3, 0, 0, smem, PdlDep{});
    __syncthreads();  // shared memory reused by the next tile
  }
}

}  // namespace hitb200
