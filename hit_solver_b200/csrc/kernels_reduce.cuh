// Reducing kernels: per-stage prepass, forcing noise transform, forcing
// synthesis and diagnostics.  See reduce.cuh for the reduction pattern.
#pragma once

#include <float.h>

#include "common.cuh"
#include "reduce.cuh"

namespace hitb200 {

constexpr unsigned kFullMask = 0xffffffffu;

// Pointers a kernel works on when it is called as an operator on caller
// arrays (use = 1) instead of on the solve's own stage buffers.
struct Bind {
  const double* qin;
  const double* q0;
  double* qout;
  const uint8_t* mask;
  double* out;
  const double* fx;
  const double* fy;
  int use;
  int terms;
  int invert_mask;
  int pad_;
};

__device__ __forceinline__ const double* stage_in(const SolveDev& s, int buf) {
  return buf == 0 ? s.q : (buf == 1 ? s.q1 : s.q2);
}
// Stage outputs: q -> q1 -> q2 -> q, except that the last stage writes q1
// when the step ends with hyperviscosity (which then reads q1 and writes q).
__device__ __forceinline__ double* stage_out(const SolveDev& s, int stage) {
  if (stage == 0) return s.q1;
  if (stage == 1) return s.q2;
  return s.scal[S_HV_STEP] != 0.0 ? s.q1 : s.q;
}

enum PreMode : int {
  PRE_STAGE = 0,   // inputs of one RHS evaluation
  PRE_STEP = 1,    // same, plus time step / Mach control / time advance of the step
  PRE_SENSOR = 2,  // sensor limits only (hyperviscosity mask, sensor API)
  PRE_CHECK = 3,   // time step and validation reductions only (API)
};

__device__ __forceinline__ int pre_op(int slot) { return slot < R_FIXED ? red_op(slot) : OP_SUM; }

// Step-level control of the HIT loop body (OOP/hit2d.py:828-845) and of the
// fixed-dt Riemann loop (riemann_config3.py:728-741).
__device__ void step_control(const SolveDev& S, const double* red, double* sc) {
  const double N = (double)S.nx * (double)S.ny;
  const double t = sc[S_TIME], step = sc[S_STEP], maxs = sc[S_MAX_STEPS];
  bool active = (maxs < 0.0 || step < maxs);
  if (!S.fixed_dt) active = active && (t < S.tfinal);
  sc[S_ACTIVE] = active ? 1.0 : 0.0;
  sc[S_HV_STEP] = 0.0;
  if (!active) return;
  double dt;
  if (S.fixed_dt) {
    dt = sc[S_DT];
  } else {
    // stable_time_step (OOP/spatial_operator.py:369-377) + viscous limit
    const double rem = S.tfinal - t;
    dt = S.cfl / red[R_SR];
    dt = fmin(dt, rem);
    if (S.mu > 0.0) {
      const double h = fmin(S.dx, S.dy);
      dt = fmin(fmin(dt, 0.25 * (h * h) / S.mu), rem);
    }
  }
  // update_mach_controlled_power (OOP/hit2d.py:293-349)
  const double mach = sqrt(red[R_VEL2] / N) / (red[R_CSUM] / N);
  sc[S_MACH] = mach;
  double power = sc[S_POWER];
  double desired = power;
  if (S.mach_control && !isnan(power)) {
    const double ratio = pow(S.mach_target / fmax(mach, 1.0e-8), S.mach_exponent);
    desired = power * ratio;
    if (S.has_mach_min) desired = fmax(desired, S.mach_min_power);
    if (S.has_mach_max) desired = fmin(desired, S.mach_max_power);
    power = S.mach_memory * power + (1.0 - S.mach_memory) * desired;
  }
  sc[S_POWER] = power;
  sc[S_POWER_DESIRED] = desired;
  if (S.forcing_on) {
    const double decay = exp(-dt / S.f_tau);
    sc[S_F_DECAY] = decay;
    sc[S_XI_SCALE] = sqrt(fmax(1.0 - decay * decay, 0.0));  // OU increment scale
  }
  sc[S_DT] = dt;
  sc[S_TIME] = t + dt;
  sc[S_STEP] = step + 1.0;
  const long long ns = (long long)(step + 1.0);
  sc[S_HV_STEP] = (S.hv_interval > 0 && ns % S.hv_interval == 0) ? 1.0 : 0.0;
}

// Prepass: one pass over a stage state computing every global quantity the
// RHS needs before its flux pass.  One CTA per 32 x 32 tile, 256 threads,
// each thread owning one column's 4 cells (rows warp, warp + 8, ...).
//   enf = 1: sensor/LF quantities on enforce_physical_state(q), as
//   PeriodicHybridEuler2DOperator.rhs does (OOP/spatial_operator.py:345-346).
// T is the arithmetic type of the sensor/Lax-Friedrichs quantities (float in
// the FP32-bulk form); the raw-state reductions that drive the time step,
// Mach control and validation are FP64 in both forms, and every sum is
// accumulated in FP64.
constexpr int kPreThreads = 256;
// CTAs per SM of the prepass's throughput variant (OCC = 1; the latency
// variant keeps 2).
#ifndef HITB200_PRE_MIN_BLOCKS
#define HITB200_PRE_MIN_BLOCKS 4
#endif
constexpr int kPreWarps = kPreThreads / 32;
constexpr int kPreRows = kTileY / kPreWarps;  // own cells per thread

// Enforced-state primitives of one node (enforce_physical_state followed by
// primitive_from_conservative) in T arithmetic; rinv64 is the node's FP64
// 1 / rho when the caller has it (FP64 form), else ignored.
template <typename T>
struct EnfPrim {
  T u, v, p, rinv, rho;
};
template <typename T>
__device__ __forceinline__ EnfPrim<T> enforced_prim(double q0, double q1, double q2, double q3,
                                                    double g, int enf) {
  EnfPrim<T> r;
  if constexpr (sizeof(T) == 8) {
    const double rho = q0 > kRhoFloor ? q0 : kRhoFloor;
    const double rinv = 1.0 / rho;
    const double ur = q1 * rinv, vr = q2 * rinv;
    const double kin = 0.5 * rho * (ur * ur + vr * vr);
    const double p_raw = (g - 1.0) * (q3 - kin);
    double ue = ur, ve = vr, pe = p_raw;
    if (enf) {
      const double e1 = rho * ur, e2 = rho * vr;
      const double e3 = p_raw > kPFloor ? q3 : kPFloor / (g - 1.0) + kin;
      ue = e1 * rinv;
      ve = e2 * rinv;
      pe = (g - 1.0) * (e3 - 0.5 * rho * (ue * ue + ve * ve));
    }
    r.u = ue;
    r.v = ve;
    r.p = pe > kPFloor ? pe : kPFloor;
    r.rinv = rinv;
    r.rho = rho;
  } else {
    const float gf = (float)g;
    const float rho = (float)q0 > (float)kRhoFloor ? (float)q0 : (float)kRhoFloor;
    const float rinv = __frcp_rn(rho);
    float a1 = (float)q1, a2 = (float)q2, a3 = (float)q3;
    float u = a1 * rinv, v = a2 * rinv;
    const float kin = 0.5f * rho * (u * u + v * v);
    float pr = (gf - 1.0f) * (a3 - kin);
    if (enf) {
      a1 = rho * u;
      a2 = rho * v;
      a3 = pr > (float)kPFloor ? a3 : (float)kPFloor / (gf - 1.0f) + kin;
      u = a1 * rinv;
      v = a2 * rinv;
      pr = (gf - 1.0f) * (a3 - 0.5f * rho * (u * u + v * v));
    }
    r.u = u;
    r.v = v;
    r.p = pr > (float)kPFloor ? pr : (float)kPFloor;
    r.rinv = rinv;
    r.rho = rho;
  }
  return r;
}

// Shared memory of one prepass tile.
template <typename T>
struct PreShared {
  T su[kTileY + 2][kTileX + 2];
  T sv[kTileY + 2][kTileX + 2];
  double2 tw[kTileY][kMaxKyDrag + 1];          // e^{-i k y}, k = 0..ky_drag, of the tile's rows
  double cbuf[kPreWarps][4][32];               // per-warp column partials of one k
  double ctab[kMaxKyDrag + 1][4][32];          // C_k(x) = sum_y m(x, y) e^{-i k y}
  double sm[kPreWarps * (R_FIXED + 4 * kMaxDrag)];
};

// One tile of the prepass: every quantity it reduces, for the tile's cells,
// into this CTA's row of partials (S.part_pre[w.c][*]); returns the number of
// slots.  The tile runs on the kPreThreads threads whose index minus `tofs`
// lies in [0, kPreThreads), with P as its shared memory; every thread of the
// CTA must call it (it synchronises the CTA), with the same solve, mode and
// `active` (a CTA may run two tiles at once, each half of its threads with its
// own tofs and P).
// Returns the number of reduction slots, or -1 when `active` is false: an
// inactive solve's tile stops after its loads (issued before the caller's flag
// arrives, so that they do not wait for it) and writes nothing.
template <typename T>
__device__ int prepass_tile(const SolveDev& S, const Work& w, int buf, int mode, int enf,
                            const Bind& bind, bool active, PreShared<T>& P, int tofs = 0) {
  const int tid = (int)threadIdx.x - tofs;
  const bool act = tid >= 0 && tid < kPreThreads;
  const double* q = bind.use ? bind.qin : stage_in(S, buf);
  const int nx = S.nx, ny = S.ny, per = S.periodic;
  const size_t plane = (size_t)nx * ny;
  const double g = S.gamma;
  const T gT = T(g);
  const T igm1 = T(1.0 / (g - 1.0));
  const double idx_ = 1.0 / S.dx, idy_ = 1.0 / S.dy;
  const T hx = T(S.dx), hy = T(S.dy);
  const T ih2x = T(1.0 / (2.0 * S.dx)), ih2y = T(1.0 / (2.0 * S.dy));
  const int x0 = w.a, y0 = w.b;
  // ranges the plans guarantee, stated for the index arithmetic
  __builtin_assume(nx >= 1 && nx <= kMaxLine && ny >= 1 && ny <= kMaxLine);
  __builtin_assume(x0 >= 0 && x0 < kMaxLine && y0 >= 0 && y0 < kMaxLine);
  const bool grads = mode != PRE_CHECK;
  const bool rawq = mode == PRE_STEP || mode == PRE_CHECK;  // time step, Mach, validation
  const bool psum = S.cooling_on && (mode == PRE_STAGE || mode == PRE_STEP);
  const int nslots = (mode == PRE_STAGE || mode == PRE_STEP) ? S.nred : R_FIXED;
  const int ndrag = nslots > R_FIXED ? S.n_drag : 0;

  auto& su = P.su;
  auto& sv = P.sv;
  auto& tw = P.tw;
  auto& cbuf = P.cbuf;
  auto& ctab = P.ctab;
  double* sm = P.sm;
  const int lane = threadIdx.x & 31, warp = tid >> 5;

  const int KY = ndrag > 0 ? S.ky_drag : -1;
  for (int t = tid; act && t < kTileY * (KY + 1); t += kPreThreads) {
    const int a = t / (KY + 1), k = t - a * (KY + 1);
    const int gj = min(y0 + a, ny - 1);
    tw[a][k] = S.twy[mode_index(k, gj, ny)];
  }

  double div2 = 0, vort2 = 0, ps = 0, sr = 0, vel2 = 0, cs = 0;
  // maxima in the bulk type: exact, so widening once at the end gives the
  // same doubles as widening every value
  T axT = T(0), ayT = T(0), mrT = T(0), mpT = T(0), meT = T(0);
  int bad = 0;  // validation flags: 1 non-finite, 2 rho <= 0, 4 p <= 0
  const int gi = x0 + lane;
  // one-node ring for the central differences (corners are not used), loaded
  // first so that its latency overlaps the tile's
  const bool ring = grads && act && tid < 4 * kTileX;
  int ra = 0, rb = 0;  // smem coordinates
  double rq[4] = {0.0, 0.0, 0.0, 0.0};
  if (ring) {
    const int side = tid >> 5, t = tid & 31;
    if (side == 0) { ra = 0; rb = t + 1; }
    else if (side == 1) { ra = kTileY + 1; rb = t + 1; }
    else if (side == 2) { ra = t + 1; rb = 0; }
    else { ra = t + 1; rb = kTileX + 1; }
    const int gj = fold_node(y0 + ra - 1, ny, per), gx = fold_node(x0 + rb - 1, nx, per);
    const size_t o = (size_t)gj * nx + gx;
#pragma unroll
    for (int c = 0; c < 4; ++c) rq[c] = q[o + c * plane];
  }
  double m0[kPreRows], m1[kPreRows];
#pragma unroll
  for (int k = 0; k < kPreRows; ++k) {
    const int a = warp + kPreWarps * k, gj = y0 + a;
    m0[k] = m1[k] = 0.0;
    if (!act) continue;
    if (gj >= ny || gi >= nx) {
      // beyond the grid in a partial tile: the folded node is the halo of
      // the last row / column
      if (grads) {
        const size_t o = (size_t)fold_node(gj, ny, per) * nx + fold_node(gi, nx, per);
        const EnfPrim<T> e = enforced_prim<T>(q[o], q[o + plane], q[o + 2 * plane], q[o + 3 * plane], g, enf);
        su[a + 1][lane + 1] = e.u;
        sv[a + 1][lane + 1] = e.v;
      }
      continue;
    }
    const size_t o = (size_t)gj * nx + gi;
    const double q0 = q[o], q1 = q[o + plane], q2 = q[o + 2 * plane], q3 = q[o + 3 * plane];
    m0[k] = q1;
    m1[k] = q2;
    T ep = T(0);
    if (mode != PRE_CHECK) {
      const EnfPrim<T> e = enforced_prim<T>(q0, q1, q2, q3, g, enf);
      ep = e.p;
      su[a + 1][lane + 1] = e.u;
      sv[a + 1][lane + 1] = e.v;
      const T c = sqrt(gT * e.p * e.rinv);
      axT = fmax(axT, fabs(e.u) + c);
      ayT = fmax(ayT, fabs(e.v) + c);
      mrT = fmax(mrT, e.rho);
      mpT = fmax(mpT, e.p);
      meT = fmax(meT, e.p * e.rinv * igm1);
    }
    // cooling's mean pressure: the FP32-bulk form takes it from its enforced
    // pressure (equal to the floored raw pressure up to rounding)
    const bool psum64 = psum && (sizeof(T) == 8 || rawq);
    if (psum && !psum64) ps += double(ep);
    if (rawq || psum64) {
      const double rho = q0 > kRhoFloor ? q0 : kRhoFloor;
      const double rinv = 1.0 / rho;
      const double ur = q1 * rinv, vr = q2 * rinv;
      const double p_raw = (g - 1.0) * (q3 - 0.5 * rho * (ur * ur + vr * vr));
      const double pr = p_raw > kPFloor ? p_raw : kPFloor;
      ps += pr;
      if (rawq) {
        const double cr = sqrt(g * pr * rinv);
        sr = fmax(sr, (fabs(ur) + cr) * idx_ + (fabs(vr) + cr) * idy_);
        vel2 += ur * ur + vr * vr;
        cs += cr;
        // validate_raw_physical_state: p = (g-1)(E - (m_x^2 + m_y^2) / (2 rho)) on
        // the unfloored density; its sign is that of 2 rho E - |m|^2 when rho > 0
        const bool fin = isfinite(q0) && isfinite(q1) && isfinite(q2) && isfinite(q3);
        const double pp = 2.0 * q0 * q3 - (q1 * q1 + q2 * q2);
        if (!fin || !isfinite(pp)) bad |= 1;
        if (q0 <= 0.0) bad |= 2;
        else if (pp <= 0.0) bad |= 4;
      }
    }
  }
  if (grads) {
    if (ring) {
      const EnfPrim<T> e = enforced_prim<T>(rq[0], rq[1], rq[2], rq[3], g, enf);
      su[ra][rb] = e.u;
      sv[ra][rb] = e.v;
    }
    __syncthreads();
    if (!active) return -1;
#pragma unroll
    for (int k = 0; k < kPreRows; ++k) {
      const int a0 = warp + kPreWarps * k, gj = y0 + a0;
      if (!act || gj >= ny || gi >= nx) continue;
      // sensor divergence / vorticity: central, one-sided at outflow edges
      const int a = a0 + 1, b = lane + 1;
      T dudx, dvdx, dudy, dvdy;
      if (per || (gi > 0 && gi < nx - 1)) {
        dudx = (su[a][b + 1] - su[a][b - 1]) * ih2x;
        dvdx = (sv[a][b + 1] - sv[a][b - 1]) * ih2x;
      } else if (nx == 1) {
        dudx = dvdx = T(0);
      } else if (gi == 0) {
        dudx = (su[a][b + 1] - su[a][b]) / hx;
        dvdx = (sv[a][b + 1] - sv[a][b]) / hx;
      } else {
        dudx = (su[a][b] - su[a][b - 1]) / hx;
        dvdx = (sv[a][b] - sv[a][b - 1]) / hx;
      }
      if (per || (gj > 0 && gj < ny - 1)) {
        dudy = (su[a + 1][b] - su[a - 1][b]) * ih2y;
        dvdy = (sv[a + 1][b] - sv[a - 1][b]) * ih2y;
      } else if (ny == 1) {
        dudy = dvdy = T(0);
      } else if (gj == 0) {
        dudy = (su[a + 1][b] - su[a][b]) / hy;
        dvdy = (sv[a + 1][b] - sv[a][b]) / hy;
      } else {
        dudy = (su[a][b] - su[a - 1][b]) / hy;
        dvdy = (sv[a][b] - sv[a - 1][b]) / hy;
      }
      const T dv = dudx + dvdy, vo = dvdx - dudy;
      div2 += double(dv * dv);
      vort2 += double(vo * vo);
    }
  } else {
    __syncthreads();  // tw table
    if (!active) return -1;
  }
  const double ax = double(axT), ay = double(ayT), mr = double(mrT), mp = double(mpT), me = double(meT);
  if (act) {
  warp_to_smem4<OP_MAX>(ax, ay, mr, mp, sm, make_int4(R_AX, R_AY, R_RHO, R_P), nslots, warp);
  warp_to_smem4<OP_MAX>(me, sr, 0.0, 0.0, sm, make_int4(R_E, R_SR, -1, -1), nslots, warp);
  warp_to_smem4<OP_SUM>(div2, vort2, ps, vel2, sm, make_int4(R_DIV2, R_VORT2, R_PSUM, R_VEL2), nslots, warp);
  warp_to_smem<OP_SUM>(cs, sm, R_CSUM, nslots, warp);
  bad = __reduce_or_sync(kFullMask, bad);
  if (lane == 0) {
    sm[warp * nslots + R_NONFINITE] = (bad & 1) ? 1.0 : 0.0;
    sm[warp * nslots + R_NONPOS_RHO] = (bad & 2) ? 1.0 : 0.0;
    sm[warp * nslots + R_NONPOS_P] = (bad & 4) ? 1.0 : 0.0;
  }
  }
  // low-k momentum transform of the drag band filter (OOP/hit2d.py:352-399),
  // separable: C_k(x) = sum_y m(x, y) e^{-i k y} per column for k = 0..ky_drag
  // (C_{-k} = conj C_k for real m), then per mode sum_x e^{-i kx x} C_ky(x).
  // Each mode is reduced by one warp and its partials go straight to the
  // CTA's row of partials.
  for (int k = 0; k <= KY; ++k) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};  // Re, Im of m0; Re, Im of m1
#pragma unroll
    for (int kk = 0; kk < kPreRows; ++kk) {
      if (!act) break;
      const double2 ey = tw[warp + kPreWarps * kk][k];
      v[0] += m0[kk] * ey.x;
      v[1] += m0[kk] * ey.y;
      v[2] += m1[kk] * ey.x;
      v[3] += m1[kk] * ey.y;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (act) cbuf[warp][j][lane] = v[j];
    __syncthreads();
    if (act && warp < 4) {
      double acc = cbuf[0][warp][lane];
#pragma unroll
      for (int ww = 1; ww < kPreWarps; ++ww) acc += cbuf[ww][warp][lane];
      ctab[k][warp][lane] = acc;
    }
    __syncthreads();
  }
  for (int md = warp; act && md < ndrag; md += kPreWarps) {
    const int2 km = S.modes[md];
    const int ky = abs(km.y);
    const double sy = km.y < 0 ? -1.0 : 1.0;  // conjugate for negative ky
    const double c0r = ctab[ky][0][lane], c0i = sy * ctab[ky][1][lane];
    const double c1r = ctab[ky][2][lane], c1i = sy * ctab[ky][3][lane];
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (gi < nx) {
      const double2 ex = S.twx[mode_index(km.x, gi, nx)];
      v[0] = ex.x * c0r - ex.y * c0i;
      v[1] = ex.x * c0i + ex.y * c0r;
      v[2] = ex.x * c1r - ex.y * c1i;
      v[3] = ex.x * c1i + ex.y * c1r;
    }
    // warp total of the four sums into lanes 0, 8, 16, 24 of sm row `warp`,
    // then straight to this CTA's partials
    const int sl = R_FIXED + 4 * md;
    warp_to_smem4<OP_SUM>(v[0], v[1], v[2], v[3], sm, make_int4(sl, sl + 1, sl + 2, sl + 3), nslots, warp);
    __syncwarp();
    if (lane < 4) S.part_pre[(size_t)w.c * nslots + sl + lane] = sm[warp * nslots + sl + lane];
  }
  __syncthreads();
  for (int t = tid; t < R_FIXED; t += kPreThreads) {
    if (!act) break;
    const int op = pre_op(t);
    double acc = sm[t];
    for (int ww = 1; ww < kPreWarps; ++ww) {
      const double x = sm[ww * nslots + t];
      acc = op == OP_SUM ? acc + x : fmax(acc, x);
    }
    S.part_pre[(size_t)w.c * nslots + t] = acc;
  }
  return nslots;
}

// Fixed-order final reduction of the prepass partials of solve S into red[]:
// every thread takes one slot and every C-th block (C = kPreThreads / slots),
// with many loads in flight, and the C partials of a slot are combined in a
// fixed order.  Every thread of the CTA must call it; the first kPreThreads
// work.  The result is the same whichever CTA computes it.  chunk is shared
// scratch of kPreThreads doubles.
__device__ void prepass_finalize(const SolveDev& S, int nslots, double* red, double* chunk) {
  const int C = max(1, kPreThreads / nslots);
  const int t = threadIdx.x % nslots, j = threadIdx.x / nslots;
  const int op = pre_op(t);
  double acc = op == OP_SUM ? 0.0 : -INFINITY;
  if (threadIdx.x < kPreThreads && j < C) {
    // 16 loads in flight per round (the partials come from every SM's
    // recent stores), combined in block order
    const double* base = S.part_pre + t;
    const int nb = S.nblk_pre;
    for (int b0 = j; b0 < nb; b0 += 16 * C) {
      double x[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int b = b0 + i * C;
        x[i] = b < nb ? __ldcg(base + (size_t)b * nslots) : 0.0;
      }
#pragma unroll
      for (int i = 0; i < 16; ++i)
        if (b0 + i * C < nb) acc = op == OP_SUM ? acc + x[i] : fmax(acc, x[i]);
    }
    chunk[j * nslots + t] = acc;
  }
  __syncthreads();
  if (threadIdx.x < nslots) {
    double v = chunk[threadIdx.x];
    for (int jj = 1; jj < C; ++jj) {
      const double x = chunk[jj * nslots + threadIdx.x];
      v = op == OP_SUM ? v + x : fmax(v, x);
    }
    red[threadIdx.x] = v;
  }
  __syncthreads();
}

// The scalar logic of one prepass from its reductions (one thread).
__device__ void prepass_scalars(const SolveDev& S, const double* red, double* sc, int mode,
                                bool api) {
  const double N = (double)S.nx * (double)S.ny;
  int status = 0;
  if (red[R_NONFINITE] > 0.0) status |= ST_NONFINITE;
  if (red[R_NONPOS_RHO] > 0.0) status |= ST_NONPOS_RHO;
  if (red[R_NONPOS_P] > 0.0) status |= ST_NONPOS_P;
  sc[S_STATUS] = (double)((int)sc[S_STATUS] | status);
  if (mode == PRE_CHECK) {
    sc[S_DT] = red[R_SR];  // caller turns the spectral radius into a time step
    return;
  }
  sc[S_ALPHA_X] = red[R_AX];
  sc[S_ALPHA_Y] = red[R_AY];
  const double div_rms = sqrt(red[R_DIV2] / N);
  const double vort_rms = sqrt(red[R_VORT2] / N);
  sc[S_DIV_RMS] = div_rms;
  sc[S_VORT_RMS] = vort_rms;
  sc[S_COMP_LIM] = div_rms > 1e-12 ? -S.comp_thr * div_rms : -INFINITY;
  sc[S_SHEAR_LIM] = (S.shear_on && vort_rms > 1e-12) ? S.shear_thr * vort_rms : INFINITY;
  sc[S_EPS_RHO] = 1e-14 + 1e-12 * red[R_RHO];
  sc[S_EPS_P] = 1e-14 + 1e-12 * red[R_P];
  sc[S_EPS_E] = 1e-14 + 1e-12 * red[R_E];
  if (mode == PRE_SENSOR) {
    if (!api) sc[S_HV_APPLIED] += 1.0;  // this prepass runs only on hyperviscosity steps
    return;
  }
  // cooling_source (OOP/hit2d.py:402-426)
  sc[S_COOL] = S.cooling_on
                   ? -((red[R_PSUM] / N - S.cooling_pref) / (S.gamma - 1.0)) / S.cooling_tau
                   : 0.0;
  // drag: S = -c * lowpass(momentum); store -c/N times the mode sums
  for (int m = 0; m < S.n_drag; ++m)
    for (int k = 0; k < 4; ++k) sc[S_DRAG + 4 * m + k] = (-S.drag_coef / N) * red[R_FIXED + 4 * m + k];
  if (mode == PRE_STEP) step_control(S, red, sc);
}


template <typename T, int OCC>
__global__ void __launch_bounds__(kPreThreads, OCC ? HITB200_PRE_MIN_BLOCKS : 2)
    prepass_kernel(const SolveDev* __restrict__ solves, const Work* __restrict__ work, int buf,
                   int mode, int enf, Bind bind) {
  const Work w = work[blockIdx.x];
  const SolveDev& S = solves[w.solve];
  double* sc = S.scal;
  pdl_wait();  // below: the state and scalars of the previous kernels
  if (mode == PRE_SENSOR && !bind.use && sc[S_HV_STEP] == 0.0) return;  // no hyperviscosity this step
  const bool active = !(mode == PRE_STAGE && !bind.use && sc[S_ACTIVE] == 0.0);
  __shared__ PreShared<T> ps;
  const int nslots = prepass_tile<T>(S, w, buf, mode, enf, bind, active, ps);
  if (nslots < 0) return;
  pdl_release();
  if (!last_block(&S.counters[0], S.nblk_pre)) return;
  // ---- last CTA of this solve: fixed-order final reduction + scalar logic ----
  __shared__ double red[R_FIXED + 4 * kMaxDrag];
  __shared__ double chunk[kPreThreads];
  prepass_finalize(S, nslots, red, chunk);
  if (threadIdx.x == 0) {
    prepass_scalars(S, red, sc, mode, bind.use);
    // a bounded wait of an earlier kernel of this solve that ran out
    if (atomicExch(&S.counters[6], 0u)) sc[S_STATUS] = (double)((int)sc[S_STATUS] | ST_BARRIER);
  }
}

// The hyperviscosity prepass of a batch (PRE_SENSOR on q1) as a grid-stride
// loop over its tiles: on the steps without hyperviscosity every tile is a
// no-op, and a grid of a few CTAs per SM costs a small fraction of one CTA
// per tile.  Each tile runs prepass_kernel's code with its own partial row
// and ticket, so the results are those of prepass_kernel.
template <typename T>
__global__ void __launch_bounds__(kPreThreads, HITB200_PRE_MIN_BLOCKS)
    hv_prepass_loop_kernel(const SolveDev* __restrict__ solves, const Work* __restrict__ work, int nwork) {
  __shared__ PreShared<T> ps;
  __shared__ double red[R_FIXED + 4 * kMaxDrag];
  __shared__ double chunk[kPreThreads];
  const Bind nb{};
  for (int item = blockIdx.x; item < nwork; item += gridDim.x) {
    const Work w = work[item];
    const SolveDev& S = solves[w.solve];
    double* sc = S.scal;
    if (sc[S_HV_STEP] == 0.0) continue;  // no hyperviscosity this step
    const int nslots = prepass_tile<T>(S, w, 1, PRE_SENSOR, 0, nb, true, ps);
    if (last_block(&S.counters[0], S.nblk_pre)) {
      prepass_finalize(S, nslots, red, chunk);
      if (threadIdx.x == 0) {
        prepass_scalars(S, red, sc, PRE_SENSOR, false);
        if (atomicExch(&S.counters[6], 0u)) sc[S_STATUS] = (double)((int)sc[S_STATUS] | ST_BARRIER);
      }
    }
    __syncthreads();  // shared memory reused by the next tile
  }
}

// Forward transform of the caller's white-noise field restricted to the
// forcing shell (the masked fft2 of OOP/forcing.py:77-79), then the OU update
// of the potential (forcing.py:80).
__global__ void __launch_bounds__(kRedThreads)
    noise_dft_kernel(const SolveDev* __restrict__ solves, const Work* __restrict__ work,
                     Bind bind) {
  const Work w = work[blockIdx.x];
  const SolveDev& S = solves[w.solve];
  double* sc = S.scal;
  if (!S.forcing_on) return;
  if (!bind.use && sc[S_ACTIVE] == 0.0) return;
  const double* xi = bind.use ? bind.qin : S.noise;
  const int nx = S.nx, ny = S.ny, nf = S.n_force;
  const int2* modes = S.modes + S.n_drag;
  __shared__ double sm[kRedWarps * 2 * kMaxForce];
  __shared__ double red[2 * kMaxForce];
  const int tx = threadIdx.x & 31, ty0 = threadIdx.x >> 5;
  double val[kCellsPerThread];
  int cj[kCellsPerThread], ci[kCellsPerThread];
  bool valid[kCellsPerThread];
#pragma unroll
  for (int k = 0; k < kCellsPerThread; ++k) {
    cj[k] = w.b + ty0 + kRedWarps * k;
    ci[k] = w.a + tx;
    valid[k] = cj[k] < ny && ci[k] < nx;
    val[k] = valid[k] ? xi[(size_t)cj[k] * nx + ci[k]] : 0.0;
  }
  const int nslots = 2 * nf;
  for (int m = 0; m < nf; ++m) {
    const int2 md = modes[m];
    double re = 0.0, im = 0.0;
#pragma unroll
    for (int k = 0; k < kCellsPerThread; ++k) {
      if (!valid[k]) continue;
      const double2 ex = S.twx[mode_index(md.x, ci[k], nx)], ey = S.twy[mode_index(md.y, cj[k], ny)];
      re += val[k] * cmul_re(ex, ey);
      im += val[k] * cmul_im(ex, ey);
    }
    warp_to_smem<OP_SUM>(re, sm, 2 * m, nslots);
    warp_to_smem<OP_SUM>(im, sm, 2 * m + 1, nslots);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nslots; t += blockDim.x) {
    double acc = sm[t];
    for (int ww = 1; ww < kRedWarps; ++ww) acc += sm[ww * nslots + t];
    S.part_noise[(size_t)w.c * nslots + t] = acc;
  }
  if (!last_block(&S.counters[1], S.nblk_noise)) return;
  {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int t = warp; t < nslots; t += kRedWarps) {
      double acc = 0.0;
#pragma unroll 8
      for (int b = lane; b < S.nblk_noise; b += 32)
        acc += __ldcg(S.part_noise + (size_t)b * nslots + t);
      acc = warp_sum(acc);
      if (lane == 0) red[t] = acc;
    }
    __syncthreads();
  }
  // OU update: phi <- decay phi + sqrt(1 - decay^2) xi_hat
  const double decay = sc[S_F_DECAY], inc = sc[S_XI_SCALE];
  for (int m = threadIdx.x; m < nf; m += blockDim.x) {
    sc[S_XI + 2 * m] = red[2 * m];
    sc[S_XI + 2 * m + 1] = red[2 * m + 1];
    sc[S_PHI + 2 * m] = decay * sc[S_PHI + 2 * m] + inc * red[2 * m];
    sc[S_PHI + 2 * m + 1] = decay * sc[S_PHI + 2 * m + 1] + inc * red[2 * m + 1];
  }
}

// ---- counter-based normal deviates (Philox4x32-10, Salmon et al., SC'11) ----
__device__ __forceinline__ uint4 philox4x32_10(uint4 ctr, uint2 key) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const unsigned hi0 = __umulhi(0xD2511F53u, ctr.x), lo0 = 0xD2511F53u * ctr.x;
    const unsigned hi1 = __umulhi(0xCD9E8D57u, ctr.z), lo1 = 0xCD9E8D57u * ctr.z;
    ctr = make_uint4(hi1 ^ ctr.y ^ key.x, lo1, hi0 ^ ctr.w ^ key.y, lo0);
    key.x += 0x9E3779B9u;
    key.y += 0xBB67AE85u;
  }
  return ctr;
}
__device__ __forceinline__ double u01(unsigned a, unsigned b) {
  // 53-bit uniform in (0, 1]
  const unsigned long long x = ((unsigned long long)a << 21) ^ (unsigned long long)b;
  return ((double)(x & ((1ull << 53) - 1)) + 1.0) * (1.0 / 9007199254740992.0);
}

// Device-drawn shell noise: the masked transform of N x N white noise has, for
// every conjugate pair (k, -k), independent real and imaginary parts
// ~ N(0, N/2) and Hermitian symmetry; a self-conjugate mode is real ~ N(0, N).
// Drawing these directly gives the reference's forcing statistics without the
// grid-sized noise field.  One CTA per solve; then the OU update.
__global__ void noise_rng_kernel(const SolveDev* __restrict__ solves, int nsolves,
                                 const int* __restrict__ partner) {
  const int s = blockIdx.x;
  if (s >= nsolves) return;
  const SolveDev& S = solves[s];
  double* sc = S.scal;
  if (sc[S_ACTIVE] == 0.0 || !S.forcing_on) return;
  const int nf = S.n_force;
  const double N = (double)S.nx * (double)S.ny;
  const unsigned long long step = (unsigned long long)sc[S_STEP];
  const double decay = sc[S_F_DECAY], inc = sc[S_XI_SCALE];
  const int* pt = partner + s * kMaxForce;
  for (int m = threadIdx.x; m < nf; m += blockDim.x) {
    const int pm = pt[m];
    const int lead = m < pm ? m : pm;  // the pair is drawn once, by its lower index
    const uint4 r = philox4x32_10(make_uint4((unsigned)lead, (unsigned)step, (unsigned)(step >> 32), 0x5eedu),
                                  make_uint2((unsigned)S.seed, (unsigned)(S.seed >> 32)));
    const double u1 = u01(r.x, r.y), u2 = u01(r.z, r.w);
    const double rad = sqrt(-2.0 * log(u1));
    double sn, cn;
    sincospi(2.0 * u2, &sn, &cn);
    double re, im;
    if (pm == m) {
      re = sqrt(N) * rad * cn;
      im = 0.0;
    } else {
      re = sqrt(0.5 * N) * rad * cn;
      im = sqrt(0.5 * N) * rad * sn;
      if (m != lead) im = -im;
    }
    sc[S_XI + 2 * m] = re;
    sc[S_XI + 2 * m + 1] = im;
    sc[S_PHI + 2 * m] = decay * sc[S_PHI + 2 * m] + inc * re;
    sc[S_PHI + 2 * m + 1] = decay * sc[S_PHI + 2 * m + 1] + inc * im;
  }
}

// Forcing synthesis: f_hat = (i ky phi, -i kx phi), fx = Re ifft2 (forcing.py:
// 82-85) evaluated directly on the shell modes, plus the sums the rescaling
// needs (forcing.py:87-118), then the scalar rescaling logic.  The synthesis
// is separable: each CTA covers whole rows, in chunks of about 1024 cells
// (synth_rows; w.a chunks from row w.b, at least one), each with its own row
// of partial sums (w.c, w.c + 1, ...), so that how chunks are grouped into
// CTAs changes no result; for each of a chunk's rows y the modes are first
// folded into
// P_k(y) = sum over modes with |kx| = k of c_m e^{i ky y} (conjugated for
// kx < 0), so that a cell needs only Re sum_k P_k(y) e^{i k x}, k = 0..max|kx|.
__global__ void __launch_bounds__(kRedThreads)
    force_synth_kernel(const SolveDev* __restrict__ solves, const Work* __restrict__ work,
                       Bind bind) {
  const Work w = work[blockIdx.x];
  const SolveDev& S = solves[w.solve];
  double* sc = S.scal;
  if (!S.forcing_on) return;
  if (!bind.use && sc[S_ACTIVE] == 0.0) return;
  const double* q = bind.use ? bind.qin : S.q;
  const int nx = S.nx, ny = S.ny, nf = S.n_force, K = S.kx_force;
  const size_t plane = (size_t)nx * ny;
  const int2* modes = S.modes + S.n_drag;
  const double invN = 1.0 / ((double)nx * (double)ny);
  __shared__ double2 ca[kMaxForce], cb[kMaxForce];
  __shared__ double2 px[kSynthMaxRows][kMaxKx + 1], py[kSynthMaxRows][kMaxKx + 1];
  __shared__ double sm[kRedWarps * 4];
  __shared__ double red[4];
  // the solve's mode tables in shared memory, read by every (row, mode) term
  __shared__ int2 mk[kMaxForce];  // (x bin, y bin) of the modes in |x bin| order
  __shared__ short kofs[kMaxKx + 2];
  // ca, cb and mk are indexed by the position j in that order (mode f_order[j])
  for (int j = threadIdx.x; j < nf; j += blockDim.x) {
    const int m = S.f_order[j];
    const double pr = sc[S_PHI + 2 * m], pi = sc[S_PHI + 2 * m + 1];
    const double2 kv = S.kvec[m];
    ca[j] = make_double2(-kv.y * pi * invN, kv.y * pr * invN);   // (i ky phi)/N
    cb[j] = make_double2(kv.x * pi * invN, -kv.x * pr * invN);   // (-i kx phi)/N
    mk[j] = modes[m];
  }
  for (int k = threadIdx.x; k < K + 2; k += blockDim.x) kofs[k] = S.f_kofs[k];
  __syncthreads();
  const double2* __restrict__ twy = S.twy;
  const int nch = w.a > 1 ? w.a : 1;
  for (int ch = 0; ch < nch; ++ch) {
  // this chunk: rows r0 .. r0 + rows - 1, every column
  const int r0 = w.b + ch * synth_rows(nx);
  const int rows = min(synth_rows(nx), ny - r0);
  // row tables in chunks of rows: one thread per (row, mode) term into shared
  // memory (the twiddle loads all in flight at once), then each (row, |kx|)
  // sum over its modes in mode order
  __shared__ double2 tmx[kSynthTerms], tmy[kSynthTerms];
  const int rc = max(1, min(rows, kSynthTerms / max(nf, 1)));
  for (int a0 = 0; a0 < rows; a0 += rc) {
    const int na = min(rc, rows - a0);
    for (int t = threadIdx.x; t < na * nf; t += blockDim.x) {
      const int aa = t / nf, j = t - aa * nf;
      const int2 md = mk[j];
      const double2 e = twy[mode_index(md.y, r0 + a0 + aa, ny)];  // e^{-i ky y}
      const double er = e.x, ei = -e.y;                             // e^{+i ky y}
      double ar = ca[j].x * er - ca[j].y * ei, ai = ca[j].x * ei + ca[j].y * er;
      double br = cb[j].x * er - cb[j].y * ei, bi = cb[j].x * ei + cb[j].y * er;
      if (md.x < 0) {
        ai = -ai;
        bi = -bi;
      }
      tmx[t] = make_double2(ar, ai);
      tmy[t] = make_double2(br, bi);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < na * (K + 1); t += blockDim.x) {
      const int aa = t / (K + 1), k = t - aa * (K + 1);
      double2 sx = make_double2(0.0, 0.0), sy = make_double2(0.0, 0.0);
      for (int j = kofs[k]; j < kofs[k + 1]; ++j) {
        const double2 u = tmx[aa * nf + j], v = tmy[aa * nf + j];
        sx.x += u.x;
        sx.y += u.y;
        sy.x += v.x;
        sy.y += v.y;
      }
      px[a0 + aa][k] = sx;
      py[a0 + aa][k] = sy;
    }
    __syncthreads();
  }
  double sxx = 0, syy = 0, sxy = 0, spow = 0;
  for (int idx = threadIdx.x; idx < rows * nx; idx += blockDim.x) {
    const int a = idx / nx, gi = idx - a * nx, gj = r0 + a;
    double fx = px[a][0].x, fy = py[a][0].x;
    int ix = 0;
    for (int k = 1; k <= K; ++k) {
      ix += gi;
      if (ix >= nx) ix -= nx;                 // (k x) mod nx
      const double2 e = S.twx[ix];             // e^{-i k x}
      const double er = e.x, ei = -e.y;       // e^{+i k x}
      fx += px[a][k].x * er - px[a][k].y * ei;
      fy += py[a][k].x * er - py[a][k].y * ei;
    }
    const size_t o = (size_t)gj * nx + gi;
    if (S.precision == 1) {
      static_cast<float*>(S.fx)[o] = (float)fx;
      static_cast<float*>(S.fy)[o] = (float)fy;
    } else {
      static_cast<double*>(S.fx)[o] = fx;
      static_cast<double*>(S.fy)[o] = fy;
    }
    const Prim<double> p = primitives(q[o], q[o + plane], q[o + 2 * plane], q[o + 3 * plane], S.gamma);
    sxx += fx * fx;
    syy += fy * fy;
    sxy += fx * fy;
    spow += p.rho * (fx * p.u + fy * p.v);
  }
  warp_to_smem4<OP_SUM>(sxx, syy, sxy, spow, sm, make_int4(0, 1, 2, 3), 4);
  __syncthreads();
  if (threadIdx.x < 4) {
    double acc = sm[threadIdx.x];
    for (int ww = 1; ww < kRedWarps; ++ww) acc += sm[ww * 4 + threadIdx.x];
    S.part_synth[(size_t)(w.c + ch) * 4 + threadIdx.x] = acc;
  }
  __syncthreads();  // sm, px, py reused by the next chunk
  }
  // ticket over chunks: the CTA finishing the solve's last ones reduces them
  __shared__ bool s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned t = atomicAdd(&S.counters[2], (unsigned)nch);
    s_last = t + (unsigned)nch == (unsigned)S.nblk_synth;
    if (s_last) S.counters[2] = 0u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp < 4) {
      double acc = 0.0;
      for (int b = lane; b < S.nblk_synth; b += 32) acc += __ldcg(S.part_synth + (size_t)b * 4 + warp);
      acc = warp_sum(acc);
      if (lane == 0) red[warp] = acc;
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  // rms normalisation and power rescaling (OOP/forcing.py:87-118)
  const double mxx = red[0] * invN, myy = red[1] * invN, mxy = red[2] * invN, mp = red[3] * invN;
  const double rms = sqrt((red[0] + red[1]) * invN);
  double s = 1.0;
  if (S.f_rms <= 0.0) s = 0.0;
  else if (rms > DBL_EPSILON) s = S.f_rms / rms;
  const double p_before = s * mp;
  double alpha = sc[S_F_ALPHA];
  double alpha_t = alpha;
  const double target = sc[S_POWER];
  if (!isnan(target) && fabs(p_before) > S.f_min_power) {
    alpha_t = target / p_before;
    if (S.f_has_max_rescale) alpha_t = fmin(fmax(alpha_t, -S.f_max_rescale), S.f_max_rescale);
    alpha = S.f_alpha_memory * alpha + (1.0 - S.f_alpha_memory) * alpha_t;
  } else if (isnan(target)) {
    alpha = 1.0;
  }
  const double fs = s * alpha;
  const double fxx = fs * fs * mxx, fyy = fs * fs * myy, fxy = fs * fs * mxy;
  const double den = fxx + fyy;
  sc[S_F_SCALE] = fs;
  sc[S_F_ALPHA] = alpha;
  sc[S_F_ALPHA_TARGET] = alpha_t;
  sc[S_F_POWER_BEFORE] = p_before;
  sc[S_F_INJECTED] = fs * mp;
  sc[S_F_FXX] = fxx;
  sc[S_F_FYY] = fyy;
  sc[S_F_FXY] = fxy;
  sc[S_F_AF] = den > 0.0 ? fabs(fxx - fyy) / den : 0.0;
}

// Conservation and flow diagnostics: plain sums over the raw state, combined
// on the host (OOP/hit2d.py:471-514 moments, plus momentum / energy sums).
enum DiagSlot : int {
  D_RHO = 0, D_U, D_V, D_RU, D_RV, D_RUU, D_RVV, D_RUV, D_VEL2, D_C, D_P, D_Q0, D_Q1, D_Q2, D_Q3,
  D_RHOMIN, D_RHOMAX, D_PMIN, D_PMAX, NDIAG
};
__global__ void __launch_bounds__(kRedThreads)
    diag_kernel(const SolveDev* __restrict__ solves, const Work* __restrict__ work, Bind bind) {
  const Work w = work[blockIdx.x];
  const SolveDev& S = solves[w.solve];
  const double* q = bind.use ? bind.qin : S.q;
  const int nx = S.nx, ny = S.ny;
  const size_t plane = (size_t)nx * ny;
  __shared__ double sm[kRedWarps * NDIAG];
  __shared__ double red[NDIAG];
  double acc[NDIAG];
#pragma unroll
  for (int k = 0; k < NDIAG; ++k) acc[k] = 0.0;
  acc[D_RHOMIN] = acc[D_PMIN] = INFINITY;
  acc[D_RHOMAX] = acc[D_PMAX] = -INFINITY;
  const int tx = threadIdx.x & 31, ty0 = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kCellsPerThread; ++k) {
    const int gj = w.b + ty0 + kRedWarps * k, gi = w.a + tx;
    if (gj >= ny || gi >= nx) continue;
    const size_t o = (size_t)gj * nx + gi;
    const double q0 = q[o], q1 = q[o + plane], q2 = q[o + 2 * plane], q3 = q[o + 3 * plane];
    const Prim<double> p = primitives(q0, q1, q2, q3, S.gamma);
    acc[D_RHO] += p.rho;
    acc[D_U] += p.u;
    acc[D_V] += p.v;
    acc[D_RU] += p.rho * p.u;
    acc[D_RV] += p.rho * p.v;
    acc[D_RUU] += p.rho * p.u * p.u;
    acc[D_RVV] += p.rho * p.v * p.v;
    acc[D_RUV] += p.rho * p.u * p.v;
    acc[D_VEL2] += p.u * p.u + p.v * p.v;
    acc[D_C] += sqrt(S.gamma * p.p / p.rho);
    acc[D_P] += p.p;
    acc[D_Q0] += q0;
    acc[D_Q1] += q1;
    acc[D_Q2] += q2;
    acc[D_Q3] += q3;
    const double ur = q1 / q0, vr = q2 / q0;
    const double praw = (S.gamma - 1.0) * (q3 - 0.5 * q0 * (ur * ur + vr * vr));
    acc[D_RHOMIN] = fmin(acc[D_RHOMIN], q0);
    acc[D_RHOMAX] = fmax(acc[D_RHOMAX], q0);
    acc[D_PMIN] = fmin(acc[D_PMIN], praw);
    acc[D_PMAX] = fmax(acc[D_PMAX], praw);
  }
#pragma unroll
  for (int k = 0; k < D_RHOMIN; ++k) warp_to_smem<OP_SUM>(acc[k], sm, k, NDIAG);
  warp_to_smem<OP_MAX>(-acc[D_RHOMIN], sm, D_RHOMIN, NDIAG);
  warp_to_smem<OP_MAX>(acc[D_RHOMAX], sm, D_RHOMAX, NDIAG);
  warp_to_smem<OP_MAX>(-acc[D_PMIN], sm, D_PMIN, NDIAG);
  warp_to_smem<OP_MAX>(acc[D_PMAX], sm, D_PMAX, NDIAG);
  __syncthreads();
  for (int t = threadIdx.x; t < NDIAG; t += blockDim.x) {
    const bool mx = t >= D_RHOMIN;
    double a = sm[t];
    for (int ww = 1; ww < kRedWarps; ++ww) a = mx ? fmax(a, sm[ww * NDIAG + t]) : a + sm[ww * NDIAG + t];
    S.part_diag[(size_t)w.c * NDIAG + t] = a;
  }
  if (!last_block(&S.counters[3], S.nblk_diag)) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int t = warp; t < NDIAG; t += kRedWarps) {
    const bool mx = t >= D_RHOMIN;
    double a = mx ? -INFINITY : 0.0;
    for (int b = lane; b < S.nblk_diag; b += 32) {
      const double x = __ldcg(S.part_diag + (size_t)b * NDIAG + t);
      a = mx ? fmax(a, x) : a + x;
    }
    a = mx ? warp_max(a) : warp_sum(a);
    if (lane == 0) red[t] = a;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < NDIAG; t += blockDim.x) {
    double v = red[t];
    if (t == D_RHOMIN || t == D_PMIN) v = -v;
    S.diag_out[t] = v;
  }
}

}  // namespace hitb200
