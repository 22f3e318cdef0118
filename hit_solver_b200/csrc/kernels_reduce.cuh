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
// RHS needs before its flux pass.
//   ENF = 1: sensor/LF quantities on enforce_physical_state(q), as
//   PeriodicHybridEuler2DOperator.rhs does (OOP/spatial_operator.py:345-346).
__global__ void __launch_bounds__(kRedThreads, 2)
    prepass_kernel(const SolveDev* __restrict__ solves, const Work* __restrict__ work, int buf,
                   int mode, int enf, Bind bind) {
  const Work w = work[blockIdx.x];
  const SolveDev& S = solves[w.solve];
  double* sc = S.scal;
  if (mode == PRE_SENSOR && !bind.use && sc[S_HV_STEP] == 0.0) return;  // no hyperviscosity this step
  if (mode == PRE_STAGE && !bind.use && sc[S_ACTIVE] == 0.0) return;
  const double* q = bind.use ? bind.qin : stage_in(S, buf);
  const int nx = S.nx, ny = S.ny, per = S.periodic;
  const size_t plane = (size_t)nx * ny;
  const double g = S.gamma;
  const double igm1 = 1.0 / (g - 1.0), idx_ = 1.0 / S.dx, idy_ = 1.0 / S.dy;
  const double ih2x = 1.0 / (2.0 * S.dx), ih2y = 1.0 / (2.0 * S.dy);
  const int x0 = w.a, y0 = w.b;

  __shared__ double su[kTileY + 2][kTileX + 2];
  __shared__ double sv[kTileY + 2][kTileX + 2];
  __shared__ double sm[kRedWarps * (R_FIXED + 4 * kMaxDrag)];
  __shared__ double red[R_FIXED + 4 * kMaxDrag];
  const bool need_grad = (mode != PRE_CHECK);
  const int tx = threadIdx.x & 31, ty0 = threadIdx.x >> 5;

  double ax = 0, ay = 0, div2 = 0, vort2 = 0, mr = 0, mp = 0, me = 0, ps = 0, sr = 0, vel2 = 0,
         cs = 0;
  int bad = 0;  // validation flags: 1 non-finite, 2 rho <= 0, 4 p <= 0
  // Every node of the tile and its one-node halo is loaded once; tile nodes
  // also feed the pointwise reductions here.
  for (int a = ty0; a < kTileY + 2; a += kRedWarps) {
    const int gy = y0 + a - 1;
    const int gj = fold_node(gy, ny, per);
    for (int b = tx; b < kTileX + 2; b += 32) {
      const int gx = x0 + b - 1;
      const bool own = a >= 1 && a <= kTileY && b >= 1 && b <= kTileX && gy < ny && gx < nx;
      if (!need_grad && !own) continue;
      const int gi = fold_node(gx, nx, per);
      const size_t o = (size_t)gj * nx + gi;
      const double q0 = q[o], q1 = q[o + plane], q2 = q[o + 2 * plane], q3 = q[o + 3 * plane];
      // One reciprocal and one square root per node serve the enforced state
      // (sensor / Lax-Friedrichs quantities) and the raw state (time step,
      // Mach, cooling); both share the floored density.
      const double rho = q0 > kRhoFloor ? q0 : kRhoFloor;
      const double rinv = 1.0 / rho;
      const double ur = q1 * rinv, vr = q2 * rinv;
      const double kin = 0.5 * rho * (ur * ur + vr * vr);
      const double p_raw = (g - 1.0) * (q3 - kin);
      double ue = ur, ve = vr, pe = p_raw;
      if (need_grad && enf) {
        const double e1 = rho * ur, e2 = rho * vr;
        const double e3 = p_raw > kPFloor ? q3 : kPFloor / (g - 1.0) + kin;
        ue = e1 * rinv;
        ve = e2 * rinv;
        pe = (g - 1.0) * (e3 - 0.5 * rho * (ue * ue + ve * ve));
      }
      pe = pe > kPFloor ? pe : kPFloor;
      const double pr = p_raw > kPFloor ? p_raw : kPFloor;
      const double cr = sqrt(g * pr * rinv);
      if (need_grad) {
        su[a][b] = ue;
        sv[a][b] = ve;
        if (own) {
          const double c = enf ? sqrt(g * pe * rinv) : cr;
          ax = fmax(ax, fabs(ue) + c);
          ay = fmax(ay, fabs(ve) + c);
          mr = fmax(mr, rho);
          mp = fmax(mp, pe);
          me = fmax(me, pe * rinv * igm1);
        }
      }
      if (!own) continue;
      // raw state: time step, Mach, cooling, validation
      ps += pr;
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
  if (need_grad) __syncthreads();
  int cj[kCellsPerThread], ci[kCellsPerThread];
  bool valid[kCellsPerThread];
#pragma unroll
  for (int k = 0; k < kCellsPerThread; ++k) {
    const int ty = ty0 + kRedWarps * k;
    const int gj = y0 + ty, gi = x0 + tx;
    cj[k] = gj;
    ci[k] = gi;
    valid[k] = (gj < ny && gi < nx);
    if (!valid[k] || !need_grad) continue;
    // sensor divergence / vorticity: central, one-sided at outflow edges
    const int a = ty + 1, b = tx + 1;
    double dudx, dvdx, dudy, dvdy;
    if (per || (gi > 0 && gi < nx - 1)) {
      dudx = (su[a][b + 1] - su[a][b - 1]) * ih2x;
      dvdx = (sv[a][b + 1] - sv[a][b - 1]) * ih2x;
    } else if (nx == 1) {
      dudx = dvdx = 0.0;
    } else if (gi == 0) {
      dudx = (su[a][b + 1] - su[a][b]) * idx_;
      dvdx = (sv[a][b + 1] - sv[a][b]) * idx_;
    } else {
      dudx = (su[a][b] - su[a][b - 1]) * idx_;
      dvdx = (sv[a][b] - sv[a][b - 1]) * idx_;
    }
    if (per || (gj > 0 && gj < ny - 1)) {
      dudy = (su[a + 1][b] - su[a - 1][b]) * ih2y;
      dvdy = (sv[a + 1][b] - sv[a - 1][b]) * ih2y;
    } else if (ny == 1) {
      dudy = dvdy = 0.0;
    } else if (gj == 0) {
      dudy = (su[a + 1][b] - su[a][b]) * idy_;
      dvdy = (sv[a + 1][b] - sv[a][b]) * idy_;
    } else {
      dudy = (su[a][b] - su[a - 1][b]) * idy_;
      dvdy = (sv[a][b] - sv[a - 1][b]) * idy_;
    }
    const double dv = dudx + dvdy, vo = dvdx - dudy;
    div2 += dv * dv;
    vort2 += vo * vo;
  }
  const int nslots = (mode == PRE_STAGE || mode == PRE_STEP) ? S.nred : R_FIXED;
  warp_to_smem<OP_MAX>(ax, sm, R_AX, nslots);
  warp_to_smem<OP_MAX>(ay, sm, R_AY, nslots);
  warp_to_smem<OP_SUM>(div2, sm, R_DIV2, nslots);
  warp_to_smem<OP_SUM>(vort2, sm, R_VORT2, nslots);
  warp_to_smem<OP_MAX>(mr, sm, R_RHO, nslots);
  warp_to_smem<OP_MAX>(mp, sm, R_P, nslots);
  warp_to_smem<OP_MAX>(me, sm, R_E, nslots);
  warp_to_smem<OP_SUM>(ps, sm, R_PSUM, nslots);
  warp_to_smem<OP_MAX>(sr, sm, R_SR, nslots);
  warp_to_smem<OP_SUM>(vel2, sm, R_VEL2, nslots);
  warp_to_smem<OP_SUM>(cs, sm, R_CSUM, nslots);
  bad = __reduce_or_sync(kFullMask, bad);
  if ((threadIdx.x & 31) == 0) {
    sm[(threadIdx.x >> 5) * nslots + R_NONFINITE] = (bad & 1) ? 1.0 : 0.0;
    sm[(threadIdx.x >> 5) * nslots + R_NONPOS_RHO] = (bad & 2) ? 1.0 : 0.0;
    sm[(threadIdx.x >> 5) * nslots + R_NONPOS_P] = (bad & 4) ? 1.0 : 0.0;
  }
  if (nslots > R_FIXED) {
    // low-k momentum transform of the drag band filter (OOP/hit2d.py:352-399)
    for (int m = 0; m < S.n_drag; ++m) {
      const int2 md = S.modes[m];
      double v[4] = {0, 0, 0, 0};
#pragma unroll
      for (int k = 0; k < kCellsPerThread; ++k) {
        if (!valid[k]) continue;
        const size_t o = (size_t)cj[k] * nx + ci[k];
        const double m0 = q[o + plane], m1 = q[o + 2 * plane];
        const double2 ex = S.twx[mode_index(md.x, ci[k], nx)], ey = S.twy[mode_index(md.y, cj[k], ny)];
        const double2 e = make_double2(cmul_re(ex, ey), cmul_im(ex, ey));  // e^{-i theta}
        v[0] += m0 * e.x;
        v[1] += m0 * e.y;
        v[2] += m1 * e.x;
        v[3] += m1 * e.y;
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) warp_to_smem<OP_SUM>(v[k], sm, R_FIXED + 4 * m + k, nslots);
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nslots; t += blockDim.x) {
    const int op = pre_op(t);
    double acc = sm[t];
    for (int ww = 1; ww < kRedWarps; ++ww) {
      const double x = sm[ww * nslots + t];
      acc = op == OP_SUM ? acc + x : fmax(acc, x);
    }
    S.part_pre[(size_t)w.c * nslots + t] = acc;
  }
  if (!last_block(&S.counters[0], S.nblk_pre)) return;

  // ---- last CTA of this solve: fixed-order final reduction + scalar logic ----
  {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int t = warp; t < nslots; t += kRedWarps) {
      const int op = pre_op(t);
      double acc = op == OP_SUM ? 0.0 : -INFINITY;
#pragma unroll 8
      for (int b = lane; b < S.nblk_pre; b += 32) {
        const double x = __ldcg(S.part_pre + (size_t)b * nslots + t);
        acc = op == OP_SUM ? acc + x : fmax(acc, x);
      }
      acc = op == OP_SUM ? warp_sum(acc) : warp_max(acc);
      if (lane == 0) red[t] = acc;
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const double N = (double)nx * (double)ny;
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
    if (!bind.use) sc[S_HV_APPLIED] += 1.0;  // this prepass runs only on hyperviscosity steps
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
// needs (forcing.py:87-118), then the scalar rescaling logic.
__global__ void __launch_bounds__(kRedThreads)
    force_synth_kernel(const SolveDev* __restrict__ solves, const Work* __restrict__ work,
                       Bind bind) {
  const Work w = work[blockIdx.x];
  const SolveDev& S = solves[w.solve];
  double* sc = S.scal;
  if (!S.forcing_on) return;
  if (!bind.use && sc[S_ACTIVE] == 0.0) return;
  const double* q = bind.use ? bind.qin : S.q;
  const int nx = S.nx, ny = S.ny, nf = S.n_force;
  const size_t plane = (size_t)nx * ny;
  const int2* modes = S.modes + S.n_drag;
  const double invN = 1.0 / ((double)nx * (double)ny);
  __shared__ double2 ca[kMaxForce], cb[kMaxForce];
  __shared__ double sm[kRedWarps * 4];
  __shared__ double red[4];
  for (int m = threadIdx.x; m < nf; m += blockDim.x) {
    const double pr = sc[S_PHI + 2 * m], pi = sc[S_PHI + 2 * m + 1];
    const double2 kv = S.kvec[m];
    ca[m] = make_double2(-kv.y * pi * invN, kv.y * pr * invN);   // (i ky phi)/N
    cb[m] = make_double2(kv.x * pi * invN, -kv.x * pr * invN);   // (-i kx phi)/N
  }
  __syncthreads();
  const int tx = threadIdx.x & 31, ty0 = threadIdx.x >> 5;
  double sxx = 0, syy = 0, sxy = 0, spow = 0;
#pragma unroll
  for (int k = 0; k < kCellsPerThread; ++k) {
    const int gj = w.b + ty0 + kRedWarps * k, gi = w.a + tx;
    if (gj >= ny || gi >= nx) continue;
    double fx = 0.0, fy = 0.0;
    for (int m = 0; m < nf; ++m) {
      const int2 md = modes[m];
      const double2 ex = S.twx[mode_index(md.x, gi, nx)], ey = S.twy[mode_index(md.y, gj, ny)];
      // e^{+i theta} = conj(e^{-i theta})
      const double er = cmul_re(ex, ey), ei = -cmul_im(ex, ey);
      fx += ca[m].x * er - ca[m].y * ei;
      fy += cb[m].x * er - cb[m].y * ei;
    }
    const size_t o = (size_t)gj * nx + gi;
    S.fx[o] = fx;
    S.fy[o] = fy;
    const Prim<double> p = primitives(q[o], q[o + plane], q[o + 2 * plane], q[o + 3 * plane], S.gamma);
    sxx += fx * fx;
    syy += fy * fy;
    sxy += fx * fy;
    spow += p.rho * (fx * p.u + fy * p.v);
  }
  warp_to_smem<OP_SUM>(sxx, sm, 0, 4);
  warp_to_smem<OP_SUM>(syy, sm, 1, 4);
  warp_to_smem<OP_SUM>(sxy, sm, 2, 4);
  warp_to_smem<OP_SUM>(spow, sm, 3, 4);
  __syncthreads();
  if (threadIdx.x < 4) {
    double acc = sm[threadIdx.x];
    for (int ww = 1; ww < kRedWarps; ++ww) acc += sm[ww * 4 + threadIdx.x];
    S.part_synth[(size_t)w.c * 4 + threadIdx.x] = acc;
  }
  if (!last_block(&S.counters[2], S.nblk_synth)) return;
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
