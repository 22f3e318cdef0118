// Initial states built on the device.
//   hit_psi_kernel      the low-k streamfunction of initialize_hit_2d
//                       (OOP/hit2d.py:158-189), O(modes x cells)
//   hit_ic_sum_kernel   per-CTA partial sums for the velocity means and rms
//   hit_ic_compose_kernel  the scaled velocity and the conservative state
//                       (OOP/hit2d.py:191-204)
//   quadrant_kernel     the four-quadrant Riemann states
//                       (OOP/problems/riemann_config3.py:59-99)
// Cell centres are x_min + dx (i + 1/2) as the reference's Domain2D forms
// them, and every product and sum that the reference evaluates as separate
// NumPy operations is rounded separately here (no contraction).
#pragma once

#include "common.cuh"

namespace hitb200 {

constexpr int kInitThreads = 256;
constexpr int kInitSumBlocks = 128;  // partial-sum CTAs of the HIT initial state

__device__ __forceinline__ double cell_centre(double lo, double d, int i) {
  return __dadd_rn(lo, __dmul_rn(d, (double)i + 0.5));
}

// psi[j][i] = sum_m amp_m cos(kx_m x_i + ky_m y_j + phase_m), modes in the
// caller's order (the order in which the reference draws their phases), each
// term added to the running sum as psi += amplitude * cos(...).
__global__ void __launch_bounds__(kInitThreads)
    hit_psi_kernel(const double* __restrict__ modes, int n_modes, int nx, int ny, double x_min,
                   double dx, double y_min, double dy, double* __restrict__ psi) {
  const long long n = (long long)nx * ny;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride) {
    const int j = (int)(c / nx), i = (int)(c - (long long)j * nx);
    const double x = cell_centre(x_min, dx, i), y = cell_centre(y_min, dy, j);
    double acc = 0.0;
    for (int m = 0; m < n_modes; ++m) {
      const double* md = modes + 4 * m;  // (kx, ky, amplitude, phase)
      const double th =
          __dadd_rn(__dadd_rn(__dmul_rn(__ldg(md), x), __dmul_rn(__ldg(md + 1), y)), __ldg(md + 3));
      acc = __dadd_rn(acc, __dmul_rn(__ldg(md + 2), cos(th)));
    }
    psi[c] = acc;
  }
}

// pass 0: part[blk] = (sum u, sum v, 0); pass 1 (means from pass 0's
// partials): part[blk][2] = sum (u - mean u)^2 + (v - mean v)^2.
template <int PASS>
__global__ void __launch_bounds__(kInitThreads)
    hit_ic_sum_kernel(const double* __restrict__ u, const double* __restrict__ v, long long n,
                      double* __restrict__ part) {
  __shared__ double sm[kInitThreads / 32][2];
  __shared__ double mean[2];
  if (PASS == 1) {
    if (threadIdx.x == 0) {
      double su = 0.0, sv = 0.0;
      for (int b = 0; b < kInitSumBlocks; ++b) {
        su += part[3 * b];
        sv += part[3 * b + 1];
      }
      mean[0] = su / (double)n;
      mean[1] = sv / (double)n;
    }
    __syncthreads();
  }
  double a = 0.0, b = 0.0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride) {
    if (PASS == 0) {
      a += u[c];
      b += v[c];
    } else {
      const double up = u[c] - mean[0], vp = v[c] - mean[1];
      a += __dadd_rn(__dmul_rn(up, up), __dmul_rn(vp, vp));
    }
  }
  a = warp_sum(a);
  b = warp_sum(b);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sm[warp][0] = a;
    sm[warp][1] = b;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double acc = 0.0;
    for (int w = 0; w < kInitThreads / 32; ++w) acc += sm[w][threadIdx.x];
    if (PASS == 0) part[3 * blockIdx.x + threadIdx.x] = acc;
    else if (threadIdx.x == 0) part[3 * blockIdx.x + 2] = acc;
  }
}

// q = (1, s u', s v', p / (gamma - 1) + 1/2 (s u'^2 + s v'^2)) with u' the
// mean-free velocity, p = 1 / gamma and s = target_mach * c_mean / rms; every
// CTA re-forms the means and the rms from the partials in the same order.
// vrms_out (CTA 0) receives the rms for the caller's zero-velocity check.
__global__ void __launch_bounds__(kInitThreads)
    hit_ic_compose_kernel(const double* __restrict__ u, const double* __restrict__ v, long long n,
                          const double* __restrict__ part, double gamma, double target_mach,
                          double c_mean, double* __restrict__ q, double* __restrict__ vrms_out) {
  __shared__ double sh[3];
  if (threadIdx.x == 0) {
    double su = 0.0, sv = 0.0, s2 = 0.0;
    for (int b = 0; b < kInitSumBlocks; ++b) {
      su += part[3 * b];
      sv += part[3 * b + 1];
      s2 += part[3 * b + 2];
    }
    const double rms = sqrt(s2 / (double)n);
    sh[0] = su / (double)n;
    sh[1] = sv / (double)n;
    sh[2] = rms > 0.0 ? target_mach * c_mean / rms : 0.0;
    if (blockIdx.x == 0) *vrms_out = rms;
  }
  __syncthreads();
  const double mu = sh[0], mv = sh[1], s = sh[2];
  const double p = 1.0 / gamma;
  const double e0 = p / (gamma - 1.0);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride) {
    const double uu = __dmul_rn(u[c] - mu, s), vv = __dmul_rn(v[c] - mv, s);
    q[c] = 1.0;
    q[n + c] = uu;  // rho u with rho = 1
    q[2 * n + c] = vv;
    q[3 * n + c] = __dadd_rn(e0, __dmul_rn(0.5, __dadd_rn(__dmul_rn(uu, uu), __dmul_rn(vv, vv))));
  }
}

// Quadrant primitive states (rho, u, v, p): lower-left, lower-right,
// upper-left, upper-right.
struct QuadStates {
  double s[4][4];
};

// q of the quadrant holding each cell centre (upper when y >= y_split, right
// when x >= x_split), through conservative_from_primitive with the density
// and pressure floors.
__global__ void __launch_bounds__(kInitThreads)
    quadrant_kernel(QuadStates st, int nx, int ny, double x_min, double dx, double y_min, double dy,
                    double x_split, double y_split, double gamma, double* __restrict__ q) {
  const long long n = (long long)nx * ny;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride) {
    const int j = (int)(c / nx), i = (int)(c - (long long)j * nx);
    const int k = (cell_centre(y_min, dy, j) >= y_split ? 2 : 0) +
                  (cell_centre(x_min, dx, i) >= x_split ? 1 : 0);
    const double rho = fmax(st.s[k][0], kRhoFloor), u = st.s[k][1], v = st.s[k][2];
    const double p = fmax(st.s[k][3], kPFloor);
    q[c] = rho;
    q[n + c] = __dmul_rn(rho, u);
    q[2 * n + c] = __dmul_rn(rho, v);
    q[3 * n + c] = __dadd_rn(p / (gamma - 1.0),
                             __dmul_rn(__dmul_rn(0.5, rho), __dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v))));
  }
}

}  // namespace hitb200
