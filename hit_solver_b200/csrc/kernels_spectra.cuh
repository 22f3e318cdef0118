// Shell-averaged kinetic-energy and enstrophy spectra of HIT snapshots
// (HIT2DSpectra.compute, OOP/postprocess/spectra.py:48-149), batched over
// snapshots.  The forward transforms are the caller's (a real-to-complex 2-D
// FFT of the four fields); around them:
//   spectra_mean_kernel    per-snapshot partial sums for the fluctuation means
//                          (spectra.py:199-210)
//   spectra_fields_kernel  the transform inputs sqrt(rho) u', sqrt(rho) v',
//                          u', v' (spectra.py:93-104)
//   spectra_shell_kernel   mode energies and enstrophies of the half spectrum
//                          binned by shell rint(|k| / dk) (spectra.py:85-121)
//   spectra_final_kernel   fixed-order sum of the per-CTA shell partials
// Every sum runs in a fixed order, so results do not depend on scheduling.
#pragma once

#include "common.cuh"

namespace hitb200 {

constexpr int kSpecThreads = 256;
constexpr int kSpecWarps = kSpecThreads / 32;
constexpr int kSpecMeanBlocks = 64;   // partial-sum CTAs per snapshot
constexpr int kSpecMaxShells = 1025;  // min(nx, ny) / 2 + 1 for grids up to 2048

// 2 pi fftfreq(n, d)[j] formed the way numpy forms it: the signed bin times
// 1 / (n d) (inv_nd, computed by the host), times 2 pi.  No contraction.
__device__ __forceinline__ double spec_wavenumber(int j, int n, double inv_nd) {
  const int half = (n - 1) / 2 + 1;
  const int b = j < half ? j : j - n;
  return __dmul_rn(2.0 * M_PI, __dmul_rn((double)b, inv_nd));
}

// Snapshot s, cell i: rho, u, v from primitive arrays (CONS = false) or from a
// conservative state [4][ny][nx] with the density floor of
// primitive_from_conservative (OOP/equations.py:136-145; CONS = true).
template <bool CONS>
__device__ __forceinline__ void spec_load(const double* a, const double* u, const double* v,
                                          size_t s, long long ncell, long long i, double& rho,
                                          double& uu, double& vv) {
  if (CONS) {
    const double* q = a + s * 4 * (size_t)ncell;
    const double q0 = q[i];
    rho = q0 > kRhoFloor ? q0 : kRhoFloor;
    uu = q[ncell + i] / rho;
    vv = q[2 * ncell + i] / rho;
  } else {
    const size_t o = s * (size_t)ncell + i;
    rho = a[o];
    uu = u[o];
    vv = v[o];
  }
}

// grid (kSpecMeanBlocks, snapshots).  part[s][blk][3] = (sum rho, sum w u,
// sum w v) with w = rho for Favre means, w = 1 for Reynolds means.
template <bool CONS>
__global__ void __launch_bounds__(kSpecThreads)
    spectra_mean_kernel(const double* __restrict__ a, const double* __restrict__ u,
                        const double* __restrict__ v, long long ncell, int favre,
                        double* __restrict__ part) {
  __shared__ double sm[kSpecWarps][3];
  const size_t s = blockIdx.y;
  double sr = 0.0, su = 0.0, sv = 0.0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ncell; i += stride) {
    double rho, uu, vv;
    spec_load<CONS>(a, u, v, s, ncell, i, rho, uu, vv);
    sr += rho;
    su += favre ? rho * uu : uu;
    sv += favre ? rho * vv : vv;
  }
  sr = warp_sum(sr);
  su = warp_sum(su);
  sv = warp_sum(sv);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sm[warp][0] = sr;
    sm[warp][1] = su;
    sm[warp][2] = sv;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double acc = 0.0;
    for (int w = 0; w < kSpecWarps; ++w) acc += sm[w][threadIdx.x];
    part[(s * gridDim.x + blockIdx.x) * 3 + threadIdx.x] = acc;
  }
}

// grid (cell blocks, snapshots).  out[s] = [sqrt(rho) u', sqrt(rho) v', u', v']
// ([4][ny][nx]); the means come from the nmb partial rows of the snapshot,
// summed in a fixed order by the first warp of every CTA.
template <bool CONS>
__global__ void __launch_bounds__(kSpecThreads)
    spectra_fields_kernel(const double* __restrict__ a, const double* __restrict__ u,
                          const double* __restrict__ v, long long ncell, int favre,
                          const double* __restrict__ part, int nmb, double* __restrict__ out) {
  __shared__ double mean[2];
  const size_t s = blockIdx.y;
  if (threadIdx.x < 32) {
    // warp 0: lane l sums partials l, l + 32, ...; then a fixed butterfly
    double sr = 0.0, su = 0.0, sv = 0.0;
    const double* p = part + s * nmb * 3;
    for (int k = threadIdx.x; k < nmb; k += 32) {
      sr += p[3 * k];
      su += p[3 * k + 1];
      sv += p[3 * k + 2];
    }
    sr = warp_sum(sr);
    su = warp_sum(su);
    sv = warp_sum(sv);
    if (threadIdx.x == 0) {
      const double n = (double)ncell;
      if (favre) {
        const double rm = sr / n;  // mean(rho); then mean(rho u) / mean(rho)
        mean[0] = (su / n) / rm;
        mean[1] = (sv / n) / rm;
      } else {
        mean[0] = su / n;
        mean[1] = sv / n;
      }
    }
  }
  __syncthreads();
  const double mu = mean[0], mv = mean[1];
  double* o = out + s * 4 * (size_t)ncell;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ncell; i += stride) {
    double rho, uu, vv;
    spec_load<CONS>(a, u, v, s, ncell, i, rho, uu, vv);
    const double up = uu - mu, vp = vv - mv, w = sqrt(rho);
    o[i] = w * up;
    o[ncell + i] = w * vp;
    o[2 * ncell + i] = up;
    o[3 * ncell + i] = vp;
  }
}

// grid (row blocks, snapshots); dynamic shared memory kSpecWarps * 2 * ns
// doubles.  spec[s][c][ny][nh] (nh = nx / 2 + 1) is the half spectrum of the
// four fields.  Warp w of the CTA walks rows j = j0 + w, j0 + w + 8, ... of
// the CTA's block in 32-mode chunks.  Along a row |kx| grows with the column,
// so the shell index is non-decreasing and equal shells form contiguous
// runs: a segmented warp scan sums each run, and the run's last lane adds it
// to the warp's own bins.  Columns 1 .. nh-1 stand for themselves and their
// mirror, the conjugate mode at (-kx, -ky) in the same shell (the Nyquist
// column of an even nx is its own mirror); in the Nyquist row of an even ny
// the mirror's ky is the row's own, which changes its vorticity but not its
// energy.  The CTA then sums its warps' bins in warp order into
// part[s][blk][2][ns].
__global__ void __launch_bounds__(kSpecThreads)
    spectra_shell_kernel(const double2* __restrict__ spec, int nx, int ny, double inv_nxdx,
                         double inv_nydy, double dk, double inv_norm, int ns, int rows_per_cta,
                         double* __restrict__ part) {
  extern __shared__ double bins[];  // [kSpecWarps][2][ns]
  const unsigned full = 0xffffffffu;
  const size_t s = blockIdx.y;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nh = nx / 2 + 1;
  const size_t plane = (size_t)ny * nh;
  const double2* sp = spec + s * 4 * plane;
  for (int t = threadIdx.x; t < kSpecWarps * 2 * ns; t += blockDim.x) bins[t] = 0.0;
  __syncthreads();
  double* eb = bins + (size_t)warp * 2 * ns;
  double* zb = eb + ns;
  const int nyq = (nx & 1) ? -1 : nx / 2;
  const int nyq_row = (ny & 1) ? -1 : ny / 2;
  const int j0 = blockIdx.x * rows_per_cta;
  const int j1 = min(ny, j0 + rows_per_cta);
  for (int j = j0 + warp; j < j1; j += kSpecWarps) {
    const double ky = spec_wavenumber(j, ny, inv_nydy);
    const double ky2 = __dmul_rn(ky, ky);
    const double2* row = sp + (size_t)j * nh;
    for (int c0 = 0; c0 < nh; c0 += 32) {
      const int i = c0 + lane;
      int key = 0x7fffffff;  // beyond every shell: dropped
      double e = 0.0, z = 0.0;
      if (i < nh) {
        const double kx = spec_wavenumber(i, nx, inv_nxdx);
        const double km = __dsqrt_rn(__dadd_rn(__dmul_rn(kx, kx), ky2));
        key = (int)rint(__ddiv_rn(km, dk));
        const double2 fa = row[i], fb = row[plane + i];
        const double2 fc = row[2 * plane + i], fd = row[3 * plane + i];
        const bool single = i == 0 || i == nyq;
        const double wt = single ? 0.5 : 1.0;  // 1/2 |.|^2, doubled for the mirror
        e = wt * (fa.x * fa.x + fa.y * fa.y + fb.x * fb.x + fb.y * fb.y) * inv_norm;
        // omega_hat = i (kx v_hat - ky u_hat)
        const double wr = kx * fd.x - ky * fc.x, wi = kx * fd.y - ky * fc.y;
        if (single || j != nyq_row) {
          z = wt * (wr * wr + wi * wi) * inv_norm;
        } else {
          // Nyquist row of an even ny: the mirror (-kx, ky) keeps ky (fftfreq
          // gives -ny/2 for both), so its vorticity is kx V + ky U (conjugated)
          const double mr = kx * fd.x + ky * fc.x, mi = kx * fd.y + ky * fc.y;
          z = 0.5 * ((wr * wr + wi * wi) + (mr * mr + mi * mi)) * inv_norm;
        }
      }
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const int k2 = __shfl_up_sync(full, key, off);
        const double e2 = __shfl_up_sync(full, e, off);
        const double z2 = __shfl_up_sync(full, z, off);
        if (lane >= off && k2 == key) {
          e += e2;
          z += z2;
        }
      }
      const int knext = __shfl_down_sync(full, key, 1);
      if ((lane == 31 || knext != key) && key < ns) {
        eb[key] += e;
        zb[key] += z;
      }
      __syncwarp();
    }
  }
  __syncthreads();
  double* o = part + (s * gridDim.x + blockIdx.x) * 2 * (size_t)ns;
  for (int t = threadIdx.x; t < 2 * ns; t += blockDim.x) {
    double acc = 0.0;
    for (int w = 0; w < kSpecWarps; ++w) acc += bins[(size_t)w * 2 * ns + t];
    o[t] = acc;
  }
}

// grid (ceil(2 ns / threads), snapshots): energy[s][k], enstrophy[s][k] as the
// sum over the nblk CTA partials of the snapshot in CTA order.
__global__ void __launch_bounds__(kSpecThreads)
    spectra_final_kernel(const double* __restrict__ part, int nblk, int ns,
                         double* __restrict__ energy, double* __restrict__ enstrophy) {
  const size_t s = blockIdx.y;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * ns) return;
  const double* p = part + s * nblk * 2 * (size_t)ns + t;
  double acc = 0.0;
#pragma unroll 8
  for (int b = 0; b < nblk; ++b) acc += p[(size_t)b * 2 * ns];
  if (t < ns) energy[s * ns + t] = acc;
  else enstrophy[s * ns + t - ns] = acc;
}

}  // namespace hitb200
