// Discrete Fourier transforms of grid lines, for the spectral parts of the
// diagnostics (OOP/hit2d.py:146-155, 429-468), the initial condition's
// spectral derivatives (OOP/hit2d.py:186-188) and the shell spectra's real
// transform (OOP/postprocess/spectra.py:84-121); NumPy's fft conventions:
// forward sum_m x_m e^{-2 pi i j m / n}, inverse with +i and the 1/n scale.
//
// Each line (n <= 1024 complex doubles) is transformed inside shared memory
// by a self-sorting (Stockham) mixed-radix algorithm: n = R_0 R_1 ... with
// radices 4, 2, 3, 5, 7 and then any remaining prime; the stage of radix R
// with Ns points already combined maps output o = t m + j (m = n / R,
// k = j mod Ns) to
//     b[(j / Ns) Ns R + k + t Ns] = sum_r a[j + r m] W^{r (k n / (Ns R) + t m)},
// W = e^{-2 pi i / n} (forward) read from a table of the n roots, staged in
// shared memory.  A CTA transforms C adjacent lines at once (C > 1 for
// columns, so that every row access covers C consecutive elements).  The
// work per stage is n R complex multiply-adds per line (a prime n falls back
// to the n^2 transform), negligible next to the line's memory traffic.
// Power-of-two lengths take a faster kernel (fft_p2_kernel, below): radix-8
// passes on points held in registers, real rows packed two to a complex
// line.  Measured on a B200, rfft2 of 256 fields of 512^2: 2.0 ms with the
// mixed-radix kernel, 0.594 ms with the radix-8 one (cuFFT: 0.47 ms).
#pragma once

#include "common.cuh"

namespace hitb200 {

constexpr int kFftMaxN = 1024;
constexpr int kFftThreads = 256;
constexpr int kFftMaxButterfly = 7;  // radices up to this are whole butterflies per thread

struct FftRadices {
  int count;
  int r[16];
};

// Radices of n: 4s, then 2, 3, 5, 7, then the remaining primes.
inline FftRadices fft_radices(int n) {
  FftRadices f{};
  for (int p : {4, 2, 3, 5, 7})
    while (n % p == 0 && f.count < 16) {
      f.r[f.count++] = p;
      n /= p;
    }
  for (int q = 11; n > 1 && f.count < 16; q += 2)
    while (n % q == 0) {
      f.r[f.count++] = q;
      n /= q;
    }
  return f;
}

// Lines: element e of line l of field f sits at
//   base + f * field + l * line + e * elem.
struct FftLines {
  long long field, line, elem;
};

// Transform C lines per CTA (grid: fields * ceil(lines / C)).  IN_REAL: the
// input holds doubles (imaginary part zero).  sign -1 forward, +1 inverse
// (unscaled; the output is multiplied by `scale`).  Only the first out_count
// outputs of each line are stored (n, or n / 2 + 1 for a half spectrum).
// OUT_REAL: only the real parts are stored (doubles).  W: the n roots
// e^{-2 pi i m / n}.
template <bool IN_REAL, bool OUT_REAL, int C>
__global__ void __launch_bounds__(kFftThreads)
    fft_lines_kernel(const void* __restrict__ in, void* __restrict__ out, int n, int lines,
                     FftLines li, FftLines lo, int out_count, int sign,
                     const double2* __restrict__ W, FftRadices rad, double scale) {
  extern __shared__ __align__(16) double2 fbuf[];
  double2* a = fbuf;
  double2* b = fbuf + (size_t)n * C;
  double2* w = fbuf + (size_t)2 * n * C;
  const int groups = (lines + C - 1) / C;
  const int f = blockIdx.x / groups, l0 = (blockIdx.x - f * groups) * C;
  const int nc = min(C, lines - l0);
  for (int m = threadIdx.x; m < n; m += blockDim.x) {
    double2 v = W[m];
    if (sign > 0) v.y = -v.y;
    w[m] = v;
  }
  // element e of line l0 + c at a[e C + c]: consecutive threads take the C
  // lines of one element (adjacent in memory for columns)
  for (int idx = threadIdx.x; idx < n * C; idx += blockDim.x) {
    const int e = idx / C, c = idx - e * C;
    double2 v = make_double2(0.0, 0.0);
    if (c < nc) {
      const long long o = f * li.field + (long long)(l0 + c) * li.line + (long long)e * li.elem;
      if constexpr (IN_REAL) v.x = static_cast<const double*>(in)[o];
      else v = static_cast<const double2*>(in)[o];
    }
    a[idx] = v;
  }
  __syncthreads();
  int Ns = 1;
  for (int s = 0; s < rad.count; ++s) {
    const int R = rad.r[s], m = n / R, step = n / (Ns * R);
    if (R <= kFftMaxButterfly) {
      // one butterfly per thread: the R inputs j + r m, twiddled by
      // W^{r k step}, transformed together, written to the R outputs
      for (int idx = threadIdx.x; idx < m * C; idx += blockDim.x) {
        const int j = idx / C, c = idx - j * C;
        const int k = j % Ns;
        const int out0 = (j - k) * R + k;  // (j / Ns) Ns R + k
        double2 v[kFftMaxButterfly];
        v[0] = a[j * C + c];
        const int tk = k * step;  // r tk < n for r < R
#pragma unroll
        for (int r = 1; r < kFftMaxButterfly; ++r) {
          if (r >= R) break;
          const double2 x = a[(j + r * m) * C + c];
          const double2 tw = w[r * tk];
          v[r] = make_double2(fma(x.x, tw.x, -x.y * tw.y), fma(x.x, tw.y, x.y * tw.x));
        }
        if (R == 2) {
          b[out0 * C + c] = make_double2(v[0].x + v[1].x, v[0].y + v[1].y);
          b[(out0 + Ns) * C + c] = make_double2(v[0].x - v[1].x, v[0].y - v[1].y);
        } else if (R == 4) {
          // W_4 = -i (forward) / +i (inverse), applied exactly
          const double2 s0 = make_double2(v[0].x + v[2].x, v[0].y + v[2].y);
          const double2 s1 = make_double2(v[0].x - v[2].x, v[0].y - v[2].y);
          const double2 s2 = make_double2(v[1].x + v[3].x, v[1].y + v[3].y);
          const double2 d = make_double2(v[1].x - v[3].x, v[1].y - v[3].y);
          const double2 s3 = sign < 0 ? make_double2(d.y, -d.x) : make_double2(-d.y, d.x);
          b[out0 * C + c] = make_double2(s0.x + s2.x, s0.y + s2.y);
          b[(out0 + Ns) * C + c] = make_double2(s1.x + s3.x, s1.y + s3.y);
          b[(out0 + 2 * Ns) * C + c] = make_double2(s0.x - s2.x, s0.y - s2.y);
          b[(out0 + 3 * Ns) * C + c] = make_double2(s1.x - s3.x, s1.y - s3.y);
        } else {
          // small odd radix: y_t = sum_r v_r W^{r t m}
          for (int t = 0; t < R; ++t) {
            double re = 0.0, im = 0.0;
            int e = 0;
            for (int r = 0; r < R; ++r) {
              const double2 tw = w[e];
              re = fma(v[r].x, tw.x, fma(-v[r].y, tw.y, re));
              im = fma(v[r].x, tw.y, fma(v[r].y, tw.x, im));
              e += t * m;
              if (e >= n) e -= n;
            }
            b[(out0 + t * Ns) * C + c] = make_double2(re, im);
          }
        }
      }
    } else {
      // a large prime radix: one output per thread, R terms each
      for (int idx = threadIdx.x; idx < n * C; idx += blockDim.x) {
        const int o = idx / C, c = idx - o * C;
        const int j = o % m, t = o / m;
        const int k = j % Ns;
        const int e1 = k * step + t * m;  // < n
        double re = 0.0, im = 0.0;
        int e = 0;
        for (int r = 0; r < R; ++r) {
          const double2 x = a[(j + r * m) * C + c];
          const double2 tw = w[e];
          re = fma(x.x, tw.x, fma(-x.y, tw.y, re));
          im = fma(x.x, tw.y, fma(x.y, tw.x, im));
          e += e1;
          if (e >= n) e -= n;
        }
        b[((j / Ns) * Ns * R + k + t * Ns) * C + c] = make_double2(re, im);
      }
    }
    __syncthreads();
    double2* tmp = a;
    a = b;
    b = tmp;
    Ns *= R;
  }
  for (int idx = threadIdx.x; idx < out_count * C; idx += blockDim.x) {
    const int e = idx / C, c = idx - e * C;
    if (c >= nc) continue;
    const double2 v = a[e * C + c];
    const long long o = f * lo.field + (long long)(l0 + c) * lo.line + (long long)e * lo.elem;
    if constexpr (OUT_REAL) static_cast<double*>(out)[o] = v.x * scale;
    else static_cast<double2*>(out)[o] = make_double2(v.x * scale, v.y * scale);
  }
}

inline size_t fft_smem_bytes(int n, int C) { return (size_t)(2 * C + 1) * n * sizeof(double2); }

// ---- power-of-two lines ----------------------------------------------------------
// n = 2^p, 8 <= n <= kFftMaxN: radix-8 Stockham passes (after one twiddle-free
// radix-2 or radix-4 pass when p is not a multiple of 3), each thread holding
// 8 points of one line in registers between passes, with one shared buffer
// of the CTA's lines (read, barrier, write, barrier).  A CTA of kFftThreads
// threads takes L = 8 kFftThreads / n lines: L adjacent rows, or L adjacent
// columns (COLS; every row access then covers L consecutive elements).
// IN_REAL (rows only): two real rows ride as one complex line
// z = x_a + i x_b and are separated after the transform,
// X_a[k] = (Z[k] + conj Z[n-k]) / 2, X_b[k] = -i (Z[k] - conj Z[n-k]) / 2.
constexpr int kFftP2Points = 8 * kFftThreads;  // points of a CTA's lines
// Shared-memory slot of point e of the CTA's line l: one pad slot after
// every 8 points (the first pass's stride-8 stores fall on different banks)
// and 2 more per line (the 8 lanes of a quarter-warp that take 4 columns'
// points of 2 rows fall on different banks).
__device__ __forceinline__ int fslot(int l, int e, int lstr) { return l * lstr + e + (e >> 3); }
__host__ __device__ inline int fft_p2_lstr(int n) { return n + n / 8 + 2; }

__host__ __device__ inline bool fft_pow2_ok(int n) { return n >= 8 && n <= kFftMaxN && (n & (n - 1)) == 0; }
inline size_t fft_p2_smem_bytes(int n) {
  return (size_t)((kFftP2Points / n) * fft_p2_lstr(n) + n) * sizeof(double2);
}

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 w) {
  return make_double2(fma(a.x, w.x, -a.y * w.y), fma(a.x, w.y, a.y * w.x));
}
// a times -i (forward, sign < 0) or +i (inverse), exact
__device__ __forceinline__ double2 cmul_mi(double2 a, int sign) {
  return sign < 0 ? make_double2(a.y, -a.x) : make_double2(-a.y, a.x);
}

// 8-point DFT in place: y_t = sum_r x_r e^{sign 2 pi i r t / 8}
__device__ __forceinline__ void dft8(double2 (&x)[8], int sign) {
  constexpr double c = 0.70710678118654752440;  // sqrt(2) / 2
  double2 a[4], b[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    a[r] = cadd(x[r], x[r + 4]);
    b[r] = csub(x[r], x[r + 4]);
  }
  // b_r times e^{sign 2 pi i r / 8}
  if (sign < 0) {
    b[1] = make_double2(c * (b[1].x + b[1].y), c * (b[1].y - b[1].x));
    b[3] = make_double2(c * (b[3].y - b[3].x), -c * (b[3].x + b[3].y));
  } else {
    b[1] = make_double2(c * (b[1].x - b[1].y), c * (b[1].x + b[1].y));
    b[3] = make_double2(-c * (b[3].x + b[3].y), c * (b[3].x - b[3].y));
  }
  b[2] = cmul_mi(b[2], sign);
  const double2 a02 = cadd(a[0], a[2]), d02 = csub(a[0], a[2]);
  const double2 a13 = cadd(a[1], a[3]), d13 = cmul_mi(csub(a[1], a[3]), sign);
  const double2 b02 = cadd(b[0], b[2]), e02 = csub(b[0], b[2]);
  const double2 b13 = cadd(b[1], b[3]), e13 = cmul_mi(csub(b[1], b[3]), sign);
  x[0] = cadd(a02, a13);
  x[4] = csub(a02, a13);
  x[2] = cadd(d02, d13);
  x[6] = csub(d02, d13);
  x[1] = cadd(b02, b13);
  x[5] = csub(b02, b13);
  x[3] = cadd(e02, e13);
  x[7] = csub(e02, e13);
}

template <bool IN_REAL, bool OUT_REAL, bool COLS>
__global__ void __launch_bounds__(kFftThreads, 4)
    fft_p2_kernel(const void* in, void* out, int n, int logn, int lines,
                  FftLines li, FftLines lo, int out_count, int sign, const double2* __restrict__ W,
                  double scale) {
  static_assert(!(IN_REAL && COLS), "real input is packed along rows only");
  extern __shared__ __align__(16) double2 fbuf[];
  const int L = kFftP2Points >> logn;  // complex lines of the CTA
  const int lstr = fft_p2_lstr(n);
  double2* buf = fbuf;                 // the CTA's lines, point (l, e) at fslot(l, e, lstr)
  double2* w = fbuf + L * lstr;        // the passes' twiddles (at most n)
  const int logL = 3 + 8 - logn;       // log2 L (kFftThreads = 256)
  const int clines = IN_REAL ? (lines + 1) >> 1 : lines;  // complex lines of a field
  const int groups = (clines + L - 1) / L;
  const int f = blockIdx.x / groups, g = blockIdx.x - f * groups;
  // Twiddles of the radix-8 passes, one table per pass (Ns = r0 8^i) laid
  // out [r - 1][k] (r = 1..7, k < Ns): the lanes of a warp read consecutive
  // k for each r, free of bank conflicts.  At most n entries in all.
  const int r0 = logn % 3;  // a first radix-2 (1) or radix-4 (2) pass
  {
    int base = 0;
    for (int ns = 1 << r0; ns < n; ns <<= 3) {
      const int step = n / (8 * ns);
      for (int e = threadIdx.x; e < 7 * ns; e += blockDim.x) {
        const int r = e / ns + 1, k = e - (r - 1) * ns;
        double2 v = W[r * k * step];  // r k step < n
        if (sign > 0) v.y = -v.y;
        w[base + e] = v;
      }
      base += 7 * ns;
    }
  }
  // ---- load ----
  // The CTA's lines hold kFftP2Points complex points (2 kFftP2Points real
  // values): a fixed number per thread, all loads issued before their
  // shared-memory stores.
  if constexpr (IN_REAL) {
    // real rows g 2L .. g 2L + 2L - 1: point e of line l is
    // (row 2l, row 2l + 1)[e]; a thread loads both rows' values of its points
    // and stores each point whole (16 bytes, no bank conflicts)
    const double* src = static_cast<const double*>(in) + f * li.field;
    constexpr int K = kFftP2Points / kFftThreads;
    double va[K], vb[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
      const int idx = threadIdx.x + i * kFftThreads;
      const int l = idx >> logn, e = idx & (n - 1);
      const int row = g * 2 * L + 2 * l;
      const long long o = (long long)row * li.line + (long long)e * li.elem;
      va[i] = row < lines ? src[o] : 0.0;
      vb[i] = row + 1 < lines ? src[o + li.line] : 0.0;
    }
#pragma unroll
    for (int i = 0; i < K; ++i) {
      const int idx = threadIdx.x + i * kFftThreads;
      buf[fslot(idx >> logn, idx & (n - 1), lstr)] = make_double2(va[i], vb[i]);
    }
  } else {
    const double2* src = static_cast<const double2*>(in) + f * li.field;
    constexpr int K = kFftP2Points / kFftThreads;
    double2 v[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
      const int idx = threadIdx.x + i * kFftThreads;
      if constexpr (COLS) {
        const int e = idx >> logL, c = idx & (L - 1);
        const int col = g * L + c;
        v[i] = col < lines ? src[(long long)col * li.line + (long long)e * li.elem] : make_double2(0.0, 0.0);
      } else {
        const int l = idx >> logn, e = idx & (n - 1);
        const int row = g * L + l;
        v[i] = row < lines ? src[(long long)row * li.line + (long long)e * li.elem] : make_double2(0.0, 0.0);
      }
    }
#pragma unroll
    for (int i = 0; i < K; ++i) {
      const int idx = threadIdx.x + i * kFftThreads;
      if constexpr (COLS) buf[fslot(idx & (L - 1), idx >> logL, lstr)] = v[i];
      else buf[fslot(idx >> logn, idx & (n - 1), lstr)] = v[i];
    }
  }
  __syncthreads();
  // ---- passes ----
  const int T = n >> 3;  // threads of a line
  const int lt = threadIdx.x >> (logn - 3), j = threadIdx.x & (T - 1);
  int Ns = 1;
  if (r0 != 0) {
    const int R = 1 << r0;
    double2 x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = buf[fslot(lt, j + i * T, lstr)];  // the 8 / R butterflies of this thread
    __syncthreads();
    if (R == 2) {
      // butterflies b = j + s T (s < 4): inputs b, b + n / 2 = x[s], x[s + 4]
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int b = j + s * T;
        buf[fslot(lt, 2 * b, lstr)] = cadd(x[s], x[s + 4]);
        buf[fslot(lt, 2 * b + 1, lstr)] = csub(x[s], x[s + 4]);
      }
    } else {
      // butterflies b = j + s T (s < 2): inputs b + r n / 4 = x[s + 2 r]
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const int b = j + s * T;
        const double2 s0 = cadd(x[s], x[s + 4]), s1 = csub(x[s], x[s + 4]);
        const double2 s2 = cadd(x[s + 2], x[s + 6]);
        const double2 s3 = cmul_mi(csub(x[s + 2], x[s + 6]), sign);
        buf[fslot(lt, 4 * b, lstr)] = cadd(s0, s2);
        buf[fslot(lt, 4 * b + 1, lstr)] = cadd(s1, s3);
        buf[fslot(lt, 4 * b + 2, lstr)] = csub(s0, s2);
        buf[fslot(lt, 4 * b + 3, lstr)] = csub(s1, s3);
      }
    }
    Ns = R;
    __syncthreads();
  }
  for (int wb = 0; Ns < n; wb += 7 * Ns, Ns <<= 3) {
    double2 x[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) x[r] = buf[fslot(lt, j + r * T, lstr)];
    const int k = j & (Ns - 1);
    const double2* wp = w + wb + k;  // this pass's table, column k
#pragma unroll
    for (int r = 1; r < 8; ++r) x[r] = cmul(x[r], wp[(r - 1) * Ns]);
    dft8(x, sign);
    __syncthreads();
    const int o = (j - k) * 8 + k;
#pragma unroll
    for (int t = 0; t < 8; ++t) buf[fslot(lt, o + t * Ns, lstr)] = x[t];
    __syncthreads();
  }
  // ---- store ----
  if constexpr (IN_REAL) {
    // both rows of line l from the same two points Z[k], Z[n - k]
    double2* dst = static_cast<double2*>(out) + f * lo.field;
    for (int idx = threadIdx.x; idx < L * out_count; idx += blockDim.x) {
      const int l = idx / out_count, k = idx - l * out_count;
      const int row = g * 2 * L + 2 * l;
      if (row >= lines) continue;
      const double2 zk = buf[fslot(l, k & (n - 1), lstr)], zm = buf[fslot(l, (n - k) & (n - 1), lstr)];
      const long long o = (long long)row * lo.line + (long long)k * lo.elem;
      dst[o] = make_double2(0.5 * (zk.x + zm.x) * scale, 0.5 * (zk.y - zm.y) * scale);
      if (row + 1 < lines)
        dst[o + lo.line] = make_double2(0.5 * (zk.y + zm.y) * scale, -0.5 * (zk.x - zm.x) * scale);
    }
  } else if constexpr (COLS) {
    for (int idx = threadIdx.x; idx < L * out_count; idx += blockDim.x) {
      const int e = idx >> logL, c = idx & (L - 1);
      const int col = g * L + c;
      if (col >= lines) continue;
      const double2 v = buf[fslot(c, e, lstr)];
      const long long o = f * lo.field + (long long)col * lo.line + (long long)e * lo.elem;
      if constexpr (OUT_REAL) static_cast<double*>(out)[o] = v.x * scale;
      else static_cast<double2*>(out)[o] = make_double2(v.x * scale, v.y * scale);
    }
  } else {
    for (int idx = threadIdx.x; idx < L * out_count; idx += blockDim.x) {
      const int l = idx / out_count, e = idx - l * out_count;
      const int row = g * L + l;
      if (row >= lines) continue;
      const double2 v = buf[fslot(l, e, lstr)];
      const long long o = f * lo.field + (long long)row * lo.line + (long long)e * lo.elem;
      if constexpr (OUT_REAL) static_cast<double*>(out)[o] = v.x * scale;
      else static_cast<double2*>(out)[o] = make_double2(v.x * scale, v.y * scale);
    }
  }
}

// 2 pi fftfreq(n, d)[j] as NumPy forms it: bin * (1 / (n d)), times 2 pi.
__device__ __forceinline__ double fft_wavenumber(int j, int n, double d) {
  const int bin = j < (n + 1) / 2 ? j : j - n;
  return 2.0 * 3.141592653589793 * ((double)bin * (1.0 / ((double)n * d)));
}

// ---- spectral diagnostics (OOP/hit2d.py:146-155, 429-468) -------------------
// rho, u, v of primitive_from_conservative (OOP/equations.py:136-145):
// fields [3][ny][nx].
__global__ void spec_prims_kernel(const double* __restrict__ q, double* __restrict__ ruv, long long n,
                                  double gamma) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    const Prim<double> p = primitives(q[c], q[n + c], q[2 * n + c], q[3 * n + c], gamma);
    ruv[c] = p.rho;
    ruv[n + c] = p.u;
    ruv[2 * n + c] = p.v;
  }
}

// From the transforms U, V [2][ny][nx]: i (KX U + KY V) (divergence),
// i (KX V - KY U) (vorticity) and U, V restricted to 0 < |k| <= kmax (the
// low-k band of the kinetic fraction) -> out [4][ny][nx].
__global__ void spec_multiply_kernel(const double2* __restrict__ uv, double2* __restrict__ out, int nx,
                                     int ny, double dx, double dy, double kmax) {
  const long long n = (long long)nx * ny;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(c / nx), i = (int)(c - (long long)j * nx);
    const double kx = fft_wavenumber(i, nx, dx), ky = fft_wavenumber(j, ny, dy);
    const double2 U = uv[c], V = uv[n + c];
    // i z = (-z.y, z.x)
    const double dre = kx * U.x + ky * V.x, dim = kx * U.y + ky * V.y;
    const double wre = kx * V.x - ky * U.x, wim = kx * V.y - ky * U.y;
    out[c] = make_double2(-dim, dre);
    out[n + c] = make_double2(-wim, wre);
    const double k2 = kx * kx + ky * ky;
    const double mag = sqrt(k2);
    const bool keep = k2 > 0.0 && mag <= kmax;
    out[2 * n + c] = keep ? U : make_double2(0.0, 0.0);
    out[3 * n + c] = keep ? V : make_double2(0.0, 0.0);
  }
}

// Sums of div^2, vort^2, rho (ul^2 + vl^2) and rho (u'^2 + v'^2) (u' = u -
// mean u, the mean from the transform's zero mode) into per-CTA partials;
// the last CTA (ticket in part_n[0]) writes the four totals to res.
// div / vort fields are copied out when the pointers are given.
__global__ void __launch_bounds__(256)
    spec_reduce_kernel(const double* __restrict__ ruv, const double* __restrict__ dwb,
                       const double2* __restrict__ uv, long long n, double* __restrict__ part,
                       unsigned* ticket, double* __restrict__ res, double* __restrict__ div_out,
                       double* __restrict__ vort_out) {
  const double mu = uv[0].x / (double)n, mv = uv[n].x / (double)n;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    const double d = dwb[c], w = dwb[n + c], ul = dwb[2 * n + c], vl = dwb[3 * n + c];
    const double rho = ruv[c], uf = ruv[n + c] - mu, vf = ruv[2 * n + c] - mv;
    s[0] += d * d;
    s[1] += w * w;
    s[2] += rho * (ul * ul + vl * vl);
    s[3] += rho * (uf * uf + vf * vf);
    if (div_out) div_out[c] = d;
    if (vort_out) vort_out[c] = w;
  }
  __shared__ double sm[8][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double v = warp_sum(s[k]);
    if (lane == 0) sm[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double acc = 0.0;
    for (int w = 0; w < 8; ++w) acc += sm[w][threadIdx.x];
    part[blockIdx.x * 4 + threadIdx.x] = acc;
  }
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned t = atomicAdd(ticket, 1u);
    last = t == gridDim.x - 1u;
    if (last) *ticket = 0u;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < 4) {
    double acc = 0.0;
    for (unsigned b = 0; b < gridDim.x; ++b) acc += __ldcg(part + b * 4 + threadIdx.x);
    res[threadIdx.x] = acc;
  }
}

// i KY P and -i KX P (the initial condition's u = d psi / dy, v = -d psi / dx,
// OOP/hit2d.py:186-188) -> out [2][ny][nx].
__global__ void spec_velocity_kernel(const double2* __restrict__ ph, double2* __restrict__ out, int nx,
                                     int ny, double dx, double dy) {
  const long long n = (long long)nx * ny;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(c / nx), i = (int)(c - (long long)j * nx);
    const double kx = fft_wavenumber(i, nx, dx), ky = fft_wavenumber(j, ny, dy);
    const double2 P = ph[c];
    out[c] = make_double2(-ky * P.y, ky * P.x);
    out[n + c] = make_double2(kx * P.y, -kx * P.x);
  }
}

}  // namespace hitb200
