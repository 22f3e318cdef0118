// The reference's forcing-noise stream on the device (noise_mode 2): the
// field np.random.default_rng(seed).standard_normal((ny, nx)) of each step
// (OOP/forcing.py:66,77), draw for draw, from the stream's PCG64 state kept
// in the solve's scalar block.
//
// NumPy's normal sampler consumes a variable number of 64-bit draws per
// normal: one on the ziggurat's fast path, two for a wedge test (which may
// reject and start over), 1 + 2t for the tail.  The field is built in five
// passes over P raw positions (P = N + N / 8 + 4096 >= the draws N normals
// need, with overwhelming margin; a shortfall sets ST_NOISE):
//   classify  every position p as the start of an attempt: its draw count
//             cons[p], whether it yields a normal, and that normal (slow
//             attempts read the draws after p themselves); per-CTA counts
//             of the slow positions (cons != 1);
//   scan      the counts' offsets (one CTA);
//   compact   the slow positions, in order;
//   resolve   which slow positions the chain of attempts from position 0
//             visits (a visited attempt skips the draws it consumed; fast
//             positions never skip), the deficit of outputs before each, and
//             the furthest draw each visited span reaches (one CTA);
//   scatter   each visited output-producing position p writes its normal to
//             index p - (draws skipped or rejected before p); the thread of
//             the last normal advances the PCG64 state past its draws.
// Transcendentals of the slow paths use CUDA's log1p / exp; they decide
// about 1.2 % of the draws, and a decision could flip only for a draw within
// an ulp of its wedge boundary.
#pragma once

#include "common.cuh"
#include "reduce.cuh"

namespace hitb200 {

namespace zig {
#include "ziggurat_table.inc"
}

constexpr int kNoiseChunk = 8;      // positions per thread (classify, scatter)
constexpr int kNoiseThreads = 256;
constexpr int kNoiseResolveThreads = 1024;
constexpr double kZigR = 3.6541528853610088;

__device__ double g_zig_w[256];
__device__ unsigned long long g_zig_k[256];
__device__ double g_zig_f[256];

struct U128 {
  unsigned long long lo, hi;
};
__device__ __forceinline__ U128 u128_mul(U128 a, U128 b) {
  U128 r;
  r.lo = a.lo * b.lo;
  r.hi = __umul64hi(a.lo, b.lo) + a.lo * b.hi + a.hi * b.lo;
  return r;
}
__device__ __forceinline__ U128 u128_add(U128 a, U128 b) {
  U128 r;
  r.lo = a.lo + b.lo;
  r.hi = a.hi + b.hi + (r.lo < a.lo ? 1ull : 0ull);
  return r;
}
__device__ __forceinline__ U128 pcg_mult() { return U128{4865540595714422341ull, 2549297995355413924ull}; }
// PCG64 step: s <- s M + inc (mod 2^128)
__device__ __forceinline__ U128 pcg_step(U128 s, U128 inc) { return u128_add(u128_mul(s, pcg_mult()), inc); }
// XSL-RR output of a state
__device__ __forceinline__ unsigned long long pcg_out(U128 s) {
  const unsigned rot = (unsigned)(s.hi >> 58);
  const unsigned long long x = s.hi ^ s.lo;
  return (x >> rot) | (x << ((64u - rot) & 63u));
}
// The state after `delta` steps (Brown's LCG skip-ahead).
__device__ U128 pcg_advance(U128 s, U128 inc, unsigned long long delta) {
  U128 am{1ull, 0ull}, ap{0ull, 0ull}, cm = pcg_mult(), cp = inc;
  while (delta) {
    if (delta & 1ull) {
      am = u128_mul(am, cm);
      ap = u128_add(u128_mul(ap, cm), cp);
    }
    cp = u128_mul(u128_add(cm, U128{1ull, 0ull}), cp);
    cm = u128_mul(cm, cm);
    delta >>= 1;
  }
  return u128_add(u128_mul(am, s), ap);
}
__device__ __forceinline__ double u53(unsigned long long r) {
  return (double)(r >> 11) * (1.0 / 9007199254740992.0);
}

// The stream state in the scalar block: 4 slots holding the bit patterns of
// state.lo, state.hi, inc.lo, inc.hi.
__device__ __forceinline__ U128 noise_state(const double* sc, int slot) {
  return U128{(unsigned long long)__double_as_longlong(sc[slot]),
              (unsigned long long)__double_as_longlong(sc[slot + 1])};
}

// Per-solve buffers of the generator (arena of a noise_mode 2 plan).
struct NoiseBufs {
  unsigned char* cons;   // [P] draws of the attempt starting at p
  unsigned char* outf;   // [P] 1 if that attempt yields a normal
  double* val;           // [P] its normal
  unsigned* cta_count;   // [nblk] slow positions per classify CTA
  unsigned* cta_off;     // [nblk + 1]
  unsigned* slow;        // [P] compacted slow positions
  long long* deficit;    // [P] outputs missing before slow entry i (exclusive)
  unsigned char* visited;  // [P] slow entry i visited by the chain
  unsigned* reach;         // [P] furthest draw reached by visited spans before entry i
  unsigned* nslow;         // [1]
  long long P;
};

__global__ void __launch_bounds__(kNoiseThreads)
    npnoise_classify_kernel(const SolveDev* __restrict__ solves, NoiseBufs b, int slot) {
  const SolveDev& S = solves[0];
  const double* sc = S.scal;
  if (sc[S_ACTIVE] == 0.0) return;
  __shared__ double zw[256], zf[256];
  __shared__ unsigned long long zk[256];
  for (int t = threadIdx.x; t < 256; t += blockDim.x) {
    zw[t] = g_zig_w[t];
    zf[t] = g_zig_f[t];
    zk[t] = g_zig_k[t];
  }
  __syncthreads();
  const U128 s0 = noise_state(sc, slot), inc = noise_state(sc, slot + 2);
  const long long p0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * kNoiseChunk;
  unsigned nslow = 0;
  if (p0 < b.P) {
    U128 s = pcg_advance(s0, inc, (unsigned long long)p0 + 1ull);  // state of draw p0
    for (int c = 0; c < kNoiseChunk && p0 + c < b.P; ++c) {
      const long long p = p0 + c;
      unsigned long long r = pcg_out(s);
      const int idx = (int)(r & 0xff);
      r >>= 8;
      const int sign = (int)(r & 1ull);
      const unsigned long long rabs = (r >> 1) & 0x000fffffffffffffull;
      double x = (double)rabs * zw[idx];
      if (sign) x = -x;
      unsigned cons = 1, out = 1;
      if (!(rabs < zk[idx])) {
        U128 t = pcg_step(s, inc);  // draws after p
        if (idx == 0) {
          // tail beyond r0 (Marsaglia's method with two uniforms per try)
          for (;;) {
            const double u1 = u53(pcg_out(t));
            t = pcg_step(t, inc);
            const double u2 = u53(pcg_out(t));
            t = pcg_step(t, inc);
            cons += 2;
            const double xx = __dmul_rn(-(1.0 / kZigR), log1p(-u1));
            const double yy = -log1p(-u2);
            if (__dadd_rn(yy, yy) > __dmul_rn(xx, xx)) {
              x = ((rabs >> 8) & 1ull) ? -__dadd_rn(kZigR, xx) : __dadd_rn(kZigR, xx);
              break;
            }
            if (cons > 250) {  // impossible in practice: report, never loop on
              out = 0;
              break;
            }
          }
        } else {
          const double u = u53(pcg_out(t));
          cons = 2;
          // separately rounded product and sum, as NumPy's C evaluates it
          const double lhs = __dadd_rn(__dmul_rn(__dsub_rn(zf[idx - 1], zf[idx]), u), zf[idx]);
          out = (lhs < exp(__dmul_rn(__dmul_rn(-0.5, x), x))) ? 1u : 0u;
        }
        ++nslow;
      }
      b.cons[p] = (unsigned char)cons;
      b.outf[p] = (unsigned char)out;
      b.val[p] = x;
      s = pcg_step(s, inc);
    }
  }
  // slow positions of this CTA
  __shared__ unsigned wsum[kNoiseThreads / 32];
  const unsigned tot = warp_sum(nslow);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = tot;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned a = 0;
    for (int w = 0; w < kNoiseThreads / 32; ++w) a += wsum[w];
    b.cta_count[blockIdx.x] = a;
  }
}

// Exclusive offsets of the per-CTA counts (one CTA).
__global__ void __launch_bounds__(1024)
    npnoise_scan_kernel(const SolveDev* __restrict__ solves, NoiseBufs b, int nblk) {
  if (solves[0].scal[S_ACTIVE] == 0.0) return;
  __shared__ unsigned carry, wsum[32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base = 0; base < nblk; base += 1024) {
    const int i = base + threadIdx.x;
    const unsigned v = i < nblk ? b.cta_count[i] : 0u;
    unsigned x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      unsigned w = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      wsum[lane] = w;
    }
    __syncthreads();
    const unsigned excl = carry + (warp > 0 ? wsum[warp - 1] : 0u) + x - v;
    if (i < nblk) b.cta_off[i] = excl;
    __syncthreads();
    if (threadIdx.x == 0) carry += wsum[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    b.cta_off[nblk] = carry;
    *b.nslow = carry;
  }
}

// The slow positions in order: each CTA rescans its classify range.
__global__ void __launch_bounds__(kNoiseThreads)
    npnoise_compact_kernel(const SolveDev* __restrict__ solves, NoiseBufs b) {
  if (solves[0].scal[S_ACTIVE] == 0.0) return;
  const long long p0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * kNoiseChunk;
  unsigned mine = 0;
  for (int c = 0; c < kNoiseChunk; ++c)
    if (p0 + c < b.P && b.cons[p0 + c] != 1) ++mine;
  // exclusive prefix of `mine` over the CTA, in thread order
  __shared__ unsigned wsum[kNoiseThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned x = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  unsigned before = 0;
  for (int w = 0; w < warp; ++w) before += wsum[w];
  unsigned pos = b.cta_off[blockIdx.x] + before + x - mine;
  for (int c = 0; c < kNoiseChunk; ++c)
    if (p0 + c < b.P && b.cons[p0 + c] != 1) b.slow[pos++] = (unsigned)(p0 + c);
}

// Which slow positions the chain from position 0 visits (one CTA): a slow
// entry starts a cluster when no earlier span reaches it; each cluster is
// walked by the thread of its start.  Then, over visited entries, the
// exclusive prefix of output deficits ((cons - 1) skipped draws, plus one for
// a rejected wedge) and of the furthest draw reached.
__global__ void __launch_bounds__(kNoiseResolveThreads)
    npnoise_resolve_kernel(const SolveDev* __restrict__ solves, NoiseBufs b) {
  if (solves[0].scal[S_ACTIVE] == 0.0) return;
  const unsigned n = *b.nslow;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ unsigned long long wred[32];
  __shared__ unsigned long long carry_u;  // running max of (slow + cons) over all entries
  __shared__ long long carry_d;
  // pass 1: all-entry reach (exclusive prefix max of slow + cons) -> cluster starts
  if (threadIdx.x == 0) carry_u = 0ull;
  __syncthreads();
  for (unsigned base = 0; base < n; base += blockDim.x) {
    const unsigned i = base + threadIdx.x;
    const unsigned long long e = i < n ? (unsigned long long)b.slow[i] + b.cons[b.slow[i]] : 0ull;
    unsigned long long x = e;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x = x > y ? x : y;
    }
    if (lane == 31) wred[warp] = x;
    __syncthreads();
    unsigned long long before = carry_u;
    for (int w = 0; w < warp; ++w) before = before > wred[w] ? before : wred[w];
    unsigned long long prev = __shfl_up_sync(0xffffffffu, x, 1);
    if (lane == 0) prev = 0ull;
    const unsigned long long excl = before > prev ? before : prev;
    // cluster starts, kept apart from the visited flags the walks write
    if (i < n) b.reach[i] = excl <= b.slow[i] ? 1u : 0u;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long m = carry_u;
      for (int w = 0; w < 32; ++w) m = m > wred[w] ? m : wred[w];
      carry_u = m;
    }
    __syncthreads();
  }
  // pass 2: walk each cluster from its start
  for (unsigned i = threadIdx.x; i < n; i += blockDim.x) {
    if (b.reach[i] != 1u) continue;
    unsigned long long end = (unsigned long long)b.slow[i] + b.cons[b.slow[i]];
    b.visited[i] = 1;
    for (unsigned j = i + 1; j < n && b.reach[j] != 1u; ++j) {
      const unsigned sj = b.slow[j];
      const bool vis = sj >= end;
      b.visited[j] = vis ? 1 : 0;
      if (vis) end = (unsigned long long)sj + b.cons[sj];
    }
  }
  __syncthreads();
  // pass 3: exclusive prefix sums of deficits and prefix max of spans over visited entries
  if (threadIdx.x == 0) {
    carry_d = 0;
    carry_u = 0ull;
  }
  __syncthreads();
  __shared__ long long wd[32];
  for (unsigned base = 0; base < n; base += blockDim.x) {
    const unsigned i = base + threadIdx.x;
    long long d = 0;
    unsigned long long e = 0ull;
    if (i < n && b.visited[i] == 1) {
      const unsigned si = b.slow[i];
      d = (long long)b.cons[si] - 1 + (b.outf[si] ? 0 : 1);
      e = (unsigned long long)si + b.cons[si];
    }
    long long xd = d;
    unsigned long long xe = e;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long yd = __shfl_up_sync(0xffffffffu, xd, o);
      const unsigned long long ye = __shfl_up_sync(0xffffffffu, xe, o);
      if (lane >= o) {
        xd += yd;
        xe = xe > ye ? xe : ye;
      }
    }
    if (lane == 31) {
      wd[warp] = xd;
      wred[warp] = xe;
    }
    __syncthreads();
    long long bd = carry_d;
    unsigned long long be = carry_u;
    for (int w = 0; w < warp; ++w) {
      bd += wd[w];
      be = be > wred[w] ? be : wred[w];
    }
    unsigned long long pe = __shfl_up_sync(0xffffffffu, xe, 1);
    if (lane == 0) pe = 0ull;
    if (i < n) {
      b.deficit[i] = bd + xd - d;
      b.reach[i] = (unsigned)(be > pe ? be : pe);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 0; w < 32; ++w) {
        carry_d += wd[w];
        carry_u = carry_u > wred[w] ? carry_u : wred[w];
      }
    }
    __syncthreads();
  }
  // normals available in [0, P): every position minus the skipped and
  // rejected ones (a span reaching past P skipped draws beyond it too)
  if (threadIdx.x == 0) {
    const long long over = (long long)carry_u > b.P ? (long long)carry_u - b.P : 0;
    const long long avail = b.P - carry_d + over;
    const SolveDev& S = solves[0];
    if (avail < (long long)S.nx * S.ny) S.scal[S_STATUS] = (double)((int)S.scal[S_STATUS] | ST_NOISE);
  }
}

// Scatter the normals of visited positions into out[0, N); the thread of
// output N - 1 advances the stream state past its draws.
__global__ void __launch_bounds__(kNoiseThreads)
    npnoise_scatter_kernel(const SolveDev* __restrict__ solves, NoiseBufs b, double* __restrict__ out,
                           long long N, int slot) {
  const SolveDev& S = solves[0];
  double* sc = S.scal;
  if (sc[S_ACTIVE] == 0.0) return;
  const unsigned n = *b.nslow;
  const long long p0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * kNoiseChunk;
  if (p0 >= b.P) return;
  // entries before p0: j = number of slow positions < p0
  unsigned lo = 0, hi = n;
  while (lo < hi) {
    const unsigned mid = (lo + hi) >> 1;
    if (b.slow[mid] < (unsigned)p0) lo = mid + 1;
    else hi = mid;
  }
  unsigned j = lo;
  for (int c = 0; c < kNoiseChunk && p0 + c < b.P; ++c) {
    const long long p = p0 + c;
    long long oi = -1;
    if (j < n && b.slow[j] == (unsigned)p) {
      // a slow position: its own entry
      if (b.visited[j] == 1 && b.outf[p]) oi = p - b.deficit[j];
      ++j;
    } else {
      // a fast position: skipped when a visited span before it reaches past it
      const long long reach = j < n ? (long long)b.reach[j] : -1;
      long long rmax = reach;
      if (j >= n && n > 0) {
        // beyond the last slow entry: the furthest span of all visited entries
        const unsigned k = n - 1;
        rmax = b.reach[k];
        if (b.visited[k] == 1) {
          const long long e = (long long)b.slow[k] + b.cons[b.slow[k]];
          rmax = rmax > e ? rmax : e;
        }
      }
      if (rmax <= p) {
        long long dsum;
        if (j < n) dsum = b.deficit[j];
        else if (n > 0) {
          const unsigned k = n - 1;
          dsum = b.deficit[k] + (b.visited[k] == 1 ? (long long)b.cons[b.slow[k]] - 1 + (b.outf[b.slow[k]] ? 0 : 1) : 0);
        } else dsum = 0;
        oi = p - dsum;
      }
    }
    if (oi >= 0 && oi < N) {
      out[oi] = b.val[p];
      if (oi == N - 1) {
        const U128 s0 = noise_state(sc, slot), inc = noise_state(sc, slot + 2);
        const U128 s1 = pcg_advance(s0, inc, (unsigned long long)(p + b.cons[p]));
        sc[slot] = __longlong_as_double((long long)s1.lo);
        sc[slot + 1] = __longlong_as_double((long long)s1.hi);
      }
    }
  }
}

}  // namespace hitb200
