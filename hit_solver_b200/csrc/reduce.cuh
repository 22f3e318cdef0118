// Grid reductions of the hot path and the scalar logic that consumes them.
//
// Every reducing kernel follows one deterministic pattern: each CTA reduces
// its tile (warp shuffles, then across warps in shared memory) and writes one
// row of per-block partials; the last CTA of the solve to finish (atomic
// ticket) sums the partials in a fixed order and runs the scalar logic in one
// thread.  Results therefore do not depend on scheduling, and no value ever
// travels to the host: time step, Lax-Friedrichs speeds, sensor limits,
// Mach control and forcing scales stay in the solve's scalar block.
#pragma once

#include "common.cuh"

namespace hitb200 {

constexpr int kRedThreads = 512;
constexpr int kRedWarps = kRedThreads / 32;
constexpr int kTileX = 32;   // prepass / noise / synth / diagnostics tile: 32 x 32 cells
constexpr int kTileY = 32;
constexpr int kCellsPerThread = kTileY / kRedWarps;  // rows of the tile per thread

enum RedOp : int { OP_SUM = 0, OP_MAX = 1 };

// Reduce `v` over the CTA into sm[row][slot] (call from all threads); row is
// the warp's index in the CTA unless the caller names it.
template <int OP>
__device__ __forceinline__ void warp_to_smem(double v, double* sm, int slot, int nslots, int row = -1) {
  v = OP == OP_SUM ? warp_sum(v) : warp_max(v);
  if ((threadIdx.x & 31) == 0) sm[(row < 0 ? (int)(threadIdx.x >> 5) : row) * nslots + slot] = v;
}

// Reduce four values over the warp with 6 exchanges instead of 20: after two
// halving steps each lane carries one of the four partial sums, then a
// butterfly over the low three lane bits completes it.  Lanes 0, 8, 16 and 24
// hold the totals of v0, v1, v2 and v3 and store them in sm[row][slot_j]
// (slot_j < 0: not stored; row as in warp_to_smem).
template <int OP>
__device__ __forceinline__ void warp_to_smem4(double v0, double v1, double v2, double v3, double* sm,
                                              int4 slot, int nslots, int row = -1) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  auto op = [](double a, double b) { return OP == OP_SUM ? a + b : fmax(a, b); };
  const bool hi4 = lane & 16, hi3 = lane & 8;
  double a0 = hi4 ? v2 : v0, a1 = hi4 ? v3 : v1;
  const double s0 = hi4 ? v0 : v2, s1 = hi4 ? v1 : v3;
  a0 = op(a0, __shfl_xor_sync(full, s0, 16));
  a1 = op(a1, __shfl_xor_sync(full, s1, 16));
  double b = hi3 ? a1 : a0;
  const double t = hi3 ? a0 : a1;
  b = op(b, __shfl_xor_sync(full, t, 8));
  b = op(b, __shfl_xor_sync(full, b, 4));
  b = op(b, __shfl_xor_sync(full, b, 2));
  b = op(b, __shfl_xor_sync(full, b, 1));
  if ((lane & 7) == 0) {
    const int j = lane >> 3;
    const int sl = j == 0 ? slot.x : j == 1 ? slot.y : j == 2 ? slot.z : slot.w;
    if (sl >= 0) sm[(row < 0 ? (int)(threadIdx.x >> 5) : row) * nslots + sl] = b;
  }
}

// After __syncthreads: threads t < nslots combine the warps and store row `blk`.
__device__ __forceinline__ void smem_to_partials(const double* sm, int nslots,
                                                 const int* ops, double* part, int blk) {
  for (int t = threadIdx.x; t < nslots; t += blockDim.x) {
    double acc = sm[t];
    const int op = ops ? ops[t] : OP_SUM;
    for (int w = 1; w < kRedWarps; ++w) {
      double x = sm[w * nslots + t];
      acc = op == OP_SUM ? acc + x : fmax(acc, x);
    }
    part[(size_t)blk * nslots + t] = acc;
  }
}

// Ticket: returns true in the last CTA of the solve.  Resets the counter.
__device__ __forceinline__ bool last_block(unsigned* counter, int nblk) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned t = atomicAdd(counter, 1u);
    is_last = (t == (unsigned)nblk - 1u);
    if (is_last) *counter = 0u;
  }
  __syncthreads();
  if (is_last) __threadfence();
  return is_last;
}

// Test hook of the grid barrier (set by hitb200_set_barrier_test): the number
// of arrivals the barrier waits for beyond its launch's CTAs (0 in normal use;
// 1 makes every wait run out) and the wait limit in nanoseconds.
__device__ unsigned g_barrier_extra = 0u;
__device__ unsigned long long g_barrier_limit_ns = 2000000000ull;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Barrier over every CTA of a cooperative launch (which guarantees that all
// of them are resident).  count and gen are zero-initialised words of the
// solve's counters; the last CTA to arrive resets count and advances gen.
// A CTA that waits longer than the limit (about 2 s of the global timer, or
// 2^26 polls) gives up: it withdraws its arrival, sets *err and continues, so
// that a failed launch cannot hang the GPU.
__device__ __forceinline__ void grid_barrier(unsigned* count, unsigned* gen, unsigned nblocks,
                                             unsigned* err) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = gen;
    const unsigned target = nblocks - 1u + *(volatile unsigned*)&g_barrier_extra;
    const unsigned long long limit = *(volatile unsigned long long*)&g_barrier_limit_ns;
    const unsigned g0 = *vgen;
    __threadfence();
    if (atomicAdd(count, 1u) == target) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      const unsigned long long t0 = global_ns();
      unsigned long long it = 0;
      while (*vgen == g0) {
        __nanosleep(100);
        if (++it > (1ull << 26) || ((it & 31) == 0 && global_ns() - t0 > limit)) {
          atomicSub(count, 1u);
          atomicOr(err, 1u);
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
}

__device__ __forceinline__ int red_op(int slot) {
  switch (slot) {
    case R_AX: case R_AY: case R_RHO: case R_P: case R_E: case R_SR:
    case R_NONFINITE: case R_NONPOS_RHO: case R_NONPOS_P:
      return OP_MAX;
    default:
      return OP_SUM;
  }
}

}  // namespace hitb200
