// One persistent launch per SSP-RK3 stage of a batch (the stage's prepass,
// sensor, y sweep and x sweep of every member in one kernel).
//
// The launch keeps a fixed number of CTAs resident (2 per SM) and each CTA
// takes work items from a queue (an atomic ticket) until it runs dry.  The
// queue holds, phase after phase, the prepass tiles (two per item), sensor
// tiles, y panels of 4 columns and x groups of 4 rows of the members.  An item
// of one phase of a solve needs that solve's previous phase complete (the
// prepass's reductions before the sensor's thresholds, the whole mask before
// the y sweep's WENO faces, the whole partial rhs before the x sweep's
// epilogue); it stages its inputs first and then waits on the solve's counter
// of finished items of that phase, exactly where the kernels of the per-phase
// launches wait for their predecessor.  The x sweep also reads, before that
// wait, what the per-phase launches wrote two kernels earlier (the mask, the
// Lax-Friedrichs speed): its items first wait, after staging their rows, for
// all of the solve's sensor tiles (which themselves waited for the prepass).  Every item an item waits for was
// queued before it, so the queue cannot deadlock whatever the residency: the
// oldest unfinished item never waits.  Each wait is bounded (the grid
// barrier's limit, about 2 s): one that runs out sets the queue's abort flag,
// which ends the launch's remaining waits at once; every solve whose wait
// ended unmet gets its bounded-wait flag, reported as ST_BARRIER by its next
// prepass.
//
// The items run the same device code as the per-phase kernels (prepass_tile,
// sensor_step_body, sweep_body) on the same tiles, lines and partials, so the
// results are bit for bit those of the per-phase launches.
#pragma once

#include "kernels_reduce.cuh"
#include "kernels_stencil.cuh"
#include "sensor_step.cuh"

namespace hitb200 {

constexpr int kStageThreads = 512;
constexpr int kStageLines = kStageThreads / kLineThreads;  // lines of a sweep item

enum QKind : int { Q_PRE = 0, Q_SEN = 1, Q_SWY = 2, Q_SWX = 3 };

// A work item: n consecutive entries from idx of its kind's work list (tiles
// for the prepass and the sensor, 4-column panels for the y sweep, 4-row
// groups for the x sweep; n is 1 or 2 for the prepass, 1 otherwise), the
// number of finished items of the previous phase of its solve that it waits
// for (sensor: 1, the prepass's completion flag, or 0 in the first stage,
// whose prepass is the step's own launch), and for x groups the number of
// the solve's sensor tiles (their early wait).
struct QItem {
  int kind, idx, n, target, early;
};

// Queue of one launch: next ticket, CTAs that have left, abort flag.  A CTA
// holds one ticket ahead of the item it runs; the oldest unfinished item is
// still always running or about to run, since the CTA holding it finishes its
// current (older) item first.
struct QCtl {
  unsigned head, exitc, abort, pad;
};

// Per-solve counters of one launch (QDEP_* words of 4): prepass complete,
// then finished sensor, y and x items.  All zero between launches.
enum QDep : int { QDEP_PRE = 0, QDEP_SEN = 1, QDEP_SWY = 2, QDEP_SWX = 3 };

// Wait of an item for `target` finished items of the previous phase of its
// solve (wait), and for `etarget` finished items of an earlier phase whose
// output it reads before that (early); the item's first thread polls, the
// item's threads then continue together.  The grid barrier's test hook adds
// its extra arrivals to the targets.  SUB: the item runs on one of the CTA's
// four groups of kLineThreads threads (one x line each, with the group's own
// named barrier); otherwise on the whole CTA.
template <bool SUB>
struct QueueDepT {
  static constexpr bool kQueued = true;
  static constexpr int kXR = SUB ? 1 : kStageLines;
  const unsigned* cnt;
  unsigned target;
  const unsigned* ecnt;
  unsigned etarget;
  unsigned* abort;
  unsigned* err;
  // first reads of the counters, issued when the item starts so that their
  // latency overlaps the item's staging; a wait polls only if its counter
  // had not reached the target then
  unsigned seen = 0u, eseen = 0u;
  __device__ __forceinline__ QueueDepT(const unsigned* c, unsigned t, const unsigned* ec, unsigned et,
                                       unsigned* ab, unsigned* e)
      : cnt(c), target(t), ecnt(ec), etarget(et), abort(ab), err(e) {
    if (tid() == 0) {
      if (t > 0u) seen = *(const volatile unsigned*)c;
      if (et > 0u) eseen = *(const volatile unsigned*)ec;
    }
  }
  __device__ __forceinline__ unsigned tid() const { return SUB ? threadIdx.x % kLineThreads : threadIdx.x; }
  __device__ __forceinline__ unsigned nthreads() const { return SUB ? (unsigned)kLineThreads : blockDim.x; }
  __device__ __forceinline__ unsigned group() const { return 1u + threadIdx.x / kLineThreads; }
  __device__ __forceinline__ void sync() const {
    if constexpr (SUB) group_sync(group(), kLineThreads);
    else __syncthreads();
  }
  __device__ __forceinline__ bool sync_or(bool p) const {
    if constexpr (SUB) return group_sync_or(group(), kLineThreads, p);
    else return __syncthreads_or(p) != 0;
  }
  __device__ __forceinline__ void wait() const { wait_for(cnt, target, seen); }
  __device__ __forceinline__ void early() const { wait_for(ecnt, etarget, eseen); }
  __device__ __forceinline__ void release() const {}
  __device__ __forceinline__ void wait_for(const unsigned* counter, unsigned target, unsigned first) const {
    if (tid() == 0 && target > 0u) {
      const volatile unsigned* c = counter;
      const volatile unsigned* ab = abort;
      const unsigned tgt = target + *(volatile unsigned*)&g_barrier_extra;
      if (first < tgt && *c < tgt) {
        const unsigned long long limit = *(volatile unsigned long long*)&g_barrier_limit_ns;
        const unsigned long long t0 = global_ns();
        unsigned long long it = 0;
        while (*c < tgt && *ab == 0u) {
          __nanosleep(64);
          if (++it > (1ull << 26) || ((it & 15) == 0 && global_ns() - t0 > limit)) {
            atomicOr(abort, 1u);
            break;
          }
        }
        // gave up (here or after another wait of the launch): this step of
        // the solve is not valid, and its next prepass reports ST_BARRIER
        if (*c < tgt) atomicOr(err, 1u);
      }
      __threadfence();
    }
    sync();
  }
};
using QueueDep = QueueDepT<false>;

// Dynamic shared memory of the prepass items: two tiles' scratch.
template <typename T>
__host__ __device__ constexpr size_t stage_pre_smem_bytes() {
  return 2 * sizeof(PreShared<T>);
}
// Layout of the dynamic shared memory: the largest item's region from 0 (two
// prepass tiles; a sensor tile; a y panel of 4 columns; four x lines, each
// group's at a multiple of `xstride`, the largest one-line x region), then
// from sh_off the four groups' statically sized sweep memory (the y items use
// group 0's).  The prepass's final reduction reuses the start of the region.
template <typename T>
using StageSweepShared = SweepShared<T, 1>;

#ifdef HITB200_STAGE_INLINE_ITEMS
#define HB_STAGE_ITEM __forceinline__
#else
#define HB_STAGE_ITEM __noinline__
#endif

// Each kind of item is a function of its own (not inlined), so that each
// gets its own register allocation at the launch's 64 registers per thread;
// they name the dynamic shared memory directly, which keeps their accesses in
// the shared state space.

// Two prepass tiles of one solve, one per half of the CTA (the prepass
// kernel's arithmetic and partial rows); the item finishing the solve's last
// tiles reduces the partials and marks the prepass complete.
template <typename T>
__device__ HB_STAGE_ITEM void stage_pre_item(const SolveDev* __restrict__ solves, const Work* __restrict__ tiles32,
                                             int idx, int n, unsigned* dep, int stage) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_last;
  const int half = threadIdx.x >= kPreThreads ? 1 : 0;
  const bool mine = half < n;
  const Work w = tiles32[idx + (mine ? half : 0)];
  const SolveDev& S = solves[w.solve];
  const bool active = __ldcg(&S.scal[S_ACTIVE]) != 0.0;
  PreShared<T>* P = reinterpret_cast<PreShared<T>*>(smem) + half;
  const int nslots = prepass_tile<T>(S, w, stage, PRE_STAGE, 1, Bind{}, active, *P,
                                     mine ? half * kPreThreads : kStageThreads);
  if (nslots < 0) {  // a finished solve: nothing to reduce
    if (threadIdx.x == 0) atomicExch(&dep[4 * w.solve + QDEP_PRE], 1u);
    return;
  }
  __syncthreads();  // also: every thread is done with the tiles' shared memory
  if (threadIdx.x == 0) {
    __threadfence();  // the partial rows visible before the ticket
    const unsigned old = atomicAdd(&S.counters[0], (unsigned)n);
    s_last = old + (unsigned)n == (unsigned)S.nblk_pre;
    if (s_last) S.counters[0] = 0u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double* chunk = reinterpret_cast<double*>(smem);
  double* red = chunk + kPreThreads;
  prepass_finalize(S, nslots, red, chunk);
  if (threadIdx.x == 0) {
    double* sc = S.scal;
    prepass_scalars(S, red, sc, PRE_STAGE, false);
    if (atomicExch(&S.counters[6], 0u)) sc[S_STATUS] = (double)((int)sc[S_STATUS] | ST_BARRIER);
    __threadfence();
    atomicExch(&dep[4 * w.solve + QDEP_PRE], 1u);
  }
}

template <typename T, int W>
__device__ HB_STAGE_ITEM void stage_sensor_item(const SolveDev* __restrict__ solves, Work w, unsigned* dep,
                                                unsigned* abort, int stage) {
  extern __shared__ __align__(16) unsigned char smem[];
  const unsigned pre_target = stage > 0 ? 1u : 0u;
  const QueueDep d(&dep[4 * w.solve + QDEP_PRE], pre_target, nullptr, 0u, abort, &solves[w.solve].counters[6]);
  sensor_step_body<T, W>(solves, w, stage, 1, 1, smem, d);
}

// A y panel of up to 4 columns on the whole CTA.
template <typename T, int MN>
__device__ HB_STAGE_ITEM void stage_y_item(const SolveDev* __restrict__ solves, Work w, unsigned* dep,
                                           unsigned* abort, unsigned target, int stage, unsigned sh_off) {
  extern __shared__ __align__(16) unsigned char smem[];
  StageSweepShared<T>& sh = *reinterpret_cast<StageSweepShared<T>*>(smem + sh_off);
  const int s = w.solve;
  const QueueDep d(&dep[4 * s + QDEP_SEN], target, nullptr, 0u, abort, &solves[s].counters[6]);
  sweep_body<T, 1, MN>(solves, w, stage, SW_STAGE, Bind{}, smem, sh, d);
}

// Up to 4 x lines of one solve, one per group of kLineThreads threads, each
// group with its own shared memory and barrier (as the one-line CTAs of the
// x sweep kernel); target: the solve's y panels, early: its sensor tiles.
template <typename T, int MN>
__device__ HB_STAGE_ITEM void stage_x_item(const SolveDev* __restrict__ solves, Work w, unsigned* dep,
                                           unsigned* abort, unsigned target, unsigned early, int stage,
                                           unsigned sh_off, unsigned xstride) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int g = threadIdx.x / kLineThreads;
  if (g >= w.b) return;  // no line for this group (the solve's last group of rows)
  StageSweepShared<T>* shg = reinterpret_cast<StageSweepShared<T>*>(smem + sh_off) + g;
  const int s = w.solve;
  const QueueDepT<true> d(&dep[4 * s + QDEP_SWY], target, &dep[4 * s + QDEP_SEN], early, abort,
                          &solves[s].counters[6]);
  const Work line{s, w.a + g, 1, 0};
  sweep_body<T, 0, MN>(solves, line, stage, SW_STAGE, Bind{}, smem + (size_t)g * xstride, *shg, d);
}

// One stage (0, 1, 2) of the members [s0, s1) of a batch: items[0, nitems)
// (the first stage's list starts after the prepass items).  T is the bulk
// type, W the members' sensor width, MN the sweeps' nodes per thread; sh_off
// and xstride place the sweep items' shared memory (see StageSweepShared).
template <typename T, int W, int MN>
__global__ void __launch_bounds__(kStageThreads, 2)
    stage_kernel(const SolveDev* __restrict__ solves, const Work* __restrict__ tiles32,
                 const Work* __restrict__ ylist, const Work* __restrict__ xlist,
                 const QItem* __restrict__ items, int nitems, QCtl* ctl, unsigned* dep, int s0, int s1,
                 int stage, unsigned sh_off, unsigned xstride) {
  __shared__ int s_item, s_flag;
  // thread 0 takes the next ticket when an item starts and hands it over when
  // the item ends, so that the atomic's latency overlaps the item
  unsigned next = 0u;
  if (threadIdx.x == 0) next = atomicAdd(&ctl->head, 1u);
  for (;;) {
    __syncthreads();  // the previous item is done with the shared memory
    if (threadIdx.x == 0) s_item = (int)next;
    __syncthreads();
    const int t = s_item;
    if (t >= nitems) break;
    if (threadIdx.x == 0) next = atomicAdd(&ctl->head, 1u);
    const QItem it = items[t];
    if (it.kind == Q_PRE) {
      stage_pre_item<T>(solves, tiles32, it.idx, it.n, dep, stage);
      continue;
    }
    int sidx;
    if (it.kind == Q_SEN) {
      const Work w = tiles32[it.idx];
      sidx = w.solve;
      stage_sensor_item<T, W>(solves, w, dep, &ctl->abort, stage);
    } else if (it.kind == Q_SWY) {
      const Work w = ylist[it.idx];
      sidx = w.solve;
      stage_y_item<T, MN>(solves, w, dep, &ctl->abort, (unsigned)it.target, stage, sh_off);
    } else {
      const Work w = xlist[it.idx];
      sidx = w.solve;
      stage_x_item<T, MN>(solves, w, dep, &ctl->abort, (unsigned)it.target, (unsigned)it.early, stage, sh_off,
                          xstride);
    }
    // this item's writes visible before it counts as finished: the CTA's
    // barrier, then one fence (cumulative over what the barrier ordered
    // before it) and the count
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(&dep[4 * sidx + it.kind], 1u);
    }
  }
  // The last CTA to leave (every item finished) clears the queue and the
  // members' counters for the next launch.
  if (threadIdx.x == 0) {
    __threadfence();
    s_flag = atomicAdd(&ctl->exitc, 1u) == gridDim.x - 1u;
  }
  __syncthreads();
  if (s_flag) {
    __threadfence();
    for (int i = threadIdx.x; i < 4 * (s1 - s0); i += blockDim.x) dep[4 * s0 + i] = 0u;
    if (threadIdx.x == 0) {
      ctl->head = 0u;
      ctl->abort = 0u;
      ctl->exitc = 0u;
    }
  }
}

}  // namespace hitb200
