// Persistent traversal kernels' work loop, shared by the frame (frame.cu) and
// the spectral mode (spectral.cu).
#pragma once

#include "traverse.cuh"

namespace ap {

APD uint32_t lane_id() {
  uint32_t l;
  asm volatile("mov.u32 %0, %%laneid;" : "=r"(l));
  return l;
}

// Persistent traversal with per-lane refill: a lane that finishes its ray
// takes the next one through a warp-aggregated atomic on `cursor`, so warps
// stay full until the batch drains.  Lanes check for a refill every
// kStepBudget steps.  load(i, o, d, tmax) fetches ray i, store(i, trav,
// visits) writes its result.  The traversal kernels run with the child tests
// unrolled and are register-capped for kTraceMinBlocks resident blocks of
// kBlock threads per SM.  Measured on the 1080p benchmark frame with the packed
// box test (CUDA events, frame time): 5, 6, 7, 8 blocks with an 8-step refill
// 42.9, 41.1, 39.8, 39.6 ms; 7 blocks with 6 and 10 steps 39.6, 40.2 ms; 8
// blocks with 6 steps 39.3-39.5 ms.
#ifndef AP_TRACE_MIN_BLOCKS
#define AP_TRACE_MIN_BLOCKS 8
#endif
#ifndef AP_STEP_BUDGET
#define AP_STEP_BUDGET 6
#endif
constexpr int kStepBudget = AP_STEP_BUDGET;
constexpr int kTraceMinBlocks = AP_TRACE_MIN_BLOCKS;

template <bool kAny, bool kCount, class Load, class Store>
APD void persistent_trace(const DevScene& s, uint32_t count, uint32_t* cursor, Load load, Store store) {
  if (count == 0) return;  // an empty queue: no warp needs the cursor
  const uint32_t lane = lane_id();
  uint2 stack[kTraversalStack];
  Trav t;
  Visits vc;
  uint32_t cur = 0;
  bool active = false, exhausted = false;
  while (true) {
    if (!exhausted) {
      const unsigned need = __ballot_sync(0xffffffffu, !active);
      if (need) {
        const int leader = __ffs(need) - 1;
        uint32_t base = 0;
        if ((int)lane == leader) base = atomicAdd(cursor, (uint32_t)__popc(need));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (base + (uint32_t)__popc(need) >= count) exhausted = true;
        if (!active) {
          const uint32_t idx = base + __popc(need & ((1u << lane) - 1u));
          if (idx < count) {
            float3 o, d;
            float tmax;
            load(idx, o, d, tmax);
            trav_init(t, o, d, tmax);
            vc = Visits();
            cur = idx;
            active = true;
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) break;
    if (active && trav_step<kAny, kCount, true>(s, t, stack, kStepBudget, &vc)) {
      store(cur, t, vc);
      active = false;
    }
  }
}

// persistent_trace over the rays of several independent jobs at once (a
// batch of frames sharing one launch): the combined index range is split by
// the jobs' first indices start[0..nj] (start[nj] = count); a lane that takes
// ray i traces it through its own job's BVH.  load(job, i, o, d, tmax) and
// store(job, i, trav) get the job and the ray's index within it.
template <bool kAny, class Load, class Store>
APD void persistent_trace_batch(const BvhView* bvh, int nj, const uint32_t* start, uint32_t count, uint32_t* cursor,
                                Load load, Store store) {
  if (count == 0) return;  // an empty queue: no warp needs the cursor
  const uint32_t lane = lane_id();
  uint2 stack[kTraversalStack];
  Trav t;
  Visits vc;
  BvhView view{nullptr, nullptr};
  uint32_t cur = 0;
  int job = 0;
  bool active = false, exhausted = false;
  while (true) {
    if (!exhausted) {
      const unsigned need = __ballot_sync(0xffffffffu, !active);
      if (need) {
        const int leader = __ffs(need) - 1;
        uint32_t base = 0;
        if ((int)lane == leader) base = atomicAdd(cursor, (uint32_t)__popc(need));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (base + (uint32_t)__popc(need) >= count) exhausted = true;
        if (!active) {
          const uint32_t idx = base + __popc(need & ((1u << lane) - 1u));
          if (idx < count) {
            job = 0;
            while (job + 1 < nj && idx >= start[job + 1]) ++job;
            cur = idx - start[job];
            view = bvh[job];
            float3 o, d;
            float tmax;
            load(job, cur, o, d, tmax);
            trav_init(t, o, d, tmax);
            active = true;
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) break;
    if (active && trav_step<kAny, false, true>(view, t, stack, kStepBudget, &vc)) {
      store(job, cur, t);
      active = false;
    }
  }
}

}  // namespace ap
