// Two-level traversal: a top-level wide BVH (TLAS) over instances, each an
// object-space wide BVH (BLAS) of its model under a 3x4 transform, as the
// reference's scenes are built (TLAS of BLAS instances, TlasInstance with a
// 4x3 transform, crates/appearance-path-tracer-gpu/src/scene_resources/
// mod.rs:159-276).
//
// A ray reaching an instance leaf continues in that instance's BLAS with its
// origin and direction mapped to object space (the direction is not
// renormalised, so a distance t means the same point in both spaces); when
// the BLAS is done the world-space ray resumes the TLAS.  Both levels share
// one stack: BLAS entries sit above the height at which the BLAS was entered.
// A hit's global triangle id is the instance's first id plus the model's
// triangle index, and the closest hit is the minimum of (t, id) over every
// triangle the watertight test accepts in object space, so the traversal
// order does not change it.  Box tests are those of the one-level traversal
// (conservative in any space); the TLAS boxes are the transformed model
// bounds, widened at build time.
#pragma once

#include "persistent.cuh"
#include "traverse.cuh"

namespace ap {

// The two-level part of a scene (DevScene holds the BLAS pool in nodes / tris,
// whose triangle records carry the model-local triangle index).
struct TwoLevel {
  const uint4* tlas_nodes;    // 5 per WideNode
  const float4* tlas_leaves;  // 3 per leaf record (TriRec layout), v0.w = instance index
  const InstRec* insts;
  uint32_t num_insts;
};

struct Trav2 {
  Trav t;                 // the current level's state (ray in that level's space)
  float3 wo, wd;          // world-space ray
  uint32_t inst_base, inst_mask;  // pending instance leaves of the current TLAS node
  uint32_t tri_base_id;   // first global triangle id of the current instance
  int sp0;                // stack height at BLAS entry
  bool blas;              // traversing a BLAS
};

APD void trav2_init(Trav2& t, float3 o, float3 d, float tmax) {
  trav_init(t.t, o, d, tmax);
  t.wo = o;
  t.wd = d;
  t.inst_base = 0;
  t.inst_mask = 0;
  t.tri_base_id = 0;
  t.sp0 = 0;
  t.blas = false;
}

// Object-space ray of instance `in`: w2o (row-major 3x4) times (o, 1) and
// times (d, 0), each row summed left to right.
APD void to_object(const InstRec& in, float3 o, float3 d, float3* oo, float3* od) {
  const float* m = in.w2o;
  *oo = f3(m[0] * o.x + m[1] * o.y + m[2] * o.z + m[3], m[4] * o.x + m[5] * o.y + m[6] * o.z + m[7],
           m[8] * o.x + m[9] * o.y + m[10] * o.z + m[11]);
  *od = f3(m[0] * d.x + m[1] * d.y + m[2] * d.z, m[4] * d.x + m[5] * d.y + m[6] * d.z,
           m[8] * d.x + m[9] * d.y + m[10] * d.z);
}

// One node of either level: child boxes against the current ray, nearest
// inner child next, the others pushed; leaf children become a pending mask
// at *leaf_base.
template <bool kAny>
APD void visit_node2(const uint4* nodes, Trav& t, uint2* stack, uint32_t* leaf_base, uint32_t* leaf_mask) {
  const uint4* np = nodes + 5 * (size_t)t.node;
  const uint4 w0 = __ldg(np + 0), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3), w4 = __ldg(np + 4);
  const float range_grown = (kAny ? t.tmax : t.hit.t) * kGrow;
  uint32_t mask = 0;
  float best_t = __uint_as_float(0x7f800000u);
  uint32_t best_node = 0;
  t.have = false;
  float tns[8];
  child_entries(w0, w2, w3, w4, t.r, 0.0f, range_grown, tns);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const uint32_t meta = meta_of(w1, i);
    if (meta == 0u) continue;
    const float tn = tns[i];
    if (!(tn < __uint_as_float(0x7f800000u))) continue;
    if (meta & 0xe0u) {
      mask |= (meta >> 5) << (meta & 0x1fu);
    } else {
      const uint32_t child = w1.x + (meta & 7u);
      if (tn < best_t) {
        if (t.have && t.sp < kTraversalStack) stack[t.sp++] = make_uint2(best_node, __float_as_uint(best_t));
        best_t = tn;
        best_node = child;
        t.have = true;
      } else if (t.sp < kTraversalStack) {
        stack[t.sp++] = make_uint2(child, __float_as_uint(tn));
      }
    }
  }
  t.node = best_node;
  t.node_t = best_t;
  *leaf_base = w1.y;
  *leaf_mask = mask;
}

// Runs up to `budget` steps (a node of either level, one triangle, or one
// instance entry); returns true when the ray is finished.  Both levels' node
// visits go through one call site (the level picks the node array and where
// the leaf mask goes), so lanes of a warp at different levels share it.
template <bool kAny, bool kCount>
APD bool trav2_step(const DevScene& s, const TwoLevel& tl, Trav2& q, uint2* stack, int budget, Visits* vc) {
  Trav& t = q.t;
  for (int step = 0; step < budget; ++step) {
    if (q.blas && t.tri_mask) {
      const int j = __ffs(t.tri_mask) - 1;
      t.tri_mask &= t.tri_mask - 1;
      if (kCount) vc->tris++;
      const float4* tp = s.tris + 3 * (size_t)(t.tri_base + j);
      const float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
      float th, u, v;
      const float lim = kAny ? t.tmax : t.hit.t;
      if (intersect_tri(t.r, f3(a.x, a.y, a.z), f3(b.x, b.y, b.z), f3(c.x, c.y, c.z), 0.0f, lim, th, u, v)) {
        const uint32_t gid = q.tri_base_id + __float_as_uint(a.w);
        if (kAny) {
          t.hit.tri = gid;
          return true;
        }
        if (th < t.hit.t || gid < t.hit.tri) {
          t.hit.t = th;
          t.hit.u = u;
          t.hit.v = v;
          t.hit.tri = gid;
        }
      }
      continue;
    }
    if (!q.blas && q.inst_mask) {  // enter the next pending instance
      const int j = __ffs(q.inst_mask) - 1;
      q.inst_mask &= q.inst_mask - 1;
      const uint32_t ii = __float_as_uint(__ldg(tl.tlas_leaves + 3 * (size_t)(q.inst_base + j)).w);
      const InstRec& in = tl.insts[ii];
      // the TLAS node to visit next waits on the stack below the BLAS
      if (t.have && t.sp < kTraversalStack) stack[t.sp++] = make_uint2(t.node, __float_as_uint(t.node_t));
      float3 oo, od;
      to_object(in, q.wo, q.wd, &oo, &od);
      t.r = ray_pre(oo, od);
      q.tri_base_id = in.tri_base;
      q.sp0 = t.sp;
      q.blas = true;
      t.node = in.blas_root;
      t.node_t = 0.0f;
      t.have = true;
      t.tri_mask = 0;
      continue;
    }
    // a node of the current level
    if (t.have && !kAny && t.node_t > t.hit.t * kGrow) t.have = false;
    if (!t.have) {
      const int floor = q.blas ? q.sp0 : 0;
      bool got = false;
      while (t.sp > floor) {
        const uint2 e = stack[--t.sp];
        if (kAny || __uint_as_float(e.y) <= t.hit.t * kGrow) {
          t.node = e.x;
          got = true;
          break;
        }
      }
      if (!got) {
        if (!q.blas) return true;
        q.blas = false;  // this instance is done: back to the world-space ray
        t.r = ray_pre(q.wo, q.wd);
        continue;
      }
    }
    if (kCount) vc->nodes++;
    uint32_t base, mask;
    visit_node2<kAny>(q.blas ? s.nodes : tl.tlas_nodes, t, stack, &base, &mask);
    if (q.blas) {
      t.tri_base = base;
      t.tri_mask = mask;
    } else {
      q.inst_base = base;
      q.inst_mask = mask;
    }
  }
  return false;
}

// persistent_trace (persistent.cuh) over the two-level scene.
template <bool kAny, bool kCount, class Load, class Store>
APD void persistent_trace2(const DevScene& s, const TwoLevel& tl, uint32_t count, uint32_t* cursor, Load load,
                           Store store) {
  if (count == 0) return;  // an empty queue: no warp needs the cursor
  const uint32_t lane = lane_id();
  uint2 stack[kTraversalStack];
  Trav2 t;
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
            trav2_init(t, o, d, tmax);
            vc = Visits();
            cur = idx;
            active = true;
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) break;
    if (active && trav2_step<kAny, kCount>(s, tl, t, stack, kStepBudget, &vc)) {
      store(cur, t.t, vc);
      active = false;
    }
  }
}

}  // namespace ap
