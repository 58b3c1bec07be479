// Oracle (test infrastructure only): binned-SAH binary BVH over the flattened
// world-space triangles.  Its result does not depend on the tree: closest hit
// is the minimum of (t, global triangle id) over all triangles that pass the
// watertight test, and the box test is widened so no such triangle is culled.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "oracle_scene.h"

namespace orc {

namespace {

struct Box {
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
  float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  void grow(const float* p) {
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], p[k]);
      hi[k] = std::max(hi[k], p[k]);
    }
  }
  void grow(const Box& b) {
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], b.lo[k]);
      hi[k] = std::max(hi[k], b.hi[k]);
    }
  }
  float area() const {
    float e0 = hi[0] - lo[0], e1 = hi[1] - lo[1], e2 = hi[2] - lo[2];
    if (e0 < 0) return 0.0f;
    return 2.0f * (e0 * e1 + e1 * e2 + e2 * e0);
  }
};

}  // namespace

void OracleBvh::build(const Scene& s) {
  const uint32_t n = s.num_tris();
  std::vector<Box> tb(n);
  std::vector<float> cen(3 * (size_t)n);
  for (uint32_t i = 0; i < n; ++i) {
    V3 a, b, c;
    s.tri_verts(i, a, b, c);
    float pa[3] = {a.x, a.y, a.z}, pb[3] = {b.x, b.y, b.z}, pc[3] = {c.x, c.y, c.z};
    tb[i].grow(pa);
    tb[i].grow(pb);
    tb[i].grow(pc);
    for (int k = 0; k < 3; ++k) cen[3 * (size_t)i + k] = 0.5f * (tb[i].lo[k] + tb[i].hi[k]);
  }
  order_.resize(n);
  for (uint32_t i = 0; i < n; ++i) order_[i] = i;
  nodes_.clear();
  nodes_.reserve(2 * (size_t)n + 1);
  struct Task { uint32_t node, first, count; };
  std::vector<Task> stack;
  nodes_.push_back(Node{});
  stack.push_back({0, 0, n});
  const int BINS = 16;
  while (!stack.empty()) {
    Task t = stack.back();
    stack.pop_back();
    Box nb, cb;
    for (uint32_t i = t.first; i < t.first + t.count; ++i) {
      nb.grow(tb[order_[i]]);
      cb.grow(&cen[3 * (size_t)order_[i]]);
    }
    Node& node = nodes_[t.node];
    for (int k = 0; k < 3; ++k) { node.lo[k] = nb.lo[k]; node.hi[k] = nb.hi[k]; }
    if (t.count <= 4) {
      node.left_or_first = t.first;
      node.count = t.count;
      continue;
    }
    int best_axis = -1, best_split = 0;
    float best_cost = FLT_MAX;
    for (int ax = 0; ax < 3; ++ax) {
      float ext = cb.hi[ax] - cb.lo[ax];
      if (!(ext > 0.0f)) continue;
      Box bins[BINS];
      uint32_t cnt[BINS] = {0};
      for (uint32_t i = t.first; i < t.first + t.count; ++i) {
        uint32_t p = order_[i];
        int b = (int)((cen[3 * (size_t)p + ax] - cb.lo[ax]) / ext * BINS);
        b = std::min(std::max(b, 0), BINS - 1);
        bins[b].grow(tb[p]);
        cnt[b]++;
      }
      float la[BINS], ra[BINS];
      uint32_t lc[BINS], rc[BINS];
      Box acc;
      uint32_t c = 0;
      for (int i = 0; i < BINS; ++i) {
        acc.grow(bins[i]);
        c += cnt[i];
        la[i] = acc.area();
        lc[i] = c;
      }
      acc = Box();
      c = 0;
      for (int i = BINS - 1; i >= 0; --i) {
        acc.grow(bins[i]);
        c += cnt[i];
        ra[i] = acc.area();
        rc[i] = c;
      }
      for (int i = 0; i < BINS - 1; ++i) {
        if (lc[i] == 0 || rc[i + 1] == 0) continue;
        float cost = la[i] * lc[i] + ra[i + 1] * rc[i + 1];
        if (cost < best_cost) { best_cost = cost; best_axis = ax; best_split = i; }
      }
    }
    uint32_t mid;
    if (best_axis < 0) {
      mid = t.first + t.count / 2;
    } else {
      float ext = cb.hi[best_axis] - cb.lo[best_axis];
      auto it = std::partition(order_.begin() + t.first, order_.begin() + t.first + t.count,
                               [&](uint32_t p) {
                                 int b = (int)((cen[3 * (size_t)p + best_axis] - cb.lo[best_axis]) /
                                               ext * BINS);
                                 b = std::min(std::max(b, 0), BINS - 1);
                                 return b <= best_split;
                               });
      mid = (uint32_t)(it - order_.begin());
      if (mid == t.first || mid == t.first + t.count) mid = t.first + t.count / 2;
    }
    uint32_t left = (uint32_t)nodes_.size();
    nodes_[t.node].left_or_first = left;
    nodes_[t.node].count = 0;
    nodes_.push_back(Node{});
    nodes_.push_back(Node{});
    stack.push_back({left, t.first, mid - t.first});
    stack.push_back({left + 1, mid, t.first + t.count - mid});
  }
}

namespace {
// Slab test in double, widened per slab by 2^-19 of the distance scale of the
// box from the origin (|lo - o| + |hi - o|) / |d| and by a relative 1e-6, so that
// every triangle that the watertight test accepts inside [tmin, tmax] (whose
// inside test rounds at the scale of the vertex distances) lies in an accepted box.
inline bool box_hit(const float* lo, const float* hi, const double* o, const double* inv,
                    double tmin, double tmax) {
  double t0 = tmin, t1 = tmax;
  for (int k = 0; k < 3; ++k) {
    double a = (lo[k] - o[k]) * inv[k];
    double b = (hi[k] - o[k]) * inv[k];
    if (a > b) std::swap(a, b);
    if (std::isnan(a) || std::isnan(b)) continue;  // ray parallel and on a slab plane
    double slack = (std::fabs(a) + std::fabs(b)) * 1.9073486328125e-06 + 1e-12;
    if (std::isinf(slack)) continue;
    a = a - 1e-6 * std::fabs(a) - slack;
    b = b + 1e-6 * std::fabs(b) + slack;
    t0 = std::max(t0, a);
    t1 = std::min(t1, b);
  }
  return t0 <= t1;
}
}  // namespace

Hit OracleBvh::closest(const Scene& s, V3 o, V3 d, float tmin, float tmax, uint64_t* nodes_visited,
                       uint64_t* tris_tested) const {
  Hit best{tmax, 0.0f, 0.0f, 0xFFFFFFFFu};
  if (nodes_.empty()) return best;
  RayPre rp = ray_pre(o, d);
  double od[3] = {o.x, o.y, o.z};
  double inv[3] = {1.0 / (double)d.x, 1.0 / (double)d.y, 1.0 / (double)d.z};
  uint32_t stack[128];
  int sp = 0;
  stack[sp++] = 0;
  while (sp) {
    const Node& nd = nodes_[stack[--sp]];
    if (nodes_visited) ++*nodes_visited;
    if (!box_hit(nd.lo, nd.hi, od, inv, tmin, best.t)) continue;
    if (nd.count) {
      for (uint32_t i = 0; i < nd.count; ++i) {
        uint32_t g = order_[nd.left_or_first + i];
        V3 a, b, c;
        s.tri_verts(g, a, b, c);
        if (tris_tested) ++*tris_tested;
        float t, u, v;
        if (intersect_tri(rp, a, b, c, tmin, best.t, t, u, v)) {
          if (t < best.t || (t == best.t && g < best.tri)) best = Hit{t, u, v, g};
        }
      }
    } else {
      stack[sp++] = nd.left_or_first;
      stack[sp++] = nd.left_or_first + 1;
    }
  }
  return best;
}

bool OracleBvh::any(const Scene& s, V3 o, V3 d, float tmin, float tmax) const {
  if (nodes_.empty()) return false;
  RayPre rp = ray_pre(o, d);
  double od[3] = {o.x, o.y, o.z};
  double inv[3] = {1.0 / (double)d.x, 1.0 / (double)d.y, 1.0 / (double)d.z};
  uint32_t stack[128];
  int sp = 0;
  stack[sp++] = 0;
  while (sp) {
    const Node& nd = nodes_[stack[--sp]];
    if (!box_hit(nd.lo, nd.hi, od, inv, tmin, tmax)) continue;
    if (nd.count) {
      for (uint32_t i = 0; i < nd.count; ++i) {
        V3 a, b, c;
        s.tri_verts(order_[nd.left_or_first + i], a, b, c);
        float t, u, v;
        if (intersect_tri(rp, a, b, c, tmin, tmax, t, u, v)) return true;
      }
    } else {
      stack[sp++] = nd.left_or_first;
      stack[sp++] = nd.left_or_first + 1;
    }
  }
  return false;
}

}  // namespace orc
