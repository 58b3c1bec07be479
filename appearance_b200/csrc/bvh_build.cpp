// Compressed 8-wide BVH build: binned-SAH binary tree, greedy collapse into
// 8-wide nodes (largest-area child opened first, down to single binary leaves
// while a node has free slots: the traversal tests all 8 slots of a node
// anyway, so a filled slot costs nothing and culls triangles at a finer
// grain), 8-bit conservative quantisation of child boxes against a per-node
// origin and power-of-two scale.  A child of at most 3 triangles that is not
// opened becomes a leaf child.
#include "bvh_build.h"

#include <algorithm>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstring>

namespace ap {

namespace {

struct Aabb {
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
  float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  void grow(const Aabb& b) {
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], b.lo[k]);
      hi[k] = std::max(hi[k], b.hi[k]);
    }
  }
  void grow_pt(const float* p) {
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], p[k]);
      hi[k] = std::max(hi[k], p[k]);
    }
  }
  double area() const {
    if (lo[0] > hi[0]) return 0.0;
    double e0 = (double)hi[0] - lo[0], e1 = (double)hi[1] - lo[1], e2 = (double)hi[2] - lo[2];
    return 2.0 * (e0 * e1 + e1 * e2 + e2 * e0);
  }
};

struct BNode {
  Aabb box;
  uint32_t left = 0, right = 0;  // children (inner)
  uint32_t first = 0, count = 0;  // leaf range in `order`
  uint32_t ntris = 0;             // triangles in subtree
  bool leaf() const { return count > 0; }
};

class BinaryBuilder {
 public:
  BinaryBuilder(const float* v, uint32_t n) : v_(v), n_(n) {}

  void build() {
    boxes_.resize(n_);
    cent_.resize(3 * (size_t)n_);
    for (uint32_t i = 0; i < n_; ++i) {
      Aabb b;
      for (int j = 0; j < 3; ++j) b.grow_pt(v_ + 9 * (size_t)i + 3 * j);
      boxes_[i] = b;
      for (int k = 0; k < 3; ++k) cent_[3 * (size_t)i + k] = 0.5f * (b.lo[k] + b.hi[k]);
    }
    order_.resize(n_);
    for (uint32_t i = 0; i < n_; ++i) order_[i] = i;
    nodes_.reserve(2 * (size_t)n_);
    nodes_.push_back(BNode{});
    struct Task { uint32_t node, first, count; };
    std::vector<Task> st;
    st.push_back({0, 0, n_});
    while (!st.empty()) {
      Task t = st.back();
      st.pop_back();
      Aabb nb, cb;
      for (uint32_t i = t.first; i < t.first + t.count; ++i) {
        nb.grow(boxes_[order_[i]]);
        cb.grow_pt(&cent_[3 * (size_t)order_[i]]);
      }
      nodes_[t.node].box = nb;
      nodes_[t.node].ntris = t.count;
      uint32_t mid = 0;
      if (t.count <= 2 || !split(t.first, t.count, nb, cb, &mid)) {
        nodes_[t.node].first = t.first;
        nodes_[t.node].count = t.count;
        continue;
      }
      uint32_t l = (uint32_t)nodes_.size();
      nodes_.push_back(BNode{});
      nodes_.push_back(BNode{});
      nodes_[t.node].left = l;
      nodes_[t.node].right = l + 1;
      st.push_back({l, t.first, mid - t.first});
      st.push_back({l + 1, mid, t.first + t.count - mid});
    }
  }

  const std::vector<BNode>& nodes() const { return nodes_; }
  const std::vector<uint32_t>& order() const { return order_; }

 private:
  // Binned SAH (16 bins per axis).  Falls back to a median split when every
  // centroid coincides; returns false only for a leaf-worthy range.
  bool split(uint32_t first, uint32_t count, const Aabb& nb, const Aabb& cb, uint32_t* mid) {
    const int B = 16;
    int best_axis = -1, best_bin = 0;
    double best = DBL_MAX;
    for (int ax = 0; ax < 3; ++ax) {
      float ext = cb.hi[ax] - cb.lo[ax];
      if (!(ext > 0.0f)) continue;
      Aabb bins[B];
      uint32_t cnt[B] = {0};
      float k = (float)B / ext;
      for (uint32_t i = first; i < first + count; ++i) {
        uint32_t p = order_[i];
        int b = std::min(B - 1, std::max(0, (int)((cent_[3 * (size_t)p + ax] - cb.lo[ax]) * k)));
        bins[b].grow(boxes_[p]);
        cnt[b]++;
      }
      double la[B];
      uint32_t lc[B];
      Aabb acc;
      uint32_t c = 0;
      for (int i = 0; i < B; ++i) {
        acc.grow(bins[i]);
        c += cnt[i];
        la[i] = acc.area();
        lc[i] = c;
      }
      acc = Aabb();
      c = 0;
      for (int i = B - 1; i > 0; --i) {
        acc.grow(bins[i]);
        c += cnt[i];
        if (lc[i - 1] == 0 || c == 0) continue;
        double cost = la[i - 1] * lc[i - 1] + acc.area() * c;
        if (cost < best) {
          best = cost;
          best_axis = ax;
          best_bin = i - 1;
        }
      }
    }
    if (best_axis < 0) {
      if (count <= 3) return false;
      *mid = first + count / 2;
      return true;
    }
    float ext = cb.hi[best_axis] - cb.lo[best_axis];
    float k = (float)B / ext;
    auto it = std::partition(order_.begin() + first, order_.begin() + first + count, [&](uint32_t p) {
      int b = std::min(B - 1, std::max(0, (int)((cent_[3 * (size_t)p + best_axis] - cb.lo[best_axis]) * k)));
      return b <= best_bin;
    });
    *mid = (uint32_t)(it - order_.begin());
    if (*mid == first || *mid == first + count) *mid = first + count / 2;
    return true;
  }

  const float* v_;
  uint32_t n_;
  std::vector<Aabb> boxes_;
  std::vector<float> cent_;
  std::vector<uint32_t> order_;
  std::vector<BNode> nodes_;
};

struct Collapser {
  const std::vector<BNode>& bn;
  const std::vector<uint32_t>& order;
  const float* verts;
  WideBvh* out;

  void collect_tris(uint32_t b, std::vector<uint32_t>& tris) const {
    const BNode& n = bn[b];
    if (n.leaf()) {
      for (uint32_t i = 0; i < n.count; ++i) tris.push_back(order[n.first + i]);
      return;
    }
    collect_tris(n.left, tris);
    collect_tris(n.right, tris);
  }

  static void quantize_axis(float lo, float hi, float* p, uint8_t* e) {
    *p = lo;
    double ext = (double)hi - (double)lo;
    int ex = -120;
    if (ext > 0.0) ex = (int)std::ceil(std::log2(ext / 255.0));
    ex = std::max(-126, std::min(127, ex));
    *e = (uint8_t)(ex + 127);
  }

  // Fills wide node `wi` from binary node `b`; returns the worst-case stack
  // need of its subtree and the subtree depth.
  void emit(uint32_t wi, uint32_t b, uint32_t depth, uint32_t* stack_need) {
    std::vector<uint32_t> kids;
    const BNode& root = bn[b];
    if (root.leaf()) {
      kids.push_back(b);
    } else {
      kids.push_back(root.left);
      kids.push_back(root.right);
      while (kids.size() < 8) {
        int pick = -1;
        double best = -1.0;
        for (size_t i = 0; i < kids.size(); ++i) {
          const BNode& c = bn[kids[i]];
          if (c.leaf()) continue;  // small subtrees split too while slots are free
          double a = c.box.area();
          if (a > best) { best = a; pick = (int)i; }
        }
        if (pick < 0) break;
        uint32_t c = kids[pick];
        kids[pick] = bn[c].left;
        kids.push_back(bn[c].right);
      }
    }
    Aabb nb;
    for (uint32_t k : kids) nb.grow(bn[k].box);
    float p[3];
    uint8_t e[3];
    for (int ax = 0; ax < 3; ++ax) quantize_axis(nb.lo[ax], nb.hi[ax], &p[ax], &e[ax]);

    uint8_t meta[8] = {0}, qlo[3][8] = {{0}}, qhi[3][8] = {{0}};
    uint8_t imask = 0;
    std::vector<uint32_t> inner;
    uint32_t tri_base = (uint32_t)out->tris.size();
    uint32_t tri_off = 0;
    for (size_t s = 0; s < kids.size(); ++s) {
      const BNode& c = bn[kids[s]];
      for (int ax = 0; ax < 3; ++ax) {
        double scale = std::ldexp(1.0, (int)e[ax] - 127);
        double ql = std::floor(((double)c.box.lo[ax] - (double)p[ax]) / scale);
        double qh = std::ceil(((double)c.box.hi[ax] - (double)p[ax]) / scale);
        qlo[ax][s] = (uint8_t)std::max(0.0, std::min(255.0, ql));
        qhi[ax][s] = (uint8_t)std::max(0.0, std::min(255.0, qh));
      }
      if (c.leaf() || c.ntris <= 3) {
        std::vector<uint32_t> tris;
        collect_tris(kids[s], tris);
        uint32_t cnt = (uint32_t)tris.size();
        meta[s] = (uint8_t)((((1u << cnt) - 1u) << 5) | tri_off);
        for (uint32_t g : tris) {
          TriRec r;
          const float* v = verts + 9 * (size_t)g;
          r.v[0] = v[0]; r.v[1] = v[1]; r.v[2] = v[2];
          std::memcpy(&r.v[3], &g, 4);
          r.v[4] = v[3]; r.v[5] = v[4]; r.v[6] = v[5]; r.v[7] = 0.0f;
          r.v[8] = v[6]; r.v[9] = v[7]; r.v[10] = v[8]; r.v[11] = 0.0f;
          out->tris.push_back(r);
        }
        tri_off += cnt;
      } else {
        meta[s] = (uint8_t)(0x10u | (uint32_t)inner.size());
        imask |= (uint8_t)(1u << s);
        inner.push_back(kids[s]);
      }
    }
    uint32_t child_base = (uint32_t)out->nodes.size();
    out->nodes.resize(out->nodes.size() + inner.size());
    WideNode& n = out->nodes[wi];
    std::memset(&n, 0, sizeof(n));
    std::memcpy(&n.w[0], &p[0], 4);
    std::memcpy(&n.w[1], &p[1], 4);
    std::memcpy(&n.w[2], &p[2], 4);
    n.w[3] = (uint32_t)e[0] | ((uint32_t)e[1] << 8) | ((uint32_t)e[2] << 16) | ((uint32_t)imask << 24);
    n.w[4] = child_base;
    n.w[5] = tri_base;
    std::memcpy(&n.w[6], meta, 8);
    std::memcpy(&n.w[8], qlo[0], 8);
    std::memcpy(&n.w[10], qlo[1], 8);
    std::memcpy(&n.w[12], qlo[2], 8);
    std::memcpy(&n.w[14], qhi[0], 8);
    std::memcpy(&n.w[16], qhi[1], 8);
    std::memcpy(&n.w[18], qhi[2], 8);
    out->stats.max_depth = std::max(out->stats.max_depth, depth + 1);
    uint32_t need_child = 0;
    for (size_t k = 0; k < inner.size(); ++k) {
      uint32_t sn = 0;
      emit(child_base + (uint32_t)k, inner[k], depth + 1, &sn);
      need_child = std::max(need_child, sn);
    }
    *stack_need = (inner.empty() ? 0u : (uint32_t)inner.size() - 1u) + need_child;
  }
};

}  // namespace

bool build_wide_bvh(const float* tri_verts, uint32_t num_tris, uint32_t max_stack, WideBvh* out,
                    std::string* err) {
  auto t0 = std::chrono::steady_clock::now();
  out->nodes.clear();
  out->tris.clear();
  out->stats = BvhStats{};
  if (num_tris == 0) {
    // an empty scene: one node without children
    out->nodes.resize(1);
    std::memset(&out->nodes[0], 0, sizeof(WideNode));
    out->nodes[0].w[3] = 127u | (127u << 8) | (127u << 16);
    out->stats.num_nodes = 1;
    return true;
  }
  BinaryBuilder bb(tri_verts, num_tris);
  bb.build();
  out->nodes.resize(1);
  out->tris.reserve(num_tris);
  Collapser c{bb.nodes(), bb.order(), tri_verts, out};
  uint32_t need = 0;
  c.emit(0, 0, 0, &need);
  out->stats.num_nodes = (uint32_t)out->nodes.size();
  out->stats.num_tris = (uint32_t)out->tris.size();
  out->stats.max_stack = need;
  out->stats.build_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (need > max_stack) {
    if (err) *err = "BVH needs " + std::to_string(need) + " traversal stack entries, limit " +
                    std::to_string(max_stack);
    return false;
  }
  return true;
}

}  // namespace ap
