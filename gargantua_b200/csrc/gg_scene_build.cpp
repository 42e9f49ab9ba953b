// gg_scene_build.cpp -- the scene of gg_set_scene on the host: primitive
// checks, the materials' one-sample shading resolved to a fixed rule, and the
// bounding-volume hierarchy the trace kernel walks.
//
// The hierarchy is built like the reference's BvhNode::build
// (crates/raytracer/src/accel/bvh.rs:26-160): objects sorted by bounding-box
// centre along the longest axis of their union, split where the
// surface-area cost (traversal 1 + intersection 1 per object, weighted by
// child over parent box area) is lowest.  Leaves hold up to kLeafMax objects
// (the nearest hit does not depend on the tree's shape), children of an
// inner node sit next to each other, and beyond depth kSahDepth the split
// is the median, so the depth stays below the kernel's traversal stack.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/gargantua_gpu.h"
#include "gg_params.h"
#include "gg_scene_host.h"

namespace gg {

namespace {

constexpr int kLeafMax = 2;
constexpr int kSahDepth = 32;
constexpr uint32_t kMaxPrims = 1u << 20;  // median splits then add at most 20 levels

struct Item {
  double lo[3], hi[3], mid[3];
  int prim;
};

bool finite3(const double* a) {
  return std::isfinite(a[0]) && std::isfinite(a[1]) && std::isfinite(a[2]);
}

double area(const double lo[3], const double hi[3]) {
  const double dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
  return 2.0 * (dx * dy + dy * dz + dz * dx);
}

void grow(double lo[3], double hi[3], const Item& it) {
  for (int a = 0; a < 3; ++a) {
    lo[a] = std::min(lo[a], it.lo[a]);
    hi[a] = std::max(hi[a], it.hi[a]);
  }
}

struct Builder {
  std::vector<Item>& items;
  std::vector<SceneNode>& nodes;
  int max_depth = 0;

  // Fills nodes[self] for items [b, e).
  void build(int self, int b, int e, int depth) {
    max_depth = std::max(max_depth, depth);
    SceneNode& N = nodes[self];
    for (int a = 0; a < 3; ++a) {
      N.lo[a] = INFINITY;
      N.hi[a] = -INFINITY;
    }
    for (int i = b; i < e; ++i) grow(N.lo, N.hi, items[i]);
    const int n = e - b;
    if (n <= kLeafMax) {
      N.first = b;
      N.count = n;
      return;
    }
    int axis = 0;
    double ext = -1.0;
    for (int a = 0; a < 3; ++a) {
      if (N.hi[a] - N.lo[a] > ext) {
        ext = N.hi[a] - N.lo[a];
        axis = a;
      }
    }
    std::stable_sort(items.begin() + b, items.begin() + e,
                     [axis](const Item& x, const Item& y) { return x.mid[axis] < y.mid[axis]; });
    int split = b + n / 2;
    if (depth < kSahDepth) {
      // prefix boxes from the left, suffix boxes swept from the right
      std::vector<double> left_area(n);
      double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (int i = 0; i < n; ++i) {
        grow(lo, hi, items[b + i]);
        left_area[i] = area(lo, hi);
      }
      const double parent = area(N.lo, N.hi);
      double rlo[3] = {INFINITY, INFINITY, INFINITY}, rhi[3] = {-INFINITY, -INFINITY, -INFINITY};
      double best = INFINITY;
      for (int i = n - 1; i >= 1; --i) {
        grow(rlo, rhi, items[b + i]);
        const double cost =
            parent > 0.0 ? 1.0 + (left_area[i - 1] * i + area(rlo, rhi) * (n - i)) / parent
                         : (double)n;
        if (cost < best) {
          best = cost;
          split = b + i;
        }
      }
    }
    const int kids = (int)nodes.size();
    nodes.resize(nodes.size() + 2);
    nodes[self].first = kids;
    nodes[self].count = 0;
    build(kids, b, split, depth + 1);
    build(kids + 1, split, e, depth + 1);
  }
};

// Every node's box holds its children's boxes and its objects' boxes, and
// every object sits in exactly one leaf.
bool consistent(const std::vector<SceneNode>& nodes, const std::vector<Item>& items) {
  std::vector<int> seen(items.size(), 0);
  std::vector<int> todo{0};
  auto inside = [](const double lo[3], const double hi[3], const double* plo, const double* phi) {
    for (int a = 0; a < 3; ++a)
      if (lo[a] < plo[a] || hi[a] > phi[a]) return false;
    return true;
  };
  while (!todo.empty()) {
    const SceneNode& N = nodes[todo.back()];
    todo.pop_back();
    if (N.count > 0) {
      for (int i = N.first; i < N.first + N.count; ++i) {
        if (i < 0 || i >= (int)items.size() || !inside(items[i].lo, items[i].hi, N.lo, N.hi))
          return false;
        seen[i] += 1;
      }
    } else {
      if (N.first < 1 || N.first + 1 >= (int)nodes.size()) return false;
      for (int k = 0; k < 2; ++k) {
        const SceneNode& C = nodes[N.first + k];
        if (!inside(C.lo, C.hi, N.lo, N.hi)) return false;
        todo.push_back(N.first + k);
      }
    }
  }
  for (int s : seen)
    if (s != 1) return false;
  return true;
}

}  // namespace

int build_scene(const gg_prim_t* prims, uint32_t n, std::vector<ScenePrim>* out_prims,
                std::vector<SceneNode>* out_nodes, uint32_t* depth) {
  if (!prims || n == 0) return GG_ERR_INVALID_ARG;
  if (n > kMaxPrims) return GG_ERR_INVALID_ARG;
  std::vector<ScenePrim> ps(n);
  std::vector<Item> items(n);
  for (uint32_t k = 0; k < n; ++k) {
    const gg_prim_t& s = prims[k];
    ScenePrim& p = ps[k];
    std::memset(&p, 0, sizeof(p));
    if (!finite3(s.p) || !finite3(s.color)) return GG_ERR_INVALID_ARG;
    switch (s.material) {
      case GG_MAT_LAMBERTIAN:  // lambertian.rs:42-56: scatters with its albedo
        p.shade = kShadeAlbedo;
        for (int c = 0; c < 3; ++c) p.albedo[c] = s.color[c];
        break;
      case GG_MAT_DIFFUSE_LIGHT:  // diffuse_light.rs:22-35: no scatter, emits
        p.shade = kShadeEmit;
        for (int c = 0; c < 3; ++c) p.emit[c] = s.color[c];
        break;
      case GG_MAT_METAL:  // metal.rs:40-57
        if (s.fuzz != 0.0) return GG_ERR_UNSUPPORTED;  // a random direction decides
        p.shade = kShadeMirror;
        for (int c = 0; c < 3; ++c) p.albedo[c] = s.color[c];
        break;
      case GG_MAT_DIELECTRIC:  // dielectric.rs:65-95: always scatters, white
        if (!(std::isfinite(s.ior) && s.ior > 0.0)) return GG_ERR_INVALID_ARG;
        p.shade = kShadeAlbedo;
        for (int c = 0; c < 3; ++c) p.albedo[c] = 1.0;
        break;
      default:
        return GG_ERR_INVALID_ARG;
    }
    Item& it = items[k];
    it.prim = (int)k;
    for (int a = 0; a < 3; ++a) p.c[a] = s.p[a];
    if (s.kind == GG_PRIM_SPHERE) {
      if (!(std::isfinite(s.radius) && s.radius > 0.0)) return GG_ERR_INVALID_ARG;
      p.kind = kPrimSphere;
      p.radius = s.radius;
      for (int a = 0; a < 3; ++a) {  // sphere.rs:17-27
        it.lo[a] = s.p[a] - s.radius;
        it.hi[a] = s.p[a] + s.radius;
      }
    } else if (s.kind == GG_PRIM_QUAD) {
      if (!finite3(s.u) || !finite3(s.v)) return GG_ERR_INVALID_ARG;
      p.kind = kPrimQuad;
      // Quad::with_arc_material (quad.rs:36-79): n = u x v, normal = n/|n|,
      // D = normal . Q, w = n / (n . n), e_alpha = v x w, e_beta = w x u
      const double* u = s.u;
      const double* v = s.v;
      const double nn[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2],
                            u[0] * v[1] - u[1] * v[0]};
      const double n2 = nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2];
      if (!(n2 > 0.0) || !std::isfinite(n2)) return GG_ERR_INVALID_ARG;  // degenerate
      const double len = std::sqrt(n2);
      for (int a = 0; a < 3; ++a) p.n[a] = nn[a] / len;
      p.d = p.n[0] * s.p[0] + p.n[1] * s.p[1] + p.n[2] * s.p[2];
      const double w[3] = {nn[0] / n2, nn[1] / n2, nn[2] / n2};
      p.ea[0] = v[1] * w[2] - v[2] * w[1];
      p.ea[1] = v[2] * w[0] - v[0] * w[2];
      p.ea[2] = v[0] * w[1] - v[1] * w[0];
      p.eb[0] = w[1] * u[2] - w[2] * u[1];
      p.eb[1] = w[2] * u[0] - w[0] * u[2];
      p.eb[2] = w[0] * u[1] - w[1] * u[0];
      for (int a = 0; a < 3; ++a) {  // the four corners, padded by 1e-4
        const double c0 = s.p[a], c1 = s.p[a] + u[a], c2 = s.p[a] + v[a],
                     c3 = s.p[a] + u[a] + v[a];
        it.lo[a] = std::min(std::min(c0, c1), std::min(c2, c3)) - 1e-4;
        it.hi[a] = std::max(std::max(c0, c1), std::max(c2, c3)) + 1e-4;
      }
    } else {
      return GG_ERR_INVALID_ARG;
    }
    for (int a = 0; a < 3; ++a) it.mid[a] = 0.5 * (it.lo[a] + it.hi[a]);
  }
  std::vector<SceneNode> nodes(1);
  Builder B{items, nodes};
  B.build(0, 0, (int)n, 0);
  if (B.max_depth + 2 > kSceneStack || !consistent(nodes, items)) return GG_ERR_INVALID_ARG;
  out_prims->resize(n);
  for (uint32_t i = 0; i < n; ++i) (*out_prims)[i] = ps[items[i].prim];
  *out_nodes = std::move(nodes);
  if (depth) *depth = (uint32_t)B.max_depth;
  return GG_OK;
}

}  // namespace gg
