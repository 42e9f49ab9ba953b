// gg_scene.cuh -- geodesic chords against a scene of objects in the spatial
// slice: trace_ray_with_scene / trace_ray_with_disk_and_scene
// (crates/raytracer/src/curved/tracer.rs:206-249, 262-366).
//
// After every step that moved the ray, the straight Cartesian chord from the
// old to the new position is tested against the scene for t in (0, 1); the
// nearest hit ends the ray with the surface's one-sample shading times the
// static-emitter redshift g^4.  The scene is a bounding-volume hierarchy
// built on the host; every lane of a warp walks it from the same root, so
// the small node and primitive arrays stay in L1.  Products and sums are
// rounded one by one (no contraction into FMAs), as the reference computes
// them.
#pragma once

#include "gg_device.cuh"

namespace gg {

GG_DEV double dot3_nc(const double a[3], const double b[3]) {
  return add_rn(add_rn(mul_rn(a[0], b[0]), mul_rn(a[1], b[1])), mul_rn(a[2], b[2]));
}

// spherical_to_cartesian (tracer.rs:11-18)
GG_DEV void sph_to_cart(const double x[4], double p[3]) {
  const double r = x[1];
  double st, ct, sp, cp;
  sincos(x[2], &st, &ct);
  sincos(x[3], &sp, &cp);
  p[0] = mul_rn(mul_rn(r, st), cp);
  p[1] = mul_rn(mul_rn(r, st), sp);
  p[2] = mul_rn(r, ct);
}

// Aabb::hit (core/aabb.rs:57-82): slab test against (t_min, t_max).
GG_DEV bool node_hit(const SceneNode& N, const double o[3], const double inv[3], double t_min,
                     double t_max) {
  double enter = t_min, exit = t_max;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double t1 = mul_rn(sub_rn(N.lo[a], o[a]), inv[a]);
    const double t2 = mul_rn(sub_rn(N.hi[a], o[a]), inv[a]);
    enter = fmax(enter, fmin(t1, t2));
    exit = fmin(exit, fmax(t1, t2));
  }
  return enter < exit;
}

// Sphere::hit (sphere.rs:53-87): the nearer root inside (t_min, t_max).
GG_DEV bool sphere_hit(const ScenePrim& S, const double o[3], const double d[3], double t_min,
                       double t_max, double& t) {
  const double oc[3] = {sub_rn(o[0], S.c[0]), sub_rn(o[1], S.c[1]), sub_rn(o[2], S.c[2])};
  const double a = dot3_nc(d, d);
  const double half_b = dot3_nc(oc, d);
  const double c = sub_rn(dot3_nc(oc, oc), mul_rn(S.radius, S.radius));
  const double disc = sub_rn(mul_rn(half_b, half_b), mul_rn(a, c));
  if (disc < 0.0) return false;
  const double sq = __dsqrt_rn(disc);
  double root = __ddiv_rn(sub_rn(-half_b, sq), a);
  if (!(t_min < root && root < t_max)) {
    root = __ddiv_rn(add_rn(-half_b, sq), a);
    if (!(t_min < root && root < t_max)) return false;
  }
  t = root;
  return true;
}

// Quad::hit (quad.rs:85-125): plane hit inside (t_min, t_max) whose planar
// coordinates (alpha, beta) lie in [0, 1].
GG_DEV bool quad_hit(const ScenePrim& Q, const double o[3], const double d[3], double t_min,
                     double t_max, double& t) {
  const double denom = dot3_nc(Q.n, d);
  if (fabs(denom) < 1e-8) return false;
  const double tt = __ddiv_rn(sub_rn(Q.d, dot3_nc(Q.n, o)), denom);
  if (!(t_min < tt && tt < t_max)) return false;
  double planar[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) planar[i] = sub_rn(add_rn(o[i], mul_rn(d[i], tt)), Q.c[i]);
  const double alpha = dot3_nc(planar, Q.ea);
  const double beta = dot3_nc(planar, Q.eb);
  if (alpha < 0.0 || alpha > 1.0 || beta < 0.0 || beta > 1.0) return false;
  t = tt;
  return true;
}

// Nearest hit of the chord o + t d, t in (0, 1), over the hierarchy
// (BvhNode::hit, accel/bvh.rs:184-254: t_max shrinks to each hit found).
// Returns the primitive index or -1.
GG_DEV int scene_nearest(const DevParams& P, const double o[3], const double d[3], double& t_hit) {
  const double inv[3] = {1.0 / d[0], 1.0 / d[1], 1.0 / d[2]};
  const double t_min = 0.0;
  double t_max = 1.0;
  int best = -1;
  int stack[kSceneStack];
  int top = 0;
  stack[top++] = 0;
  while (top > 0) {
    const SceneNode& N = P.nodes[stack[--top]];
    if (!node_hit(N, o, inv, t_min, t_max)) continue;
    if (N.count > 0) {
      for (int k = N.first; k < N.first + N.count; ++k) {
        const ScenePrim& S = P.prims[k];
        double t;
        const bool h = S.kind == kPrimSphere ? sphere_hit(S, o, d, t_min, t_max, t)
                                             : quad_hit(S, o, d, t_min, t_max, t);
        if (h) {
          t_max = t;
          best = k;
        }
      }
    } else if (top + 2 <= kSceneStack) {  // the host bounds the depth below the stack
      stack[top++] = N.first + 1;
      stack[top++] = N.first;
    }
  }
  t_hit = t_max;
  return best;
}

// shade_hit (tracer.rs:369-384) times redshift_g4_static (tracer.rs:40-52)
// at the hit point, for primitive k hit at chord parameter t.
template <int METRIC>
GG_DEV void scene_shade(const DevParams& P, int k, double t, const double o[3], const double d[3],
                        double lin[3]) {
  const ScenePrim& S = P.prims[k];
  double point[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) point[i] = add_rn(o[i], mul_rn(d[i], t));
  double outward[3];
  if (S.kind == kPrimSphere) {
#pragma unroll
    for (int i = 0; i < 3; ++i) outward[i] = __ddiv_rn(sub_rn(point[i], S.c[i]), S.radius);
  } else {
#pragma unroll
    for (int i = 0; i < 3; ++i) outward[i] = S.n[i];
  }
  // HitRecord::new (core/hit.rs): the normal faces the incoming chord
  const bool front = dot3_nc(d, outward) < 0.0;
  double nrm[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) nrm[i] = front ? outward[i] : -outward[i];
  const double len = __dsqrt_rn(dot3_nc(d, d));
  double unit[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) unit[i] = __ddiv_rn(d[i], len);
  bool scatters = S.shade == kShadeAlbedo;
  if (S.shade == kShadeMirror) {  // Metal::scatter (metal.rs:40-57), fuzz 0
    const double two_dot = mul_rn(2.0, dot3_nc(unit, nrm));
    double refl[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) refl[i] = sub_rn(unit[i], mul_rn(two_dot, nrm[i]));
    scatters = dot3_nc(refl, nrm) > 0.0;
  }
  const double neg_unit[3] = {-unit[0], -unit[1], -unit[2]};
  const double facing = add_rn(0.5, mul_rn(0.5, fmax(dot3_nc(neg_unit, nrm), 0.0)));
  // cartesian_to_spherical (tracer.rs:20-28) of the hit point, then g^4
  const double r = fmax(__dsqrt_rn(dot3_nc(point, point)), 1e-10);
  const double th = acos(fmin(fmax(__ddiv_rn(point[2], r), -1.0), 1.0));
  const Gmet g = metric_tensor<METRIC>(P, r, th);
  const double g_tt_emit = -g.tt, g_tt_obs = -P.cam_g_tt;
  double g4 = 0.0;
  if (!(g_tt_emit <= 0.0 || g_tt_obs <= 0.0)) {
    const double gg = __dsqrt_rn(__ddiv_rn(g_tt_emit, g_tt_obs));
    const double g2 = mul_rn(gg, gg);
    g4 = mul_rn(g2, g2);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double lit = add_rn(mul_rn(scatters ? S.albedo[c] : 0.0, facing), S.emit[c]);
    lin[c] = mul_rn(lit, g4);
  }
}

}  // namespace gg
