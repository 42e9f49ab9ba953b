// ggo_capi.cpp -- C entry points of the CPU oracle (liboracle_gg.so).
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, the smoke check and the
// CPU-baseline leg of bench.py, never by the product.  The parameter structs
// are the product's public POD structs (include/gargantua_gpu.h) so the same
// inputs reach both; the arithmetic is this directory's own restatement of
// the reference (gg_oracle.hpp).
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "../include/gargantua_gpu.h"
#include "gg_counting.hpp"
#include "gg_oracle.hpp"

#define GGO_API extern "C" __attribute__((visibility("default")))

namespace {

using namespace ggo;

Camera make_camera(const gg_camera_t* c) {
  Camera cam;
  for (int i = 0; i < 4; ++i) cam.position[i] = c->position[i];
  for (int i = 0; i < 3; ++i) cam.look_at[i] = c->look_at[i];
  for (int i = 0; i < 3; ++i) cam.up[i] = c->up[i];
  cam.fov_y_radians = c->fov_y_radians;
  cam.aspect = c->aspect;
  return cam;
}

RK45 make_rk45(const gg_integrator_t* in) {
  RK45 k;
  k.initial_step = in->initial_step;
  k.min_step = in->min_step;
  k.max_step = in->max_step;
  k.tolerance = in->tolerance;
  k.max_radius = in->max_radius;
  k.horizon_buffer = in->horizon_buffer;
  k.rtol = in->rtol;
  k.atol = in->atol;
  k.stepper = in->stepper;
  return k;
}

// The sky map GG_SKY_HDRI renders sample (ggo_set_hdri); one per process.
std::vector<float> g_hdri_px;
HdriMap g_hdri;
// The objects of opts.scene renders (ggo_set_scene); one per process.
std::vector<SceneObj> g_scene;

TraceSetup make_setup(const gg_disk_t* disk, const gg_integrator_t* integ,
                      const gg_render_opts_t* opts) {
  TraceSetup S;
  S.integ = make_rk45(integ);
  S.max_steps = integ->max_steps;
  S.disk_kind = disk ? disk->kind : kDiskNone;
  if (disk) {
    S.vdisk.r_inner = disk->r_inner;
    S.vdisk.r_outer = disk->r_outer;
    S.vdisk.scale_height = disk->scale_height;
    S.vdisk.density_0 = disk->density_0;
    S.vdisk.temperature_0 = disk->temperature_0;
    S.tdisk.r_inner = disk->r_inner;
    S.tdisk.r_outer = disk->r_outer;
    S.tdisk.emissivity_index = disk->emissivity_index;
  }
  S.sky = opts->sky;
  S.sky_rows = opts->sky_rows;
  S.sky_cols = opts->sky_cols;
  S.sky_seed = opts->sky_seed;
  S.hdri = g_hdri;
  if (opts->scene) S.scene = &g_scene;
  return S;
}

uint32_t samples_per_pixel(const gg_render_opts_t* o) {
  if (o->jitter_spp > 0) return o->jitter_spp;
  uint32_t spa = o->samples_per_axis < 1 ? 1 : o->samples_per_axis;
  return spa * spa;
}

// EXTENSION: seeded uniform sub-pixel offset of sample `key`.
inline double jitter_unit(uint64_t seed, uint64_t key) {
  return (double)(splitmix64(seed ^ splitmix64(key)) >> 11) * (1.0 / 9007199254740992.0);
}

// Image-plane point of sample s of pixel (px, py): the reference's stratified
// sub-pixel centres (renderer.rs:327-331 with ray.rs:22-23), or jitter.
void sample_uv(const gg_render_opts_t* o, uint32_t w, uint32_t h, uint32_t px, uint32_t py,
               uint32_t s, double* u, double* v) {
  if (o->jitter_spp > 0) {
    uint64_t key = ((uint64_t)py * w + px) * o->jitter_spp + s;
    double ox = jitter_unit(o->seed, 2 * key);
    double oy = jitter_unit(o->seed, 2 * key + 1);
    *u = ((double)px + ox) / (double)w * 2.0 - 1.0;
    *v = 1.0 - ((double)py + oy) / (double)h * 2.0;
    return;
  }
  uint32_t spa = o->samples_per_axis < 1 ? 1 : o->samples_per_axis;
  uint32_t sy = s / spa, sx = s % spa;
  pixel_uv(px * spa + sx, py * spa + sy, w * spa, h * spa, u, v);
}

template <class M>
Sample trace_one(const M& metric, const Camera& cam, const TraceSetup& S,
                 const gg_render_opts_t* o, uint32_t w, uint32_t h, uint64_t index) {
  uint32_t spp = samples_per_pixel(o);
  uint64_t pix = index / spp;
  uint32_t s = (uint32_t)(index % spp);
  uint32_t px = (uint32_t)(pix % w), py = (uint32_t)(pix / w);
  double u, v;
  sample_uv(o, w, h, px, py, s, &u, &v);
  State<double> st = from_camera_uv(metric, cam, u, v);
  return trace(metric, S, cam.position, st);
}

void store(const gg_ray_out_t* r, uint64_t n, uint64_t i, const Sample& o) {
  if (!r) return;
  if (r->cls) r->cls[i] = o.cls;
  if (r->x) for (int c = 0; c < 4; ++c) r->x[c * n + i] = o.st.position[c];
  if (r->v) for (int c = 0; c < 4; ++c) r->v[c * n + i] = o.st.velocity[c];
  if (r->lambda) r->lambda[i] = o.st.lambda;
  if (r->attempts) r->attempts[i] = o.attempts;
  if (r->accepted) r->accepted[i] = o.accepted;
  if (r->intensity) r->intensity[i] = o.intensity;
  if (r->color_temp) r->color_temp[i] = o.color_temp;
  if (r->rgb) for (int c = 0; c < 3; ++c) r->rgb[3 * i + c] = o.rgb[c];
  if (r->cross) for (int c = 0; c < 8; ++c) r->cross[c * n + i] = o.cross[c];
}

template <class F>
void parallel_for(uint64_t n, int threads, F&& body) {
  if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
  if (threads < 1) threads = 1;
  std::atomic<uint64_t> next{0};
  auto worker = [&]() {
    for (;;) {
      uint64_t i = next.fetch_add(1);
      if (i >= n) break;
      body(i);
    }
  };
  if (threads == 1) { worker(); return; }
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
  for (auto& t : pool) t.join();
}

template <class M>
void render_impl(const M& metric, const gg_camera_t* camera, const gg_disk_t* disk,
                 const gg_integrator_t* integ, const gg_render_opts_t* opts, uint32_t w,
                 uint32_t h, uint8_t* rgb, const gg_ray_out_t* rays, int threads) {
  Camera cam = make_camera(camera);
  TraceSetup S = make_setup(disk, integ, opts);
  uint32_t spp = samples_per_pixel(opts);
  uint64_t n = (uint64_t)w * h * spp;
  double inv_spp = 1.0 / (double)spp;
  // rows in parallel, pixels of a row in order (render_inner, renderer.rs:286-296)
  parallel_for(h, threads, [&](uint64_t py) {
    for (uint32_t px = 0; px < w; ++px) {
      double acc[3] = {0.0, 0.0, 0.0};
      for (uint32_t s = 0; s < spp; ++s) {
        uint64_t idx = ((uint64_t)py * w + px) * spp + s;
        Sample o = trace_one(metric, cam, S, opts, w, h, idx);
        store(rays, n, idx, o);
        acc[0] = acc[0] + o.rgb[0];
        acc[1] = acc[1] + o.rgb[1];
        acc[2] = acc[2] + o.rgb[2];
      }
      if (rgb) {
        uint8_t* p = rgb + 3 * ((uint64_t)py * w + px);
        for (int c = 0; c < 3; ++c) p[c] = encode_channel(acc[c] * inv_spp);
      }
    }
  });
}

template <class F>
int with_metric(const gg_metric_t* m, F&& f) {
  if (!m || !(m->mass > 0.0)) return GG_ERR_INVALID_ARG;
  if (m->kind == GG_METRIC_SCHWARZSCHILD) { f(Schwarzschild(m->mass)); return GG_OK; }
  if (m->kind == GG_METRIC_KERR) { f(Kerr(m->mass, m->spin)); return GG_OK; }
  return GG_ERR_INVALID_ARG;
}

void pack_g(const G<double>& g, double out[16]) {
  for (int i = 0; i < 16; ++i) out[i] = 0.0;
  out[0] = g.tt; out[5] = g.rr; out[10] = g.thth; out[15] = g.phph;
  out[3] = g.tph; out[12] = g.tph;
}

}  // namespace

GGO_API int ggo_render(const gg_metric_t* metric, const gg_camera_t* camera,
                       const gg_disk_t* disk, const gg_integrator_t* integ,
                       const gg_render_opts_t* opts, uint32_t w, uint32_t h, uint8_t* rgb,
                       const gg_ray_out_t* rays, int threads) {
  if (!camera || !integ || !opts || w == 0 || h == 0) return GG_ERR_INVALID_ARG;
  return with_metric(metric, [&](const auto& M) {
    render_impl(M, camera, disk, integ, opts, w, h, rgb, rays, threads);
  });
}

// Traces the listed sample indices; output arrays are indexed by list position.
GGO_API int ggo_trace_samples(const gg_metric_t* metric, const gg_camera_t* camera,
                              const gg_disk_t* disk, const gg_integrator_t* integ,
                              const gg_render_opts_t* opts, uint32_t w, uint32_t h,
                              const uint64_t* index, uint64_t n, const gg_ray_out_t* rays,
                              int threads) {
  if (!camera || !integ || !opts || !index || w == 0 || h == 0) return GG_ERR_INVALID_ARG;
  return with_metric(metric, [&](const auto& M) {
    Camera cam = make_camera(camera);
    TraceSetup S = make_setup(disk, integ, opts);
    parallel_for(n, threads, [&](uint64_t i) {
      Sample o = trace_one(M, cam, S, opts, w, h, index[i]);
      store(rays, n, i, o);
    });
  });
}

// Crossing state (escape sphere or disk plane) of the listed samples, 8*n
// component-major; NaN where the ray ended elsewhere.
GGO_API int ggo_trace_cross(const gg_metric_t* metric, const gg_camera_t* camera,
                            const gg_disk_t* disk, const gg_integrator_t* integ,
                            const gg_render_opts_t* opts, uint32_t w, uint32_t h,
                            const uint64_t* index, uint64_t n, double* cross, int threads) {
  if (!camera || !integ || !opts || !index || !cross) return GG_ERR_INVALID_ARG;
  return with_metric(metric, [&](const auto& M) {
    Camera cam = make_camera(camera);
    TraceSetup S = make_setup(disk, integ, opts);
    parallel_for(n, threads, [&](uint64_t i) {
      Sample o = trace_one(M, cam, S, opts, w, h, index[i]);
      for (int c = 0; c < 8; ++c) cross[c * n + i] = o.cross[c];
    });
  });
}

// Trace from an explicit initial state (9 doubles: x[4], v[4], lambda).
GGO_API int ggo_trace_state(const gg_metric_t* metric, const gg_camera_t* camera,
                            const gg_disk_t* disk, const gg_integrator_t* integ,
                            const gg_render_opts_t* opts, const double* state9,
                            const gg_ray_out_t* rays) {
  if (!camera || !integ || !opts || !state9) return GG_ERR_INVALID_ARG;
  return with_metric(metric, [&](const auto& M) {
    Camera cam = make_camera(camera);
    TraceSetup S = make_setup(disk, integ, opts);
    State<double> st;
    for (int i = 0; i < 4; ++i) st.position[i] = state9[i];
    for (int i = 0; i < 4; ++i) st.velocity[i] = state9[4 + i];
    st.lambda = state9[8];
    Sample o = trace(M, S, cam.position, st);
    store(rays, 1, 0, o);
  });
}

// Trace from image-plane point (u, v) (used to probe class boundaries).
GGO_API int ggo_trace_uv(const gg_metric_t* metric, const gg_camera_t* camera,
                         const gg_disk_t* disk, const gg_integrator_t* integ,
                         const gg_render_opts_t* opts, double u, double v,
                         const gg_ray_out_t* rays) {
  if (!camera || !integ || !opts) return GG_ERR_INVALID_ARG;
  return with_metric(metric, [&](const auto& M) {
    Camera cam = make_camera(camera);
    TraceSetup S = make_setup(disk, integ, opts);
    State<double> st = from_camera_uv(M, cam, u, v);
    Sample o = trace(M, S, cam.position, st);
    store(rays, 1, 0, o);
  });
}

GGO_API int ggo_metric_tensor(const gg_metric_t* m, const double pos[4], double g[16]) {
  return with_metric(m, [&](const auto& M) {
    V4<double> p{{pos[0], pos[1], pos[2], pos[3]}};
    pack_g(M.metric_tensor(p), g);
  });
}

GGO_API int ggo_christoffel(const gg_metric_t* m, const double pos[4], double gamma[64]) {
  return with_metric(m, [&](const auto& M) {
    V4<double> p{{pos[0], pos[1], pos[2], pos[3]}};
    double gm[4][4][4];
    M.christoffel(p, gm);
    std::memcpy(gamma, gm, sizeof(gm));
  });
}

GGO_API int ggo_numerical_christoffel(const gg_metric_t* m, const double pos[4], double h,
                                      double gamma[64]) {
  return with_metric(m, [&](const auto& M) {
    V4<double> p{{pos[0], pos[1], pos[2], pos[3]}};
    double gm[4][4][4];
    numerical_christoffel(M, p, h, gm);
    std::memcpy(gamma, gm, sizeof(gm));
  });
}

GGO_API int ggo_geodesic_acceleration(const gg_metric_t* m, const double pos[4],
                                      const double vel[4], double acc[4]) {
  return with_metric(m, [&](const auto& M) {
    V4<double> p{{pos[0], pos[1], pos[2], pos[3]}};
    V4<double> v{{vel[0], vel[1], vel[2], vel[3]}};
    V4<double> a = M.geodesic_acceleration(p, v);
    for (int i = 0; i < 4; ++i) acc[i] = a[i];
  });
}

GGO_API int ggo_event_horizon(const gg_metric_t* m, double* rh) {
  int has = 0;
  int st = with_metric(m, [&](const auto& M) { has = M.event_horizon(rh) ? 1 : 0; });
  return st == GG_OK ? has : st;
}

GGO_API int ggo_orbital_four_velocity(const gg_metric_t* m, const double pos[4], double u[4]) {
  int has = 0;
  int st = with_metric(m, [&](const auto& M) {
    V4<double> p{{pos[0], pos[1], pos[2], pos[3]}};
    V4<double> uu;
    has = M.orbital_four_velocity(p, &uu) ? 1 : 0;
    if (has) for (int i = 0; i < 4; ++i) u[i] = uu[i];
  });
  return st == GG_OK ? has : st;
}

// nsteps calls of RK4Integrator::step with results ignored, as the reference
// tests do (geodesic.rs:378-380, kerr.rs:600-602).  state9: x[4], v[4], lambda.
GGO_API int ggo_rk4_run(const gg_metric_t* m, double* state9, double step_size,
                        uint64_t nsteps) {
  return with_metric(m, [&](const auto& M) {
    RK4 k;
    k.step_size = step_size;
    State<double> st;
    for (int i = 0; i < 4; ++i) st.position[i] = state9[i];
    for (int i = 0; i < 4; ++i) st.velocity[i] = state9[4 + i];
    st.lambda = state9[8];
    for (uint64_t i = 0; i < nsteps; ++i) k.step(M, st);
    for (int i = 0; i < 4; ++i) state9[i] = st.position[i];
    for (int i = 0; i < 4; ++i) state9[4 + i] = st.velocity[i];
    state9[8] = st.lambda;
  });
}

// One RK45Integrator::step.  Returns the StepResult (>= 0) or a status (< 0).
GGO_API int ggo_rk45_step(const gg_metric_t* m, const gg_integrator_t* integ, double* state9,
                          double* h, int* accepted) {
  int res = 0;
  int st = with_metric(m, [&](const auto& M) {
    RK45 k = make_rk45(integ);
    State<double> s;
    for (int i = 0; i < 4; ++i) s.position[i] = state9[i];
    for (int i = 0; i < 4; ++i) s.velocity[i] = state9[4 + i];
    s.lambda = state9[8];
    bool acc = false;
    res = k.step(M, s, *h, &acc);
    if (accepted) *accepted = acc ? 1 : 0;
    for (int i = 0; i < 4; ++i) state9[i] = s.position[i];
    for (int i = 0; i < 4; ++i) state9[4 + i] = s.velocity[i];
    state9[8] = s.lambda;
  });
  return st == GG_OK ? res : st;
}

// Operation counts of one accepted RK45 attempt from `state9` with step h:
// out[0..9] = add, mul, div, neg, sqrt, sin, cos, pow, exp, other.
GGO_API int ggo_count_attempt_ops(const gg_metric_t* m, const gg_integrator_t* integ,
                                  const double* state9, double h, uint64_t out[10]) {
  return with_metric(m, [&](const auto& M) {
    RK45 k = make_rk45(integ);
    State<CountingDouble> s;
    for (int i = 0; i < 4; ++i) s.position[i] = CountingDouble(state9[i]);
    for (int i = 0; i < 4; ++i) s.velocity[i] = CountingDouble(state9[4 + i]);
    s.lambda = CountingDouble(state9[8]);
    CountingDouble hh(h);
    op_counts() = OpCounts();
    k.step(M, s, hh);
    OpCounts c = op_counts();
    uint64_t v[10] = {c.add, c.mul, c.div, c.neg, c.sqrt, c.sin, c.cos, c.pow, c.exp, c.other};
    for (int i = 0; i < 10; ++i) out[i] = v[i];
  });
}

GGO_API void ggo_pixel_direction(const gg_camera_t* camera, double u, double v, double dir[3]) {
  V3 d = make_camera(camera).pixel_direction(u, v);
  for (int i = 0; i < 3; ++i) dir[i] = d[i];
}

GGO_API int ggo_from_camera(const gg_metric_t* m, const gg_camera_t* camera, uint32_t px,
                            uint32_t py, uint32_t w, uint32_t h, double* state9) {
  return with_metric(m, [&](const auto& M) {
    double u, v;
    pixel_uv(px, py, w, h, &u, &v);
    State<double> s = from_camera_uv(M, make_camera(camera), u, v);
    for (int i = 0; i < 4; ++i) state9[i] = s.position[i];
    for (int i = 0; i < 4; ++i) state9[4 + i] = s.velocity[i];
    state9[8] = s.lambda;
  });
}

// ggo_from_camera for n pixel centres, pixel index i = py * w + px in
// index[k], state k in states[9 k .. 9 k + 8].
GGO_API int ggo_from_camera_n(const gg_metric_t* m, const gg_camera_t* camera, uint32_t w,
                              uint32_t h, const uint64_t* index, uint64_t n, double* states) {
  for (uint64_t k = 0; k < n; ++k) {
    const int st = ggo_from_camera(m, camera, (uint32_t)(index[k] % w), (uint32_t)(index[k] / w),
                                   w, h, states + 9 * k);
    if (st != 0) return st;
  }
  return 0;
}

GGO_API double ggo_redshift_factor(const gg_metric_t* m, const double pos[4], const double p[4],
                                   double sqrt_neg_gtt_obs) {
  double g = 0.0;
  with_metric(m, [&](const auto& M) {
    V4<double> x{{pos[0], pos[1], pos[2], pos[3]}};
    V4<double> k{{p[0], p[1], p[2], p[3]}};
    g = redshift_factor(M, x, k, sqrt_neg_gtt_obs);
  });
  return g;
}

GGO_API void ggo_procedural_sky(const double dir[3], double rgb[3]) {
  procedural_sky(V3{{dir[0], dir[1], dir[2]}}, rgb);
}

// spatial_dir (tracer.rs:185-189) of a velocity 4-vector.
GGO_API void ggo_spatial_dir(const double v[4], double dir[3]) {
  const V3 d = spatial_dir(V4<double>{{v[0], v[1], v[2], v[3]}});
  dir[0] = d[0];
  dir[1] = d[1];
  dir[2] = d[2];
}

// Batched forms of the two above over n inputs (rows of 3 and 4 doubles).
GGO_API void ggo_procedural_sky_n(const double* dirs, double* rgb, uint64_t n) {
  for (uint64_t i = 0; i < n; ++i)
    procedural_sky(V3{{dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]}}, rgb + 3 * i);
}

GGO_API void ggo_spatial_dir_n(const double* v, double* dirs, uint64_t n) {
  for (uint64_t i = 0; i < n; ++i) ggo_spatial_dir(v + 4 * i, dirs + 3 * i);
}

GGO_API void ggo_checker_sky(double theta, double phi, uint32_t rows, uint32_t cols,
                             uint64_t seed, double rgb[3]) {
  checker_sky(theta, phi, rows, cols, seed, rgb);
}

// Sets the map of GG_SKY_HDRI renders (copied); returns 0, or -1 for no texels.
GGO_API int ggo_set_hdri(const float* rgb, uint32_t width, uint32_t height, float intensity) {
  if (!rgb || width < 1 || height < 1) return -1;
  g_hdri_px.assign(rgb, rgb + (size_t)width * height * 3);
  g_hdri.px = g_hdri_px.data();
  g_hdri.width = width;
  g_hdri.height = height;
  g_hdri.intensity = intensity;
  return 0;
}

// Sets the objects of opts.scene renders: spheres and quads with Lambertian,
// DiffuseLight, Metal (fuzz 0) or Dielectric materials.  Returns 0, or -1
// for an unknown kind or material.
GGO_API int ggo_set_scene(const gg_prim_t* prims, uint32_t n) {
  std::vector<SceneObj> objs;
  for (uint32_t k = 0; k < n; ++k) {
    const gg_prim_t& p = prims[k];
    if (p.material < kMatLambertian || p.material > kMatDielectric) return -1;
    V3 a{{p.p[0], p.p[1], p.p[2]}}, color{{p.color[0], p.color[1], p.color[2]}};
    if (p.kind == kObjSphere) {
      SceneObj o;
      o.kind = kObjSphere;
      o.material = p.material;
      o.center = a;
      o.radius = p.radius;
      o.color = color;
      objs.push_back(o);
    } else if (p.kind == kObjQuad) {
      objs.push_back(make_quad(a, V3{{p.u[0], p.u[1], p.u[2]}}, V3{{p.v[0], p.v[1], p.v[2]}},
                               p.material, color));
    } else {
      return -1;
    }
  }
  g_scene = std::move(objs);
  return 0;
}

// The nearest hit of the chord o + t d, t in (0, 1), over the objects set by
// ggo_set_scene: returns the object's index or -1, with t and the shaded
// (unredshifted) colour.
GGO_API int ggo_scene_hit(const double o[3], const double d[3], double* t, double rgb[3]) {
  Hit h;
  V3 dir{{d[0], d[1], d[2]}};
  if (!scene_hit(g_scene, V3{{o[0], o[1], o[2]}}, dir, 0.0, 1.0, h)) return -1;
  *t = h.t;
  shade_hit(dir, h, rgb);
  return (int)(h.obj - g_scene.data());
}

// HdriSky::sample of the map set by ggo_set_hdri at direction dir.
GGO_API void ggo_hdri_sky(const double dir[3], double rgb[3]) {
  hdri_sky(g_hdri, V3{{dir[0], dir[1], dir[2]}}, rgb);
}

GGO_API void ggo_disk_color(double intensity, double rgb[3]) { disk_color(intensity, rgb); }

GGO_API void ggo_encode_srgb(const double lin[3], uint8_t out[3]) {
  for (int i = 0; i < 3; ++i) out[i] = encode_channel(lin[i]);
}

GGO_API uint64_t ggo_splitmix64(uint64_t x) { return splitmix64(x); }

GGO_API void ggo_sample_uv(const gg_render_opts_t* o, uint32_t w, uint32_t h, uint32_t px,
                           uint32_t py, uint32_t s, double uv[2]) {
  sample_uv(o, w, h, px, py, s, &uv[0], &uv[1]);
}

// EXTENSION: prograde ISCO, Bardeen, Press & Teukolsky (1972) eq. 2.21.
GGO_API double ggo_kerr_isco(double mass, double spin) {
  double a = spin / mass;
  double z1 = 1.0 + std::cbrt(1.0 - a * a) * (std::cbrt(1.0 + a) + std::cbrt(1.0 - a));
  double z2 = std::sqrt(3.0 * a * a + z1 * z1);
  return mass * (3.0 + z2 - std::sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2)));
}

// EXTENSION: prograde circular photon orbit, r = 2M (1 + cos(2/3 acos(-a/M))).
GGO_API double ggo_kerr_photon_orbit(double mass, double spin) {
  return 2.0 * mass * (1.0 + std::cos((2.0 / 3.0) * std::acos(-spin / mass)));
}
