/*
 * ORACLE — test infrastructure, not product code.
 *
 * Voxel-grid form of the cloud march and its gradient, on the CPU, as the
 * checker for the CUDA forward and adjoint kernels.  The reference has no
 * voxel density source (its clouds are procedural: sample_density,
 * shaders/clouds/cloud_march.wgsl:432-530), so this restates the reference's
 * march loop (:808-1000) with the grid as the density and the three changes
 * the library documents for the differentiable form: no density gate, the
 * step integral (1 - e^-x)/x without the 1e-6 floor, no aerial perspective.
 * Light march (:543-578), Beer-powder and octaves (:888-927), sun
 * transmittance (:328-354), phase (:256-296), sky ambient (:672-700) and
 * lightning (:968-977) are the reference's, through oracle_march_core.h.
 *
 * The gradient here is an independent implementation: a plain reverse sweep
 * over every stored step in FP64 (no checkpoints).  Central finite
 * differences evaluate the FP64 loss over exactly the pixels whose samples
 * (primary or light taps, every step) touch the perturbed voxel's
 * interpolation support; no other pixel can change.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"
#include "oracle_common.h"
#include "oracle_march_core.h"

using namespace oracle_core;

namespace {

template <class R>
struct Corners {
  int64_t idx[8];  // -1 = outside the grid
  R w[8];
};

template <class R>
struct GridMarch {
  March<R> m;
  const PscDensityGrid* G;
  const float* vals;
  R min_x, min_z, base, top, cell_x, cell_y, cell_z;
  R k;  // density = k * value
  R inv_sigma_bar;
  R exit_t;
  V3<R> sigma_t;
  Layer<R> L;

  void init(const OracleScene* s, const PscDensityGrid* g, const float* values) {
    m.init(s, 0);
    G = g;
    vals = values;
    L = m.layers[0];
    base = L.base;
    top = L.top;
    min_x = R(g->min_x_m);
    min_z = R(g->min_z_m);
    cell_x = R(g->size_x_m) / R(g->nx);
    cell_z = R(g->size_z_m) / R(g->nz);
    cell_y = (top - base) / R(g->ny);
    sigma_t = (m.sigma_s + m.sigma_a) * March<R>::chromatic(L.droplet);
    inv_sigma_bar = R(3) / (sigma_t.x + sigma_t.y + sigma_t.z);
    k = R(g->density_scale) * inv_sigma_bar;
    exit_t = R(g->exit_transmittance);
  }

  // Trilinear weights between cell centres; corners outside read as zero.
  Corners<R> corners(R x, R alt, R z) const {
    Corners<R> c;
    const R fx = (x - min_x) / cell_x - R(0.5);
    const R fy = (alt - base) / cell_y - R(0.5);
    const R fz = (z - min_z) / cell_z - R(0.5);
    const R cx = std::floor(std::fmin(std::fmax(fx, R(-2)), R(G->nx + 1)));
    const R cy = std::floor(std::fmin(std::fmax(fy, R(-2)), R(G->ny + 1)));
    const R cz = std::floor(std::fmin(std::fmax(fz, R(-2)), R(G->nz + 1)));
    const R wx = fx - cx, wy = fy - cy, wz = fz - cz;
    const int ix = (int)cx, iy = (int)cy, iz = (int)cz;
    int n = 0;
    for (int dy = 0; dy < 2; ++dy)
      for (int dz = 0; dz < 2; ++dz)
        for (int dx = 0; dx < 2; ++dx, ++n) {
          const int X = ix + dx, Y = iy + dy, Z = iz + dz;
          const bool in = X >= 0 && X < (int)G->nx && Y >= 0 && Y < (int)G->ny && Z >= 0 &&
                          Z < (int)G->nz;
          c.idx[n] = in ? ((int64_t)Y * G->nz + Z) * G->nx + X : -1;
          c.w[n] = (dx ? wx : R(1) - wx) * (dy ? wy : R(1) - wy) * (dz ? wz : R(1) - wz);
        }
    return c;
  }
  R fetch(const Corners<R>& c) const {
    R v = 0;
    for (int i = 0; i < 8; ++i)
      if (c.idx[i] >= 0) v += c.w[i] * R(vals[c.idx[i]]);
    return v;
  }

  // Light-march geometry (cloud_march.wgsl:543-578): tap j at distance
  // (j + 0.5) * delta toward the sun.
  R light_delta(R alt) const {
    const R cos_sun = std::fmax(m.sun.y, R(0.05));
    return std::fmax((top - alt) / cos_sun, R(1)) / R(m.light_steps);
  }
  void light_tap(V3<R> p, R alt, R delta, uint32_t j, R* qx, R* qa, R* qz) const {
    const R r0 = m.planet_r + alt;
    const R cv = dot((p - m.centre()) / std::fmax(r0, R(1)), m.sun);
    const R t = (R(j) + R(0.5)) * delta;
    const V3<R> q = p + m.sun * t;
    *qx = q.x;
    *qz = q.z;
    *qa = m.altitude_from_entry(q, r0, cv, alt, t);
  }
  R light_sum(V3<R> p, R alt, R delta) const {  // sum of grid values * delta
    R s = 0;
    for (uint32_t j = 0; j < m.light_steps; ++j) {
      R qx, qa, qz;
      light_tap(p, alt, delta, j, &qx, &qa, &qz);
      s += fetch(corners(qx, qa, qz)) * delta;
    }
    return s;
  }

  struct Ray {
    V3<R> org, dir;
    R cos_theta, fwd, jitter, t0, step, r0, cos_view, h0;
    bool hit;
  };
  Ray ray(uint32_t px, uint32_t py, uint32_t width, const float* depth) const {
    Ray r{};
    const typename March<R>::ViewRay vr = m.view_ray(px, py, depth, width);
    r.org = vr.org;
    r.dir = vr.dir;
    r.cos_theta = vr.cos_theta;
    r.fwd = vr.fwd;
    r.jitter = vr.jitter;
    R t0 = 0, t1 = 0;
    r.hit = m.layer_intersect(r.org, r.dir, L, &t0, &t1);
    if (r.hit) {
      t1 = std::fmin(t1, vr.depth_t_max);
      r.hit = t1 > t0;
    }
    r.t0 = t0;
    r.step = r.hit ? (t1 - t0) / R(m.cloud_steps) : R(0);
    r.r0 = length(r.org - m.centre());
    r.cos_view = dot((r.org - m.centre()) / std::fmax(r.r0, R(1)), r.dir);
    r.h0 = r.r0 - m.planet_r;
    return r;
  }
  V3<R> pos(const Ray& r, uint32_t s, R* alt) const {
    const R t = r.t0 + (R(s) + r.jitter) * r.step;
    const V3<R> p = r.org + r.dir * t;
    *alt = m.altitude_from_entry(p, r.r0, r.cos_view, r.h0, t);
    return p;
  }

  // Per-position lighting: the in-scatter source X(od) = sun(od) * energy(od)
  // + ambient + lightning and its derivative in the light optical depth.
  struct Light {
    V3<R> sun_k;      // sun illuminance * sun transmittance * forward gain
    R coef[8];        // a^n * phase_n
    V3<R> amb;        // ambient + lightning
  };
  Light lighting(const Ray& r, V3<R> p, R alt) const {
    Light l{};
    const R hn = clampv<R>((alt - base) / std::fmax(top - base, R(1)), R(0), R(1));
    const typename March<R>::PhaseC pc = m.phase_constants(L, hn);
    R a = 1, c = 1;
    for (uint32_t n = 0; n < m.octaves; ++n) {
      l.coef[n] = a * m.phase_with(r.cos_theta, c, pc);
      a = a * m.ms_a;
      c = c * m.ms_c;
    }
    const R gain = m.forward_bias > R(0) ? R(1) + m.forward_bias * r.fwd : R(1);
    l.sun_k = (m.sun_illum * m.sun_transmittance_at(p)) * gain;
    l.amb = (m.sky_ambient(p) * m.ambient) * mix<R>(R(0.3), R(1), hn);
    if (m.lightning_radius > R(0)) {
      const R dx = p.x - m.lightning_origin.x, dz = p.z - m.lightning_origin.z;
      const R fo = clampv<R>(R(1) - std::sqrt(dx * dx + dz * dz) / m.lightning_radius, R(0), R(1));
      l.amb = l.amb + m.lightning_rgb * (fo * fo * (R(3) - R(2) * fo));
    }
    return l;
  }
  // channel c: X and dX/dod
  void source(const Light& l, int c, R od, R* X, R* dX) const {
    const R st = c == 0 ? sigma_t.x : c == 1 ? sigma_t.y : sigma_t.z;
    const R sk = c == 0 ? l.sun_k.x : c == 1 ? l.sun_k.y : l.sun_k.z;
    const R am = c == 0 ? l.amb.x : c == 1 ? l.amb.y : l.amb.z;
    R S = 0, dS = 0, b = 1;
    for (uint32_t n = 0; n < m.octaves; ++n) {
      const R e = std::exp(-st * od * b);
      S += l.coef[n] * e;
      dS += -l.coef[n] * st * b * e;
      b = b * m.ms_b;
    }
    S *= sk;
    dS *= sk;
    const R B = std::exp(-st * od), P = R(1) - std::exp(R(-2) * st * od);
    const R dB = -st * B, dP = R(2) * st * std::exp(R(-2) * st * od);
    const R ps = m.powder;
    const R E = (R(1) - ps) * B + ps * (R(2) * B * P);
    const R dE = (R(1) - ps) * dB + ps * R(2) * (dB * P + B * dP);
    *X = S * E + am;
    *dX = dS * E + S * dE;
  }
  static R phi(R x) {  // (1 - e^-x) / x
    if (std::fabs(x) < R(1e-4)) return R(1) - x * (R(0.5) - x / R(6));
    return -std::expm1(-x) / x;
  }
  R sigt(int c) const { return c == 0 ? sigma_t.x : c == 1 ? sigma_t.y : sigma_t.z; }
  R sigs(int c) const { return c == 0 ? m.sigma_s.x : c == 1 ? m.sigma_s.y : m.sigma_s.z; }

  struct Rec {
    V3<R> p;
    R alt, g, gl, T[3];
  };
  // Forward march of one pixel; fills `recs` (executed steps) if given.
  void forward(const Ray& r, R Lo[3], R To[3], std::vector<Rec>* recs) const {
    Lo[0] = Lo[1] = Lo[2] = 0;
    To[0] = To[1] = To[2] = 1;
    if (recs) recs->clear();
    if (!r.hit || r.step <= R(0)) return;
    for (uint32_t s = 0; s < m.cloud_steps; ++s) {
      R alt;
      const V3<R> p = pos(r, s, &alt);
      const R g = fetch(corners(p.x, alt, p.z));
      const R delta = light_delta(alt);
      const R gl = light_sum(p, alt, delta);
      if (recs) recs->push_back(Rec{p, alt, g, gl, {To[0], To[1], To[2]}});
      const R rho = k * g, od = k * gl;
      const Light l = lighting(r, p, alt);
      for (int c = 0; c < 3; ++c) {
        R X, dX;
        source(l, c, od, &X, &dX);
        const R x = rho * sigt(c) * r.step;
        const R s_int = rho * sigs(c) * X * r.step * phi(x);
        Lo[c] += To[c] * s_int;
        To[c] *= std::exp(-x);
      }
      if (std::fmax(To[0], std::fmax(To[1], To[2])) < exit_t) break;
    }
  }

  static R pixel_loss(const R Lo[3], const R To[3], const float* bg, const float* tgt, R inv_n,
                      R gI[3]) {
    R loss = 0;
    for (int c = 0; c < 3; ++c) {
      const R d = (Lo[c] + R(bg[c]) * To[c]) - R(tgt[c]);
      loss += d * d * inv_n;
      gI[c] = R(2) * d * inv_n;
    }
    return loss;
  }

  // Reverse sweep over the stored steps; gradient into `grad` (dense).
  R backward(const Ray& r, const std::vector<Rec>& recs, const R gI[3], const float* bg,
             double* grad) const {
    R lam[3] = {gI[0] * R(bg[0]), gI[1] * R(bg[1]), gI[2] * R(bg[2])};
    R dk = 0;
    for (size_t si = recs.size(); si-- > 0;) {
      const Rec& q = recs[si];
      const R rho = k * q.g, od = k * q.gl;
      const Light l = lighting(r, q.p, q.alt);
      R drho = 0, dod = 0;
      for (int c = 0; c < 3; ++c) {
        R X, dX;
        source(l, c, od, &X, &dX);
        const R x = rho * sigt(c) * r.step;
        const R e = std::exp(-x), ph = phi(x);
        const R s_int = rho * sigs(c) * X * r.step * ph;
        drho += gI[c] * q.T[c] * sigs(c) * X * r.step * e + lam[c] * q.T[c] * (-sigt(c) * r.step * e);
        dod += gI[c] * q.T[c] * rho * sigs(c) * r.step * ph * dX;
        lam[c] = lam[c] * e + gI[c] * s_int;
      }
      const Corners<R> cp = corners(q.p.x, q.alt, q.p.z);
      for (int i = 0; i < 8; ++i)
        if (cp.idx[i] >= 0) grad[cp.idx[i]] += double(k * cp.w[i] * drho);
      const R delta = light_delta(q.alt);
      for (uint32_t j = 0; j < m.light_steps; ++j) {
        R qx, qa, qz;
        light_tap(q.p, q.alt, delta, j, &qx, &qa, &qz);
        const Corners<R> cl = corners(qx, qa, qz);
        for (int i = 0; i < 8; ++i)
          if (cl.idx[i] >= 0) grad[cl.idx[i]] += double(k * delta * cl.w[i] * dod);
      }
      dk += q.g * drho + q.gl * dod;
    }
    return dk * inv_sigma_bar;  // d loss / d density_scale
  }

  // Every voxel any sample of this pixel interpolates from (all steps,
  // ignoring the early exit: a superset of what can change the pixel).
  template <class F>
  void touched(const Ray& r, F&& fn) const {
    if (!r.hit || r.step <= R(0)) return;
    for (uint32_t s = 0; s < m.cloud_steps; ++s) {
      R alt;
      const V3<R> p = pos(r, s, &alt);
      const Corners<R> cp = corners(p.x, alt, p.z);
      for (int i = 0; i < 8; ++i)
        if (cp.idx[i] >= 0) fn(cp.idx[i]);
      const R delta = light_delta(alt);
      for (uint32_t j = 0; j < m.light_steps; ++j) {
        R qx, qa, qz;
        light_tap(p, alt, delta, j, &qx, &qa, &qz);
        const Corners<R> cl = corners(qx, qa, qz);
        for (int i = 0; i < 8; ++i)
          if (cl.idx[i] >= 0) fn(cl.idx[i]);
      }
    }
  }
};

bool grid_ok(const OracleScene* s, const PscDensityGrid* g) {
  return s && g && g->values && g->nx && g->ny && g->nz && s->blue_noise && s->lut_transmittance &&
         s->lut_skyview && s->params.cloud_layer_count == 1 && s->params.cone_light_sampling == 0 &&
         s->params.multi_scatter_octaves >= 1 && s->params.multi_scatter_octaves <= 8;
}

int set_threads(int threads) {
#ifdef _OPENMP
  return threads > 0 ? threads : omp_get_max_threads();
#else
  (void)threads;
  return 1;
#endif
}

template <class R>
int grid_render_t(const OracleScene* s, const PscDensityGrid* g, uint32_t w, uint32_t h, int threads,
                  float* lum, float* tr) {
  GridMarch<R> gm;
  gm.init(s, g, g->values);
  const int nt = set_threads(threads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (int64_t y = 0; y < (int64_t)h; ++y)
    for (uint32_t x = 0; x < w; ++x) {
      R Lo[3], To[3];
      gm.forward(gm.ray(x, (uint32_t)y, w, s->depth), Lo, To, nullptr);
      const size_t i = ((size_t)y * w + x) * 4;
      for (int c = 0; c < 3; ++c) {
        lum[i + c] = (float)Lo[c];
        tr[i + c] = (float)To[c];
      }
      lum[i + 3] = 1.0f;
      tr[i + 3] = 1.0f;
    }
  return 0;
}

double subset_loss(const GridMarch<double>& gm, const OracleScene* s, uint32_t w, uint32_t h,
                   const float* bg, const float* tgt, const uint32_t* pix, uint32_t n, int nt) {
  const double inv_n = 1.0 / (3.0 * (double)w * (double)h);
  double total = 0.0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : total) num_threads(nt)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    const uint32_t p = pix ? pix[i] : (uint32_t)i;
    const uint32_t x = p % w, y = p / w;
    double Lo[3], To[3], gI[3];
    gm.forward(gm.ray(x, y, w, s->depth), Lo, To, nullptr);
    total += GridMarch<double>::pixel_loss(Lo, To, bg + (size_t)p * 4, tgt + (size_t)p * 4, inv_n, gI);
  }
  return total;
}

}  // namespace

extern "C" {

int oracle_grid_render(const OracleScene* s, const PscDensityGrid* g, uint32_t w, uint32_t h,
                       int precision, int threads, float* lum, float* tr) {
  if (!grid_ok(s, g) || !lum || !tr || !w || !h) return -1;
  return precision == ORACLE_FP32 ? grid_render_t<float>(s, g, w, h, threads, lum, tr)
                                  : grid_render_t<double>(s, g, w, h, threads, lum, tr);
}

int oracle_grid_loss(const OracleScene* s, const PscDensityGrid* g, uint32_t w, uint32_t h,
                     const float* bg, const float* tgt, const uint32_t* pixels, uint32_t n_pixels,
                     int threads, double* loss) {
  if (!grid_ok(s, g) || !bg || !tgt || !loss) return -1;
  GridMarch<double> gm;
  gm.init(s, g, g->values);
  *loss = subset_loss(gm, s, w, h, bg, tgt, pixels, pixels ? n_pixels : w * h, set_threads(threads));
  return 0;
}

int oracle_grid_adjoint(const OracleScene* s, const PscDensityGrid* g, uint32_t w, uint32_t h,
                        const float* bg, const float* tgt, uint32_t row0, uint32_t row1,
                        int threads, double* grad, double* grad_scale, double* loss) {
  if (!grid_ok(s, g) || !bg || !tgt || !grad || !grad_scale || !loss) return -1;
  if (row1 == 0 || row1 > h) row1 = h;
  if (row0 >= row1) return -1;
  GridMarch<double> gm;
  gm.init(s, g, g->values);
  const size_t nvox = (size_t)g->nx * g->ny * g->nz;
  const int nt = set_threads(threads);
  const double inv_n = 1.0 / (3.0 * (double)w * (double)h);
  std::vector<std::vector<double>> part(nt);
  double total_loss = 0.0, total_ds = 0.0;
#pragma omp parallel num_threads(nt) reduction(+ : total_loss, total_ds)
  {
#ifdef _OPENMP
    const int tid = omp_get_thread_num();
#else
    const int tid = 0;
#endif
    std::vector<double>& acc = part[tid];
    acc.assign(nvox, 0.0);
    std::vector<GridMarch<double>::Rec> recs;
    recs.reserve(gm.m.cloud_steps);
#pragma omp for schedule(dynamic, 1)
    for (int64_t y = row0; y < (int64_t)row1; ++y)
      for (uint32_t x = 0; x < w; ++x) {
        const auto r = gm.ray(x, (uint32_t)y, w, s->depth);
        double Lo[3], To[3], gI[3];
        gm.forward(r, Lo, To, &recs);
        const size_t p = (size_t)y * w + x;
        total_loss += GridMarch<double>::pixel_loss(Lo, To, bg + p * 4, tgt + p * 4, inv_n, gI);
        total_ds += gm.backward(r, recs, gI, bg + p * 4, acc.data());
      }
  }
  for (size_t i = 0; i < nvox; ++i) {
    double v = 0.0;
    for (int t = 0; t < nt; ++t) v += part[t][i];
    grad[i] = v;
  }
  *grad_scale = total_ds;
  *loss = total_loss;
  return 0;
}

int oracle_grid_counts(const OracleScene* s, const PscDensityGrid* g, uint32_t w, uint32_t h,
                       int threads, uint64_t* out) {
  if (!grid_ok(s, g) || !out) return -1;
  GridMarch<double> gm;
  gm.init(s, g, g->values);
  uint64_t steps = 0, prim = 0, light = 0, hit = 0;
  const int nt = set_threads(threads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt) reduction(+ : steps, prim, light, hit)
  for (int64_t y = 0; y < (int64_t)h; ++y) {
    std::vector<GridMarch<double>::Rec> recs;
    for (uint32_t x = 0; x < w; ++x) {
      const auto r = gm.ray(x, (uint32_t)y, w, s->depth);
      double Lo[3], To[3];
      gm.forward(r, Lo, To, &recs);
      hit += recs.empty() ? 0 : 1;
      steps += recs.size();
      for (const auto& q : recs) {
        const Corners<double> cp = gm.corners(q.p.x, q.alt, q.p.z);
        for (int i = 0; i < 8; ++i) prim += cp.idx[i] >= 0;
        const double delta = gm.light_delta(q.alt);
        for (uint32_t j = 0; j < gm.m.light_steps; ++j) {
          double qx, qa, qz;
          gm.light_tap(q.p, q.alt, delta, j, &qx, &qa, &qz);
          const Corners<double> cl = gm.corners(qx, qa, qz);
          for (int i = 0; i < 8; ++i) light += cl.idx[i] >= 0;
        }
      }
    }
  }
  out[0] = (uint64_t)w * h;
  out[1] = hit;
  out[2] = steps;
  out[3] = prim;
  out[4] = light;
  return 0;
}

int oracle_grid_fd(const OracleScene* s, const PscDensityGrid* g, uint32_t w, uint32_t h,
                   const float* bg, const float* tgt, const uint64_t* voxels, uint32_t n_vox,
                   double eps, int threads, double* out, uint32_t* n_pixels_out) {
  if (!grid_ok(s, g) || !bg || !tgt || !voxels || !out) return -1;
  const size_t nvox = (size_t)g->nx * g->ny * g->nz;
  std::vector<int32_t> slot(nvox, -1);
  for (uint32_t i = 0; i < n_vox; ++i) {
    if (voxels[i] >= nvox) return -1;
    slot[voxels[i]] = (int32_t)i;
  }
  const int nt = set_threads(threads);
  std::vector<float> copy(g->values, g->values + nvox);
  PscDensityGrid gg = *g;
  gg.values = copy.data();
  GridMarch<double> gm;
  gm.init(s, &gg, copy.data());
  // pixels touching each listed voxel
  std::vector<std::vector<std::vector<uint32_t>>> hits(nt, std::vector<std::vector<uint32_t>>(n_vox));
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (int64_t y = 0; y < (int64_t)h; ++y) {
#ifdef _OPENMP
    const int tid = omp_get_thread_num();
#else
    const int tid = 0;
#endif
    for (uint32_t x = 0; x < w; ++x) {
      const uint32_t p = (uint32_t)y * w + x;
      gm.touched(gm.ray(x, (uint32_t)y, w, s->depth), [&](int64_t v) {
        const int32_t k = slot[(size_t)v];
        if (k >= 0 && (hits[tid][k].empty() || hits[tid][k].back() != p)) hits[tid][k].push_back(p);
      });
    }
  }
  for (uint32_t i = 0; i < n_vox; ++i) {
    std::vector<uint32_t> px;
    for (int t = 0; t < nt; ++t) px.insert(px.end(), hits[t][i].begin(), hits[t][i].end());
    std::sort(px.begin(), px.end());
    px.erase(std::unique(px.begin(), px.end()), px.end());
    if (n_pixels_out) n_pixels_out[i] = (uint32_t)px.size();
    const float v0 = copy[voxels[i]];
    copy[voxels[i]] = (float)((double)v0 + eps);
    const double lp = subset_loss(gm, s, w, h, bg, tgt, px.data(), (uint32_t)px.size(), nt);
    copy[voxels[i]] = (float)((double)v0 - eps);
    const double lm = subset_loss(gm, s, w, h, bg, tgt, px.data(), (uint32_t)px.size(), nt);
    copy[voxels[i]] = v0;
    // the perturbation actually applied, after rounding to the FP32 grid
    const double hi = (double)(float)((double)v0 + eps), lo = (double)(float)((double)v0 - eps);
    out[i] = (lp - lm) / (hi - lo);
  }
  return 0;
}

}  // extern "C"
