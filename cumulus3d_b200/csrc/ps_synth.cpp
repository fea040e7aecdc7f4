// ps_synth.cpp — seeded synthetic aerial scenes for PatchStereo workloads (libps_synth.so, host code).
//
// Scene: a heightfield terrain built from 4 octaves of seeded value noise (relief 0..`relief` metres), optionally
// raised by axis-aligned box structures (building-like steps), stored as a height grid of `cell` metres and defined
// everywhere by bilinear interpolation of that grid.  Albedo: seeded value noise at three scales plus a blocky hash
// pattern (the idea of crates/dense/src/synthetic.rs:52-74, re-derived here for terrain).  Shading: Lambertian with
// a fixed sun.  Images are ray cast through each pixel centre (integer-centre convention, K = [fx fy cx cy]) in
// binary64 and receive seeded Gaussian noise (Box–Muller on splitmix64).  Ground-truth camera-z depth and
// camera-frame normals (facing the camera) are written alongside.
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

extern "C" {

struct SynthScene {
  uint64_t seed;
  double relief;      // metres (terrain height range 0..relief)
  double wavelength;  // metres, base period of the terrain noise
  double cell;        // metres, height-grid resolution
  double x0, y0, x1, y1;  // grid extent (world xy)
  double noise_sigma;     // image noise σ
  int num_boxes;
  double box_hmin, box_hmax;      // box heights (metres)
  double box_smin, box_smax;      // box side lengths (metres)
  double albedo_scale;            // multiplies all texture periods
};

}  // extern "C"

namespace {

inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
inline double hash2(int64_t ix, int64_t iy, uint64_t seed) {
  uint64_t z = (uint64_t)ix * 0x9e3779b97f4a7c15ULL ^ (uint64_t)iy * 0xc2b2ae3d27d4eb4fULL ^ seed;
  return (double)(mix64(z) >> 11) / (double)(1ULL << 53);
}
inline double value_noise(double x, double y, uint64_t seed) {
  double fx = floor(x), fy = floor(y);
  double tx = x - fx, ty = y - fy;
  double sx = tx * tx * (3.0 - 2.0 * tx), sy = ty * ty * (3.0 - 2.0 * ty);
  int64_t ix = (int64_t)fx, iy = (int64_t)fy;
  double a = hash2(ix, iy, seed), b = hash2(ix + 1, iy, seed), c = hash2(ix, iy + 1, seed), d = hash2(ix + 1, iy + 1, seed);
  double top = a + (b - a) * sx, bot = c + (d - c) * sx;
  return top + (bot - top) * sy;
}

struct Grid {
  int nx = 0, ny = 0;
  double x0 = 0, y0 = 0, cell = 1;
  std::vector<float> h;
  double hmax = 0, hmin = 0;
  double at(int i, int j) const {
    i = std::min(std::max(i, 0), nx - 1);
    j = std::min(std::max(j, 0), ny - 1);
    return h[(size_t)j * nx + i];
  }
  // bilinear height and gradient
  double height(double x, double y, double* gx = nullptr, double* gy = nullptr) const {
    double u = (x - x0) / cell, v = (y - y0) / cell;
    double fu = floor(u), fv = floor(v);
    int i = (int)fu, j = (int)fv;
    double a = u - fu, b = v - fv;
    double h00 = at(i, j), h10 = at(i + 1, j), h01 = at(i, j + 1), h11 = at(i + 1, j + 1);
    if (gx) *gx = ((h10 - h00) * (1 - b) + (h11 - h01) * b) / cell;
    if (gy) *gy = ((h01 - h00) * (1 - a) + (h11 - h10) * a) / cell;
    return (h00 * (1 - a) + h10 * a) * (1 - b) + (h01 * (1 - a) + h11 * a) * b;
  }
};

Grid build_grid(const SynthScene& s) {
  Grid g;
  g.cell = s.cell;
  g.x0 = s.x0;
  g.y0 = s.y0;
  g.nx = (int)ceil((s.x1 - s.x0) / s.cell) + 2;
  g.ny = (int)ceil((s.y1 - s.y0) / s.cell) + 2;
  g.h.assign((size_t)g.nx * g.ny, 0.0f);
  // boxes: seeded positions inside the extent
  struct Box {
    double x0, y0, x1, y1, top;
  };
  std::vector<Box> boxes;
  uint64_t bs = s.seed ^ 0xb0c5ULL;
  auto rnd = [&]() {
    bs += 0x9e3779b97f4a7c15ULL;
    return (double)(mix64(bs) >> 11) / (double)(1ULL << 53);
  };
  for (int k = 0; k < s.num_boxes; ++k) {
    double sx = s.box_smin + (s.box_smax - s.box_smin) * rnd();
    double sy = s.box_smin + (s.box_smax - s.box_smin) * rnd();
    double cx = s.x0 + (s.x1 - s.x0) * rnd(), cy = s.y0 + (s.y1 - s.y0) * rnd();
    double hh = s.box_hmin + (s.box_hmax - s.box_hmin) * rnd();
    boxes.push_back({cx - sx / 2, cy - sy / 2, cx + sx / 2, cy + sy / 2, hh});
  }
  double hmin = 1e30, hmax = -1e30;
#pragma omp parallel for schedule(static) reduction(min : hmin) reduction(max : hmax)
  for (int j = 0; j < g.ny; ++j)
    for (int i = 0; i < g.nx; ++i) {
      double x = g.x0 + i * g.cell, y = g.y0 + j * g.cell;
      double acc = 0, norm = 0, amp = 1, freq = 1.0 / s.wavelength;
      for (int o = 0; o < 4; ++o) {
        acc += amp * value_noise(x * freq, y * freq, s.seed + 101 * o);
        norm += amp;
        amp *= 0.5;
        freq *= 2.0;
      }
      double h = s.relief * acc / norm;
      for (const Box& b : boxes)
        if (x >= b.x0 && x <= b.x1 && y >= b.y0 && y <= b.y1) {
          // building: flat roof at terrain height at its centre + box height
          h = std::max(h, b.top + s.relief * 0.5);
        }
      g.h[(size_t)j * g.nx + i] = (float)h;
      hmin = std::min(hmin, h);
      hmax = std::max(hmax, h);
    }
  g.hmin = hmin;
  g.hmax = hmax;
  return g;
}

double albedo(double x, double y, const SynthScene& s) {
  const double k = s.albedo_scale > 0 ? s.albedo_scale : 1.0;
  double blocks = hash2((int64_t)floor(x / (0.3 * k)), (int64_t)floor(y / (0.3 * k)), s.seed ^ 0x55);
  double fine = value_noise(x / (0.2 * k), y / (0.2 * k), s.seed ^ 0x77);
  double mid = value_noise(x / (0.7 * k), y / (0.7 * k), s.seed + 7);
  double coarse = value_noise(x / (3.0 * k), y / (3.0 * k), s.seed + 13);
  double a = 0.30 * blocks + 0.30 * fine + 0.20 * mid + 0.20 * coarse;
  return std::min(std::max(a, 0.0), 1.0);
}

// First hit of the ray o + t·d (|d| = 1) with the height field; returns false on a miss.
bool cast(const Grid& g, const double* o, const double* d, double* thit) {
  if (!(d[2] < -1e-9)) return false;
  double ttop = (o[2] - (g.hmax + 1e-3)) / -d[2];
  double tbot = (o[2] - (g.hmin - 1e-3)) / -d[2];
  if (ttop < 0) ttop = 0;
  double dxy = sqrt(d[0] * d[0] + d[1] * d[1]);
  double dt = 0.5 * g.cell / std::max(dxy, 1e-6);
  dt = std::min(dt, 0.25 / std::max(-d[2], 1e-6));
  double t0 = ttop;
  double f0 = o[2] + t0 * d[2] - g.height(o[0] + t0 * d[0], o[1] + t0 * d[1]);
  if (f0 <= 0) {
    *thit = t0;
    return true;
  }
  for (double t = ttop + dt;; t += dt) {
    bool last = t >= tbot;
    if (last) t = tbot;
    double f = o[2] + t * d[2] - g.height(o[0] + t * d[0], o[1] + t * d[1]);
    if (f <= 0) {
      double a = t0, b = t;
      for (int k = 0; k < 40; ++k) {
        double m = 0.5 * (a + b);
        double fm = o[2] + m * d[2] - g.height(o[0] + m * d[0], o[1] + m * d[1]);
        if (fm > 0) a = m;
        else b = m;
      }
      *thit = 0.5 * (a + b);
      return true;
    }
    if (last) return false;
    t0 = t;
  }
}

}  // namespace

extern "C" {

// Renders `nviews` cameras of size w×h; per view 16 doubles: fx, fy, cx, cy, R[9] (world -> camera, row-major),
// t[3] (camera = R·world + t).  images: nviews*w*h floats; depth (nullable): nviews*w*h; normal (nullable): nviews*w*h*3.
int synth_render(const SynthScene* s, const double* cams, int nviews, int w, int h, float* images, float* depth,
                 float* normal) {
  if (!s || !cams || nviews < 0 || w < 1 || h < 1 || !images) return 1;
  Grid g = build_grid(*s);
  const double sun[3] = {0.30 / 0.9985, -0.40 / 0.9985, 0.866 / 0.9985};
  for (int v = 0; v < nviews; ++v) {
    const double* c = cams + (size_t)v * 16;
    const double fx = c[0], fy = c[1], cx = c[2], cy = c[3];
    const double* R = c + 4;
    const double* t = c + 13;
    // camera centre C = -Rᵀ t
    double C[3];
    for (int i = 0; i < 3; ++i) C[i] = -(R[0 * 3 + i] * t[0] + R[1 * 3 + i] * t[1] + R[2 * 3 + i] * t[2]);
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        const size_t p = (size_t)v * w * h + (size_t)y * w + x;
        double rc[3] = {(x - cx) / fx, (y - cy) / fy, 1.0};
        double d[3];
        for (int i = 0; i < 3; ++i) d[i] = R[0 * 3 + i] * rc[0] + R[1 * 3 + i] * rc[1] + R[2 * 3 + i] * rc[2];
        double l = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        for (double& q : d) q /= l;
        double th;
        double val = 0.0;
        float dep = 0.0f, nc[3] = {0, 0, 0};
        if (cast(g, C, d, &th)) {
          double X[3] = {C[0] + th * d[0], C[1] + th * d[1], C[2] + th * d[2]};
          double gx, gy;
          g.height(X[0], X[1], &gx, &gy);
          double n[3] = {-gx, -gy, 1.0};
          double nl = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
          for (double& q : n) q /= nl;
          double shade = 0.55 + 0.45 * std::max(0.0, n[0] * sun[0] + n[1] * sun[1] + n[2] * sun[2]);
          val = 0.08 + 0.85 * albedo(X[0], X[1], *s) * shade;
          double zc = R[6] * X[0] + R[7] * X[1] + R[8] * X[2] + t[2];
          dep = (float)zc;
          double ncam[3];
          for (int i = 0; i < 3; ++i) ncam[i] = R[i * 3 + 0] * n[0] + R[i * 3 + 1] * n[1] + R[i * 3 + 2] * n[2];
          if (ncam[0] * rc[0] + ncam[1] * rc[1] + ncam[2] * rc[2] > 0)
            for (double& q : ncam) q = -q;
          for (int i = 0; i < 3; ++i) nc[i] = (float)ncam[i];
        }
        // Gaussian noise (Box–Muller), seeded per (scene, view, pixel)
        uint64_t z = mix64(s->seed ^ mix64(0x6e6f697365ULL + (uint64_t)v) ^ (uint64_t)(y * w + x));
        double u1 = ((double)(z >> 11) + 1.0) / (double)(1ULL << 53);
        double u2 = (double)(mix64(z) >> 11) / (double)(1ULL << 53);
        double gn = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
        images[p] = (float)(val + s->noise_sigma * gn);
        if (depth) depth[p] = dep;
        if (normal) {
          normal[3 * p] = nc[0];
          normal[3 * p + 1] = nc[1];
          normal[3 * p + 2] = nc[2];
        }
      }
  }
  return 0;
}

}  // extern "C"
