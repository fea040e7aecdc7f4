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

// ============================================================================================ reference test scene
// The synthetic scene of the reference's accuracy tests (crates/dense/src/synthetic.rs:108-290, make_scene with
// SynthConfig): a textured floor z = 0 plus axis-aligned boxes, ray cast in binary64; cameras on a gx × gy grid at
// `altitude`, each looking at half its own xy position on the floor; the 8-bit image is the mean of four quarter-pixel
// samples (value · 230 + 15, rounded), stored as gray of the RGB (v, v, trunc(0.8·v)) with the Rec. 709 weights
// (crates/dense/src/scene.rs:163-174); ground truth (camera z, camera-frame normal) from the pixel-centre ray; sparse
// points from seeded pixels of the ground truth, observed by every view whose ground-truth depth agrees within 1 %.

namespace {

struct RefBox {
  double mn[3], mx[3];
};

// texture(u, v, seed) (synthetic.rs:67-73)
double ref_texture(double u, double v, uint64_t seed) {
  const double blocks = hash2((int64_t)floor(u / 0.18), (int64_t)floor(v / 0.18), seed ^ 0x55);
  const double fine = value_noise(u / 0.09, v / 0.09, seed);
  const double coarse = value_noise(u / 1.5, v / 1.5, seed + 7);
  return std::min(std::max(0.45 * blocks + 0.3 * fine + 0.25 * coarse, 0.0), 1.0);
}

// cast (synthetic.rs:136-188): first hit (distance, world normal, texture value) of the ray o + t·d.
bool ref_cast(const double* o, const double* d, const RefBox* boxes, int nb, uint64_t seed, double* tout, double* nout,
              double* val) {
  bool have = false;
  double bt = 0.0, bn[3] = {0, 0, 0}, bv = 0.0;
  if (d[2] < -1e-12) {
    const double t = -o[2] / d[2];
    if (t > 0.0) {
      const double p0 = o[0] + t * d[0], p1 = o[1] + t * d[1];
      have = true;
      bt = t;
      bn[0] = 0.0;
      bn[1] = 0.0;
      bn[2] = 1.0;
      bv = ref_texture(p0, p1, seed);
    }
  }
  for (int bi = 0; bi < nb; ++bi) {
    const RefBox& b = boxes[bi];
    double t0 = 0.0, t1 = INFINITY;
    int axis = 0;
    double sign = 0.0;
    bool ok = true;
    for (int a = 0; a < 3; ++a) {
      if (fabs(d[a]) < 1e-12) {
        if (o[a] < b.mn[a] || o[a] > b.mx[a]) ok = false;
        continue;
      }
      double ta = (b.mn[a] - o[a]) / d[a], tb = (b.mx[a] - o[a]) / d[a];
      double s = -1.0;
      if (ta > tb) {
        std::swap(ta, tb);
        s = 1.0;
      }
      if (ta > t0) {
        t0 = ta;
        axis = a;
        sign = s;
      }
      t1 = std::min(t1, tb);
    }
    if (!ok || t0 > t1 || t0 <= 0.0) continue;
    if (have && bt <= t0) continue;
    const double p[3] = {o[0] + t0 * d[0], o[1] + t0 * d[1], o[2] + t0 * d[2]};
    double n[3] = {0.0, 0.0, 0.0};
    n[axis] = sign;
    double u, v;
    if (axis == 0) {
      u = p[1];
      v = p[2];
    } else if (axis == 1) {
      u = p[0];
      v = p[2];
    } else {
      u = p[0];
      v = p[1];
    }
    have = true;
    bt = t0;
    bn[0] = n[0];
    bn[1] = n[1];
    bn[2] = n[2];
    bv = ref_texture(u + 17.0 * (double)bi, v - 5.0 * (double)axis, seed + 3);
  }
  if (have) {
    *tout = bt;
    nout[0] = bn[0];
    nout[1] = bn[1];
    nout[2] = bn[2];
    *val = bv;
  }
  return have;
}

inline double rdot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline void runit(double* a) {
  const double n = sqrt(rdot(a, a));
  a[0] /= n;
  a[1] /= n;
  a[2] /= n;
}

}  // namespace

extern "C" {

struct RefSceneConfig {
  int width, height;
  double focal;
  int grid_x, grid_y;
  double spacing, altitude;
  uint64_t seed;
  int num_points;
  int num_boxes;         // at most 8
  double boxes[8][6];    // min xyz, max xyz
};

// Renders the scene.  Outputs (caller-allocated, nviews = grid_x·grid_y, views in the reference's order j-major):
// cams: nviews × 16 doubles (fx, fy, cx, cy, R[9] world -> camera row-major, t[3]); gray: nviews·w·h bytes;
// depth, normal (3 per pixel): ground truth; points: up to num_points × 3 doubles, track_off: num_points + 1,
// track_views: num_points · nviews; *npoints receives the number of points kept.
int synth_reference_scene(const RefSceneConfig* cfg, double* cams, unsigned char* gray, float* depth, float* normal,
                          double* points, uint32_t* track_off, uint32_t* track_views, int* npoints) {
  if (!cfg || !cams || !gray || !depth || !normal || cfg->width < 1 || cfg->height < 1 || cfg->num_boxes < 0 ||
      cfg->num_boxes > 8)
    return 1;
  const int w = cfg->width, h = cfg->height, gx = cfg->grid_x, gy = cfg->grid_y;
  const double f = cfg->focal, cx = ((double)w - 1.0) / 2.0, cy = ((double)h - 1.0) / 2.0;
  RefBox boxes[8];
  for (int b = 0; b < cfg->num_boxes; ++b)
    for (int a = 0; a < 3; ++a) {
      boxes[b].mn[a] = cfg->boxes[b][a];
      boxes[b].mx[a] = cfg->boxes[b][3 + a];
    }
  const int nv = gx * gy;
  std::vector<double> R(nv * 9), T(nv * 3), Cc(nv * 3);
  for (int j = 0; j < gy; ++j)
    for (int i = 0; i < gx; ++i) {
      const int v = j * gx + i;
      const double c[3] = {((double)i - ((double)gx - 1.0) / 2.0) * cfg->spacing,
                           ((double)j - ((double)gy - 1.0) / 2.0) * cfg->spacing, cfg->altitude};
      const double target[3] = {c[0] * 0.5, c[1] * 0.5, 0.0};
      double zc[3] = {target[0] - c[0], target[1] - c[1], target[2] - c[2]};
      runit(zc);
      const double up[3] = {0.0, 1.0, 0.0};
      double xc[3] = {zc[1] * up[2] - zc[2] * up[1], zc[2] * up[0] - zc[0] * up[2], zc[0] * up[1] - zc[1] * up[0]};
      runit(xc);
      const double yc[3] = {zc[1] * xc[2] - zc[2] * xc[1], zc[2] * xc[0] - zc[0] * xc[2], zc[0] * xc[1] - zc[1] * xc[0]};
      for (int k = 0; k < 3; ++k) {
        R[v * 9 + k] = xc[k];
        R[v * 9 + 3 + k] = yc[k];
        R[v * 9 + 6 + k] = zc[k];
        Cc[v * 3 + k] = c[k];
      }
      T[v * 3 + 0] = -rdot(xc, c);
      T[v * 3 + 1] = -rdot(yc, c);
      T[v * 3 + 2] = -rdot(zc, c);
      double* o = cams + (size_t)v * 16;
      o[0] = f;
      o[1] = f;
      o[2] = cx;
      o[3] = cy;
      for (int k = 0; k < 9; ++k) o[4 + k] = R[v * 9 + k];
      for (int k = 0; k < 3; ++k) o[13 + k] = T[v * 3 + k];
    }
  static const double subs[5][2] = {{-0.25, -0.25}, {0.25, -0.25}, {-0.25, 0.25}, {0.25, 0.25}, {0.0, 0.0}};
  for (int v = 0; v < nv; ++v) {
    const double* xc = &R[v * 9];
    const double* yc = &R[v * 9 + 3];
    const double* zc = &R[v * 9 + 6];
    const double* c = &Cc[v * 3];
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        double acc = 0.0;
        const size_t p = (size_t)v * w * h + (size_t)y * w + x;
        depth[p] = 0.0f;
        normal[3 * p] = normal[3 * p + 1] = normal[3 * p + 2] = 0.0f;
        for (int s = 0; s < 5; ++s) {
          const double rc[3] = {((double)x + subs[s][0] - cx) / f, ((double)y + subs[s][1] - cy) / f, 1.0};
          double dw[3];
          for (int k = 0; k < 3; ++k) dw[k] = xc[k] * rc[0] + yc[k] * rc[1] + zc[k] * rc[2];
          runit(dw);
          double tt, nw[3], val = 0.0;
          const bool hit = ref_cast(c, dw, boxes, cfg->num_boxes, cfg->seed, &tt, nw, &val);
          if (s == 4) {
            if (hit) {
              const double pw[3] = {c[0] + tt * dw[0], c[1] + tt * dw[1], c[2] + tt * dw[2]};
              depth[p] = (float)(rdot(zc, pw) + T[v * 3 + 2]);
              normal[3 * p] = (float)rdot(xc, nw);
              normal[3 * p + 1] = (float)rdot(yc, nw);
              normal[3 * p + 2] = (float)rdot(zc, nw);
            }
          } else {
            acc += hit ? val : 0.0;
          }
        }
        const double q = std::min(std::max(round(acc / 4.0 * 230.0 + 15.0), 0.0), 255.0);
        const unsigned char g = (unsigned char)q;
        const unsigned char b = (unsigned char)((double)g * 0.8);
        const double gr = 0.2126 * (double)g + 0.7152 * (double)g + 0.0722 * (double)b;
        gray[p] = (unsigned char)std::min(std::max(round(gr), 0.0), 255.0);
      }
  }
  // sparse points (synthetic.rs:255-287)
  int np = 0;
  if (points && track_off && track_views && npoints) {
    uint64_t s = cfg->seed ^ 0xabcULL;
    auto rnd = [&]() {
      s += 0x9e3779b97f4a7c15ULL;
      return (double)(mix64(s) >> 11) / (double)(1ULL << 53);
    };
    uint32_t nobs = 0;
    track_off[0] = 0;
    for (int k = 0; k < cfg->num_points; ++k) {
      const int v = k % nv;
      const double xr = round(rnd() * (double)(w - 1)), yr = round(rnd() * (double)(h - 1));
      const int x = (int)xr, y = (int)yr;
      const double d = (double)depth[(size_t)v * w * h + (size_t)y * w + x];
      if (d <= 0.0) continue;
      const double pc[3] = {((double)x - cx) / f * d, ((double)y - cy) / f * d, d};
      const double dd[3] = {pc[0] - T[v * 3], pc[1] - T[v * 3 + 1], pc[2] - T[v * 3 + 2]};
      const double* r = &R[v * 9];
      const double pw[3] = {r[0] * dd[0] + r[3] * dd[1] + r[6] * dd[2], r[1] * dd[0] + r[4] * dd[1] + r[7] * dd[2],
                            r[2] * dd[0] + r[5] * dd[1] + r[8] * dd[2]};
      uint32_t cnt = 0;
      for (int o = 0; o < nv; ++o) {
        const double* ro = &R[o * 9];
        const double cc[3] = {ro[0] * pw[0] + ro[1] * pw[1] + ro[2] * pw[2] + T[o * 3],
                              ro[3] * pw[0] + ro[4] * pw[1] + ro[5] * pw[2] + T[o * 3 + 1],
                              ro[6] * pw[0] + ro[7] * pw[1] + ro[8] * pw[2] + T[o * 3 + 2]};
        if (cc[2] <= 0.0) continue;
        const double u = f * cc[0] / cc[2] + cx, vv = f * cc[1] / cc[2] + cy, z = cc[2];
        const double ui = round(u), vi = round(vv);
        if (ui < 0.0 || vi < 0.0 || ui >= (double)w || vi >= (double)h) continue;
        const double dt = (double)depth[(size_t)o * w * h + (size_t)vi * w + (size_t)ui];
        if (fabs(dt - z) < 0.01 * z) track_views[nobs + cnt++] = (uint32_t)o;
      }
      if (cnt >= 2) {
        points[3 * np] = pw[0];
        points[3 * np + 1] = pw[1];
        points[3 * np + 2] = pw[2];
        nobs += cnt;
        track_off[++np] = nobs;
      }
    }
    *npoints = np;
  }
  return 0;
}

}  // extern "C"
