// Host-side derivation of the per-session and per-iteration constants of a PatchStereo run.  Shared by the
// engine's runtime and by the CPU oracle so that both start from the same binary32 constants.
//
// Session constants follow Session::new (crates/cuda/src/patchmatch.rs:496-521); per-iteration constants follow
// Session::run (crates/cuda/src/patchmatch.rs:767-774); the emission model follows crates/dense/src/math.rs:49-82.
#pragma once
#include <math.h>
#include <stdint.h>
#include "../../include/patchstereo.h"

struct PsConsts {
  float tau_bad, inv2beta2, prev_w;
  int n1, n2, topk;
  float inv2s, inv2c, cos_tri_min, inv2inc, lambda, gmax;
  float cos_filter_tri, q_min, ncc_norm, inv2ncc, filter_gmax, weak_var;
};

// An 8-bit gray value as the unit-range f32 the engine computes with: the correctly rounded u/255 (the value an
// 8-bit normalized texture fetch returns, so texture and plane sampling agree bit for bit).
static inline float ps_u8_unit(unsigned char u) { return (float)((double)u / 255.0); }

// Rust's f64::to_radians: x * (PI / 180) with the quotient taken in binary64.
static inline double ps_to_radians_f64(double deg) { return deg * (3.14159265358979323846 / 180.0); }

// Rust's f32::to_radians: x * (PI_f32 / 180) with the quotient taken in binary32.
static inline float ps_to_radians_f32(float deg) {
  const float pi = 3.14159265358979323846f;
  const float rpd = pi / 180.0f;
  return deg * rpd;
}

// erf by its Maclaurin series (crates/dense/src/math.rs:49-66).
static inline double ps_erf(double x) {
  if (fabs(x) > 5.0) return x > 0 ? 1.0 : (x < 0 ? -1.0 : x);
  double sum = 0.0, term = x, x2 = x * x;
  for (int n = 0; n < 200; ++n) {
    double t = term / (double)(2 * n + 1);
    sum += t;
    double as = fabs(sum) > 1e-300 ? fabs(sum) : 1e-300;
    if (fabs(t) < 1e-17 * as) break;
    term *= -x2 / (double)(n + 1);
  }
  return sum * 2.0 / sqrt(3.14159265358979323846);
}
// Normalisation A(σ) of the half-normal density truncated to [0,2] (math.rs:68-71).
static inline double ps_emission_norm(double sigma) {
  return 2.0 / (sqrt(2.0 * 3.14159265358979323846) * sigma * ps_erf(2.0 / (sigma * 1.4142135623730951)));
}
// E(c) = A·exp(-c²/(2σ²)) (math.rs:73-76).
static inline double ps_emission(double cost, double sigma) {
  return ps_emission_norm(sigma) * exp(-cost * cost / (2.0 * sigma * sigma));
}

static inline float ps_sigma_s(const ps_pm_params* p) {
  return p->sigma_spatial > 0.0f ? p->sigma_spatial : (float)p->window_radius;
}

static inline PsConsts ps_session_consts(const ps_pm_params* p, const ps_filter_params* f) {
  PsConsts c;
  const float sc = ps_sigma_s(p);
  c.topk = (int)p->top_k;
  c.tau_bad = p->tau1;
  c.inv2beta2 = 1.0f / (2.0f * p->beta * p->beta);
  c.prev_w = p->prev_view_weight;
  c.n1 = (int)p->n1;
  c.n2 = (int)p->n2;
  c.inv2s = 1.0f / (2.0f * sc * sc);
  c.inv2c = 1.0f / (2.0f * p->sigma_color * p->sigma_color);
  c.cos_tri_min = cosf(ps_to_radians_f32(p->min_triangulation_angle_deg));
  c.inv2inc = 1.0f / (2.0f * p->incident_angle_sigma * p->incident_angle_sigma);
  c.lambda = p->geom_lambda;
  c.gmax = p->geom_max_cost;
  c.cos_filter_tri = cosf(ps_to_radians_f32(f->min_triangulation_angle_deg));
  c.q_min = (float)ps_emission(1.0 - (double)f->min_ncc, (double)f->ncc_sigma);
  c.ncc_norm = (float)ps_emission_norm((double)f->ncc_sigma);
  c.inv2ncc = 1.0f / (2.0f * f->ncc_sigma * f->ncc_sigma);
  c.filter_gmax = f->geom_max_cost;
  c.weak_var = p->weak_texture_var;
  return c;
}

// Per-iteration schedule: τ(t) = τ0·exp(-t²/α), ε_t = max(ε0·2^-t, ε_min), φ_t = max(φ0·2^-t, φ_min) in radians.
static inline void ps_iter_consts(const ps_pm_params* p, int geometric, int t, float* tau_good, float* eps,
                                  float* phi) {
  const float tf = (float)t;
  *tau_good = p->tau0 * expf(-tf * tf / p->tau_alpha);
  const float eps0 = geometric ? p->eps0_geometric : p->eps0_photometric;
  const float phi0 = geometric ? p->phi0_geometric_deg : p->phi0_photometric_deg;
  float half = 1.0f;
  for (int k = 0; k < t; ++k) half *= 0.5f;  // 0.5f32.powi(t), exact for t < 150
  const float e = eps0 * half, f = phi0 * half;
  *eps = e > p->eps_min ? e : p->eps_min;
  *phi = ps_to_radians_f32(f > p->phi_min_deg ? f : p->phi_min_deg);
}

static inline void ps_default_pm(ps_pm_params* o) {
  o->window_radius = 5;
  o->window_step = 2;
  o->sigma_spatial = -1.0f;
  o->sigma_color = 0.2f;
  o->tau0 = 0.8f;
  o->tau_alpha = 90.0f;
  o->tau1 = 1.2f;
  o->beta = 0.3f;
  o->n1 = 2;
  o->n2 = 3;
  o->prev_view_weight = 0.2f;
  o->min_triangulation_angle_deg = 1.0f;
  o->incident_angle_sigma = 0.9f;
  o->geom_lambda = 0.2f;
  o->geom_max_cost = 3.0f;
  o->top_k = 3;
  o->eps0_photometric = 0.2f;
  o->eps0_geometric = 0.05f;
  o->phi0_photometric_deg = 30.0f;
  o->phi0_geometric_deg = 10.0f;
  o->eps_min = 0.005f;
  o->phi_min_deg = 1.0f;
  o->weak_texture_var = 0.0f;
}

static inline void ps_default_filter(ps_filter_params* o) {
  o->min_ncc = 0.1f;
  o->min_triangulation_angle_deg = 3.0f;
  o->min_num_consistent = 2;
  o->geom_max_cost = 1.0f;
  o->ncc_sigma = 0.6f;
  o->median_filter = 1;
}
