// Oracle (test infrastructure only): pbf.rs step_coupled and helpers, mac/lubrication.rs subset,
// dem.rs step_recorded. Each function cites the reference lines it restates.
#include <algorithm>
#include <cstring>

#include "oracle_core.hpp"

namespace orc {

static const Real GRAVITY = -Real(9.81);

// ------------------------------------------------------------------ pbf.rs:45-116 constants
static const Real EPSILON_RELAX = Real(200.0);
static const uint32_t ADAPTIVE_MAX_EXTRA_ITERATIONS = 6;
static const Real COMPRESSION_CONVERGENCE_TOLERANCE = Real(0.02);
static const Real OVERLAP_PUSH_MARGIN = Real(0.05);
static const Real REFERENCE_SURFACE_TENSION_N_M = Real(0.072);
static const Real COHESION_ACCEL_FACTOR = Real(2.0);
static const Real ADHESION_ACCEL_FACTOR = Real(2.0);
static const Real VISCOSITY_CG_TOLERANCE = Real(1e-3);
static const uint32_t VISCOSITY_CG_MAX_ITERS = 50;
static const Real VISCOSITY_ETA_FACTOR = Real(0.01);
static const Real BALL_FORM_DRAG_COEFFICIENT = Real(1.0);
static const Real CENTRAL_VISCOSITY_FACTOR = Real(4.0);
static const Real BALL_BC_GAIN = Real(0.5);
static const Real BINGHAM_PLASTIC_RATIO = Real(100.0);
static const Real SQUEEZE_GAIN = Real(1.0);
static const Real SQUEEZE_STIFFNESS_CAP = Real(8.0);
static const double MIN_FILM_GAP_RATIO = 0.02;
static const Real F_CLAMP_G_MULTIPLE = Real(60.0);
static const Real FLUID_SPEED_SAFETY_FACTOR = Real(5.0);

// pbf.rs:119-181 kernels
static Real poly6(Real r2, Real h) {
  if (r2 >= h * h || r2 < Real(0.0)) return Real(0.0);
  Real h2 = h * h;
  Real term = h2 - r2;
  return Real(4.0) / (PI_F * powi8(h)) * term * term * term;
}
static Vec2 spiky_grad(Vec2 delta, Real r, Real h) {
  if (r <= Real(1e-9) || r >= h) return Vec2();
  Real coeff = -Real(30.0) / (PI_F * powi5(h)) * (h - r) * (h - r);
  return (delta / r) * coeff;
}
static Real cohesion_kernel(Real r, Real h) {
  if (r <= Real(0.0) || r >= h) return Real(0.0);
  Real coeff = Real(35840.0) / (Real(209.0) * PI_F * powi8(h));
  Real term = powi3(h - r) * powi3(r);
  if (r <= Real(0.5) * h) return coeff * (Real(2.0) * term - powi6(h) / Real(64.0));
  return coeff * term;
}
static Real adhesion_kernel(Real r, Real h) {
  if (r <= Real(0.5) * h || r >= h) return Real(0.0);
  Real coeff = Real(35840.0) / (Real(163.0) * PI_F * powi8(h));
  return coeff * powi3(h - r) * powi3(r);
}

// pbf.rs:190-219
static uint32_t boundary_points_per_ball(Real ball_radius, Real dx) {
  Real circumference = TAU_F * ball_radius;
  return std::max(f2u_sat(std::round(circumference / dx)), 6u);
}
static std::vector<Vec2> ball_boundary_particles(const Balls& b, Real dx) {
  std::vector<Vec2> out;
  if (b.len() == 0 || b.radius <= Real(0.0) || dx <= Real(0.0)) return out;
  uint32_t count = boundary_points_per_ball(b.radius, dx);
  std::vector<Vec2> offsets(count);
  for (uint32_t k = 0; k < count; ++k) {
    Real angle = TAU_F * (Real)k / (Real)count;
    offsets[k] = Vec2(cosf_r(angle), sinf_r(angle)) * b.radius;
  }
  out.reserve(b.len() * count);
  for (size_t i = 0; i < b.len(); ++i)
    for (uint32_t k = 0; k < count; ++k) out.push_back(b.x[i] + offsets[k]);
  return out;
}

// pbf.rs:262-288
void neighbor_lists(const std::vector<Vec2>& x, Real h, std::vector<uint32_t>* offsets,
                    std::vector<uint32_t>* nbrs) {
  UniformGrid g = UniformGrid::build(x, h);
  size_t n = x.size();
  std::vector<std::pair<uint32_t, uint32_t>> edges;
  g.for_each_candidate_pair([&](uint32_t i, uint32_t j) {
    if ((x[i] - x[j]).length_squared() <= h * h) {
      edges.push_back({i, j});
      edges.push_back({j, i});
    }
  });
  offsets->assign(n + 1, 0);
  for (auto& e : edges) (*offsets)[e.first + 1] += 1;
  for (size_t k = 1; k < offsets->size(); ++k) (*offsets)[k] += (*offsets)[k - 1];
  std::vector<uint32_t> cursor = *offsets;
  nbrs->assign(edges.size(), 0);
  for (auto& e : edges) { (*nbrs)[cursor[e.first]] = e.second; cursor[e.first] += 1; }
}

struct Nbr {
  std::vector<uint32_t> off, idx;
  size_t b(size_t i) const { return off[i]; }
  size_t e(size_t i) const { return off[i + 1]; }
};

// pbf.rs:292-294 (sequential f32 sum) and its f64 counterpart
static Real dot_f32(const std::vector<Vec2>& a, const std::vector<Vec2>& b) {
  Real s = Real(0.0);
  for (size_t i = 0; i < a.size(); ++i) s += a[i].dot(b[i]);
  return s;
}
static double dot_f64(const std::vector<Vec2>& a, const std::vector<Vec2>& b) {
  double s = 0.0;
  for (size_t i = 0; i < a.size(); ++i) s += (double)a[i].x * (double)b[i].x + (double)a[i].y * (double)b[i].y;
  return s;
}

// pbf.rs:312-351
struct ViscWeights { std::vector<Real> w; std::vector<Vec2> dir; };
static ViscWeights morris_weights(const std::vector<Vec2>& x, const Nbr& nb, const std::vector<Real>& density,
                                  Real mass, const std::vector<Real>& mu, Real h) {
  Real eta2 = VISCOSITY_ETA_FACTOR * h * h;
  ViscWeights vw;
  vw.w.assign(nb.idx.size(), Real(0.0));
  vw.dir.assign(nb.idx.size(), Vec2());
  for (size_t i = 0; i < x.size(); ++i) {
    Real rho_i = fmax_r(density[i], Real(1e-6));
    for (size_t k = nb.b(i); k < nb.e(i); ++k) {
      size_t ju = nb.idx[k];
      Real rho_j = fmax_r(density[ju], Real(1e-6));
      Vec2 delta = x[i] - x[ju];
      Real r = delta.length();
      Vec2 grad = spiky_grad(delta, r, h);
      Real numerator = (mass * (mu[i] + mu[ju]) / (rho_i * rho_j)) * std::fabs(delta.dot(grad));
      vw.w[k] = numerator / (delta.length_squared() + eta2);
      vw.dir[k] = r > Real(1e-9) ? delta / r : Vec2(Real(1.0), Real(0.0));
    }
  }
  return vw;
}

// pbf.rs:359-377
static void laplacian_apply_into(const Nbr& nb, const ViscWeights& w, const Vec2* v, size_t n, Vec2* out) {
  for (size_t i = 0; i < n; ++i) {
    Vec2 sum;
    for (size_t k = nb.b(i); k < nb.e(i); ++k) {
      size_t j = nb.idx[k];
      Vec2 e = w.dir[k];
      sum += (CENTRAL_VISCOSITY_FACTOR * w.w[k] * e.dot(v[i] - v[j])) * e;
    }
    out[i] = sum;
  }
}
static Real viscosity_diag(Real sum_w) { return Real(0.5) * CENTRAL_VISCOSITY_FACTOR * sum_w; }

// pbf.rs:423-480 (fluid-only CG); `fp64` selects f64 inner products and norms.
static uint32_t solve_implicit_viscosity(const Nbr& nb, const ViscWeights& w, std::vector<Vec2>* vp, Real dt,
                                         bool fp64) {
  std::vector<Vec2>& v = *vp;
  size_t n = v.size();
  double b_norm = fp64 ? std::sqrt(dot_f64(v, v)) : (double)std::sqrt(dot_f32(v, v));
  if (b_norm <= 0.0 || !std::isfinite(b_norm)) return 0;
  Real target_f = VISCOSITY_CG_TOLERANCE * (Real)b_norm;
  double target_d = (double)VISCOSITY_CG_TOLERANCE * b_norm;
  std::vector<Vec2> lv(n), ax(n), r(n), p, ap(n);
  auto apply = [&](const std::vector<Vec2>& in, std::vector<Vec2>& out) {
    laplacian_apply_into(nb, w, in.data(), n, lv.data());
    for (size_t i = 0; i < n; ++i) out[i] = in[i] + dt * lv[i];
  };
  apply(v, ax);
  for (size_t i = 0; i < n; ++i) r[i] = v[i] - ax[i];
  p = r;
  if (!fp64) {
    Real rs_old = dot_f32(r, r);
    if (std::sqrt(rs_old) <= target_f) return 0;
    for (uint32_t iter = 1; iter <= VISCOSITY_CG_MAX_ITERS; ++iter) {
      apply(p, ap);
      Real p_ap = dot_f32(p, ap);
      if (p_ap <= Real(0.0) || !std::isfinite(p_ap)) return iter;
      Real alpha = rs_old / p_ap;
      for (size_t i = 0; i < n; ++i) { v[i] += alpha * p[i]; r[i] -= alpha * ap[i]; }
      Real rs_new = dot_f32(r, r);
      if (std::sqrt(rs_new) <= target_f) return iter;
      Real beta = rs_new / rs_old;
      for (size_t i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
      rs_old = rs_new;
    }
  } else {
    double rs_old = dot_f64(r, r);
    if (std::sqrt(rs_old) <= target_d) return 0;
    for (uint32_t iter = 1; iter <= VISCOSITY_CG_MAX_ITERS; ++iter) {
      apply(p, ap);
      double p_ap = dot_f64(p, ap);
      if (p_ap <= 0.0 || !std::isfinite(p_ap)) return iter;
      Real alpha = (Real)(rs_old / p_ap);
      for (size_t i = 0; i < n; ++i) { v[i] += alpha * p[i]; r[i] -= alpha * ap[i]; }
      double rs_new = dot_f64(r, r);
      if (std::sqrt(rs_new) <= target_d) return iter;
      Real beta = (Real)(rs_new / rs_old);
      for (size_t i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
      rs_old = rs_new;
    }
  }
  return VISCOSITY_CG_MAX_ITERS;
}

struct BoundaryGroup { uint32_t fluid, ball; Real c; Vec2 lever_c; Real lever2_c; };
struct SqueezeLink { uint32_t ball, other; Vec2 n; Real c; };

// mac/lubrication.rs:19-115 (the subset pbf.rs:544-625 uses)
static const double H_START = 8.0;
struct SqueezeFilm {
  double r, c1, c2, prefactor;
  SqueezeFilm(double k1, double k2, double nu) {
    r = 1.0 / (k1 + k2);
    double r3 = r * (r * r);
    double q = r3 * (k1 * (k1 * k1) + k2 * (k2 * k2));
    c1 = 0.788 + 0.265 * q;
    c2 = dmax_r(0.006 + 0.057 * (q - 0.25), 0.0);
    prefactor = 3.0 * std::sqrt(2.0) * M_PI * nu * std::pow(r, 1.5);
  }
  double coefficient(double h) const {
    double eps = h / r;
    return prefactor / (h * std::sqrt(h)) * (1.0 + c1 * eps + c2 * eps * eps);
  }
};
static double resolved_ratio(double h_cells) {
  static const double T[6][2] = {{0.0, 0.0}, {0.5, 0.06}, {1.0, 0.25}, {2.0, 0.90}, {4.0, 0.99}, {8.0, 1.0}};
  if (h_cells >= 8.0) return 1.0;
  double h = dmax_r(h_cells, 0.0);
  for (int k = 0; k < 5; ++k) {
    if (h <= T[k + 1][0]) {
      double t = (h - T[k][0]) / (T[k + 1][0] - T[k][0]);
      return T[k][1] + t * (T[k + 1][1] - T[k][1]);
    }
  }
  return 1.0;
}

// pbf.rs:544-625
static std::vector<SqueezeLink> squeeze_links(const Balls& balls, Real drum_radius, Real dx, Real mu, Real dt,
                                              const std::vector<Vec2>* closing, size_t* in_range_out) {
  std::vector<SqueezeLink> out;
  size_t in_range = 0;
  Real r = balls.radius;
  *in_range_out = 0;
  if (balls.len() == 0 || r <= Real(0.0) || mu <= Real(0.0)) return out;
  double a = (double)r, b = (double)drum_radius, dxd = (double)dx, mud = (double)mu;
  Real gain = SQUEEZE_GAIN;
  Real reach = (Real)(H_START * dxd);
  Real c_max = SQUEEZE_STIFFNESS_CAP * balls.mass / fmax_r(dt, Real(1e-12));
  UniformGrid grid = UniformGrid::build(balls.x, Real(2.0) * r + reach);
  Real range2 = (Real(2.0) * r + reach) * (Real(2.0) * r + reach) * (Real(1.0) + Real(1e-4));
  SqueezeFilm pair_film(1.0 / a, 1.0 / a, mud);
  SqueezeFilm wall_film(1.0 / a, -1.0 / b, mud);
  for (size_t i = 0; i < balls.len(); ++i) {
    Vec2 xi = balls.x[i];
    if (!xi.is_finite()) continue;
    grid.for_each_near(xi, [&](uint32_t j) {
      if ((size_t)j <= i) return;
      Vec2 e = balls.x[j] - xi;
      if (e.length_squared() >= range2 || !e.is_finite()) return;
      Real dist = e.length();
      Real gap = dist - Real(2.0) * r;
      if (gap >= reach || dist < Real(1e-9)) return;
      in_range += 1;
      Vec2 n = e / dist;
      if (closing && n.dot((*closing)[i] - (*closing)[j]) <= Real(0.0)) return;
      double weight = 1.0 - resolved_ratio((double)gap / dxd);
      double hh = dmax_r((double)gap, MIN_FILM_GAP_RATIO * a);
      double c = weight * pair_film.coefficient(hh);
      out.push_back({(uint32_t)i, j, n, fmin_r(gain * (Real)c, c_max)});
    });
    Real dist = xi.length();
    Real gap = drum_radius - r - dist;
    if (gap < reach && dist > Real(1e-9)) {
      in_range += 1;
      Vec2 n = xi / dist;
      if (closing && n.dot((*closing)[i]) <= Real(0.0)) continue;
      double weight = 1.0 - resolved_ratio((double)gap / dxd);
      double hh = dmax_r((double)gap, MIN_FILM_GAP_RATIO * a);
      double c = weight * wall_film.coefficient(hh);
      out.push_back({(uint32_t)i, WALL_ID, n, fmin_r(gain * (Real)c, c_max)});
    }
  }
  *in_range_out = in_range;
  return out;
}

// pbf.rs:641-791 (joint fluid + ball Jacobi-PCG); `fp64` selects f64 inner products and norms.
static uint32_t solve_viscosity_with_balls(const Nbr& nb, const ViscWeights& weights,
                                           const std::vector<BoundaryGroup>& groups,
                                           const std::vector<SqueezeLink>& links, Real mass, Real ball_mass_,
                                           Real ball_inertia_, Real dt, const std::vector<Vec2>& guess,
                                           std::vector<Vec2>* vp, std::vector<Vec2>* ball_vp,
                                           std::vector<Real>* ball_wp, bool fp64) {
  std::vector<Vec2>& v = *vp;
  std::vector<Vec2>& ball_v = *ball_vp;
  std::vector<Real>& ball_w = *ball_wp;
  size_t n = v.size(), nbn = ball_v.size(), len = n + 2 * nbn;
  auto perp = [](Vec2 l) { return Vec2(-l.y, l.x); };
  std::vector<Vec2> x;
  x.reserve(len);
  if (guess.size() == n) {
    for (size_t i = 0; i < n; ++i) x.push_back(v[i] + guess[i]);
  } else {
    for (size_t i = 0; i < n; ++i) x.push_back(v[i]);
  }
  for (size_t i = 0; i < nbn; ++i) x.push_back(ball_v[i]);
  for (size_t i = 0; i < nbn; ++i) x.push_back(Vec2(ball_w[i], Real(0.0)));
  std::vector<Vec2> b;
  b.reserve(len);
  for (size_t i = 0; i < n; ++i) b.push_back(mass * v[i]);
  for (size_t i = 0; i < nbn; ++i) b.push_back(ball_mass_ * ball_v[i]);
  for (size_t i = 0; i < nbn; ++i) b.push_back(Vec2(ball_inertia_ * ball_w[i], Real(0.0)));
  std::vector<Real> diag(len, Real(0.0));
  for (size_t i = 0; i < n; ++i) {
    Real sw = Real(0.0);
    for (size_t k = nb.b(i); k < nb.e(i); ++k) sw += weights.w[k];
    diag[i] = mass * (Real(1.0) + dt * viscosity_diag(sw));
  }
  for (size_t bi = 0; bi < nbn; ++bi) { diag[n + bi] = ball_mass_; diag[n + nbn + bi] = ball_inertia_; }
  for (const auto& g : groups) {
    Real d = dt * mass * g.c;
    diag[g.fluid] += d;
    diag[n + g.ball] += d;
    diag[n + nbn + g.ball] += dt * mass * g.lever2_c;
  }
  for (const auto& l : links) {
    Real d = dt * l.c;
    diag[n + l.ball] += d;
    if (l.other != WALL_ID) diag[n + l.other] += d;
  }
  std::vector<Real> inv_diag(len);
  for (size_t i = 0; i < len; ++i) inv_diag[i] = Real(1.0) / fmax_r(diag[i], Real(1e-20));
  std::vector<Vec2> lv(n);
  auto apply = [&](const std::vector<Vec2>& xx, std::vector<Vec2>& out) {
    laplacian_apply_into(nb, weights, xx.data(), n, lv.data());
    for (size_t i = 0; i < n; ++i) out[i] = mass * (xx[i] + dt * lv[i]);
    for (size_t bi = 0; bi < nbn; ++bi) {
      out[n + bi] = ball_mass_ * xx[n + bi];
      out[n + nbn + bi] = Vec2(ball_inertia_ * xx[n + nbn + bi].x, Real(0.0));
    }
    for (const auto& g : groups) {
      size_t i = g.fluid, bi = g.ball;
      Vec2 vb = xx[n + bi];
      Real w = xx[n + nbn + bi].x;
      Vec2 rel = xx[i] - vb;
      Real k = dt * mass;
      Vec2 d = k * (g.c * rel - w * perp(g.lever_c));
      out[i] += d;
      out[n + bi] -= d;
      out[n + nbn + bi].x -= k * (cross2(g.lever_c, rel) - w * g.lever2_c);
    }
    for (const auto& l : links) {
      size_t i = l.ball;
      Vec2 rel = xx[n + l.ball];
      if (l.other != WALL_ID) rel = rel - xx[n + l.other];
      Vec2 d = (dt * l.c * l.n.dot(rel)) * l.n;
      out[n + i] += d;
      if (l.other != WALL_ID) out[n + l.other] -= d;
    }
  };
  auto res_norm_f = [&](const std::vector<Vec2>& r) {
    Real s = Real(0.0);
    for (size_t i = 0; i < r.size(); ++i) s += inv_diag[i] * r[i].length_squared();
    return std::sqrt(s);
  };
  auto res_norm_d = [&](const std::vector<Vec2>& r) {
    double s = 0.0;
    for (size_t i = 0; i < r.size(); ++i)
      s += (double)inv_diag[i] * ((double)r[i].x * (double)r[i].x + (double)r[i].y * (double)r[i].y);
    return std::sqrt(s);
  };
  std::vector<Vec2> ax(len);
  apply(x, ax);
  std::vector<Vec2> r(len), z(len);
  for (size_t i = 0; i < len; ++i) r[i] = b[i] - ax[i];
  for (size_t i = 0; i < len; ++i) z[i] = r[i] * inv_diag[i];
  uint32_t iters = 0;
  if (!fp64) {
    Real b_norm = res_norm_f(b);
    if (b_norm > Real(0.0) && std::isfinite(b_norm) && res_norm_f(r) > VISCOSITY_CG_TOLERANCE * b_norm) {
      Real target = VISCOSITY_CG_TOLERANCE * b_norm;
      std::vector<Vec2> p = z, ap(len);
      Real rz_old = dot_f32(r, z);
      for (uint32_t iter = 1; iter <= 4 * VISCOSITY_CG_MAX_ITERS; ++iter) {
        iters = iter;
        apply(p, ap);
        Real p_ap = dot_f32(p, ap);
        if (p_ap <= Real(0.0) || !std::isfinite(p_ap)) break;
        Real alpha = rz_old / p_ap;
        for (size_t i = 0; i < len; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * ap[i]; }
        if (res_norm_f(r) <= target) break;
        for (size_t i = 0; i < len; ++i) z[i] = r[i] * inv_diag[i];
        Real rz_new = dot_f32(r, z);
        Real beta = rz_new / rz_old;
        for (size_t i = 0; i < len; ++i) p[i] = z[i] + beta * p[i];
        rz_old = rz_new;
      }
    }
  } else {
    double b_norm = res_norm_d(b);
    if (b_norm > 0.0 && std::isfinite(b_norm) && res_norm_d(r) > (double)VISCOSITY_CG_TOLERANCE * b_norm) {
      double target = (double)VISCOSITY_CG_TOLERANCE * b_norm;
      std::vector<Vec2> p = z, ap(len);
      double rz_old = dot_f64(r, z);
      for (uint32_t iter = 1; iter <= 4 * VISCOSITY_CG_MAX_ITERS; ++iter) {
        iters = iter;
        apply(p, ap);
        double p_ap = dot_f64(p, ap);
        if (p_ap <= 0.0 || !std::isfinite(p_ap)) break;
        Real alpha = (Real)(rz_old / p_ap);
        for (size_t i = 0; i < len; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * ap[i]; }
        if (res_norm_d(r) <= target) break;
        for (size_t i = 0; i < len; ++i) z[i] = r[i] * inv_diag[i];
        double rz_new = dot_f64(r, z);
        Real beta = (Real)(rz_new / rz_old);
        for (size_t i = 0; i < len; ++i) p[i] = z[i] + beta * p[i];
        rz_old = rz_new;
      }
    }
  }
  for (size_t i = 0; i < n; ++i) v[i] = x[i];
  for (size_t i = 0; i < nbn; ++i) ball_v[i] = x[n + i];
  for (size_t i = 0; i < nbn; ++i) ball_w[i] = x[n + nbn + i].x;
  return iters;
}

// pbf.rs:800-868
static std::vector<Real> shear_rates(const std::vector<Vec2>& x, const std::vector<Vec2>& v, const Nbr& nb,
                                      const std::vector<Real>& density, Real mass, Real h) {
  size_t n = x.size();
  std::vector<Real> out(n, Real(0.0));
  for (size_t i = 0; i < n; ++i) {
    Real gxx = Real(0.0), gxy = Real(0.0), gyx = Real(0.0), gyy = Real(0.0);
    for (size_t k = nb.b(i); k < nb.e(i); ++k) {
      size_t ju = nb.idx[k];
      Vec2 delta = x[i] - x[ju];
      Real r = delta.length();
      Vec2 grad = spiky_grad(delta, r, h);
      Real coeff = mass / fmax_r(density[ju], Real(1e-6));
      Vec2 dv = v[ju] - v[i];
      gxx += coeff * dv.x * grad.x;
      gxy += coeff * dv.x * grad.y;
      gyx += coeff * dv.y * grad.x;
      gyy += coeff * dv.y * grad.y;
    }
    Real dxy = Real(0.5) * (gxy + gyx);
    out[i] = std::sqrt(Real(2.0) * (gxx * gxx + gyy * gyy + Real(2.0) * dxy * dxy));
  }
  return out;
}
static Real mean_shear_rate(const std::vector<Vec2>& x, const std::vector<Vec2>& v, const Nbr& nb,
                             const std::vector<Real>& density, Real mass, Real h) {
  std::vector<Real> rates = shear_rates(x, v, nb, density, mass, h);
  Real sum = Real(0.0);
  uint32_t count = 0;
  for (Real g : rates)
    if (std::isfinite(g)) { sum += g; count += 1; }
  return count == 0 ? Real(0.0) : sum / (Real)count;
}
static std::vector<Real> bingham_viscosity(const std::vector<Real>& rates, Real mu, Real tau_y) {
  Real gamma0 = tau_y / (BINGHAM_PLASTIC_RATIO * mu);
  std::vector<Real> out(rates.size());
  for (size_t i = 0; i < rates.size(); ++i) {
    Real g = std::isfinite(rates[i]) ? rates[i] : Real(0.0);
    Real extra = g < Real(1e-4) * gamma0 ? tau_y / gamma0 : tau_y * (Real(1.0) - expf_r(-g / gamma0)) / g;
    out[i] = mu + extra;
  }
  return out;
}

// pbf.rs:924-926, 957-996
static double kinetic_energy_f64(const std::vector<Vec2>& v, Real mass) {
  double s = 0.0;
  for (const Vec2& q : v) s += (double)q.length_squared();
  return 0.5 * (double)mass * s;
}
static Real impulse_clamp(Real ball_mass_, Real dt) { return F_CLAMP_G_MULTIPLE * ball_mass_ * Real(9.81) * dt; }
static Real fluid_speed_clamp_v_max(const Drum& d) {
  return FLUID_SPEED_SAFETY_FACTOR * (std::fabs(d.omega) * d.radius_m + std::sqrt(Real(4.0) * std::fabs(GRAVITY) * d.radius_m));
}
static void clamp_fluid_speed(std::vector<Vec2>* v, Real v_max) {
  for (Vec2& q : *v) {
    Real speed = q.length();
    if (!std::isfinite(speed)) q = Vec2();
    else if (speed > v_max) q *= v_max / speed;
  }
}

// pbf.rs:1124-1150
std::vector<Real> fluid_densities(const Fluid& f) {
  size_t n = f.len();
  std::vector<Real> density(n, Real(0.0));
  if (n == 0) return density;
  UniformGrid g = UniformGrid::build(f.x, f.h);
  Real self_c = f.particle_mass * poly6(Real(0.0), f.h);
  std::fill(density.begin(), density.end(), self_c);
  g.for_each_candidate_pair([&](uint32_t i, uint32_t j) {
    Real r2 = (f.x[i] - f.x[j]).length_squared();
    Real w = poly6(r2, f.h);
    density[i] += f.particle_mass * w;
    density[j] += f.particle_mass * w;
  });
  return density;
}
double fluid_mechanical_energy(const Fluid& f) {
  double py = 0.0;
  for (const Vec2& p : f.x) py += (double)p.y;
  double potential = py * (double)f.particle_mass * (double)std::fabs(GRAVITY);
  return kinetic_energy_f64(f.v, f.particle_mass) + potential;
}

// pbf.rs:1174-2365
void fluid_step_coupled(Fluid* fl, const Drum& drum, Real drum_angle, const SlurryParams& slurry,
                        uint32_t iterations, Real dt, const Balls& balls, CouplingImpulses* coupling,
                        FluidStepStats* stats_out, StepCounters* ctr, Debug* dbg, const SolveOptions& opt) {
  size_t n = fl->len();
  coupling->zeros(balls.len());
  *stats_out = FluidStepStats();
  if (n == 0 || dt <= Real(0.0)) return;
  std::vector<Vec2>& X = fl->x;
  std::vector<Vec2>& V = fl->v;
  // step 0: sanitize
  for (size_t i = 0; i < n; ++i)
    if (!X[i].is_finite() || !V[i].is_finite()) { X[i] = Vec2(); V[i] = Vec2(); }
  Real h = fl->h, rest_density = fl->rest_density, mass = fl->particle_mass;
  bool have_ball_grid = balls.len() > 0;
  UniformGrid ball_grid;
  if (have_ball_grid) {
    Real contact_radius = balls.radius + OVERLAP_PUSH_MARGIN * h;
    ball_grid = UniformGrid::build(balls.x, fmax_r(fmax_r(Real(2.0) * balls.radius, contact_radius), Real(1e-6)));
  }
  // step 1: predict
  std::vector<Vec2> x0 = X;
  for (size_t i = 0; i < n; ++i) {
    V[i].y += GRAVITY * dt;
    X[i] += V[i] * dt;
  }
  Real drum_angle_next = drum_angle + drum.omega * dt;
  // step 2: grid + neighbour lists
  UniformGrid grid = UniformGrid::build(X, h);
  Nbr nb;
  {
    std::vector<std::pair<uint32_t, uint32_t>> edges;
    grid.for_each_candidate_pair([&](uint32_t i, uint32_t j) {
      if ((X[i] - X[j]).length_squared() <= h * h) { edges.push_back({i, j}); edges.push_back({j, i}); }
    });
    nb.off.assign(n + 1, 0);
    for (auto& e : edges) nb.off[e.first + 1] += 1;
    for (size_t k = 1; k < nb.off.size(); ++k) nb.off[k] += nb.off[k - 1];
    std::vector<uint32_t> cursor = nb.off;
    nb.idx.assign(edges.size(), 0);
    for (auto& e : edges) { nb.idx[cursor[e.first]] = e.second; cursor[e.first] += 1; }
  }
  if (ctr) ctr->n_fluid_edges = (uint32_t)nb.idx.size();
  if (dbg) { dbg->nbr_offsets = nb.off; dbg->nbrs = nb.idx; }
  // step 3: density constraint iterations
  std::vector<Real> density(n, Real(0.0)), lambda(n, Real(0.0));
  std::vector<Vec2> delta_p(n), grad_cache(nb.idx.size());
  uint32_t base_iterations = std::max(iterations, 1u);
  uint32_t iter_count = 0;
  for (;;) {
    Real max_c = Real(0.0);
    for (size_t i = 0; i < n; ++i) {
      Real rho = mass * poly6(Real(0.0), h);
      Vec2 grad_self;
      Real sum_grad_sq = Real(0.0);
      for (size_t k = nb.b(i); k < nb.e(i); ++k) {
        size_t ju = nb.idx[k];
        Vec2 delta = X[i] - X[ju];
        Real r2 = delta.length_squared();
        rho += mass * poly6(r2, h);
        Real r = delta.length();
        Vec2 raw_grad = spiky_grad(delta, r, h);
        grad_cache[k] = raw_grad;
        Vec2 grad = raw_grad * (mass / rest_density);
        grad_self += grad;
        sum_grad_sq += grad.length_squared();
      }
      density[i] = rho;
      Real c_i = fmax_r(density[i] / rest_density - Real(1.0), Real(0.0));
      max_c = fmax_r(max_c, c_i);
      sum_grad_sq += grad_self.length_squared();
      lambda[i] = -c_i / (sum_grad_sq + EPSILON_RELAX);
    }
    for (size_t i = 0; i < n; ++i) {
      Vec2 sum;
      for (size_t k = nb.b(i); k < nb.e(i); ++k) {
        size_t ju = nb.idx[k];
        sum += (lambda[i] + lambda[ju]) * grad_cache[k];
      }
      delta_p[i] = sum * (mass / rest_density);
    }
    for (size_t i = 0; i < n; ++i) X[i] += delta_p[i];
    iter_count += 1;
    bool converged = max_c <= COMPRESSION_CONVERGENCE_TOLERANCE;
    if ((iter_count >= base_iterations && converged) || iter_count >= base_iterations + ADAPTIVE_MAX_EXTRA_ITERATIONS)
      break;
  }
  if (ctr) ctr->density_iters = iter_count;
  // step 3.5: ball overlap push
  std::vector<Vec2> push_velocity_excess(n);
  if (have_ball_grid) {
    Real contact_radius = balls.radius + OVERLAP_PUSH_MARGIN * h;
    std::vector<uint32_t> nearby;
    for (size_t i = 0; i < n; ++i) {
      nearby.clear();
      ball_grid.for_each_near(X[i], [&](uint32_t b) { nearby.push_back(b); });
      for (uint32_t bb : nearby) {
        size_t b = bb;
        Vec2 delta = X[i] - balls.x[b];
        Real dist = delta.length();
        if (std::isnan(dist) || dist >= contact_radius) continue;
        Vec2 n_hat = dist > Real(1e-9) ? delta / dist : Vec2(Real(1.0), Real(0.0));
        Real push_mag = fmin_r(contact_radius - dist, Real(0.5) * balls.radius);
        Vec2 push = push_mag * n_hat;
        X[i] += push;
        Vec2 lever = n_hat * balls.radius;
        Vec2 v_surface = balls.v[b] + balls.omega[b] * Vec2(-lever.y, lever.x);
        Real arrest_speed = fmax_r(-(V[i] - v_surface).dot(n_hat), Real(0.0));
        Real full_impulse_mag = mass * push_mag / dt;
        Real reduced_mass = balls.mass > Real(0.0) ? (mass * balls.mass) / (mass + balls.mass) : mass;
        Real impulse_mag = fmin_r(full_impulse_mag, reduced_mass * arrest_speed);
        push_velocity_excess[i] += ((full_impulse_mag - impulse_mag) / mass) * n_hat;
        Vec2 reaction = -impulse_mag * n_hat;
        coupling->impulses[b] += reaction;
        coupling->fluid_momentum_change += impulse_mag * n_hat;
        coupling->angular_impulses[b] += cross2(lever, reaction);
      }
    }
  }
  // step 3.6a: cohesion
  std::vector<Vec2> cohesion_dv(n);
  Real cohesion_accel = (fmax_r((Real)slurry.surface_tension_n_m, Real(0.0)) / REFERENCE_SURFACE_TENSION_N_M) *
                         COHESION_ACCEL_FACTOR * std::fabs(GRAVITY);
  if (cohesion_accel > Real(0.0)) {
    for (size_t i = 0; i < n; ++i) {
      Vec2 pull;
      for (size_t k = nb.b(i); k < nb.e(i); ++k) {
        size_t ju = nb.idx[k];
        Vec2 delta = X[i] - X[ju];
        Real r = delta.length();
        if (r <= Real(1e-9)) continue;
        Real w = mass * cohesion_kernel(r, h) / rest_density;
        pull -= w * (delta / r);
      }
      cohesion_dv[i] = cohesion_accel * pull * dt;
    }
  }
  // step 3.6b: adhesion (queries the stale step-2 grid)
  std::vector<Vec2> adhesion_dv(n);
  Real wettability = clamp_r((Real)slurry.wettability, Real(0.0), Real(1.0));
  if (wettability > Real(0.0) && balls.len() > 0 && balls.radius > Real(0.0)) {
    Real dx = Real(0.5) * h;
    Real h_adh = fmin_r(h, Real(2.0) * balls.radius);
    std::vector<Vec2> bpos = ball_boundary_particles(balls, dx);
    size_t count_per_ball = boundary_points_per_ball(balls.radius, dx);
    if (!bpos.empty() && h_adh > Real(0.0)) {
      Real adhesion_accel = wettability * ADHESION_ACCEL_FACTOR * std::fabs(GRAVITY);
      struct Item { size_t j; Vec2 dir; Real w; };
      std::vector<Item> items;
      std::vector<uint32_t> slot(n, UINT32_MAX);
      std::vector<uint32_t> nearby;
      Real range2 = h_adh * h_adh * (Real(1.0) + Real(1e-4));
      Real inner2 = Real(0.25) * h_adh * h_adh * (Real(1.0) - Real(1e-4));
      for (size_t b = 0; b < balls.len(); ++b) {
        if (!balls.x[b].is_finite()) continue;
        size_t start = b * count_per_ball;
        size_t end = std::min(start + count_per_ball, bpos.size());
        items.clear();
        for (size_t q = start; q < end; ++q) {
          Vec2 bp = bpos[q];
          nearby.clear();
          grid.for_each_near(bp, [&](uint32_t j) { nearby.push_back(j); });
          for (uint32_t jj : nearby) {
            size_t ju = jj;
            Vec2 delta = bp - X[ju];
            Real r2 = delta.length_squared();
            if (r2 >= range2 || r2 <= inner2) continue;
            Real r = std::sqrt(r2);
            if (!std::isfinite(r) || r <= Real(0.5) * h_adh || r >= h_adh) continue;
            Real w = mass * adhesion_kernel(r, h_adh) / rest_density;
            if (w <= Real(0.0)) continue;
            Vec2 n_hat = delta / r;
            if (slot[ju] == UINT32_MAX) {
              slot[ju] = (uint32_t)items.size();
              items.push_back({ju, w * n_hat, w});
            } else {
              Item& it = items[slot[ju]];
              it.dir += w * n_hat;
              it.w += w;
            }
          }
        }
        for (auto& it : items) slot[it.j] = UINT32_MAX;
        if (items.empty()) continue;
        Real weight_sum = Real(0.0);
        Vec2 dir_sum;
        for (auto& it : items) { dir_sum += it.dir; weight_sum += it.w; }
        if (weight_sum <= Real(1e-9)) continue;
        Real pull_len = dir_sum.length();
        if (pull_len <= Real(1e-9)) continue;
        Vec2 ball_pull_dir = -dir_sum / pull_len;
        Real coverage = fmin_r(weight_sum, Real(1.0));
        Real m_contrib = mass * weight_sum;
        Real attach = m_contrib / (balls.mass + m_contrib);
        Vec2 dv_b = ball_pull_dir * (adhesion_accel * coverage * dt * attach);
        coupling->impulses[b] += balls.mass * dv_b;
        Vec2 lever = ball_pull_dir * balls.radius;
        coupling->angular_impulses[b] += balls.mass * cross2(lever, dv_b);
        for (auto& it : items) {
          Real frac = it.w / weight_sum;
          Vec2 dv_i = -(balls.mass * frac / mass) * dv_b;
          adhesion_dv[it.j] += dv_i;
          coupling->fluid_momentum_change += mass * dv_i;
        }
      }
    }
  }
  // step 4: wall projection
  std::vector<uint8_t> touched(n, 0);
  double acct_wall_impulse[2] = {0.0, 0.0};
  double acct_wall_angular = 0.0;
  Real acct_wall_bins[WALL_IMPULSE_BINS] = {};
  for (size_t i = 0; i < n; ++i) {
    Real d;
    Vec2 normal;
    drum.sdf_world(X[i], drum_angle_next, &d, &normal);
    if (d < Real(0.0)) {
      X[i] += -d * normal;
      touched[i] = 1;
      Vec2 push = mass * (-d * normal) / dt;
      acct_wall_impulse[0] += (double)push.x;
      acct_wall_impulse[1] += (double)push.y;
      acct_wall_angular += (double)cross2(X[i], push);
      Real angle = atan2f_r(X[i].y, X[i].x);
      size_t bin = f2u_sat(((angle + PI_F) / TAU_F) * (Real)WALL_IMPULSE_BINS);
      acct_wall_bins[std::min(bin, (size_t)WALL_IMPULSE_BINS - 1)] += mass * -d / dt;
    }
  }
  // step 5: velocity reconstruction
  for (size_t i = 0; i < n; ++i) V[i] = (X[i] - x0[i]) / dt;
  for (size_t i = 0; i < n; ++i) V[i] -= push_velocity_excess[i];
  for (size_t i = 0; i < n; ++i) V[i] += cohesion_dv[i];
  for (size_t i = 0; i < n; ++i) V[i] += adhesion_dv[i];
  // step 6: wall no-slip
  Real beta = clamp_r((Real)slurry.wall_no_slip, Real(0.0), Real(1.0));
  Real wall_work_j = Real(0.0);
  double ke_before_noslip = kinetic_energy_f64(V, mass);
  if (beta > Real(0.0)) {
    for (size_t i = 0; i < n; ++i) {
      if (!touched[i]) continue;
      Vec2 v_wall = drum.wall_velocity(X[i]);
      Vec2 v_old = V[i];
      V[i] = (Real(1.0) - beta) * v_old + beta * v_wall;
      Vec2 dv = V[i] - v_old;
      wall_work_j += mass * dv.dot(v_wall);
      acct_wall_impulse[0] += (double)(mass * dv.x);
      acct_wall_impulse[1] += (double)(mass * dv.y);
      acct_wall_angular += (double)cross2(X[i], mass * dv);
    }
  }
  double ke_mark = kinetic_energy_f64(V, mass);
  double ke_delta_noslip = ke_mark - ke_before_noslip;
  // step 6.5: ball drag (Gauss-Seidel over balls)
  Real mu = fmax_r((Real)slurry.viscosity_pa_s, Real(0.0));
  if (balls.len() > 0 && balls.radius > Real(0.0) && balls.true_radius > Real(0.0) && mu > Real(1e-6)) {
    Real beta_b = clamp_r((Real)slurry.ball_no_slip, Real(0.0), Real(1.0));
    Real rot_cap = Real(0.2) * fluid_speed_clamp_v_max(drum);
    Real rho_ball = balls.mass / (PI_F * balls.radius * balls.radius);
    Real mass_true = rho_ball * PI_F * balls.true_radius * balls.true_radius;
    Real inv_tau_stokes = Real(0.0);
    if (beta_b > Real(0.0)) {
      Real h_c = balls.radius + h;
      Real w_hc0 = fmax_r(poly6(Real(0.0), h_c), Real(1e-12));
      UniformGrid cgrid = UniformGrid::build(X, fmax_r(h_c, Real(1e-6)));
      Real i_b = balls.inertia;
      std::vector<uint32_t> nearby;
      struct Item { size_t j; Vec2 r_i; Real phi; };
      std::vector<Item> items;
      for (size_t b = 0; b < balls.len(); ++b) {
        if (!balls.x[b].is_finite()) continue;
        nearby.clear();
        cgrid.for_each_near(balls.x[b], [&](uint32_t j) { nearby.push_back(j); });
        if (nearby.empty()) continue;
        items.clear();
        Real m_ent = Real(0.0), i_ent = Real(0.0), l_sum = Real(0.0);
        Vec2 r_sum, v_sum;
        for (uint32_t jj : nearby) {
          size_t ju = jj;
          Vec2 r_i = X[ju] - balls.x[b];
          Real r2 = r_i.length_squared();
          if (!std::isfinite(r2) || r2 >= h_c * h_c) continue;
          Real phi = poly6(r2, h_c) / w_hc0;
          if (phi <= Real(0.0)) continue;
          Real w = mass * phi;
          m_ent += w;
          r_sum += w * r_i;
          v_sum += w * V[ju];
          i_ent += w * r2;
          l_sum += w * cross2(r_i, V[ju]);
          items.push_back({ju, r_i, phi});
        }
        if (ctr) ctr->n_coupling_items += (uint32_t)items.size();
        if (m_ent <= Real(1e-12) || items.empty()) continue;
        Vec2 r_bar = r_sum / m_ent;
        Vec2 v_bar = v_sum / m_ent;
        Vec2 v_rel = v_bar - balls.v[b];
        Real speed_rel = v_rel.length();
        Real inv_tau_form = (speed_rel > Real(1e-6) && rest_density > Real(0.0))
                                 ? Real(0.5) * rest_density * BALL_FORM_DRAG_COEFFICIENT * (Real(2.0) * balls.true_radius) *
                                       speed_rel / mass_true
                                 : Real(0.0);
        Real bt = beta_b * (Real(1.0) - expf_r(-dt * (inv_tau_stokes + inv_tau_form)));
        Real a_lin = bt * m_ent / (balls.mass + m_ent);
        Vec2 dv_b = a_lin * v_rel;
        Real dw_b = Real(0.0), c_rot = Real(0.0);
        Vec2 p_bar;
        if (i_ent > Real(1e-12)) {
          Real omega_bar = l_sum / i_ent;
          Real a_rot = bt * i_ent / (i_b + i_ent);
          Real candidate_dw = a_rot * (omega_bar - balls.omega[b]);
          p_bar = Vec2(-r_bar.y, r_bar.x);
          Real s = Real(0.0), s_scale = Real(0.0);
          for (auto& it : items) {
            Vec2 perp_i(-it.r_i.y, it.r_i.x);
            Real phi2 = it.phi * it.phi;
            s += mass * phi2 * cross2(it.r_i, perp_i - p_bar);
            s_scale += mass * phi2 * it.r_i.length_squared();
          }
          if (std::fabs(s) > Real(0.1) * s_scale) {
            Real raw_c_rot = -i_b * candidate_dw / s;
            Real max_lever = Real(2.0) * h_c;
            Real c_rot_cap = max_lever > Real(1e-9) ? rot_cap / max_lever : Real(0.0);
            c_rot = clamp_r(raw_c_rot, -c_rot_cap, c_rot_cap);
            dw_b = -c_rot * s / i_b;
          }
        }
        for (auto& it : items) {
          Vec2 dv_i = -(balls.mass / m_ent) * dv_b * it.phi;
          if (c_rot != Real(0.0)) {
            Vec2 perp_i(-it.r_i.y, it.r_i.x);
            dv_i += c_rot * it.phi * (perp_i - p_bar);
          }
          V[it.j] += dv_i;
          coupling->fluid_momentum_change += mass * dv_i;
        }
        coupling->impulses[b] += balls.mass * dv_b;
        coupling->angular_impulses[b] += i_b * dw_b + balls.mass * cross2(r_bar, dv_b);
      }
    }
  }
  double ke_after_drag = kinetic_energy_f64(V, mass);
  double ke_delta_drag = ke_after_drag - ke_mark;
  ke_mark = ke_after_drag;
  // step 6.6: buoyancy (Gauss-Seidel over balls on the stale step-2 grid)
  if (balls.len() > 0 && balls.radius > Real(0.0)) {
    Real area = PI_F * balls.radius * balls.radius;
    std::vector<uint32_t> nearby;
    std::vector<std::pair<size_t, Real>> weights;
    for (size_t b = 0; b < balls.len(); ++b) {
      if (!balls.x[b].is_finite()) continue;
      nearby.clear();
      grid.for_each_near(balls.x[b], [&](uint32_t j) { nearby.push_back(j); });
      if (nearby.empty()) continue;
      Real rho_local = Real(0.0);
      weights.clear();
      for (uint32_t jj : nearby) {
        size_t ju = jj;
        Real r2 = (balls.x[b] - X[ju]).length_squared();
        Real w = mass * poly6(r2, h);
        if (w > Real(0.0)) { rho_local += w; weights.push_back({ju, w}); }
      }
      if (ctr && rho_local > Real(0.0)) ctr->n_coupling_items += (uint32_t)weights.size();
      if (rho_local <= Real(0.0)) continue;
      Real rho_eff = fmin_r(rho_local, rest_density);
      Real omega_num = Real(0.0), omega_den = Real(0.0);
      for (auto& jw : weights) {
        Vec2 d = X[jw.first];
        Real d2 = d.length_squared();
        if (d2 <= Real(1e-12)) continue;
        omega_num += jw.second * cross2(d, V[jw.first]) / d2;
        omega_den += jw.second;
      }
      Real omega_local = omega_den > Real(0.0)
                              ? clamp_r(omega_num / omega_den, -std::fabs(drum.omega), std::fabs(drum.omega))
                              : Real(0.0);
      Vec2 g_vec(Real(0.0), GRAVITY);
      Vec2 centripetal = omega_local * omega_local * balls.x[b];
      Vec2 g_eff = g_vec + centripetal;
      Vec2 impulse_on_ball = -rho_eff * area * g_eff * dt;
      coupling->impulses[b] += impulse_on_ball;
      for (auto& jw : weights) {
        Real frac = jw.second / rho_local;
        Vec2 dv = -(impulse_on_ball * frac) / mass;
        V[jw.first] += dv;
        coupling->fluid_momentum_change += mass * dv;
      }
    }
  }
  double ke_after_buoy = kinetic_energy_f64(V, mass);
  double ke_delta_buoy = ke_after_buoy - ke_mark;
  ke_mark = ke_after_buoy;
  // density recompute at final x over the step-2 neighbour lists
  uint32_t viscosity_iterations = 0;
  for (size_t i = 0; i < n; ++i) {
    Real rho = mass * poly6(Real(0.0), h);
    for (size_t k = nb.b(i); k < nb.e(i); ++k) {
      Real r2 = (X[i] - X[nb.idx[k]]).length_squared();
      rho += mass * poly6(r2, h);
    }
    density[i] = rho;
  }
  // step 7: implicit viscosity
  if (mu > Real(0.0)) {
    std::vector<Real> mu_eff;
    if (slurry.rheology == RHEO_BINGHAM && slurry.yield_stress_pa > Real(0.0)) {
      mu_eff = bingham_viscosity(shear_rates(X, V, nb, density, mass, h), mu, slurry.yield_stress_pa);
    } else {
      mu_eff.assign(n, mu);
    }
    ViscWeights weights = morris_weights(X, nb, density, mass, mu_eff, h);
    std::vector<BoundaryGroup> groups;
    if (balls.len() > 0 && balls.radius > Real(0.0)) {
      Real dx = Real(0.5) * h;
      size_t count = boundary_points_per_ball(balls.radius, dx);
      std::vector<Vec2> pts = ball_boundary_particles(balls, dx);
      UniformGrid grid_now = UniformGrid::build(X, h);
      Real eta2 = VISCOSITY_ETA_FACTOR * h * h;
      Real spiky_norm = -Real(30.0) / (PI_F * powi5(h));
      Real range2 = h * h * (Real(1.0) + Real(1e-4));
      std::vector<Real> fluid_factor(n);
      for (size_t j = 0; j < n; ++j)
        fluid_factor[j] = BALL_BC_GAIN * (mass * Real(2.0) * mu_eff[j] / (fmax_r(density[j], Real(1e-6)) * rest_density));
      std::vector<uint32_t> slot(n, UINT32_MAX);
      size_t group_start = 0, current_ball = SIZE_MAX;
      for (size_t k = 0; k < pts.size(); ++k) {
        Vec2 bp = pts[k];
        size_t bi = k / count;
        if (bi != current_ball) {
          for (size_t g = group_start; g < groups.size(); ++g) slot[groups[g].fluid] = UINT32_MAX;
          group_start = groups.size();
          current_ball = bi;
        }
        if (!balls.x[bi].is_finite()) continue;
        grid_now.for_each_near(bp, [&](uint32_t j) {
          Vec2 delta = X[j] - bp;
          Real r2 = delta.length_squared();
          if (r2 >= range2) return;
          Real r = std::sqrt(r2);
          if (!std::isfinite(r) || r >= h || r <= Real(1e-9)) return;
          Real dot_abs = std::fabs(spiky_norm * (h - r) * (h - r) * r);
          Real c = fluid_factor[j] * dot_abs / (r2 + eta2);
          if (c > Real(0.0)) {
            Vec2 lever = bp - balls.x[bi];
            Vec2 lever_c = c * lever;
            Real lever2_c = c * lever.length_squared();
            uint32_t s = slot[j];
            if (s == UINT32_MAX) {
              slot[j] = (uint32_t)groups.size();
              groups.push_back({j, (uint32_t)bi, c, lever_c, lever2_c});
            } else {
              BoundaryGroup& g = groups[s];
              g.c += c;
              g.lever_c += lever_c;
              g.lever2_c += lever2_c;
            }
          }
        });
      }
    }
    std::vector<Vec2> ball_v0(balls.len());
    for (size_t bi = 0; bi < balls.len(); ++bi) ball_v0[bi] = balls.v[bi] + coupling->impulses[bi] / balls.mass;
    size_t links_in_range = 0;
    std::vector<SqueezeLink> links = squeeze_links(balls, drum.radius_m, Real(0.5) * h, mu, dt, &ball_v0, &links_in_range);
    if (ctr) {
      ctr->n_groups = (uint32_t)groups.size();
      ctr->n_links = (uint32_t)links.size();
      ctr->links_in_range = (uint32_t)links_in_range;
    }
    if (groups.empty() && links_in_range == 0) {
      viscosity_iterations = solve_implicit_viscosity(nb, weights, &V, dt, opt.cg_fp64 != 0);
    } else {
      std::vector<Vec2> ball_v = ball_v0;
      std::vector<Real> ball_w(balls.len());
      for (size_t bi = 0; bi < balls.len(); ++bi)
        ball_w[bi] = balls.omega[bi] + coupling->angular_impulses[bi] / balls.inertia;
      std::vector<Real> ball_w0 = ball_w;
      std::vector<Vec2> guess;
      guess.swap(fl->viscous_guess);
      std::vector<Vec2> v_in = V;
      viscosity_iterations = solve_viscosity_with_balls(nb, weights, groups, links, mass, balls.mass, balls.inertia,
                                                        dt, guess, &V, &ball_v, &ball_w, opt.cg_fp64 != 0);
      fl->viscous_guess.resize(n);
      for (size_t i = 0; i < n; ++i) {
        Vec2 d = V[i] - v_in[i];
        fl->viscous_guess[i] = d.is_finite() ? d : Vec2();
      }
      for (size_t bi = 0; bi < balls.len(); ++bi) {
        Vec2 dv = ball_v[bi] - ball_v0[bi];
        Real dw = ball_w[bi] - ball_w0[bi];
        if (dv.is_finite() && std::isfinite(dw)) {
          coupling->impulses[bi] += balls.mass * dv;
          coupling->angular_impulses[bi] += balls.inertia * dw;
          coupling->fluid_momentum_change -= balls.mass * dv;
        }
      }
    }
  }
  if (ctr) ctr->cg_iters = viscosity_iterations;
  Real mean_shear = mean_shear_rate(X, V, nb, density, mass, h);
  double ke_after_visc = kinetic_energy_f64(V, mass);
  double ke_delta_visc = ke_after_visc - ke_mark;
  clamp_fluid_speed(&V, fluid_speed_clamp_v_max(drum));
  double ke_delta_clamp = kinetic_energy_f64(V, mass) - ke_after_visc;
  // step 8: impulse clamp
  if (balls.len() > 0) {
    Real clamp = impulse_clamp(balls.mass, dt);
    Real angular_clamp = clamp * balls.radius;
    for (size_t b = 0; b < balls.len(); ++b) {
      Real mag = coupling->impulses[b].length();
      if (mag > clamp && mag > Real(1e-9)) {
        coupling->impulses[b] *= clamp / mag;
        coupling->clamp_hits += 1;
      }
      coupling->angular_impulses[b] = clamp_r(coupling->angular_impulses[b], -angular_clamp, angular_clamp);
    }
  }
  FluidStepStats& st = *stats_out;
  st.viscosity_iterations = viscosity_iterations;
  st.mean_shear_rate_per_s = mean_shear;
  st.coupling_clamp_hits = coupling->clamp_hits;
  st.wall_work_j = wall_work_j;
  st.wall_impulse[0] = (Real)acct_wall_impulse[0];
  st.wall_impulse[1] = (Real)acct_wall_impulse[1];
  st.wall_angular_impulse = (Real)acct_wall_angular;
  for (int k = 0; k < WALL_IMPULSE_BINS; ++k) st.wall_normal_impulse_by_angle[k] = acct_wall_bins[k];
  st.ke_delta_noslip_j = (Real)ke_delta_noslip;
  st.ke_delta_drag_j = (Real)ke_delta_drag;
  st.ke_delta_buoyancy_j = (Real)ke_delta_buoy;
  st.ke_delta_viscosity_j = (Real)ke_delta_visc;
  st.ke_delta_clamp_j = (Real)ke_delta_clamp;
}

// ------------------------------------------------------------------ dem.rs
static const Real RESTITUTION_VELOCITY_THRESHOLD = Real(0.02);
static const Real RESTITUTION_THRESHOLD_FROUDE = Real(0.1428);
static const Real MAX_RECOVERY_FRACTION = Real(0.2);
static const Real CCD_CONTACT_SKIN_FRACTION = Real(1e-2);
static const Real IMPACT_ENERGY_MIN_J = Real(1e-6);
static const Real IMPACT_ENERGY_MAX_J = Real(1.0);

// dem.rs:43-46
Real restitution_velocity_threshold(Real r) {
  return RESTITUTION_THRESHOLD_FROUDE * std::sqrt(-GRAVITY * Real(2.0) * r);
}
// dem.rs:99-109
int impact_energy_bin(Real e) {
  if (!std::isfinite(e) || e <= Real(0.0)) return -1;
  Real ec = clamp_r(e, IMPACT_ENERGY_MIN_J, IMPACT_ENERGY_MAX_J);
  Real log_min = log10f_r(IMPACT_ENERGY_MIN_J);
  Real log_max = log10f_r(IMPACT_ENERGY_MAX_J);
  Real t = (log10f_r(ec) - log_min) / (log_max - log_min);
  uint32_t idx = f2u_sat(t * (Real)IMPACT_BINS);
  return (int)std::min(idx, (uint32_t)IMPACT_BINS - 1);
}
// dem.rs:127-138
Real effective_friction(Real mu_k, Real mu_s, Real v_t, Real vs) {
  if (mu_s <= mu_k) return mu_k;
  Real ratio = v_t / vs;
  Real weight = expf_r(-(ratio * ratio));
  return mu_k + (mu_s - mu_k) * weight;
}
// dem.rs:253-273
static Real mechanical_energy_j(const Balls& b) {
  Real e = Real(0.0);
  for (size_t i = 0; i < b.len(); ++i) {
    e += Real(0.5) * b.mass * b.v[i].length_squared();
    e += Real(0.5) * b.inertia * b.omega[i] * b.omega[i];
    e += b.mass * std::fabs(GRAVITY) * b.x[i].y;
  }
  return e;
}
double dem_mechanical_energy_f64(const Balls& b) {
  double e = 0.0;
  for (size_t i = 0; i < b.len(); ++i) {
    e += 0.5 * (double)b.mass * (double)b.v[i].length_squared();
    e += 0.5 * (double)b.inertia * (double)(b.omega[i] * b.omega[i]);
    e += (double)b.mass * (double)std::fabs(GRAVITY) * (double)b.x[i].y;
  }
  return e;
}
// dem.rs:1071-1080
static Real angle_diff(Real a, Real b) {
  Real d = a - b;
  while (d > PI_F) d -= Real(2.0) * PI_F;
  while (d < -PI_F) d += Real(2.0) * PI_F;
  return d;
}

// dem.rs:530-1066
DemStepStats dem_step_recorded(Balls* bp, const Drum& drum, Real drum_angle, const MediaParams& media,
                               uint32_t iterations, Real dt, const CouplingImpulses* ext,
                               std::vector<ImpactRecord>* impacts, StepCounters* ctr, Debug* dbg) {
  Balls& B = *bp;
  DemStepStats out;
  if (B.len() == 0 || dt <= Real(0.0)) return out;
  size_t n = B.len();
  Real w = B.mass > Real(0.0) ? Real(1.0) / B.mass : Real(0.0);
  Real w_rot = B.inertia > Real(0.0) ? Real(1.0) / B.inertia : Real(0.0);
  Real r = B.radius;
  Real impact_threshold = restitution_velocity_threshold(r);
  for (size_t i = 0; i < n; ++i)
    if (!B.x[i].is_finite() || !B.v[i].is_finite()) { B.x[i] = Vec2(); B.v[i] = Vec2(); }
  std::vector<Vec2> x0 = B.x;
  std::vector<Real> theta0 = B.theta;
  std::vector<Vec2> v_pre = B.v;
  std::vector<Real> omega_pre = B.omega;
  double coupling_work = 0.0;
  for (size_t i = 0; i < n; ++i) {
    B.v[i].y += GRAVITY * dt;
    if (ext) {
      double ke_before = 0.5 * (double)B.mass * (double)B.v[i].length_squared() +
                         0.5 * (double)B.inertia * (double)(B.omega[i] * B.omega[i]);
      B.v[i] += ext->impulses[i] * w;
      B.omega[i] += ext->angular_impulses[i] * w_rot;
      double ke_after = 0.5 * (double)B.mass * (double)B.v[i].length_squared() +
                        0.5 * (double)B.inertia * (double)(B.omega[i] * B.omega[i]);
      coupling_work += ke_after - ke_before;
    }
    B.x[i] += B.v[i] * dt;
    B.theta[i] += B.omega[i] * dt;
  }
  Real e_after_predict = mechanical_energy_j(B);
  Real max_disp = Real(0.0);
  for (size_t i = 0; i < n; ++i) max_disp = fmax_r(max_disp, B.v[i].length() * dt / fmax_r(Real(2.0) * r, Real(1e-12)));
  Real max_speed = Real(0.0);
  for (size_t i = 0; i < n; ++i) max_speed = fmax_r(max_speed, B.v[i].length());
  Real solve_margin = (Real)std::max(iterations, 1u) * MAX_RECOVERY_FRACTION * Real(2.0) * r;
  Real cell_size = fmax_r(fmax_r(Real(2.0) * r * Real(1.05), Real(2.0) * r + max_speed * dt + solve_margin), Real(1e-6));
  UniformGrid grid = UniformGrid::build(B.x, cell_size);
  std::vector<std::pair<uint32_t, uint32_t>> pairs;
  grid.for_each_candidate_pair([&](uint32_t i, uint32_t j) { pairs.push_back({i, j}); });
  if (ctr) ctr->n_ball_pairs = (uint32_t)pairs.size();
  if (dbg) dbg->ball_pairs = pairs;
  // step 2.5: wall CCD
  Real drum_angle_next = drum_angle + drum.omega * dt;
  std::vector<Real> toi(n, Real(1.0));
  for (size_t i = 0; i < n; ++i) {
    Real d_end;
    Vec2 nn;
    drum.sdf_world(B.x[i], drum_angle_next, &d_end, &nn);
    Real c_end = d_end - r;
    if (c_end >= -MAX_RECOVERY_FRACTION * Real(2.0) * r) continue;
    Real t;
    if (drum.toi_swept(x0[i], B.x[i], drum_angle, drum_angle_next, r, &t)) toi[i] = fmin_r(toi[i], t);
  }
  for (size_t i = 0; i < n; ++i) {
    if (toi[i] < Real(1.0)) {
      if (ctr) ctr->ccd_clamps += 1;
      Real path_len = (B.x[i] - x0[i]).length();
      Real skin = CCD_CONTACT_SKIN_FRACTION * r;
      Real t_skin = path_len > Real(1e-9) ? skin / path_len : Real(1.0);
      Real t_cl = fmin_r(toi[i] + t_skin, Real(1.0));
      B.x[i] = x0[i] + (B.x[i] - x0[i]) * t_cl;
    }
  }
  std::vector<Real> lam_bb(pairs.size(), Real(0.0)), lam_bw(n, Real(0.0));
  // step 3: projection
  for (uint32_t it = 0; it < std::max(iterations, 1u); ++it) {
    for (size_t k = 0; k < pairs.size(); ++k) {
      size_t i = pairs[k].first, j = pairs[k].second;
      Vec2 delta = B.x[i] - B.x[j];
      Real dist = delta.length();
      Real c = dist - Real(2.0) * r;
      if (c >= Real(0.0)) continue;
      Vec2 n_hat = dist > Real(1e-9) ? delta / dist : Vec2(Real(1.0), Real(0.0));
      Real w_sum = w + w;
      if (w_sum <= Real(0.0)) continue;
      Real c_eff = fmax_r(c, -MAX_RECOVERY_FRACTION * Real(2.0) * r);
      Real d_lambda = -c_eff / w_sum;
      B.x[i] += w * d_lambda * n_hat;
      B.x[j] -= w * d_lambda * n_hat;
      lam_bb[k] += d_lambda;
    }
    for (size_t i = 0; i < n; ++i) {
      Real d;
      Vec2 n_hat;
      drum.sdf_world(B.x[i], drum_angle_next, &d, &n_hat);
      Real c = d - r;
      if (c >= Real(0.0)) continue;
      if (w <= Real(0.0)) continue;
      Real c_eff = fmax_r(c, -MAX_RECOVERY_FRACTION * Real(2.0) * r);
      Real d_lambda = -c_eff / w;
      B.x[i] += w * d_lambda * n_hat;
      lam_bw[i] += d_lambda;
    }
  }
  // step 4: velocity reconstruction
  for (size_t i = 0; i < n; ++i) {
    B.v[i] = (B.x[i] - x0[i]) / dt;
    B.omega[i] = angle_diff(B.theta[i], theta0[i]) / dt;
  }
  struct C3 { uint32_t i, j; Real l; };
  std::vector<C3> bb(pairs.size());
  for (size_t k = 0; k < pairs.size(); ++k) bb[k] = {pairs[k].first, pairs[k].second, lam_bb[k]};
  std::sort(bb.begin(), bb.end(), [](const C3& a, const C3& b) { return a.i != b.i ? a.i < b.i : a.j < b.j; });
  if (ctr) {
    uint32_t act = 0;
    for (auto& c : bb) act += c.l > Real(0.0);
    ctr->n_active_contacts = act;
  }
  // step 5: friction
  for (const C3& c : bb) {
    if (c.l <= Real(0.0)) continue;
    size_t iu = c.i, ju = c.j;
    Vec2 delta = B.x[iu] - B.x[ju];
    Real dist = delta.length();
    Vec2 n_hat = dist > Real(1e-9) ? delta / dist : Vec2(Real(1.0), Real(0.0));
    Vec2 t_hat(-n_hat.y, n_hat.x);
    Real v_t = (B.v[iu] - B.v[ju]).dot(t_hat) - r * B.omega[iu] - r * B.omega[ju];
    Real w_sum_t = w + w + r * r * w_rot + r * r * w_rot;
    if (w_sum_t <= Real(0.0)) continue;
    Real raw = -v_t * dt / w_sum_t;
    Real mu = effective_friction(media.friction_ball_ball, media.friction_ball_ball_static, v_t,
                                  media.friction_velocity_scale_m_s);
    Real max_mag = mu * c.l;
    Real dlt = clamp_r(raw, -max_mag, max_mag);
    B.x[iu] += w * dlt * t_hat;
    B.x[ju] -= w * dlt * t_hat;
    B.theta[iu] -= r * w_rot * dlt;
    B.theta[ju] -= r * w_rot * dlt;
    Vec2 dv = w * dlt * t_hat / dt;
    Real domega = -r * w_rot * dlt / dt;
    B.v[iu] += dv;
    B.v[ju] -= dv;
    B.omega[iu] += domega;
    B.omega[ju] += domega;
  }
  Real wall_work_j = Real(0.0);
  for (size_t i = 0; i < n; ++i) {
    Real lambda_n = lam_bw[i];
    if (lambda_n <= Real(0.0)) continue;
    Real dd;
    Vec2 n_hat;
    drum.sdf_world(B.x[i], drum_angle_next, &dd, &n_hat);
    Vec2 t_hat(-n_hat.y, n_hat.x);
    Vec2 v_wall = drum.wall_velocity(B.x[i] - r * n_hat);
    Real v_t = (B.v[i] - v_wall).dot(t_hat) - r * B.omega[i];
    Real w_sum_t = w + r * r * w_rot;
    if (w_sum_t <= Real(0.0)) continue;
    Real raw = -v_t * dt / w_sum_t;
    Real mu = effective_friction(media.friction_ball_wall, media.friction_ball_wall_static, v_t,
                                  media.friction_velocity_scale_m_s);
    Real max_mag = mu * lambda_n;
    Real dlt = clamp_r(raw, -max_mag, max_mag);
    B.x[i] += w * dlt * t_hat;
    B.theta[i] -= r * w_rot * dlt;
    B.v[i] += w * dlt * t_hat / dt;
    B.omega[i] += -r * w_rot * dlt / dt;
    wall_work_j += (dlt / dt) * t_hat.dot(v_wall);
    wall_work_j += (lambda_n / dt) * n_hat.dot(v_wall);
  }
  // resync
  for (size_t i = 0; i < n; ++i) {
    B.v[i] = (B.x[i] - x0[i]) / dt;
    B.omega[i] = angle_diff(B.theta[i], theta0[i]) / dt;
  }
  // step 6: restitution
  uint32_t collision_count = 0;
  uint32_t hist[IMPACT_BINS] = {};
  for (const C3& c : bb) {
    if (c.l <= Real(0.0)) continue;
    size_t iu = c.i, ju = c.j;
    Vec2 delta = B.x[iu] - B.x[ju];
    Real dist = delta.length();
    Vec2 n_hat = dist > Real(1e-9) ? delta / dist : Vec2(Real(1.0), Real(0.0));
    Real v_n_pre = (v_pre[iu] - v_pre[ju]).dot(n_hat);
    bool fresh = v_n_pre < -RESTITUTION_VELOCITY_THRESHOLD;
    if (fresh) {
      collision_count += 1;
      Real e_imp = Real(0.5) * (B.mass * Real(0.5)) * v_n_pre * v_n_pre;
      int bin = impact_energy_bin(e_imp);
      if (bin >= 0) hist[bin] += 1;
    }
    Real e = fresh ? media.restitution_ball_ball : Real(0.0);
    if (-v_n_pre > impact_threshold && impacts) {
      Vec2 t_hat(-n_hat.y, n_hat.x);
      Real slip = (v_pre[iu] - v_pre[ju]).dot(t_hat) - r * omega_pre[iu] - r * omega_pre[ju];
      impacts->push_back({0u, c.i, c.j, (float)-v_n_pre, (float)std::fabs(slip), (float)e});
    }
    Real target = fmax_r(fmax_r(-e * v_n_pre, Real(0.0)), fmax_r(v_n_pre, Real(0.0)));
    Real v_n_now = (B.v[iu] - B.v[ju]).dot(n_hat);
    Real delta_v_n = target - v_n_now;
    Real w_sum = w + w;
    if (w_sum <= Real(0.0)) continue;
    Real impulse = delta_v_n / w_sum;
    B.v[iu] += w * impulse * n_hat;
    B.v[ju] -= w * impulse * n_hat;
  }
  for (size_t i = 0; i < n; ++i) {
    Real lambda_n = lam_bw[i];
    if (lambda_n <= Real(0.0)) continue;
    Real dd;
    Vec2 n_hat;
    drum.sdf_world(B.x[i], drum_angle_next, &dd, &n_hat);
    Vec2 v_wall = drum.wall_velocity(B.x[i] - r * n_hat);
    Real v_n_pre = (v_pre[i] - v_wall).dot(n_hat);
    bool fresh = v_n_pre < -RESTITUTION_VELOCITY_THRESHOLD;
    if (fresh) {
      collision_count += 1;
      Real e_imp = Real(0.5) * B.mass * v_n_pre * v_n_pre;
      int bin = impact_energy_bin(e_imp);
      if (bin >= 0) hist[bin] += 1;
    }
    Real e = fresh ? media.restitution_ball_wall : Real(0.0);
    if (-v_n_pre > impact_threshold && impacts) {
      Vec2 t_hat(-n_hat.y, n_hat.x);
      Real slip = (v_pre[i] - v_wall).dot(t_hat) - r * omega_pre[i];
      impacts->push_back({1u, (uint32_t)i, WALL_ID, (float)-v_n_pre, (float)std::fabs(slip), (float)e});
    }
    Real target = fmax_r(fmax_r(-e * v_n_pre, Real(0.0)), fmax_r(v_n_pre, Real(0.0)));
    Real v_n_now = (B.v[i] - v_wall).dot(n_hat);
    Real delta_v_n = target - v_n_now;
    if (w <= Real(0.0)) continue;
    B.v[i] += delta_v_n * n_hat;
  }
  // step 7: rolling resistance
  if (media.rolling_friction > Real(0.0) && B.inertia > Real(0.0)) {
    std::vector<Real> total(n, Real(0.0));
    for (const C3& c : bb) { total[c.i] += fmax_r(c.l, Real(0.0)); total[c.j] += fmax_r(c.l, Real(0.0)); }
    for (size_t i = 0; i < n; ++i) total[i] += fmax_r(lam_bw[i], Real(0.0));
    for (size_t i = 0; i < n; ++i) {
      Real ln = total[i];
      if (ln <= Real(0.0) || B.omega[i] == Real(0.0)) continue;
      Real normal_force = ln / dt;
      Real max_dw = media.rolling_friction * normal_force * r / B.inertia * dt;
      Real dw = fmin_r(max_dw, std::fabs(B.omega[i]));
      B.omega[i] -= signum_r(B.omega[i]) * dw;
    }
  }
  Real e_final = mechanical_energy_j(B);
  out.wall_work_j = wall_work_j;
  out.collision_count = collision_count;
  for (int k = 0; k < IMPACT_BINS; ++k) out.impact_energy_histogram[k] = hist[k];
  out.dissipated_energy_j = e_after_predict + wall_work_j - e_final;
  out.max_substep_displacement_over_diameter = max_disp;
  out.coupling_work_j = (Real)coupling_work;
  return out;
}

}  // namespace orc

// ---------------------------------------------------------------- probes of the viscosity stage
// C entry points over the functions above, for the reference unit tests that call them directly
// (pbf.rs:2428, 2476, 2513). Test infrastructure like the rest of the oracle.
extern "C" {

// morris_weights + laplacian_apply_into (pbf.rs:312-377) on caller points: the neighbour lists of
// pbf.rs:262-288 at h, per-particle densities and viscosities as given; out[2n] = (L v)_i,
// *w_max = the largest weight.
int or_probe_viscous_operator(const float* xy, const float* v, const float* density, const float* mu, uint32_t n,
                              float h, float mass, float* out, float* w_max) {
  using namespace orc;
  std::vector<Vec2> x(n), vv(n), o(n);
  for (uint32_t i = 0; i < n; ++i) { x[i] = Vec2(xy[2 * i], xy[2 * i + 1]); vv[i] = Vec2(v[2 * i], v[2 * i + 1]); }
  Nbr nb;
  neighbor_lists(x, h, &nb.off, &nb.idx);
  std::vector<Real> dens(density, density + n), m(mu, mu + n);
  ViscWeights w = morris_weights(x, nb, dens, mass, m, h);
  laplacian_apply_into(nb, w, vv.data(), n, o.data());
  Real wm = Real(0.0);
  for (Real q : w.w) wm = fmax_r(wm, q);
  for (uint32_t i = 0; i < n; ++i) { out[2 * i] = o[i].x; out[2 * i + 1] = o[i].y; }
  if (w_max) *w_max = wm;
  return 0;
}

// squeeze_links (pbf.rs:544-625) of balls at bx[2 nb] (radius r, mass ball_mass) in a drum of
// drum_radius; closing (2 nb, may be null: no approach filter) as the reference's Option. Links
// go to ball/other (other = 0xFFFFFFFF for the wall), nrm[2], c; *n_out all links (even beyond
// cap), *in_range the pairs and walls within range.
int or_probe_squeeze_links(const float* bx, uint32_t nb, float r, float ball_mass, float drum_radius, float dx,
                           float mu, float dt, const float* closing, uint32_t* ball, uint32_t* other, float* nrm,
                           float* c, uint32_t cap, uint32_t* n_out, uint32_t* in_range) {
  using namespace orc;
  Balls b;
  for (uint32_t i = 0; i < nb; ++i) b.x.push_back(Vec2(bx[2 * i], bx[2 * i + 1]));
  b.v.assign(nb, Vec2());
  b.theta.assign(nb, Real(0.0));
  b.omega.assign(nb, Real(0.0));
  b.radius = r;
  b.mass = ball_mass;
  std::vector<Vec2> cl;
  for (uint32_t i = 0; closing && i < nb; ++i) cl.push_back(Vec2(closing[2 * i], closing[2 * i + 1]));
  size_t ir = 0;
  std::vector<SqueezeLink> links = squeeze_links(b, drum_radius, dx, mu, dt, closing ? &cl : nullptr, &ir);
  for (size_t k = 0; k < links.size() && k < cap; ++k) {
    ball[k] = links[k].ball;
    other[k] = links[k].other;
    nrm[2 * k] = links[k].n.x;
    nrm[2 * k + 1] = links[k].n.y;
    c[k] = links[k].c;
  }
  *n_out = (uint32_t)links.size();
  if (in_range) *in_range = (uint32_t)ir;
  return 0;
}

// solve_viscosity_with_balls (pbf.rs:641-791) for n fluid particles without neighbours (their
// Laplacian rows are empty, as in the reference test's NeighborLists{offsets: [0; n + 1]}), no
// boundary groups, the given links and no warm start: fluid_v[2n], ball_v[2nb] and ball_w[nb]
// are solved in place; *iters receives the PCG iterations.
int or_probe_joint_solve(uint32_t n, float* fluid_v, uint32_t nb, float* ball_v, float* ball_w, uint32_t nl,
                         const uint32_t* l_ball, const uint32_t* l_other, const float* l_n, const float* l_c,
                         float mass, float ball_mass, float ball_inertia, float dt, uint32_t* iters) {
  using namespace orc;
  Nbr nbr;
  nbr.off.assign(n + 1, 0);
  ViscWeights w;
  std::vector<BoundaryGroup> groups;
  std::vector<SqueezeLink> links;
  for (uint32_t k = 0; k < nl; ++k)
    links.push_back({l_ball[k], l_other[k], Vec2(l_n[2 * k], l_n[2 * k + 1]), l_c[k]});
  std::vector<Vec2> v(n), bv(nb), guess;
  std::vector<Real> bw(ball_w, ball_w + nb);
  for (uint32_t i = 0; i < n; ++i) v[i] = Vec2(fluid_v[2 * i], fluid_v[2 * i + 1]);
  for (uint32_t i = 0; i < nb; ++i) bv[i] = Vec2(ball_v[2 * i], ball_v[2 * i + 1]);
  uint32_t it = solve_viscosity_with_balls(nbr, w, groups, links, mass, ball_mass, ball_inertia, dt, guess, &v, &bv,
                                           &bw, false);
  for (uint32_t i = 0; i < n; ++i) { fluid_v[2 * i] = v[i].x; fluid_v[2 * i + 1] = v[i].y; }
  for (uint32_t i = 0; i < nb; ++i) { ball_v[2 * i] = bv[i].x; ball_v[2 * i + 1] = bv[i].y; ball_w[i] = bw[i]; }
  if (iters) *iters = it;
  return 0;
}

}  // extern "C"
