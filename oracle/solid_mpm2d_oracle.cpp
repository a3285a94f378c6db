// CPU FP64 restatement of the reference's 2D MLS-MPM elastic solid (src/solid-mpm.js) and of the
// parts of its caller's frame loop that touch MPM solids (src/simulation.js:239-298).
//
// TEST INFRASTRUCTURE ONLY: this file is the checker. Only tests/ load it; the product library
// (libmpm_b200.so) never links, calls or falls back to it.
//
// Parity pin: the reference is JavaScript and no JS runtime exists on either machine, so this
// restatement is pinned against the reference's own tests for the path
// (tests/solid-mpm.test.mjs:9-66), restated in tests/test_solid2d.py.
//
// State layout follows the reference: F and C per particle as eight FP64 fields
// (f00 f01 f10 f11 c00 c01 c10 c11, src/solid-mpm.js:5); the caller's x, y, vx, vy, mass and
// volume are Float32 arrays (src/simulation.js:18-19), so they are read as float and every
// update is rounded back to float exactly where the JS typed-array store rounds it.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr double kDX = 8, kOrigin = -592, kArea = 12.96;  // src/solid-mpm.js:4
constexpr int kN = 149;

double clampd(double x, double a, double b) { return std::max(a, std::min(b, x)); }

struct Stencil2 {
  int bx, by;
  double fx, fy, wx[3], wy[3];
};

// src/solid-mpm.js:30-36
void stencil2(double x, double y, Stencil2& s) {
  const double px = (x - kOrigin) / kDX, py = (y - kOrigin) / kDX;
  s.bx = static_cast<int>(clampd(std::floor(px - .5), 0, kN - 3));
  s.by = static_cast<int>(clampd(std::floor(py - .5), 0, kN - 3));
  s.fx = px - s.bx;
  s.fy = py - s.by;
  auto set = [](double f, double* w) {
    w[0] = .5 * (1.5 - f) * (1.5 - f);
    w[1] = .75 - (f - 1) * (f - 1);
    w[2] = .5 * (f - .5) * (f - .5);
  };
  set(s.fx, s.wx);
  set(s.fy, s.wy);
}

}  // namespace

extern "C" {

// The caller's arrays (src/simulation.js:18-28) plus the settings and scene name the step reads.
struct Oracle2Sim {
  int32_t count;
  int32_t scene;     // 0 other, 1 'softbody', 2 'basin'
  int32_t boundary;  // settings.boundary
  int32_t gravity;   // settings.gravity: 0 'none', 1 'center', 2 'uniform'
  double stiffness;  // settings.solidStiffness
  double strength;   // settings.strength
  float *x, *y, *vx, *vy;
  const float *mass, *volume;
  const uint8_t *material, *pinned;
  const uint8_t* mpm_material;  // 256 flags: MATERIALS[m].mpm (src/solid-mpm.js:7)
};

// Deformation state owned by SolidMPM (src/solid-mpm.js:21-24): fields[8][capacity].
struct Oracle2State {
  int64_t capacity;
  double* f[8];
  int32_t substeps, active_nodes;
};

struct Oracle2Stats {
  int32_t count;
  double min_j, max_j, strain;
  int32_t nodes, substeps;
};

// src/solid-mpm.js:10-18: Kirchhoff stress P F^T of 2D fixed-corotated elasticity, closed-form polar.
void oracle2_solid_stress(double a, double b, double c, double d, double mu, double lambda, double* tau) {
  const double J = a * d - b * c, q = std::hypot(a + d, c - b);
  const double r = q > 1e-12 ? (a + d) / q : 1, t = q > 1e-12 ? (c - b) / q : 0;
  const double volume = lambda * (J - 1) * J;
  tau[0] = 2 * mu * ((a - r) * a + (b + t) * b) + volume;
  tau[1] = 2 * mu * ((a - r) * c + (b + t) * d);
  tau[2] = 2 * mu * ((c - t) * a + (d - r) * b);
  tau[3] = 2 * mu * ((c - t) * c + (d - r) * d) + volume;
}

static bool is_solid(const Oracle2Sim* s, int p) { return s->mpm_material[s->material[p]] != 0; }

// src/solid-mpm.js:37-46
double oracle2_stable_step(const Oracle2State* st, const Oracle2Sim* s) {
  double wave = 1, gradient = 0;
  const double sound = std::sqrt(19200 * s->stiffness);
  for (int p = 0; p < s->count; ++p) {
    if (!is_solid(s, p)) continue;
    const double stretch = std::max(1.0, std::sqrt(st->f[0][p] * st->f[0][p] + st->f[1][p] * st->f[1][p] +
                                                   st->f[2][p] * st->f[2][p] + st->f[3][p] * st->f[3][p]));
    wave = std::max(wave, std::hypot((double)s->vx[p], (double)s->vy[p]) + sound * stretch * stretch);
    gradient = std::max(gradient, std::fabs(st->f[4][p]) + std::fabs(st->f[5][p]) + std::fabs(st->f[6][p]) +
                                      std::fabs(st->f[7][p]));
  }
  return std::min(std::min(1.0 / 240, .18 * kDX / wave), .1 / std::max(1.0, gradient));
}

// src/solid-mpm.js:47-91: one MPM step of the solid particles. grid_out (optional) receives the
// grid after the update, as [mass, ux, uy] x N*N.
void oracle2_step(Oracle2State* st, Oracle2Sim* s, double dt, double* grid_out) {
  std::vector<double> mass(kN * kN, 0.0), ux(kN * kN, 0.0), uy(kN * kN, 0.0), fixed(kN * kN, 0.0);
  double** f = st->f;
  Stencil2 sc;
  for (int p = 0; p < s->count; ++p) {
    if (!is_solid(s, p)) continue;
    stencil2(s->x[p], s->y[p], sc);
    const double m = s->mass[p], V0 = kArea * s->volume[p], rho = m / V0, E = rho * 16000 * s->stiffness;
    double tau[4];
    oracle2_solid_stress(f[0][p], f[1][p], f[2][p], f[3][p], .4 * E, .4 * E, tau);
    const double factor = -dt * V0 * 4 / (kDX * kDX);
    const double a00 = m * f[4][p] + factor * tau[0], a01 = m * f[5][p] + factor * tau[1];
    const double a10 = m * f[6][p] + factor * tau[2], a11 = m * f[7][p] + factor * tau[3];
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) {
        const int n = (sc.by + j) * kN + sc.bx + i;
        const double w = sc.wx[i] * sc.wy[j], dx = (i - sc.fx) * kDX, dy = (j - sc.fy) * kDX;
        mass[n] += w * m;
        ux[n] += w * (m * s->vx[p] + a00 * dx + a01 * dy);
        uy[n] += w * (m * s->vy[p] + a10 * dx + a11 * dy);
        if (s->pinned[p]) fixed[n] += w * m;
      }
  }
  const bool demo = s->scene == 1, basin = s->scene == 2;
  const double bound = demo ? 170 : basin ? 245 : 555, floor_ = demo ? -145 : basin ? -175 : -555,
               top = demo ? 145 : bound;
  const bool walls = s->boundary || demo || basin;
  st->active_nodes = 0;
  for (int n = 0; n < kN * kN; ++n) {
    if (!(mass[n] > 1e-12)) continue;
    st->active_nodes++;
    ux[n] /= mass[n];
    uy[n] /= mass[n];
    if (fixed[n] > 1e-9) {
      ux[n] = uy[n] = 0;
      continue;
    }
    if (walls) {
      const double x = kOrigin + (n % kN) * kDX, y = kOrigin + (n / kN) * kDX;
      if ((x < -bound + kDX && ux[n] < 0) || (x > bound - kDX && ux[n] > 0)) ux[n] = 0;
      if ((y < floor_ + kDX && uy[n] < 0) || (y > top - kDX && uy[n] > 0)) uy[n] = 0;
    }
  }
  if (grid_out)
    for (int n = 0; n < kN * kN; ++n) {
      grid_out[3 * n] = mass[n];
      grid_out[3 * n + 1] = mass[n] > 1e-12 ? ux[n] : 0;
      grid_out[3 * n + 2] = mass[n] > 1e-12 ? uy[n] : 0;
    }
  for (int p = 0; p < s->count; ++p) {
    if (!is_solid(s, p) || s->pinned[p]) continue;
    stencil2(s->x[p], s->y[p], sc);
    double vx = 0, vy = 0, a = 0, b = 0, c = 0, d = 0;
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) {
        const int n = (sc.by + j) * kN + sc.bx + i;
        const double w = sc.wx[i] * sc.wy[j], dx = (i - sc.fx) * 4 / kDX, dy = (j - sc.fy) * 4 / kDX;
        vx += w * ux[n];
        vy += w * uy[n];
        a += w * ux[n] * dx;
        b += w * ux[n] * dy;
        c += w * uy[n] * dx;
        d += w * uy[n] * dy;
      }
    f[4][p] = a;
    f[5][p] = b;
    f[6][p] = c;
    f[7][p] = d;
    const double F0 = f[0][p], F1 = f[1][p], F2 = f[2][p], F3 = f[3][p];
    f[0][p] = (1 + dt * a) * F0 + dt * b * F2;
    f[1][p] = (1 + dt * a) * F1 + dt * b * F3;
    f[2][p] = dt * c * F0 + (1 + dt * d) * F2;
    f[3][p] = dt * c * F1 + (1 + dt * d) * F3;
    s->vx[p] = (float)vx;
    s->vy[p] = (float)vy;
    s->x[p] = (float)((double)s->x[p] + dt * vx);
    s->y[p] = (float)((double)s->y[p] + dt * vy);
    if (walls) {
      s->x[p] = (float)clampd(s->x[p], -bound + .1, bound - .1);
      s->y[p] = (float)clampd(s->y[p], floor_ + .1, top - .1);
    }
  }
}

// The MPM-solid branch of Simulation.substep before mpm.step (src/simulation.js:270-288): pinned
// particles stop; others receive the body force (no damping for MPM solids) and a +-180 clamp.
void oracle2_apply_forces(const Oracle2Sim* s, double dt) {
  for (int i = 0; i < s->count; ++i) {
    if (!is_solid(s, i)) continue;
    if (s->pinned[i]) {
      s->vx[i] = s->vy[i] = 0;
      continue;
    }
    double gx = 0, gy = 0;
    if (s->gravity == 1) {
      const double r = std::sqrt((double)s->x[i] * s->x[i] + (double)s->y[i] * s->y[i] + 400);
      gx = -s->x[i] / r;
      gy = -s->y[i] / r;
    } else if (s->gravity == 2) {
      gy = -1;
    }
    const double force = 27 * s->strength;
    const float vx = (float)(s->vx[i] + gx * force * dt), vy = (float)(s->vy[i] + gy * force * dt);
    s->vx[i] = (float)clampd(vx, -180, 180);
    s->vy[i] = (float)clampd(vy, -180, 180);
  }
}

// The MPM branch of Simulation.step (src/simulation.js:239-255) for a simulation whose moving
// particles are all MPM solids: CFL-bounded substeps until dt is solved or 96 substeps ran.
// Returns the substep count; *advanced receives the simulated time.
int oracle2_frame(Oracle2State* st, Oracle2Sim* s, double dt, double* advanced) {
  dt = clampd(dt, 0, .05);
  double remaining = dt;
  int steps = 0;
  while (remaining > 1e-9 && steps < 96) {
    const double h = std::min(remaining, oracle2_stable_step(st, s));
    if (h > 0) {
      oracle2_apply_forces(s, h);
      oracle2_step(st, s, h, nullptr);
    }
    remaining -= h;
    steps++;
  }
  st->substeps = steps;
  if (advanced) *advanced = dt - remaining;
  return steps;
}

// src/solid-mpm.js:108-116
void oracle2_stats(const Oracle2State* st, const Oracle2Sim* s, Oracle2Stats* out) {
  int count = 0;
  double mn = INFINITY, mx = 0, strain = 0;
  for (int p = 0; p < s->count; ++p) {
    if (!is_solid(s, p)) continue;
    count++;
    const double a = st->f[0][p], b = st->f[1][p], c = st->f[2][p], d = st->f[3][p], J = a * d - b * c;
    mn = std::min(mn, J);
    mx = std::max(mx, J);
    const double e0 = a * a + c * c - 1, e1 = b * b + d * d - 1, e2 = std::sqrt(2.0) * (a * b + c * d);
    strain = std::max(strain, .5 * std::sqrt(e0 * e0 + e1 * e1 + e2 * e2));
  }
  out->count = count;
  out->min_j = count ? mn : 1;
  out->max_j = count ? mx : 1;
  out->strain = strain;
  out->nodes = st->active_nodes;
  out->substeps = st->substeps;
}

}  // extern "C"
