// CPU FP64 restatement of the reference's 3D MLS-MPM solid step.
//
// TEST INFRASTRUCTURE ONLY: this file is the checker. Only tests/, the smoke
// check of __graft_entry__.py and the cpu-baseline leg of bench.py load it.
// The product library (libmpm_b200.so) never links, calls or falls back to it.
//
// Parity pin: the reference is JavaScript and no JS runtime exists on either
// machine, so this restatement is pinned against the reference's own
// known-answer tests (tests/metal-plasticity.test.mjs:12-23,
// tests/thermal-plasticity.test.mjs:12-31, tests/constitutive.test.mjs:10-25,
// tests/three.test.mjs:8-21, src/simulation/vv-mpm.js:7), restated in
// tests/test_oracle_kat.py.
//
// Units. The reference works in sandbox units with mu = lambda = 0.4 E and
// strengths given as stress / E (src/three/mpm.js:34-37,
// src/three/metal-plasticity.js:1-2). Every formula here takes mu, lambda and
// strengths as parameters, so mu = lambda = 0.4 with strengths / E reproduces
// the reference numbers exactly, and SI inputs give the SI restatement:
//   q     = sqrt(6) * mu * |dev e| / J    (reference: sqrt(6)*.4*length/J)
//   slope = 3 * mu / J                   (reference: 1.2/J)
//
// Build: oracle/build_oracle.py (g++ -O3 -fopenmp -shared).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// Material parameters. model follows src/three/constitutive.js:6-19:
// 0 fixed-corotated, 1 Neo-Hookean, 2 snow, 3 sand, 4 ideal J2, 5 linear-hardening J2,
// 6 Johnson-Cook, 7 simplified Johnson-Cook, 8 cohesive Drucker-Prager, 9 Deshpande-Fleck foam,
// 10 thermal J2, 11 Norton creep.
struct OracleMaterial {
  int32_t model;
  int32_t pad;
  double mu, lambda;
  // J2 / Johnson-Cook (src/three/metal-plasticity.js:3): A, B, n, C, rate0, Tref, Tm, m
  double A, B, n, C, rate0, Tref, Tm, m;
  // thermal (src/three/thermal-plasticity.js:3): Tref, Thot, hotRatio, A, H, rate, Q, n, stress
  double tTref, tThot, tHotRatio, tA, tH, tRate, tQ, tN, tStress;
  // plastic heating: heat fraction beta and specific heat cp (gpu/mixed_material.py:150-172)
  double beta, cp;
  // snow yield strain and sand friction angle in degrees (per particle in the reference,
  // src/three/simulation.js:40; defaults .025 and 35)
  double yieldStrain, friction;
  // pressure models (src/three/pressure-plasticity.js:2): strengths in the stress unit of mu
  double cohesion, slope, dilatancy, tension, alpha, plateau, gamma, densify, pbeta, epsD;
  // heat exchange and phase change (src/thermal.js:35-56, src/three/phase-change.js:4-18):
  // conductivity, melting point and latent heat (phase change enabled when latent > 0)
  double kcond, Tphase, latent;
};

struct OracleScene {
  double origin[3];
  double H;
  int32_t dims[3];
  int32_t sticky_floor;     // 1: nodes within one cell of lower[1] get v = 0
  double lower[3], upper[3];
  double gravity[3];
  int32_t gravity_on_grid;  // 0: v += g dt on particles before P2G (src/three/simulation.js:337-344)
  int32_t clamp_positions;  // 1: clamp x to [clamp_lo, clamp_hi] after G2P (src/three/simulation.js:358-365)
  double clamp_lo[3], clamp_hi[3];
  double mass_eps;          // grid mass threshold (src/three/mpm.js:89 uses 1e-12)
  // CFL rule (src/three/mpm.js:43-55): dt <= min(dt_max, cfl*H/max(1, |v|+c*max(1,row*col,compr)),
  // grad_limit/max(1, sum|C|)) with c = sqrt((lambda+2mu)/rho)
  double cfl, dt_max, grad_limit;
  // grid heat conduction (this project's coupled-scene extension, no reference counterpart):
  // off when cond_k <= 0; conductance k H dt min(1, min(m_i, m_j) / (rho H^3)) between face
  // neighbours that both hold mass, node increments Q_i / (m_i cp) added to particles in G2P
  double cond_k, cond_rho, cond_cp;
};

struct OracleLedger {
  double mass, kinetic, affine, potential, elastic;
  double momentum[3], angular[3];
  double min_j, max_j, max_plastic, max_von_mises;
  int64_t nonfinite, invalid_j, unsupported_elastic;
};

// ---------------------------------------------------------------------------
// 3x3 helpers: src/three/math.js:9-32
static double det3(const double* a) {
  return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
         a[2] * (a[3] * a[7] - a[4] * a[6]);
}

// math.js:10-15 inverseTranspose; returns false where |det| < 1e-10
static bool inverse_transpose(const double* a, double* out) {
  const double d = det3(a);
  if (std::fabs(d) < 1e-10) return false;
  out[0] = (a[4] * a[8] - a[5] * a[7]) / d;
  out[1] = (a[5] * a[6] - a[3] * a[8]) / d;
  out[2] = (a[3] * a[7] - a[4] * a[6]) / d;
  out[3] = (a[2] * a[7] - a[1] * a[8]) / d;
  out[4] = (a[0] * a[8] - a[2] * a[6]) / d;
  out[5] = (a[1] * a[6] - a[0] * a[7]) / d;
  out[6] = (a[1] * a[5] - a[2] * a[4]) / d;
  out[7] = (a[2] * a[3] - a[0] * a[5]) / d;
  out[8] = (a[0] * a[4] - a[1] * a[3]) / d;
  return true;
}

// math.js:16-24: polar rotation by Newton averaging R <- (R + R^-T)/2, at most 8 iterations
void oracle_rotation(const double* F, double* R) {
  double r[9], inv[9];
  std::memcpy(r, F, sizeof r);
  for (int it = 0; it < 8; ++it) {
    if (!inverse_transpose(r, inv)) {
      for (int k = 0; k < 9; ++k) R[k] = (k % 4 == 0) ? 1.0 : 0.0;
      return;
    }
    double diff = 0;
    for (int k = 0; k < 9; ++k) {
      const double v = 0.5 * (r[k] + inv[k]);
      diff += std::fabs(v - r[k]);
      r[k] = v;
    }
    if (diff < 1e-8) break;
  }
  std::memcpy(R, r, sizeof r);
}

// math.js:25-32: fixed-corotated Kirchhoff stress 2mu(F-R)F^T + lambda(J-1)J I
void oracle_stress3(const double* F, double mu, double lambda, double* t) {
  double R[9];
  oracle_rotation(F, R);
  const double J = det3(F);
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += 2 * mu * (F[a * 3 + k] - R[a * 3 + k]) * F[b * 3 + k];
      if (a == b) s += lambda * (J - 1) * J;
      t[a * 3 + b] = s;
    }
}

// constitutive.js:22-42: Jacobi diagonalisation of F^T F (at most 10 sweeps, pairs
// (0,1),(0,2),(1,2), skip threshold 1e-13*(1+|app|+|aqq|)); sigma = sqrt(max(1e-16, lambda));
// U = F V / sigma. Singular values are not sorted.
void oracle_svd3(const double* F, double* u, double* v, double* sigma) {
  double a[9] = {0};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) a[i * 3 + j] += F[k * 3 + i] * F[k * 3 + j];
  for (int k = 0; k < 9; ++k) v[k] = (k % 4 == 0) ? 1.0 : 0.0;
  static const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int sweep = 0; sweep < 10; ++sweep) {
    bool changed = false;
    for (const auto& pq : pairs) {
      const int p = pq[0], q = pq[1];
      const double apq = a[p * 3 + q];
      if (std::fabs(apq) < 1e-13 * (1 + std::fabs(a[p * 3 + p]) + std::fabs(a[q * 3 + q]))) continue;
      changed = true;
      const double theta = 0.5 * std::atan2(2 * apq, a[q * 3 + q] - a[p * 3 + p]);
      const double c = std::cos(theta), s = std::sin(theta);
      const double app = a[p * 3 + p], aqq = a[q * 3 + q];
      a[p * 3 + p] = c * c * app - 2 * s * c * apq + s * s * aqq;
      a[q * 3 + q] = s * s * app + 2 * s * c * apq + c * c * aqq;
      a[p * 3 + q] = a[q * 3 + p] = 0;
      for (int k = 0; k < 3; ++k) {
        if (k != p && k != q) {
          const double x = a[k * 3 + p], y = a[k * 3 + q];
          a[k * 3 + p] = a[p * 3 + k] = c * x - s * y;
          a[k * 3 + q] = a[q * 3 + k] = s * x + c * y;
        }
        const double x = v[k * 3 + p], y = v[k * 3 + q];
        v[k * 3 + p] = c * x - s * y;
        v[k * 3 + q] = s * x + c * y;
      }
    }
    if (!changed) break;
  }
  for (int k = 0; k < 3; ++k) sigma[k] = std::sqrt(std::max(1e-16, a[k * 3 + k]));
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += F[i * 3 + k] * v[k * 3 + j] / sigma[j];
      u[i * 3 + j] = s;
    }
}

// constitutive.js:43-47: F = U diag(sigma) V^T
void oracle_compose(const double* u, const double* v, const double* sigma, double* F) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += u[i * 3 + k] * sigma[k] * v[j * 3 + k];
      F[i * 3 + j] = s;
    }
}

// constitutive.js:88-90
double oracle_von_mises(const double* t, double J) {
  const double s = 0.5 * ((t[0] - t[4]) * (t[0] - t[4]) + (t[4] - t[8]) * (t[4] - t[8]) +
                          (t[8] - t[0]) * (t[8] - t[0])) +
                   3 * (t[1] * t[1] + t[2] * t[2] + t[5] * t[5]);
  return std::sqrt(std::max(0.0, s)) / std::max(1e-6, J);
}

// constitutive.js:92-106: models 0 and 2 use stress3 (model 2 scaled by hardening(jp), which is
// 1 at the default jp = 1, constitutive.js:48), model 1 Neo-Hookean, models >= 3 Hencky
int oracle_constitutive_stress(const double* F, int model, double mu, double lambda, double* tau) {
  if (model == 0 || model == 2) {
    oracle_stress3(F, mu, lambda, tau);
    return 0;
  }
  if (model < 0 || model > 11) return -1;
  for (int k = 0; k < 9; ++k) tau[k] = 0;
  if (model == 1) {
    const double pressure = lambda * std::log(std::max(det3(F), 1e-6));
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double s = 0;
        for (int k = 0; k < 3; ++k) s += mu * F[a * 3 + k] * F[b * 3 + k];
        if (a == b) s += pressure - mu;
        tau[a * 3 + b] = s;
      }
    return 0;
  }
  double u[9], v[9], sigma[3], e[3];
  oracle_svd3(F, u, v, sigma);
  for (int k = 0; k < 3; ++k) e[k] = std::log(std::max(sigma[k], 1e-6));
  const double trace = e[0] + e[1] + e[2];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += u[a * 3 + k] * (2 * mu * e[k] + lambda * trace) * u[b * 3 + k];
      tau[a * 3 + b] = s;
    }
  return 0;
}

// constitutive.js:81-86: Kirchhoff stress from the returned principal stretches, Hencky form
// (models other than snow): diag = 2 mu e + lambda tr e, tau = U diag U^T
void oracle_principal_stress(const double* u, const double* sigma, double mu, double lambda,
                             double* tau) {
  double e[3];
  for (int k = 0; k < 3; ++k) e[k] = std::log(sigma[k]);
  const double trace = e[0] + e[1] + e[2];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += u[a * 3 + k] * (2 * mu * e[k] + lambda * trace) * u[b * 3 + k];
      tau[a * 3 + b] = s;
    }
}

// metal-plasticity.js:12-19
double oracle_flow_stress(int model, double ep, double rate, double T, const OracleMaterial* p) {
  if (model == 4) return p->A;
  if (model == 5) return p->A + p->B * ep;
  const double rateFactor = 1 + p->C * std::log(std::max(1.0, rate / p->rate0));
  const double theta = std::max(0.0, std::min(1.0, (T - p->Tref) / (p->Tm - p->Tref)));
  return (p->A + p->B * std::pow(ep, p->n)) * rateFactor * (model == 6 ? 1 - std::pow(theta, p->m) : 1);
}

// metal-plasticity.js:20-38 (models 4-7), mu = 0.4 in reference units
void oracle_metal_return(const double* sigma, int model, double ep, double dt, double T,
                         const OracleMaterial* p, double* out, double* increment) {
  double e[3], dev[3];
  for (int k = 0; k < 3; ++k) e[k] = std::log(std::max(sigma[k], 1e-6));
  const double trace = e[0] + e[1] + e[2];
  for (int k = 0; k < 3; ++k) dev[k] = e[k] - trace / 3;
  const double length = std::sqrt(dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]);
  const double J = std::max(1e-6, std::exp(trace));
  const double q = std::sqrt(6.0) * p->mu * length / J;
  double inc = 0;
  if (q > oracle_flow_stress(model, ep, 0, T, p)) {
    const double slope = 3 * p->mu / J;
    if (model <= 5) {
      inc = (q - oracle_flow_stress(model, ep, 0, T, p)) / (slope + (model == 5 ? p->B : 0));
    } else {
      double lo = 0, hi = q / slope;
      for (int it = 0; it < 24; ++it) {
        const double mid = (lo + hi) / 2;
        if (q - slope * mid > oracle_flow_stress(model, ep + mid, mid / std::max(dt, 1e-12), T, p))
          lo = mid;
        else
          hi = mid;
      }
      inc = (lo + hi) / 2;
    }
  }
  const double scale = std::max(0.0, 1 - std::sqrt(1.5) * inc / std::max(length, 1e-20));
  for (int k = 0; k < 3; ++k) out[k] = std::exp(trace / 3 + scale * dev[k]);
  *increment = inc;
}

// thermal-plasticity.js:12-15
double oracle_thermal_strength(double ep, double T, const OracleMaterial* p) {
  const double theta = std::max(0.0, std::min(1.0, (T - p->tTref) / (p->tThot - p->tTref)));
  return (p->tA + p->tH * ep) * (1 - (1 - p->tHotRatio) * theta);
}

// thermal-plasticity.js:17-21 (temperatures in degrees C, Kelvin offset 273.15)
double oracle_creep_log_rate(double q, double T, const OracleMaterial* p) {
  if (p->tRate == 0 || q <= 0) return -INFINITY;
  const double act = std::max(-60.0, std::min(60.0, p->tQ / 8.314462618 *
                                                         (1 / (p->tTref + 273.15) -
                                                          1 / std::max(1.0, T + 273.15))));
  return std::log(p->tRate) + act + p->tN * std::log(q / p->tStress);
}

// thermal-plasticity.js:22-40 (models 10, 11)
void oracle_thermal_return(const double* sigma, int model, double ep, double dt, double T,
                           const OracleMaterial* p, double* out, double* increment) {
  double e[3], dev[3];
  for (int k = 0; k < 3; ++k) e[k] = std::log(std::max(sigma[k], 1e-6));
  const double tr = e[0] + e[1] + e[2];
  for (int k = 0; k < 3; ++k) dev[k] = e[k] - tr / 3;
  const double length = std::sqrt(dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]);
  const double J = std::max(1e-6, std::exp(tr));
  const double q = std::sqrt(6.0) * p->mu * length / J, slope = 3 * p->mu / J;
  double inc = 0;
  if (model == 10) {
    const double factor = oracle_thermal_strength(0, T, p) / p->tA;
    inc = std::max(0.0, (q - oracle_thermal_strength(ep, T, p)) / (slope + p->tH * factor));
  } else if (dt > 0 && p->tRate > 0 && q > 1e-20) {
    double lo = 0, hi = q / slope;
    for (int k = 0; k < 32; ++k) {
      const double mid = (lo + hi) / 2;
      if (std::log(mid / dt) < oracle_creep_log_rate(std::max(0.0, q - slope * mid), T, p))
        lo = mid;
      else
        hi = mid;
    }
    inc = (lo + hi) / 2;
  }
  const double scale = std::max(0.0, 1 - std::sqrt(1.5) * inc / std::max(length, 1e-20));
  for (int k = 0; k < 3; ++k) out[k] = std::exp(tr / 3 + scale * dev[k]);
  *increment = inc;
}

// constitutive.js:48
double oracle_hardening(double jp) { return std::max(0.25, std::min(4.0, std::exp(10 * (1 - jp)))); }

// pressure-plasticity.js:11-14. Fully densified foam (ep >= epsD) has strength 1e30 here (1e20 in
// the reference's E units): both stand for "cannot yield".
double oracle_foam_strength(double ep, const OracleMaterial* p) {
  const double r = ep / p->epsD;
  return r >= 1 ? 1e30
                : p->plateau + p->gamma * r - p->densify * std::log(std::max(1e-30, 1 - std::pow(r, p->pbeta)));
}

// pressure-plasticity.js:15-48 (models 8 and 9). The reference's G = 0.4 / J and K = (2/3) / J
// are mu / J and (lambda + 2 mu / 3) / J at mu = lambda = 0.4.
void oracle_pressure_return(const double* sigma, int model, double jp, double ep, const OracleMaterial* p,
                            double* out, double* jp_out, double* increment) {
  double e[3], dev[3];
  for (int k = 0; k < 3; ++k) e[k] = std::log(std::max(sigma[k], 1e-6));
  const double trace = e[0] + e[1] + e[2];
  for (int k = 0; k < 3; ++k) dev[k] = e[k] - trace / 3;
  const double length = std::sqrt(dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]);
  const double J = std::max(1e-6, std::exp(trace) * jp), G = p->mu / J, K = (p->lambda + 2 * p->mu / 3) / J;
  const double mean = K * trace, q = std::sqrt(6.0) * G * length;
  double meanNew = mean, qNew = q, inc = 0;
  if (model == 8) {
    const double t = q / std::sqrt(3.0), c = p->cohesion, a = p->slope, b = p->dilatancy, T = p->tension;
    if (mean > T && t + a * T <= c) {
      meanNew = T;
    } else if (t + a * mean > c) {
      const double dl = (t + a * mean - c) / (G + a * K * b);
      meanNew = mean - K * b * dl;
      qNew = std::sqrt(3.0) * std::max(0.0, t - G * dl);
      if (meanNew > T) {
        meanNew = T;
        qNew = std::sqrt(3.0) * std::max(0.0, c - a * T);
      }
    }
  } else {
    const double a2 = p->alpha * p->alpha, B = 1 + a2 / 9, trial = std::sqrt((q * q + a2 * mean * mean) / B);
    if (trial > oracle_foam_strength(ep, p)) {
      auto state = [&](double eta, double& qn, double& mn, double& dl) {
        qn = q / (1 + 3 * G * eta);
        mn = mean / (1 + K * a2 * eta);
        const double hat = std::sqrt((qn * qn + a2 * mn * mn) / B);
        dl = eta * B * hat;
        return hat - oracle_foam_strength(ep + dl, p);
      };
      double qn, mn, dl, lo = 0, hi = 1 / G;
      for (int k = 0; k < 32 && state(hi, qn, mn, dl) > 0; ++k) hi *= 2;
      for (int k = 0; k < 28; ++k) {
        const double mid = (lo + hi) / 2;
        if (state(mid, qn, mn, dl) > 0) lo = mid;
        else hi = mid;
      }
      state((lo + hi) / 2, qn, mn, dl);
      qNew = qn;
      meanNew = mn;
      inc = dl;
    }
  }
  const double traceNew = meanNew / K, scale = q > 1e-20 ? qNew / q : 1;
  double newE[3];
  for (int k = 0; k < 3; ++k) newE[k] = traceNew / 3 + scale * dev[k];
  if (model == 8) {
    double d2 = 0;
    for (int k = 0; k < 3; ++k) d2 += (e[k] - newE[k]) * (e[k] - newE[k]);
    inc = std::sqrt(2.0 / 3.0) * std::sqrt(d2);
  }
  for (int k = 0; k < 3; ++k) out[k] = std::exp(newE[k]);
  *jp_out = jp * std::exp(trace - traceNew);
  *increment = inc;
}

// constitutive.js:52-78 (projectPlastic); models 0, 1 return F unchanged. jp and dilation are
// MPM3.Jp and MPM3.dilation, read and updated (either may be null: 1 and 0, not returned).
// Outputs the projected F, the plastic increment (metal, thermal and pressure returns give their
// own; snow and sand |log(s / s')|), and the cached Kirchhoff stress of constitutive.js:81-86
// (principalStress with mu, lambda: snow's fixed-corotated form, Hencky for the others).
int oracle_project(const double* F, const OracleMaterial* p, double ep, double dt, double T, double* jp,
                   double* dilation, double* Fout, double* increment, double* tau_cache) {
  const int model = p->model;
  if (model < 0 || model > 11) return -1;
  if (model < 2) {
    std::memcpy(Fout, F, 9 * sizeof(double));
    *increment = 0;
    oracle_constitutive_stress(F, model, p->mu, p->lambda, tau_cache);
    return 0;
  }
  double jpv = jp ? *jp : 1.0, dil = dilation ? *dilation : 0.0;
  double u[9], v[9], s[3], proj[3], inc = -1;
  oracle_svd3(F, u, v, s);
  if (model == 2) {
    double ds = 1, dp = 1;
    for (int k = 0; k < 3; ++k) {
      proj[k] = std::max(1 - p->yieldStrain, std::min(1 + p->yieldStrain * .3, s[k]));
      ds *= s[k];
      dp *= proj[k];
    }
    jpv = std::max(.6, std::min(20.0, jpv * ds / dp));
  } else if (model >= 10) {
    oracle_thermal_return(s, model, ep, dt, T, p, proj, &inc);
  } else if (model >= 8) {
    oracle_pressure_return(s, model, jpv, ep, p, proj, &jpv, &inc);
  } else if (model >= 4) {
    oracle_metal_return(s, model, ep, dt, T, p, proj, &inc);
  } else {  // sand
    double e[3];
    for (int k = 0; k < 3; ++k) e[k] = std::log(std::max(s[k], 1e-6));
    const double trace = e[0] + e[1] + e[2] + dil;
    if (trace >= 0) {
      proj[0] = proj[1] = proj[2] = 1;
      dil = trace;
    } else {
      dil = 0;
      double dev[3];
      for (int k = 0; k < 3; ++k) dev[k] = e[k] - trace / 3;
      const double length = std::sqrt(dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]);
      const double sn = std::sin(p->friction * 3.14159265358979323846 / 180), alpha = std::sqrt(2.0 / 3) * 2 * sn / (3 - sn);
      // the reference's 2.5 = (3 lambda + 2 mu) / (2 mu) at lambda = mu
      const double delta = std::max(0.0, length + (3 * p->lambda + 2 * p->mu) / (2 * p->mu) * trace * alpha);
      for (int k = 0; k < 3; ++k) proj[k] = std::exp(e[k] - delta / (length > 0 ? length : 1) * dev[k]);
    }
  }
  if (inc < 0) {  // snow and sand: |log(s / s')|
    double d2 = 0;
    for (int k = 0; k < 3; ++k) d2 += std::log(s[k] / proj[k]) * std::log(s[k] / proj[k]);
    inc = std::sqrt(d2);
  }
  oracle_compose(u, v, proj, Fout);
  *increment = inc;
  if (jp) *jp = jpv;
  if (dilation) *dilation = dil;
  if (model == 2) {  // principalStress of snow: 2 mu (s - 1) s + lambda (J - 1) J
    const double Jp = proj[0] * proj[1] * proj[2];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double t = 0;
        for (int k = 0; k < 3; ++k)
          t += u[a * 3 + k] * (2 * p->mu * (proj[k] - 1) * proj[k] + p->lambda * (Jp - 1) * Jp) * u[b * 3 + k];
        tau_cache[a * 3 + b] = t;
      }
  } else {
    oracle_principal_stress(u, proj, p->mu, p->lambda, tau_cache);
  }
  return 0;
}

// ---------------------------------------------------------------------------
// The step. src/three/mpm.js:56-134 (updateStress, P2G, grid update, G2P + F update,
// return map), with gravity on particles as in src/three/simulation.js:337-344 or on the grid.
// Arrays: x, v (n x 3), C, F, tau_cache (n x 9), ep, T, m, V (n), mat (n, index into mats),
// pinned (n, may be null), cache_valid (n, may be null: stress recomputed from F).
// Optional outputs: grid_mass (nodes), grid_mom (nodes x 3, after P2G incl. gravity),
// grid_vel (nodes x 3, after the grid update).
static inline int64_t node_index(const OracleScene* sc, int x, int y, int z) {
  return ((int64_t)z * sc->dims[1] + y) * sc->dims[0] + x;
}

struct Stencil {
  int base[3];
  double frac[3];
  double w[3][3];
};

// mpm.js:25-32
static inline void stencil(const OracleScene* sc, const double* x, Stencil& st) {
  for (int a = 0; a < 3; ++a) {
    const double q = (x[a] - sc->origin[a]) / sc->H;
    const int b = std::max(0, std::min(sc->dims[a] - 3, (int)std::floor(q - 0.5)));
    const double t = q - b;
    st.base[a] = b;
    st.frac[a] = t;
    st.w[a][0] = 0.5 * (1.5 - t) * (1.5 - t);
    st.w[a][1] = 0.75 - (t - 1) * (t - 1);
    st.w[a][2] = 0.5 * (t - 0.5) * (t - 0.5);
  }
}

int oracle_step(const OracleScene* sc, const OracleMaterial* mats, int32_t nmat, int64_t n,
                double* x, double* v, double* C, double* F, double* ep, double* T, double* jp, double* dilation,
                const double* m, const double* V, const int32_t* mat, const uint8_t* pinned,
                double* tau_cache, uint8_t* cache_valid, double dt, double* grid_mass,
                double* grid_mom, double* grid_vel, int32_t threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
  const int64_t nodes = (int64_t)sc->dims[0] * sc->dims[1] * sc->dims[2];
  const double H = sc->H;
  std::vector<double> gm(nodes, 0.0), gv(nodes * 3, 0.0);
  const bool conduct = sc->cond_k > 0;
  std::vector<double> gh(conduct ? nodes : 0, 0.0), gdT(conduct ? nodes : 0, 0.0);
  std::vector<uint8_t> fixed(nodes, 0);
  std::vector<double> tau((size_t)n * 9);
  for (int64_t p = 0; p < n; ++p)
    if (mat[p] < 0 || mat[p] >= nmat) return -1;

  // gravity on particle velocities before the MPM step (simulation.js:337-344)
  if (!sc->gravity_on_grid) {
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; ++p) {
      if (pinned && pinned[p]) continue;
      for (int a = 0; a < 3; ++a) v[p * 3 + a] += sc->gravity[a] * dt;
    }
  }
  // updateStress (mpm.js:33-39): cached stress for models >= 2 when valid, else from F
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < n; ++p) {
    const OracleMaterial* mp = &mats[mat[p]];
    if (mp->model >= 2 && cache_valid && cache_valid[p])
      std::memcpy(&tau[p * 9], &tau_cache[p * 9], 9 * sizeof(double));
    else
      oracle_constitutive_stress(&F[p * 9], mp->model, mp->mu, mp->lambda, &tau[p * 9]);
    if (mp->model == 2) {  // snow's compaction hardening scales the stress (mpm.js:35-37)
      const double h = oracle_hardening(jp ? jp[p] : 1.0);
      for (int k = 0; k < 9; ++k) tau[p * 9 + k] *= h;
    }
  }
  // P2G (mpm.js:66-85). With threads == 1 it is serial, so the summation order is the
  // particle order; with more threads the scatter uses atomic adds (CPU baseline timing).
  auto p2g_particle = [&](int64_t p, bool atomic) {
    Stencil st;
    stencil(sc, &x[p * 3], st);
    const double mp = m[p];
    double A[9];
    for (int k = 0; k < 9; ++k) A[k] = mp * C[p * 9 + k] - dt * V[p] * 4 / (H * H) * tau[p * 9 + k];
    for (int k = 0; k < 3; ++k)
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
          const int64_t nd = node_index(sc, st.base[0] + i, st.base[1] + j, st.base[2] + k);
          const double w = st.w[0][i] * st.w[1][j] * st.w[2][k];
          const double dx = (i - st.frac[0]) * H, dy = (j - st.frac[1]) * H, dz = (k - st.frac[2]) * H;
          const double add[4] = {w * mp, w * (mp * v[p * 3 + 0] + A[0] * dx + A[1] * dy + A[2] * dz),
                                 w * (mp * v[p * 3 + 1] + A[3] * dx + A[4] * dy + A[5] * dz),
                                 w * (mp * v[p * 3 + 2] + A[6] * dx + A[7] * dy + A[8] * dz)};
          if (conduct) {
            const double hq = w * mp * T[p];
            if (atomic) {
#pragma omp atomic
              gh[nd] += hq;
            } else {
              gh[nd] += hq;
            }
          }
          if (atomic) {
#pragma omp atomic
            gm[nd] += add[0];
#pragma omp atomic
            gv[nd * 3 + 0] += add[1];
#pragma omp atomic
            gv[nd * 3 + 1] += add[2];
#pragma omp atomic
            gv[nd * 3 + 2] += add[3];
          } else {
            gm[nd] += add[0];
            gv[nd * 3 + 0] += add[1];
            gv[nd * 3 + 1] += add[2];
            gv[nd * 3 + 2] += add[3];
          }
          if (pinned && pinned[p] && w > 1e-8) fixed[nd] = 1;
        }
  };
  if (threads == 1) {
    for (int64_t p = 0; p < n; ++p) p2g_particle(p, false);
  } else {
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; ++p) p2g_particle(p, true);
  }
  if (sc->gravity_on_grid) {
    for (int64_t nd = 0; nd < nodes; ++nd)
      for (int a = 0; a < 3; ++a) gv[nd * 3 + a] += dt * gm[nd] * sc->gravity[a];
  }
  if (grid_mass) std::memcpy(grid_mass, gm.data(), nodes * sizeof(double));
  if (grid_mom) std::memcpy(grid_mom, gv.data(), nodes * 3 * sizeof(double));
  // grid update (mpm.js:89-102): v = p/m, fixed nodes and separating slip on all six faces;
  // optional sticky floor (all components zero within one cell of lower[1])
#pragma omp parallel for schedule(static)
  for (int64_t nd = 0; nd < nodes; ++nd) {
    if (!(gm[nd] > sc->mass_eps)) {
      gv[nd * 3] = gv[nd * 3 + 1] = gv[nd * 3 + 2] = 0;
      continue;
    }
    const int ix = (int)(nd % sc->dims[0]);
    const int iy = (int)((nd / sc->dims[0]) % sc->dims[1]);
    const int iz = (int)(nd / ((int64_t)sc->dims[0] * sc->dims[1]));
    const double q[3] = {sc->origin[0] + ix * H, sc->origin[1] + iy * H, sc->origin[2] + iz * H};
    const bool sticky = sc->sticky_floor && q[1] < sc->lower[1] + H;
    for (int a = 0; a < 3; ++a) {
      double vel = gv[nd * 3 + a] / gm[nd];
      if (sticky || fixed[nd] || (q[a] < sc->lower[a] + H && vel < 0) ||
          (q[a] > sc->upper[a] - H && vel > 0))
        vel = 0;
      gv[nd * 3 + a] = vel;
    }
  }
  if (grid_vel) std::memcpy(grid_vel, gv.data(), nodes * 3 * sizeof(double));
  // grid heat conduction between face-neighbour nodes that both hold mass
  if (conduct) {
    std::vector<double> Tn(nodes, 0.0);
    for (int64_t nd = 0; nd < nodes; ++nd)
      if (gm[nd] > sc->mass_eps) Tn[nd] = gh[nd] / gm[nd];
    const double g0 = sc->cond_k * H * dt, mfull = sc->cond_rho * H * H * H;
    const int64_t stride[3] = {1, sc->dims[0], (int64_t)sc->dims[0] * sc->dims[1]};
#pragma omp parallel for schedule(static)
    for (int64_t nd = 0; nd < nodes; ++nd) {
      if (!(gm[nd] > sc->mass_eps)) continue;
      const int idx[3] = {(int)(nd % sc->dims[0]), (int)((nd / sc->dims[0]) % sc->dims[1]),
                          (int)(nd / ((int64_t)sc->dims[0] * sc->dims[1]))};
      double q = 0;
      for (int a = 0; a < 3; ++a)
        for (int d = -1; d <= 1; d += 2) {
          const int pp = idx[a] + d;
          if (pp < 0 || pp >= sc->dims[a]) continue;
          const int64_t nj = nd + d * stride[a];
          if (!(gm[nj] > sc->mass_eps)) continue;
          q += g0 * std::min(1.0, std::min(gm[nd], gm[nj]) / mfull) * (Tn[nj] - Tn[nd]);
        }
      gdT[nd] = q / (gm[nd] * sc->cond_cp);
    }
  }
  // G2P + F update (mpm.js:107-123), then the return map (mpm.js:126-131)
  int status = 0;
#pragma omp parallel for schedule(static) reduction(min : status)
  for (int64_t p = 0; p < n; ++p) {
    if (pinned && pinned[p]) continue;
    Stencil st;
    stencil(sc, &x[p * 3], st);
    double vx = 0, vy = 0, vz = 0, c[9] = {0};
    for (int k = 0; k < 3; ++k)
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
          const int64_t nd = node_index(sc, st.base[0] + i, st.base[1] + j, st.base[2] + k);
          const double w = st.w[0][i] * st.w[1][j] * st.w[2][k];
          const double dx = (i - st.frac[0]) * 4 / H, dy = (j - st.frac[1]) * 4 / H,
                       dz = (k - st.frac[2]) * 4 / H;
          const double a = w * gv[nd * 3], b = w * gv[nd * 3 + 1], cc = w * gv[nd * 3 + 2];
          vx += a; vy += b; vz += cc;
          c[0] += a * dx; c[1] += a * dy; c[2] += a * dz;
          c[3] += b * dx; c[4] += b * dy; c[5] += b * dz;
          c[6] += cc * dx; c[7] += cc * dy; c[8] += cc * dz;
        }
    double Fo[9];
    std::memcpy(Fo, &F[p * 9], sizeof Fo);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double val = Fo[a * 3 + b];
        for (int k = 0; k < 3; ++k) val += dt * c[a * 3 + k] * Fo[k * 3 + b];
        F[p * 9 + a * 3 + b] = val;
      }
    std::memcpy(&C[p * 9], c, sizeof c);
    if (conduct) {
      // node temperature increments, interpolated like the velocity, and relaxation of the particle's
      // offset from the interpolated node temperature at the rate of the finest unresolved mode
      // (wavelength 2H): beta = 1 - exp(-pi^2 alpha dt / H^2). Both parts keep sum m T.
      double dT = 0, Tint = 0;
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i < 3; ++i) {
            const int64_t nd = node_index(sc, st.base[0] + i, st.base[1] + j, st.base[2] + k);
            const double w = st.w[0][i] * st.w[1][j] * st.w[2][k];
            dT += w * gdT[nd];
            Tint += w * (gm[nd] > sc->mass_eps ? gh[nd] / gm[nd] : 0.0);
          }
      const double beta = 1 - std::exp(-9.869604401089358 * sc->cond_k * dt / (sc->cond_rho * sc->cond_cp * H * H));
      T[p] += dT + beta * (Tint - T[p]);
    }
    v[p * 3] = vx; v[p * 3 + 1] = vy; v[p * 3 + 2] = vz;
    x[p * 3] += dt * vx; x[p * 3 + 1] += dt * vy; x[p * 3 + 2] += dt * vz;
    if (sc->clamp_positions)
      for (int a = 0; a < 3; ++a)
        x[p * 3 + a] = std::max(sc->clamp_lo[a], std::min(sc->clamp_hi[a], x[p * 3 + a]));
    const OracleMaterial* mp = &mats[mat[p]];
    if (mp->model >= 2) {
      double Fn[9], inc = 0, tc[9];
      if (oracle_project(&F[p * 9], mp, ep[p], dt, T[p], jp ? &jp[p] : nullptr, dilation ? &dilation[p] : nullptr, Fn,
                         &inc, tc) != 0) {
        status = -2;
        continue;
      }
      std::memcpy(&F[p * 9], Fn, sizeof Fn);
      ep[p] += inc;
      if (tau_cache) std::memcpy(&tau_cache[p * 9], tc, sizeof tc);
      if (cache_valid) cache_valid[p] = 1;
      // plastic-work heating: dT = beta * tau_eq(returned) * dep / (rho0 * cp), tau_eq the
      // Kirchhoff von Mises stress sqrt(6) mu |dev e_returned| (gpu/mixed_material.py:150-172)
      if (mp->beta > 0 && inc > 0 && ((mp->model >= 4 && mp->model <= 7) || mp->model >= 10)) {
        double u[9], vv[9], s[3], e[3];
        oracle_svd3(&F[p * 9], u, vv, s);
        for (int k = 0; k < 3; ++k) e[k] = std::log(std::max(s[k], 1e-6));
        const double tr = (e[0] + e[1] + e[2]) / 3;
        double dn = 0;
        for (int k = 0; k < 3; ++k) dn += (e[k] - tr) * (e[k] - tr);
        const double tau_eq = std::sqrt(6.0) * mp->mu * std::sqrt(dn);
        T[p] += mp->beta * tau_eq * inc * V[p] / (m[p] * mp->cp);
      }
    }
  }
  return status;
}

// src/three/mpm.js:43-55 generalised: c = sqrt((lambda + 2 mu)/rho) per particle
// (reference units: sqrt(19200 stiffness) since lambda + 2mu = 1.2 E = 1.2*16000*stiffness*rho)
double oracle_stable_dt(const OracleScene* sc, const OracleMaterial* mats, int64_t n,
                        const double* v, const double* C, const double* F, const double* m,
                        const double* V, const int32_t* mat, const double* jp) {
  double maxw = 1, grad = 1;
  for (int64_t p = 0; p < n; ++p) {
    double row = 0, col = 0, g = 0;
    for (int a = 0; a < 3; ++a) {
      double r = 0, c = 0;
      for (int b = 0; b < 3; ++b) {
        r += std::fabs(F[p * 9 + a * 3 + b]);
        c += std::fabs(F[p * 9 + b * 3 + a]);
        g += std::fabs(C[p * 9 + a * 3 + b]);
      }
      row = std::max(row, r);
      col = std::max(col, c);
    }
    const OracleMaterial* mp = &mats[mat[p]];
    const double jpp = jp ? jp[p] : 1.0;
    const bool press = mp->model == 8 || mp->model == 9;
    const double compression =
        mp->model == 1 || press ? 1 / std::max(0.05, det3(&F[p * 9]) * (press ? jpp : 1.0)) : 1;
    const double hard = mp->model == 2 ? oracle_hardening(jpp) : 1.0;
    const double c = std::sqrt((mp->lambda + 2 * mp->mu) * hard * V[p] / m[p]);
    const double speed = std::sqrt(v[p * 3] * v[p * 3] + v[p * 3 + 1] * v[p * 3 + 1] + v[p * 3 + 2] * v[p * 3 + 2]);
    maxw = std::max(maxw, speed + c * std::max(1.0, std::max(row * col, compression)));
    grad = std::max(grad, g);
  }
  double dt = std::min(sc->dt_max, std::min(sc->cfl * sc->H / maxw, sc->grad_limit / grad));
  if (sc->cond_k > 0) dt = std::min(dt, 0.9 * sc->cond_rho * sc->cond_cp * sc->H * sc->H / (6 * sc->cond_k));
  return dt;
}

// src/simulation/mechanical-diagnostics.js:9-37 (SI: no sandbox length factor) and
// src/simulation/particle-health.js:12-30. Elastic energy density per reference volume:
// model 0 mu|F-R|^2 + lambda/2 (J-1)^2; model 1 mu/2(|F|^2-3) - mu log J + lambda/2 log^2 J;
// Hencky models (an extension; the reference reports them unsupported) mu|e|^2 + lambda/2 tr^2 e.
void oracle_ledger(const OracleScene* sc, const OracleMaterial* mats, int64_t n, const double* x,
                   const double* v, const double* C, const double* F, const double* ep,
                   const double* m, const double* V, const int32_t* mat, const double* jp, OracleLedger* out) {
  OracleLedger L{};
  L.min_j = INFINITY;
  L.max_j = -INFINITY;
  const double D = sc->H * sc->H / 4;
  for (int64_t p = 0; p < n; ++p) {
    const double* Fp = &F[p * 9];
    const double* Cp = &C[p * 9];
    bool finite = std::isfinite(m[p]);
    for (int a = 0; a < 3; ++a) finite = finite && std::isfinite(x[p * 3 + a]) && std::isfinite(v[p * 3 + a]);
    for (int k = 0; k < 9; ++k) finite = finite && std::isfinite(Fp[k]) && std::isfinite(Cp[k]);
    const double J = det3(Fp);
    if (std::isfinite(J)) {
      L.min_j = std::min(L.min_j, J);
      L.max_j = std::max(L.max_j, J);
      if (J <= 0) L.invalid_j++;
    } else {
      finite = false;
    }
    if (!finite) L.nonfinite++;
    const double mp = m[p];
    const double* xp = &x[p * 3];
    const double* vp = &v[p * 3];
    L.mass += mp;
    L.kinetic += 0.5 * mp * (vp[0] * vp[0] + vp[1] * vp[1] + vp[2] * vp[2]);
    L.potential -= mp * (sc->gravity[0] * xp[0] + sc->gravity[1] * xp[1] + sc->gravity[2] * xp[2]);
    double c2 = 0;
    for (int k = 0; k < 9; ++k) c2 += Cp[k] * Cp[k];
    L.affine += 0.5 * mp * D * c2;
    const double P[3] = {mp * vp[0], mp * vp[1], mp * vp[2]};
    double Hh[3] = {xp[1] * P[2] - xp[2] * P[1], xp[2] * P[0] - xp[0] * P[2], xp[0] * P[1] - xp[1] * P[0]};
    const double spin[3] = {Cp[7] - Cp[5], Cp[2] - Cp[6], Cp[3] - Cp[1]};
    for (int k = 0; k < 3; ++k) {
      Hh[k] += mp * D * spin[k];
      L.momentum[k] += P[k];
      L.angular[k] += Hh[k];
    }
    const OracleMaterial* mt = &mats[mat[p]];
    double W = 0;
    if (!(J > 0)) {
      L.unsupported_elastic++;
    } else if (mt->model == 0 || mt->model == 2) {  // snow with its hardened moduli
      double R[9];
      oracle_rotation(Fp, R);
      double s = 0;
      for (int k = 0; k < 9; ++k) s += (Fp[k] - R[k]) * (Fp[k] - R[k]);
      W = (mt->model == 2 ? oracle_hardening(jp ? jp[p] : 1.0) : 1.0) *
          (mt->mu * s + 0.5 * mt->lambda * (J - 1) * (J - 1));
    } else if (mt->model == 1) {
      double s = 0;
      for (int k = 0; k < 9; ++k) s += Fp[k] * Fp[k];
      const double lj = std::log(J);
      W = 0.5 * mt->mu * (s - 3) - mt->mu * lj + 0.5 * mt->lambda * lj * lj;
    } else {
      double u[9], vv[9], s[3], e[3];
      oracle_svd3(Fp, u, vv, s);
      for (int k = 0; k < 3; ++k) e[k] = std::log(std::max(s[k], 1e-6));
      const double tr = e[0] + e[1] + e[2];
      W = mt->mu * (e[0] * e[0] + e[1] * e[1] + e[2] * e[2]) + 0.5 * mt->lambda * tr * tr;
    }
    L.elastic += V[p] * W;
    if (ep) L.max_plastic = std::max(L.max_plastic, ep[p]);
    double tau[9];
    oracle_constitutive_stress(Fp, mt->model <= 2 ? mt->model : 4, mt->mu, mt->lambda, tau);
    const double jpp = jp ? jp[p] : 1.0;
    if (mt->model == 2)
      for (int k = 0; k < 9; ++k) tau[k] *= oracle_hardening(jpp);
    // Cauchy von Mises over the total volume ratio J Jp for the pressure models (mpm.js:38)
    L.max_von_mises = std::max(L.max_von_mises, oracle_von_mises(tau, J * (mt->model == 8 || mt->model == 9 ? jpp : 1.0)));
  }
  *out = L;
}

// ---------------------------------------------------------------------------
// Solid position regularisation, src/three/solid-sampling.js:5-42 (regularizeSolids), in SI:
// spacing_i = spacing cbrt(clamp(V_i J_i Jp_i / volume_unit, 1/64, 8)) (the reference's 2.8 and
// volume 1), pairs of one part (here: one material index) closer than the mean of their spacings
// pushed apart by (target - r) gain / (r (1/m_i + 1/m_j)) along x_i - x_j, weighted by the inverse
// masses (pinned particles have none), coincident pairs (r below 1e-8 of the reference's units, i.e.
// spacing * 1e-8 / 2.8) along a hashed direction of their indices; gain = 1 - exp(-rate dt); every
// shift scaled by 1 / max(1, max_i |shift_i| / (max_speed dt)), applied to unpinned particles and
// clamped to [lo, hi]. Pairs are visited i < j in index order like the reference's loop over cells
// (the order changes only the rounding of the sums). jp may be null (1).
struct OracleRegularizer {
  double spacing, volume_unit, max_speed, rate;
};

void oracle_regularize(const OracleRegularizer* rg, const OracleMaterial* mats, int64_t n, double* x,
                       const double* F, const double* jp, const double* V, const double* m, const int32_t* mat,
                       const uint8_t* pinned, double dt, const double* lo, const double* hi) {
  std::vector<double> target(n), inv(n), dx((size_t)n * 3, 0.0);
  for (int64_t i = 0; i < n; ++i) {
    const int model = mats[mat[i]].model;
    const double j = (model == 2 || model == 8 || model == 9) && jp ? jp[i] : 1.0;
    const double vol = std::max(.015625, std::min(8.0, V[i] * det3(&F[i * 9]) * j / rg->volume_unit));
    target[i] = rg->spacing * std::cbrt(vol);
    inv[i] = pinned && pinned[i] ? 0.0 : 1.0 / m[i];
  }
  // cell list with cells as large as the largest possible target (2 spacing)
  const double hc = 2 * rg->spacing;
  double lo_c[3] = {INFINITY, INFINITY, INFINITY};
  for (int64_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) lo_c[a] = std::min(lo_c[a], x[i * 3 + a]);
  std::vector<std::vector<int64_t>> cells;
  std::vector<int64_t> cell_of(n);
  int dims[3] = {1, 1, 1};
  for (int64_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) dims[a] = std::max(dims[a], (int)std::floor((x[i * 3 + a] - lo_c[a]) / hc) + 1);
  cells.resize((size_t)dims[0] * dims[1] * dims[2]);
  auto coord = [&](int64_t i, int a) { return (int)std::floor((x[i * 3 + a] - lo_c[a]) / hc); };
  for (int64_t i = 0; i < n; ++i) {
    const int64_t c = ((int64_t)coord(i, 2) * dims[1] + coord(i, 1)) * dims[0] + coord(i, 0);
    cell_of[i] = c;
    cells[c].push_back(i);
  }
  const double gain = 1 - std::exp(-rg->rate * dt), eps = rg->spacing * 1e-8 / 2.8;
  for (int64_t i = 0; i < n; ++i) {
    const int ci[3] = {coord(i, 0), coord(i, 1), coord(i, 2)};
    for (int z = -1; z <= 1; ++z)
      for (int y = -1; y <= 1; ++y)
        for (int xx = -1; xx <= 1; ++xx) {
          const int cz = ci[2] + z, cy = ci[1] + y, cx = ci[0] + xx;
          if (cz < 0 || cy < 0 || cx < 0 || cz >= dims[2] || cy >= dims[1] || cx >= dims[0]) continue;
          for (int64_t j : cells[((int64_t)cz * dims[1] + cy) * dims[0] + cx]) {
            if (j <= i || mat[i] != mat[j]) continue;
            const double total = inv[i] + inv[j];
            if (!(total > 0)) continue;
            double d[3] = {x[i * 3] - x[j * 3], x[i * 3 + 1] - x[j * 3 + 1], x[i * 3 + 2] - x[j * 3 + 2]};
            double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            const double t = (target[i] + target[j]) * .5;
            if (r >= t) continue;
            double q;
            if (r < eps) {
              const uint32_t h = (uint32_t)(i + 1) * 73856093u ^ (uint32_t)(j + 1) * 19349663u;
              d[0] = (h & 1023) / 511.5 - 1;
              d[1] = ((h >> 10) & 1023) / 511.5 - 1;
              d[2] = ((h >> 20) & 1023) / 511.5 - 1;
              r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
              q = t * gain / (r * total);
            } else {
              q = (t - r) * gain / (r * total);
            }
            for (int a = 0; a < 3; ++a) {
              dx[i * 3 + a] += d[a] * q * inv[i];
              dx[j * 3 + a] -= d[a] * q * inv[j];
            }
          }
        }
  }
  double scale = 1;
  const double budget = rg->max_speed * dt;
  for (int64_t i = 0; i < n; ++i)
    scale = std::max(scale, std::sqrt(dx[i * 3] * dx[i * 3] + dx[i * 3 + 1] * dx[i * 3 + 1] + dx[i * 3 + 2] * dx[i * 3 + 2]) / budget);
  for (int64_t i = 0; i < n; ++i) {
    if (pinned && pinned[i]) continue;
    for (int a = 0; a < 3; ++a) x[i * 3 + a] = std::max(lo[a], std::min(hi[a], x[i * 3 + a] + dx[i * 3 + a] / scale));
  }
}

// ---------------------------------------------------------------------------
// Particle-pair heat exchange, src/thermal.js:35-56 (exchangeHeat), over the pairs of
// src/three/simulation.js:168-174 (r in (1e-6, H) of the reference's units: here
// (radius * 1.25e-7, radius)), then the phase decode of src/three/phase-change.js:12-18 for
// materials with latent > 0 (h <= cp Tm: solid at h / cp; h >= cp Tm + L: molten at (h - L) / cp;
// between: Tm with the previous phase) and h / cp otherwise. A phase switch resets the
// particle's deformation (MPM3.resetParticle) and unpins a molten one. Enthalpy h (J/kg) and the
// molten flags are the state; T is written from them. Returns the sum of |Q| over pairs.
struct OracleHeat {
  double radius, geometry, heat_rate;
  int32_t ambient, pad;
  double ambient_T, ambient_rate;
};

// phaseEnthalpy (src/three/phase-change.js:11)
double oracle_phase_enthalpy(double T, const OracleMaterial* p) {
  return p->cp * T + (p->latent > 0 && T > p->Tphase ? p->latent : 0.0);
}

double oracle_exchange_heat(const OracleHeat* x, const OracleMaterial* mats, int64_t n, const double* pos, double* T,
                            double* h, uint8_t* melted, const double* m, const int32_t* mat, uint8_t* pinned,
                            double* F, double* C, double* ep, double* jp, double* dilation, double dt) {
  const double R = x->radius, eps = R * 1.25e-7;
  // pairs i < j in index order (the reference collects them over neighbour cells; the pair set and
  // each pair's terms are the same)
  struct Pair { int64_t i, j; double g; };
  std::vector<Pair> pairs;
  std::vector<std::vector<int64_t>> cells;
  double lo[3] = {INFINITY, INFINITY, INFINITY};
  for (int64_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) lo[a] = std::min(lo[a], pos[i * 3 + a]);
  int dims[3] = {1, 1, 1};
  auto coord = [&](int64_t i, int a) { return (int)std::floor((pos[i * 3 + a] - lo[a]) / R); };
  for (int64_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) dims[a] = std::max(dims[a], coord(i, a) + 1);
  cells.resize((size_t)dims[0] * dims[1] * dims[2]);
  for (int64_t i = 0; i < n; ++i) cells[((int64_t)coord(i, 2) * dims[1] + coord(i, 1)) * dims[0] + coord(i, 0)].push_back(i);
  for (int64_t i = 0; i < n; ++i) {
    const int ci[3] = {coord(i, 0), coord(i, 1), coord(i, 2)};
    for (int z = -1; z <= 1; ++z)
      for (int y = -1; y <= 1; ++y)
        for (int xx = -1; xx <= 1; ++xx) {
          const int cz = ci[2] + z, cy = ci[1] + y, cx = ci[0] + xx;
          if (cz < 0 || cy < 0 || cx < 0 || cz >= dims[2] || cy >= dims[1] || cx >= dims[0]) continue;
          for (int64_t j : cells[((int64_t)cz * dims[1] + cy) * dims[0] + cx]) {
            if (j <= i) continue;
            const double d[3] = {pos[i * 3] - pos[j * 3], pos[i * 3 + 1] - pos[j * 3 + 1], pos[i * 3 + 2] - pos[j * 3 + 2]};
            const double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            if (!(r > eps && r < R)) continue;
            const double ki = mats[mat[i]].kcond, kj = mats[mat[j]].kcond;
            const double kh = ki + kj > 0 ? 2 * ki * kj / (ki + kj) : 0.0;
            pairs.push_back({i, j, (1 - r / R) * x->geometry * x->heat_rate * kh});
          }
        }
  }
  std::vector<double> budget(n, 0.0), heat(n, 0.0);
  for (const Pair& p : pairs) {
    budget[p.i] += p.g;
    budget[p.j] += p.g;
  }
  for (int64_t i = 0; i < n; ++i)
    budget[i] = budget[i] ? std::min(1.0, .45 * m[i] * mats[mat[i]].cp / (dt * budget[i])) : 1.0;
  double exchanged = 0;
  for (const Pair& p : pairs) {
    const double q = (T[p.j] - T[p.i]) * p.g * dt * std::min(budget[p.i], budget[p.j]);
    exchanged += std::fabs(q);
    heat[p.i] += q;
    heat[p.j] -= q;
  }
  for (int64_t i = 0; i < n; ++i) {
    const OracleMaterial* mp = &mats[mat[i]];
    h[i] += heat[i] / m[i];
    if (x->ambient) h[i] -= (T[i] - x->ambient_T) * mp->cp * dt * x->ambient_rate;
    bool liquid = false;
    if (mp->latent > 0) {
      const double start = mp->cp * mp->Tphase, end = start + mp->latent;
      if (h[i] <= start) {
        T[i] = h[i] / mp->cp;
      } else if (h[i] >= end) {
        liquid = true;
        T[i] = (h[i] - mp->latent) / mp->cp;
      } else {
        liquid = melted[i] != 0;
        T[i] = mp->Tphase;
      }
    } else {
      T[i] = h[i] / mp->cp;
    }
    if (liquid != (melted[i] != 0)) {
      melted[i] = liquid ? 1 : 0;
      for (int k = 0; k < 9; ++k) {
        F[i * 9 + k] = (k % 4 == 0) ? 1.0 : 0.0;
        C[i * 9 + k] = 0.0;
      }
      ep[i] = 0;
      if (jp) jp[i] = 1;
      if (dilation) dilation[i] = 0;
      if (liquid && pinned) pinned[i] = 0;
    }
  }
  return exchanged;
}

}  // extern "C"
