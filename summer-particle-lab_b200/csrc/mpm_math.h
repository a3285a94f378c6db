// Constitutive and transfer math of the MLS-MPM solid step, FP32, for device and host.
//
// Centred form. Deformation gradients are held as D = F - I, so small elastic strains keep full
// FP32 precision (F ~ 1 + 1e-3 would keep only 4 significant digits of the strain). The left
// Cauchy-Green tensor is formed as B - I = D + D^T + D D^T, its eigenvalues beta_k = sigma_k^2 - 1
// are found by cyclic Jacobi rotations, and strains use log1p/expm1.
//
// The eigen-decomposition of F F^T replaces the reference's SVD of F (src/three/constitutive.js:
// 22-42) and Newton polar iteration (src/three/math.js:16-24): with F = U S V^T the left singular
// vectors U are the eigenvectors of F F^T and
//   fixed-corotated  (F - R) F^T = (V_l - I) V_l = U diag((s-1) s) U^T      (math.js:25-32)
//   Hencky           tau = U diag(2 mu e + lambda tr e) U^T, e = log s      (constitutive.js:101-104)
//   return map       F' = U diag(s'/s) U^T F                                 (constitutive.js:77)
// so V is never needed.
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define MPM_HD __host__ __device__ __forceinline__
#define MPM_NOINLINE static __host__ __device__ __noinline__
#else
#define MPM_HD inline
#define MPM_NOINLINE static __attribute__((noinline))
#endif

namespace mpm {

struct Sym3 {
  float xx, yy, zz, xy, xz, yz;
};

MPM_HD float rsqrt_hd(float x) {
#if defined(__CUDA_ARCH__)
  return rsqrtf(x);
#else
  return 1.0f / sqrtf(x);
#endif
}

// Quadratic B-spline weights for fraction t in [0.5, 1.5) (src/three/mpm.js:28-30)
MPM_HD void bspline_weights(float t, float w[3]) {
  const float a = 1.5f - t, b = t - 1.0f, c = t - 0.5f;
  w[0] = 0.5f * a * a;
  w[1] = 0.75f - b * b;
  w[2] = 0.5f * c * c;
}

// B - I = D + D^T + D D^T
MPM_HD Sym3 cauchy_green_minus_identity(const float D[9]) {
  Sym3 b;
  b.xx = 2.f * D[0] + (D[0] * D[0] + D[1] * D[1] + D[2] * D[2]);
  b.yy = 2.f * D[4] + (D[3] * D[3] + D[4] * D[4] + D[5] * D[5]);
  b.zz = 2.f * D[8] + (D[6] * D[6] + D[7] * D[7] + D[8] * D[8]);
  b.xy = D[1] + D[3] + (D[0] * D[3] + D[1] * D[4] + D[2] * D[5]);
  b.xz = D[2] + D[6] + (D[0] * D[6] + D[1] * D[7] + D[2] * D[8]);
  b.yz = D[5] + D[7] + (D[3] * D[6] + D[4] * D[7] + D[5] * D[8]);
  return b;
}

// det(I + D) - 1 = tr D + (sum of principal 2x2 minors of D) + det D
MPM_HD float det_minus_one(const float D[9]) {
  const float tr = D[0] + D[4] + D[8];
  const float m2 = (D[0] * D[4] - D[1] * D[3]) + (D[0] * D[8] - D[2] * D[6]) + (D[4] * D[8] - D[5] * D[7]);
  const float d3 = D[0] * (D[4] * D[8] - D[5] * D[7]) - D[1] * (D[3] * D[8] - D[5] * D[6]) +
                   D[2] * (D[3] * D[7] - D[4] * D[6]);
  return tr + m2 + d3;
}

// One Jacobi rotation annihilating a_pq (Golub & Van Loan, symmetric Schur 2x2):
// theta = (a_qq - a_pp) / (2 a_pq), t = sgn(theta)/(|theta| + sqrt(theta^2 + 1)),
// c = 1/sqrt(1 + t^2), s = t c. r is the third index. U columns p, q rotate with it.
MPM_HD void jacobi_rotate(float& app, float& aqq, float& apq, float& arp, float& arq, float& u0p,
                          float& u0q, float& u1p, float& u1q, float& u2p, float& u2q) {
  if (apq == 0.f) return;
  const float theta = (aqq - app) / (2.f * apq);
  const float t = copysignf(1.f, theta) / (fabsf(theta) + sqrtf(fmaf(theta, theta, 1.f)));
  const float c = rsqrt_hd(fmaf(t, t, 1.f));
  const float s = t * c;
  app = fmaf(-t, apq, app);
  aqq = fmaf(t, apq, aqq);
  apq = 0.f;
  const float rp = arp, rq = arq;
  arp = c * rp - s * rq;
  arq = s * rp + c * rq;
  float x, y;
  x = u0p; y = u0q; u0p = c * x - s * y; u0q = s * x + c * y;
  x = u1p; y = u1q; u1p = c * x - s * y; u1q = s * x + c * y;
  x = u2p; y = u2q; u2p = c * x - s * y; u2q = s * x + c * y;
}

// Cyclic Jacobi eigen-decomposition of a symmetric 3x3 matrix: a = U diag(lam) U^T, U row-major
// with eigenvectors in columns. Stops when the off-diagonal mass is below 2^-24 of the diagonal.
MPM_HD void sym_eig3(Sym3 a, float lam[3], float U[9]) {
  float u00 = 1.f, u01 = 0.f, u02 = 0.f, u10 = 0.f, u11 = 1.f, u12 = 0.f, u20 = 0.f, u21 = 0.f,
        u22 = 1.f;
  for (int sweep = 0; sweep < 6; ++sweep) {
    const float off = fabsf(a.xy) + fabsf(a.xz) + fabsf(a.yz);
    const float dia = fabsf(a.xx) + fabsf(a.yy) + fabsf(a.zz);
    if (!(off > 5.9604645e-8f * dia) && sweep > 0) break;
    if (off == 0.f) break;
    jacobi_rotate(a.xx, a.yy, a.xy, a.xz, a.yz, u00, u01, u10, u11, u20, u21);  // (0,1), r=2
    jacobi_rotate(a.xx, a.zz, a.xz, a.xy, a.yz, u00, u02, u10, u12, u20, u22);  // (0,2), r=1
    jacobi_rotate(a.yy, a.zz, a.yz, a.xy, a.xz, u01, u02, u11, u12, u21, u22);  // (1,2), r=0
  }
  lam[0] = a.xx; lam[1] = a.yy; lam[2] = a.zz;
  U[0] = u00; U[1] = u01; U[2] = u02;
  U[3] = u10; U[4] = u11; U[5] = u12;
  U[6] = u20; U[7] = u21; U[8] = u22;
}

// S = U diag(d) U^T (symmetric)
MPM_HD Sym3 rotate_diag(const float U[9], const float d[3]) {
  Sym3 s;
  s.xx = U[0] * U[0] * d[0] + U[1] * U[1] * d[1] + U[2] * U[2] * d[2];
  s.yy = U[3] * U[3] * d[0] + U[4] * U[4] * d[1] + U[5] * U[5] * d[2];
  s.zz = U[6] * U[6] * d[0] + U[7] * U[7] * d[1] + U[8] * U[8] * d[2];
  s.xy = U[0] * U[3] * d[0] + U[1] * U[4] * d[1] + U[2] * U[5] * d[2];
  s.xz = U[0] * U[6] * d[0] + U[1] * U[7] * d[1] + U[2] * U[8] * d[2];
  s.yz = U[3] * U[6] * d[0] + U[4] * U[7] * d[1] + U[5] * U[8] * d[2];
  return s;
}

// Product of two commuting symmetric matrices (polynomials in the same B): symmetric, 6 entries.
MPM_HD Sym3 sym_mul(const Sym3& a, const Sym3& b) {
  Sym3 r;
  r.xx = a.xx * b.xx + a.xy * b.xy + a.xz * b.xz;
  r.yy = a.xy * b.xy + a.yy * b.yy + a.yz * b.yz;
  r.zz = a.xz * b.xz + a.yz * b.yz + a.zz * b.zz;
  r.xy = a.xx * b.xy + a.xy * b.yy + a.xz * b.yz;
  r.xz = a.xx * b.xz + a.xy * b.yz + a.xz * b.zz;
  r.yz = a.xy * b.xz + a.yy * b.yz + a.yz * b.zz;
  return r;
}

MPM_HD float sym_norm(const Sym3& a) {
  return sqrtf(a.xx * a.xx + a.yy * a.yy + a.zz * a.zz + 2.f * (a.xy * a.xy + a.xz * a.xz + a.yz * a.yz));
}

// Number of power-series terms for a symmetric argument of Frobenius norm r (a bound on its
// spectral radius) so that the truncation r^(n+1)/(n+1) stays below ~1e-8 r; 0 means "too large:
// use the eigen-decomposition".
constexpr float kSeriesMaxNorm = 0.15f;
MPM_HD int series_terms(float r) {
  return r <= 1e-3f ? 3 : r <= 1e-2f ? 4 : r <= 3e-2f ? 5 : r <= 6e-2f ? 6 : r <= 0.1f ? 8 : r <= kSeriesMaxNorm ? 10 : 0;
}

// The same choice from the squared norm (no square root on the per-particle path).
MPM_HD float sym_norm2(const Sym3& a) {
  return a.xx * a.xx + a.yy * a.yy + a.zz * a.zz + 2.f * (a.xy * a.xy + a.xz * a.xz + a.yz * a.yz);
}
MPM_HD int series_terms_sq(float r2) {
  return r2 <= 1e-6f ? 3 : r2 <= 1e-4f ? 4 : r2 <= 9e-4f ? 5 : r2 <= 3.6e-3f ? 6 : r2 <= 1e-2f ? 8
       : r2 <= kSeriesMaxNorm * kSeriesMaxNorm ? 10 : 0;
}

// Coefficient c_k of x^(k+1) in the series (Taylor coefficients, exact rationals):
//   kind 0  log(1 + x)      = x - x^2/2 + x^3/3 - ...          c_k = (-1)^k / (k + 1)
//   kind 1  sqrt(1 + x) - 1 = x/2 - x^2/8 + x^3/16 - ...       c_k = binom(1/2, k + 1)
//   kind 2  exp(x) - 1      = x + x^2/2 + x^3/6 + ...          c_k = 1 / (k + 1)!
MPM_HD constexpr double series_coeff(int kind, int k) {
  if (kind == 0) return ((k & 1) ? -1.0 : 1.0) / (k + 1);
  double c = 1.0;
  if (kind == 1) {
    for (int j = 0; j <= k; ++j) c *= (0.5 - j) / (j + 1);
    return c;
  }
  for (int j = 1; j <= k + 1; ++j) c /= j;
  return c;
}

// sum_{k=0..N-1} c_k B^(k+1) by Horner's scheme: B (c_0 I + B (c_1 I + ... + B c_(N-1) I)),
// fully unrolled with compile-time coefficients
template <int KIND, int N>
MPM_HD Sym3 series_n(const Sym3& B) {
  constexpr float last = static_cast<float>(series_coeff(KIND, N - 1));
  Sym3 Q{last, last, last, 0.f, 0.f, 0.f};
#pragma unroll
  for (int k = N - 2; k >= 0; --k) {
    Q = sym_mul(B, Q);
    const float ck = static_cast<float>(series_coeff(KIND, k));
    Q.xx += ck;
    Q.yy += ck;
    Q.zz += ck;
  }
  return sym_mul(B, Q);
}

template <int KIND>
MPM_HD Sym3 matrix_series(const Sym3& B, int n) {
  switch (n) {
    case 3: return series_n<KIND, 3>(B);
    case 4: return series_n<KIND, 4>(B);
    case 5: return series_n<KIND, 5>(B);
    case 6: return series_n<KIND, 6>(B);
    case 8: return series_n<KIND, 8>(B);
    default: return series_n<KIND, 10>(B);
  }
}

// Per-material constants on the device (SI). See mpm_material in include/mpm_b200.h.
struct MaterialDev {
  int model;
  float mu, lam;
  float yield_stress, hardening;
  float T_ref, inv_T_span, hot_ratio;
  float heat_per_work;   // heat_fraction / specific_heat (K per J/kg)
  float cp;              // specific heat (J/kg/K)
  float wave_modulus;    // lambda + 2 mu (CFL wave speed c = sqrt(wave_modulus V / m))
  // Johnson-Cook, models 6 and 7 (src/three/metal-plasticity.js:12-19): yield_stress = A,
  // hardening = B, flow = (A + B ep^n)(1 + C ln max(1, rate / rate0))(1 - theta^m), the last
  // factor for model 6 only, theta = clamp((T - T_ref) / (T_melt - T_ref), 0, 1)
  float jc_n, jc_C, jc_inv_rate0, jc_inv_T_span, jc_m;
  // Norton creep, model 11 (src/three/thermal-plasticity.js:17-21): log rate = log A0 +
  // clamp(Q/R (1/(T_ref + off) - 1/max(1, T + off)), -60, 60) + n log(q / stress)
  float cr_log_rate, cr_Q_over_R, cr_inv_Tref_abs, cr_T_offset, cr_n, cr_inv_stress;
  int cr_on;             // creep rate > 0
};

// Constants of the laws with a second history scalar, in their own table so the row the hot J2
// path copies stays small.
struct MaterialExt {
  // snow, model 2 (src/three/constitutive.js:48,58-60): s - 1 clamped to [snow_lo, snow_hi]
  float snow_lo, snow_hi;
  // sand, model 3 (constitutive.js:66-74): alpha (3 lambda + 2 mu) / (2 mu) with
  // alpha = sqrt(2/3) 2 sin(phi) / (3 - sin(phi))
  float sand_k;
  // pressure models 8 and 9 (src/three/pressure-plasticity.js:11-48): bulk modulus lambda + 2 mu / 3,
  // cohesive Drucker-Prager cohesion, slope, dilatancy and tension cutoff; Deshpande-Fleck alpha^2,
  // 1 + alpha^2 / 9, plateau, gamma, densification, beta and 1 / eps_D
  float bulk;
  float dp_c, dp_a, dp_b, dp_T;
  float df_a2, df_B, df_plateau, df_gamma, df_densify, df_beta, df_inv_epsd;
  // particle-pair heat exchange and enthalpy phase change (src/thermal.js:35-56,
  // src/three/phase-change.js:4-18): conductivity, melting point, latent heat (0: no phase change)
  float conductivity, melting_point, latent;
};

// Models whose state carries a second history scalar (aux): Jp - 1 for snow and the pressure
// models (the plastic volume ratio, src/three/mpm.js:9), the dilation for sand.
MPM_HD bool aux_model(int model) { return model == 2 || model == 3 || model == 8 || model == 9; }

// Johnson-Cook flow stress (src/three/metal-plasticity.js:12-19).
MPM_HD float jc_flow(const MaterialDev& mt, float ep, float rate, float T) {
  const float rf = 1.f + mt.jc_C * logf(fmaxf(1.f, rate * mt.jc_inv_rate0));
  float f = (mt.yield_stress + mt.hardening * powf(fmaxf(ep, 0.f), mt.jc_n)) * rf;
  if (mt.model == 6) {
    const float th = fminf(1.f, fmaxf(0.f, (T - mt.T_ref) * mt.jc_inv_T_span));
    f *= 1.f - powf(th, mt.jc_m);
  }
  return f;
}

// Norton creep log strain rate at von Mises stress q (src/three/thermal-plasticity.js:17-21).
MPM_HD float creep_log_rate(const MaterialDev& mt, float q, float T) {
  if (!mt.cr_on || !(q > 0.f)) return -INFINITY;
  const float act = fminf(60.f, fmaxf(-60.f, mt.cr_Q_over_R * (mt.cr_inv_Tref_abs - 1.f / fmaxf(1.f, T + mt.cr_T_offset))));
  return mt.cr_log_rate + act + mt.cr_n * logf(q * mt.cr_inv_stress);
}

// The Johnson-Cook consistency condition q - 3 mu / J dep = flow(ep + dep, dep / dt, T) for a trial
// stress above the initial flow stress: 24 bisections of [0, q J / (3 mu)], the reference's bracket
// and count (src/three/metal-plasticity.js:28-34).
MPM_HD float jc_bisect(const MaterialDev& mt, float q, float J, float ep, float T, float dt) {
  const float slope = 3.f * mt.mu / J;
  float lo = 0.f, hi = q / slope;
  const float inv_dt = 1.f / fmaxf(dt, 1e-12f);
  for (int it = 0; it < 24; ++it) {
    const float mid = 0.5f * (lo + hi);
    if (q - slope * mid > jc_flow(mt, ep + mid, mid * inv_dt, T)) lo = mid;
    else hi = mid;
  }
  return 0.5f * (lo + hi);
}

// Plastic strain increment of the J2-type returns for the trial von Mises stress q
// (src/three/metal-plasticity.js:20-27, src/three/thermal-plasticity.js:22-37): closed form for
// models 4, 5 and 10, 24 bisections of the consistency condition for Johnson-Cook (6, 7), 32
// bisections of the creep rate for Norton creep (11), with the reference's brackets.
MPM_HD float plastic_increment(const MaterialDev& mt, float q, float J, float ep, float T, float dt) {
  const float slope = 3.f * mt.mu / J;
  if (mt.model == 6 || mt.model == 7) {
    if (!(q > jc_flow(mt, ep, 0.f, T))) return 0.f;
    return jc_bisect(mt, q, J, ep, T, dt);
  }
  if (mt.model == 11) {
    if (!(dt > 0.f && mt.cr_on && q > 1e-20f)) return 0.f;
    float lo = 0.f, hi = q / slope;
    for (int it = 0; it < 32; ++it) {
      const float mid = 0.5f * (lo + hi);
      if (logf(mid / dt) < creep_log_rate(mt, fmaxf(0.f, q - slope * mid), T)) lo = mid;
      else hi = mid;
    }
    return 0.5f * (lo + hi);
  }
  float soft = 1.f;
  if (mt.model == 10) {
    const float theta = fminf(1.f, fmaxf(0.f, (T - mt.T_ref) * mt.inv_T_span));
    soft = 1.f - (1.f - mt.hot_ratio) * theta;
  }
  const float yield = (mt.yield_stress + (mt.model == 4 ? 0.f : mt.hardening * ep)) * soft;
  if (!(q > yield)) return 0.f;
  const float hard = mt.model == 4 ? 0.f : mt.hardening * soft;
  return (q - yield) / (slope + hard);
}

// ---- Learned Johnson-Cook return (models 6 and 7) ------------------------------------------
// The consistency condition of src/three/metal-plasticity.js:28-34 in dimensionless form: with
// slope = 3 mu / J, the bracket s = q / slope and dep = u s (u in [0, 1]),
//   g(u) = 1 - u - flow(ep + u s, u s / dt, T) / q,
// decreasing in u, zero at the return. The reference bisects it 24 times. The learned form takes a
// network's guess of u, refines it by Newton steps on g and accepts the result only if |g| <= tol
// (the stress residual |q - slope dep - flow| is then at most tol q); otherwise the caller runs the
// exact bisection.

// Hardware approximations for the learned return's refinement and network inputs (device), the
// libm functions on the host. Relative errors are a few 1e-7 over the arguments used here, far
// below the gate's tolerance (1e-5 of the trial stress), and the gate is evaluated with the same
// functions, so an accepted increment's true residual is within the tolerance plus that error.
MPM_HD float fast_logf(float x) {
#if defined(__CUDA_ARCH__)
  return __logf(x);
#else
  return logf(x);
#endif
}

MPM_HD float fast_expf(float x) {
#if defined(__CUDA_ARCH__)
  return __expf(x);
#else
  return expf(x);
#endif
}

// x^y for x > 0
MPM_HD float fast_powf(float x, float y) {
#if defined(__CUDA_ARCH__)
  return __powf(x, y);
#else
  return powf(x, y);
#endif
}

MPM_HD float fast_divf(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fdividef(a, b);
#else
  return a / b;
#endif
}

// Flow stress and its derivative with respect to dep at dep = d >= 0 (fast functions).
MPM_HD float jc_flow_d(const MaterialDev& mt, float ep, float d, float inv_dt, float soft, float& dflow) {
  const float e = fmaxf(ep + d, 1e-30f);
  const float pw = fast_powf(e, mt.jc_n);
  const float hard = mt.yield_stress + mt.hardening * pw;
  const float r = d * inv_dt * mt.jc_inv_rate0;
  const bool rate_on = r > 1.f;
  const float rf = 1.f + mt.jc_C * fast_logf(fmaxf(r, 1.f));
  dflow = soft * (mt.hardening * mt.jc_n * fast_divf(pw, e) * rf + (rate_on ? fast_divf(hard * mt.jc_C, d) : 0.f));
  return soft * hard * rf;
}

// Thermal softening factor of model 6 (1 for model 7).
MPM_HD float jc_soft(const MaterialDev& mt, float T) {
  if (mt.model != 6) return 1.f;
  const float th = fminf(1.f, fmaxf(0.f, (T - mt.T_ref) * mt.jc_inv_T_span));
  return 1.f - powf(th, mt.jc_m);
}

// The eight network inputs of a plastic Johnson-Cook trial state (q > flow(ep, 0, T)); all are
// dimensionless, so one network serves every material with the same B / A, n and C:
//   a = A soft / q, the hardening at ep and at ep + s relative to q, C ln max(1, s / (dt rate0)),
//   log10 of the bracket s, ep, 1 - a - h0 and the network's bias input. Fast functions: the
//   inputs only steer the guess, which the refinement and the gate check.
MPM_NOINLINE void jc_features(const MaterialDev& mt, float q, float J, float ep, float T, float dt, float x[8]) {
  const float slope = 3.f * mt.mu / J;
  const float s = q / slope;
  const float soft = jc_soft(mt, T);
  const float iq = 1.f / q;
  const float e0 = fmaxf(ep, 0.f);
  const float a = mt.yield_stress * soft * iq;
  const float h0 = mt.hardening * soft * fast_powf(fmaxf(e0, 1e-30f), mt.jc_n) * iq;
  const float h1 = mt.hardening * soft * fast_powf(e0 + s, mt.jc_n) * iq;
  const float L = fast_logf(fmaxf(1.f, s * fast_divf(mt.jc_inv_rate0, fmaxf(dt, 1e-30f))));
  x[0] = a;
  x[1] = h0;
  x[2] = h1 - h0;
  x[3] = mt.jc_C * L;
  x[4] = 0.10857362f * fast_logf(fmaxf(s, 1e-12f)) + 1.5f;  // 0.25 log10(s) + 1.5
  x[5] = ep;
  x[6] = 1.f - a - h0;
  x[7] = 1.f;
}

// Newton refinement of a predicted root u and the gate. The rate factor max(1, rate / rate0) has a
// kink at u_k = dt rate0 / s, where the slope of g jumps; g is smooth on either side, so when the
// kink lies inside the bracket the refinement first finds the side of the root (the sign of g(u_k)).
// Left of the kink Newton runs on v = u; right of it on v = ln(u / u_k), in which the logarithmic
// rate term is linear (the curvature that slows Newton on u just past the kink). Both sides share
// one loop (the side only selects the map from v to u), so the lanes of a warp do not split by
// side. At most `newton` steps, stopping as soon as |g| <= tol; a step that would leave the side's
// interval is replaced by the midpoint toward its end. Returns dep = u s, and ok when the final
// |g(u)| <= tol (returned by value: a reference output would give the caller's variable an address).
struct JcRefined {
  float dep;
  bool ok;
};
MPM_NOINLINE JcRefined jc_refine(const MaterialDev& mt, float q, float J, float ep, float T, float dt, float u_pred,
                                 float tol, int newton) {
  const float slope = 3.f * mt.mu / J;
  const float s = q / slope;
  const float soft = jc_soft(mt, T);
  const float inv_dt = 1.f / fmaxf(dt, 1e-12f);
  const float iq = 1.f / q;
  const float sq = s * iq;
  float df;
  const float uk = mt.jc_C > 0.f ? 1.f / (s * inv_dt * mt.jc_inv_rate0) : 2.f;
  bool right = false;  // the root lies past the kink (the rate term is on)
  if (uk > 0.f && uk < 1.f) right = 1.f - uk - jc_flow_d(mt, ep, uk * s, inv_dt, soft, df) * iq > 0.f;
  const float vhi = right ? -fast_logf(uk) : fminf(1.f, uk);
  float v = right ? fast_logf(fast_divf(fmaxf(u_pred, uk), uk)) : u_pred;
  v = fminf(vhi, fmaxf(0.f, v));
  float u, g;
  for (int k = 0;; ++k) {
    u = right ? uk * fast_expf(v) : v;
    g = 1.f - u - jc_flow_d(mt, ep, u * s, inv_dt, soft, df) * iq;
    if (k >= newton || fabsf(g) <= tol) break;
    const float dgu = -1.f - df * sq;  // dg / du
    float vn = v - fast_divf(g, right ? dgu * u : dgu);
    if (!(vn > 0.f)) vn = 0.5f * v;
    if (!(vn < vhi)) vn = 0.5f * (v + vhi);
    v = vn;
  }
  return {u * s, fabsf(g) <= tol};
}

struct ConstitutiveOut {
  Sym3 tau;       // Kirchhoff stress for the next P2G
  float dep;      // plastic strain increment
  float dT;       // temperature increment from plastic work
  float Jm1;      // det F - 1 after the return
};

// Deshpande-Fleck foam strength (src/three/pressure-plasticity.js:11-14); fully densified
// (ep >= eps_D) is given an effectively infinite strength.
MPM_HD float foam_strength(const MaterialExt& mt, float ep) {
  const float r = ep * mt.df_inv_epsd;
  if (r >= 1.f) return 1e30f;
  return mt.df_plateau + mt.df_gamma * r - mt.df_densify * logf(fmaxf(1e-30f, 1.f - powf(r, mt.df_beta)));
}

// Snow's compaction hardening clamp(exp(10 (1 - Jp)), 0.25, 4) with aux = Jp - 1
// (src/three/constitutive.js:48).
MPM_HD float snow_hardening(float aux) { return fminf(4.f, fmaxf(0.25f, expf(-10.f * aux))); }

// Hencky strains e_k = log(max(s_k, 1e-6)) from beta_k = s_k^2 - 1 (constitutive.js:58,
// metal-plasticity.js:21)
MPM_HD float hencky_strain(float beta) {
  return fmaxf(0.5f * log1pf(beta), -13.815510558f);
}

// Large-strain path (|B| > 0.15): Jacobi eigen-decomposition of B. Out of line so its registers do
// not count against the series path that almost every particle takes.
MPM_NOINLINE ConstitutiveOut constitutive_eigen(const MaterialDev& mt, Sym3 B, float D[9], float ep,
                                                float T, float inv_rho0, bool do_return, float dt) {
  ConstitutiveOut out;
  out.dep = 0.f;
  out.dT = 0.f;
  float beta[3], U[9];
  sym_eig3(B, beta, U);
  if (mt.model == 0) {  // fixed-corotated: U diag(2 mu (s-1) s) U^T + lambda (J-1) J I
    float d[3];
    for (int k = 0; k < 3; ++k) {
      const float sm1 = beta[k] / (1.f + sqrtf(fmaxf(1.f + beta[k], 0.f)));  // s - 1
      d[k] = 2.f * mt.mu * (beta[k] - sm1);                                  // (s - 1) s = beta - (s - 1)
    }
    const float Jm1 = det_minus_one(D);
    const float vol = mt.lam * Jm1 * (1.f + Jm1);
    out.tau = rotate_diag(U, d);
    out.tau.xx += vol;
    out.tau.yy += vol;
    out.tau.zz += vol;
    out.Jm1 = Jm1;
    return out;
  }
  // J2 family on Hencky strains
  float e[3];
  for (int k = 0; k < 3; ++k) e[k] = hencky_strain(beta[k]);
  const float tr = e[0] + e[1] + e[2];
  const float tr3 = tr * (1.f / 3.f);
  float dev[3];
  for (int k = 0; k < 3; ++k) dev[k] = e[k] - tr3;
  const float len = sqrtf(dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]);
  const float J = fmaxf(1e-6f, expf(tr));
  const float q = 2.449489742783178f * mt.mu * len / J;
  const float dep = do_return ? plastic_increment(mt, q, J, ep, T, dt) : 0.f;
  float scale = 1.f;
  if (dep > 0.f) {
    scale = fmaxf(0.f, 1.f - 1.224744871391589f * dep / fmaxf(len, 1e-20f));
    // D' = M + M D + D with M = U diag(expm1((scale - 1) dev_k)) U^T
    float r[3];
    for (int k = 0; k < 3; ++k) r[k] = expm1f((scale - 1.f) * dev[k]);
    const Sym3 M = rotate_diag(U, r);
    float Dn[9];
    const float m00 = M.xx, m01 = M.xy, m02 = M.xz, m11 = M.yy, m12 = M.yz, m22 = M.zz;
    for (int b = 0; b < 3; ++b) {
      Dn[0 * 3 + b] = m00 * D[0 * 3 + b] + m01 * D[1 * 3 + b] + m02 * D[2 * 3 + b];
      Dn[1 * 3 + b] = m01 * D[0 * 3 + b] + m11 * D[1 * 3 + b] + m12 * D[2 * 3 + b];
      Dn[2 * 3 + b] = m02 * D[0 * 3 + b] + m12 * D[1 * 3 + b] + m22 * D[2 * 3 + b];
    }
    Dn[0] += m00; Dn[1] += m01; Dn[2] += m02;
    Dn[3] += m01; Dn[4] += m11; Dn[5] += m12;
    Dn[6] += m02; Dn[7] += m12; Dn[8] += m22;
    for (int k = 0; k < 9; ++k) D[k] += Dn[k];
    // plastic work heating (gpu/mixed_material.py:150-172): dT = beta * tau_eq * dep / (rho0 cp)
    // with tau_eq = sqrt(6) mu |dev e_returned| the returned Kirchhoff von Mises stress
    out.dT = mt.heat_per_work * 2.449489742783178f * mt.mu * scale * len * dep * inv_rho0;
  }
  float d[3];
  for (int k = 0; k < 3; ++k) d[k] = 2.f * mt.mu * (tr3 + scale * dev[k]) + mt.lam * tr;
  out.tau = rotate_diag(U, d);
  out.dep = dep;
  out.Jm1 = expm1f(tr);
  return out;
}

// Snow (2), sand (3), cohesive Drucker-Prager (8) and Deshpande-Fleck foam (9): the returns of
// src/three/constitutive.js:58-74 and src/three/pressure-plasticity.js:15-48 on the principal
// stretches s_k of F (eigenvalues beta_k = s_k^2 - 1 of B), then F' = U diag(s'/s) U^T F and the
// cached stress of the returned state (constitutive.js:81-86; snow: fixed-corotated scaled by
// its hardening). aux is Jp - 1 (models 2, 8, 9) or the dilation (model 3), updated in place.
// Always on the eigen-decomposition: the snow clamp acts per principal stretch, and these laws
// are not on the benchmark path whose registers the series path keeps small. Without the law's
// constants (xp null) only the stress of the stored state is available (no return).
MPM_NOINLINE ConstitutiveOut constitutive_pressure(const MaterialDev& mt, const MaterialExt* xp, Sym3 B,
                                                   float D[9], float ep, float& aux, bool do_return) {
  if (!xp) do_return = false;
  const MaterialExt none{};
  const MaterialExt& xt = xp ? *xp : none;
  ConstitutiveOut out;
  out.dep = 0.f;
  out.dT = 0.f;
  float beta[3], U[9];
  sym_eig3(B, beta, U);
  float sm1[3], e[3], r[3] = {0.f, 0.f, 0.f};
  for (int k = 0; k < 3; ++k) {
    sm1[k] = beta[k] / (1.f + sqrtf(fmaxf(1.f + beta[k], 0.f)));  // s - 1
    e[k] = hencky_strain(beta[k]);
  }
  bool moved = false;
  float d[3];
  if (mt.model == 2) {
    float sn[3] = {sm1[0], sm1[1], sm1[2]};  // returned s - 1
    if (do_return) {
      float lr = 0.f, inc2 = 0.f;
      for (int k = 0; k < 3; ++k) {
        sn[k] = fminf(xt.snow_hi, fmaxf(xt.snow_lo, sm1[k]));
        r[k] = (sn[k] - sm1[k]) / (1.f + sm1[k]);
        const float dl = -log1pf(r[k]);  // log(s / s')
        lr += dl;
        inc2 += dl * dl;
      }
      // Jp <- clamp(Jp det F / det F', 0.6, 20)
      aux = fminf(19.f, fmaxf(-0.4f, aux * expf(lr) + expm1f(lr)));
      out.dep = sqrtf(inc2);
      moved = out.dep > 0.f;
    }
    const float h = snow_hardening(aux);
    const float Jm1 = expm1f(log1pf(sn[0]) + log1pf(sn[1]) + log1pf(sn[2]));
    const float vol = h * mt.lam * Jm1 * (1.f + Jm1);
    for (int k = 0; k < 3; ++k) d[k] = 2.f * h * mt.mu * sn[k] * (1.f + sn[k]) + vol;
    out.Jm1 = Jm1;
  } else {
    float en[3] = {e[0], e[1], e[2]};  // returned log stretches
    if (do_return && mt.model == 3) {
      const float tr = e[0] + e[1] + e[2] + aux;
      if (tr >= 0.f) {  // no tensile strength: back to the unstretched state, dilation kept
        en[0] = en[1] = en[2] = 0.f;
        aux = tr;
      } else {
        aux = 0.f;
        float dev[3];
        for (int k = 0; k < 3; ++k) dev[k] = e[k] - tr * (1.f / 3.f);
        const float len = sqrtf(dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]);
        const float delta = fmaxf(0.f, len + xt.sand_k * tr);
        const float f = delta / (len > 0.f ? len : 1.f);
        for (int k = 0; k < 3; ++k) en[k] = e[k] - f * dev[k];
      }
    } else if (do_return) {  // models 8, 9
      const float tr = e[0] + e[1] + e[2];
      float dev[3];
      for (int k = 0; k < 3; ++k) dev[k] = e[k] - tr * (1.f / 3.f);
      const float len = sqrtf(dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]);
      const float J = fmaxf(1e-6f, expf(tr) * (1.f + aux));
      const float G = mt.mu / J, K = xt.bulk / J;
      const float mean = K * tr, q = 2.449489742783178f * G * len;
      float mean_n = mean, q_n = q, inc = 0.f;
      if (mt.model == 8) {
        const float t = q * 0.5773502691896258f;
        const float c = xt.dp_c, a = xt.dp_a, b = xt.dp_b, T = xt.dp_T;
        if (mean > T && t + a * T <= c) {
          mean_n = T;
        } else if (t + a * mean > c) {
          const float dl = (t + a * mean - c) / (G + a * K * b);
          mean_n = mean - K * b * dl;
          q_n = 1.7320508075688772f * fmaxf(0.f, t - G * dl);
          if (mean_n > T) {
            mean_n = T;
            q_n = 1.7320508075688772f * fmaxf(0.f, c - a * T);
          }
        }
      } else {
        const float a2 = xt.df_a2, Bf = xt.df_B;
        const float trial = sqrtf((q * q + a2 * mean * mean) / Bf);
        if (trial > foam_strength(xt, ep)) {
          // residual of the consistency condition at plastic multiplier eta (decreasing in eta)
          auto residual = [&](float eta, float& qn, float& mn, float& dl) {
            qn = q / (1.f + 3.f * G * eta);
            mn = mean / (1.f + K * a2 * eta);
            const float hat = sqrtf((qn * qn + a2 * mn * mn) / Bf);
            dl = eta * Bf * hat;
            return hat - foam_strength(xt, ep + dl);
          };
          float qn, mn, dl;
          float lo = 0.f, hi = 1.f / G;
          for (int k = 0; k < 32 && residual(hi, qn, mn, dl) > 0.f; ++k) hi *= 2.f;
          for (int k = 0; k < 28; ++k) {
            const float mid = 0.5f * (lo + hi);
            if (residual(mid, qn, mn, dl) > 0.f) lo = mid;
            else hi = mid;
          }
          residual(0.5f * (lo + hi), qn, mn, dl);
          q_n = qn;
          mean_n = mn;
          inc = dl;
        }
      }
      const float tr_n = mean_n / K, scale = q > 1e-20f ? q_n / q : 1.f;
      for (int k = 0; k < 3; ++k) en[k] = tr_n * (1.f / 3.f) + scale * dev[k];
      if (mt.model == 8) {
        const float d0 = e[0] - en[0], d1 = e[1] - en[1], d2 = e[2] - en[2];
        inc = 0.816496580927726f * sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
      }
      // Jp <- Jp exp(tr - tr')
      const float dv = tr - tr_n;
      aux = aux * expf(dv) + expm1f(dv);
      out.dep = inc;
    }
    if (do_return) {
      float inc2 = 0.f;
      for (int k = 0; k < 3; ++k) {
        const float dk = en[k] - e[k];
        r[k] = expm1f(dk);
        inc2 += dk * dk;
        moved = moved || dk != 0.f;
      }
      if (mt.model == 3) out.dep = sqrtf(inc2);  // |log(s / s')| (constitutive.js:76)
    }
    const float tr = en[0] + en[1] + en[2];
    for (int k = 0; k < 3; ++k) d[k] = 2.f * mt.mu * en[k] + mt.lam * tr;
    out.Jm1 = expm1f(tr);
  }
  if (moved) {
    // D' = M + M D + D with M = U diag(s'/s - 1) U^T
    const Sym3 M = rotate_diag(U, r);
    float Dn[9];
    for (int b = 0; b < 3; ++b) {
      Dn[0 * 3 + b] = M.xx * D[0 * 3 + b] + M.xy * D[1 * 3 + b] + M.xz * D[2 * 3 + b];
      Dn[1 * 3 + b] = M.xy * D[0 * 3 + b] + M.yy * D[1 * 3 + b] + M.yz * D[2 * 3 + b];
      Dn[2 * 3 + b] = M.xz * D[0 * 3 + b] + M.yz * D[1 * 3 + b] + M.zz * D[2 * 3 + b];
    }
    Dn[0] += M.xx; Dn[1] += M.xy; Dn[2] += M.xz;
    Dn[3] += M.xy; Dn[4] += M.yy; Dn[5] += M.yz;
    Dn[6] += M.xz; Dn[7] += M.yz; Dn[8] += M.zz;
    for (int k = 0; k < 9; ++k) D[k] += Dn[k];
  }
  out.tau = rotate_diag(U, d);
  return out;
}

// Trial invariants of the J2-type returns on the small-strain series path (|B - I| <= 0.15):
// L = log(I + B) / 2 = log V_l, its deviator, |dev L|, J - 1 and the trial von Mises stress q.
struct J2Trial {
  Sym3 dv;
  float len, trL, tr3, em1, J, q;
};

MPM_HD J2Trial j2_trial_series(const MaterialDev& mt, const Sym3& B, int nt) {
  J2Trial t;
  Sym3 L = matrix_series<0>(B, nt);  // log(I + B) = 2 log V_l
  L.xx *= 0.5f; L.yy *= 0.5f; L.zz *= 0.5f; L.xy *= 0.5f; L.xz *= 0.5f; L.yz *= 0.5f;
  t.trL = L.xx + L.yy + L.zz;
  t.tr3 = t.trL * (1.f / 3.f);
  t.dv = L;
  t.dv.xx -= t.tr3; t.dv.yy -= t.tr3; t.dv.zz -= t.tr3;
  t.len = sym_norm(t.dv);
  t.em1 = expm1f(t.trL);  // J - 1
  t.J = fmaxf(1e-6f, 1.f + t.em1);
  t.q = 2.449489742783178f * mt.mu * t.len / t.J;
  return t;
}

// The return for a plastic strain increment dep (0: elastic) and the Hencky stress of the
// returned state: F' = exp((scale - 1) dev L) F with scale = 1 - sqrt(3/2) dep / |dev L|
// (src/three/metal-plasticity.js:24-26, src/three/constitutive.js:77-86), plastic-work heating.
MPM_HD ConstitutiveOut j2_finish(const MaterialDev& mt, const J2Trial& t, float D[9], float dep, float inv_rho0) {
  ConstitutiveOut out;
  out.dT = 0.f;
  const Sym3& dv = t.dv;
  float scale = 1.f;
  if (dep > 0.f) {
    scale = fmaxf(0.f, 1.f - 1.224744871391589f * dep / fmaxf(t.len, 1e-20f));
    const float g = scale - 1.f;
    const Sym3 M{g * dv.xx, g * dv.yy, g * dv.zz, g * dv.xy, g * dv.xz, g * dv.yz};
    const int nm = series_terms(sym_norm(M));
    const Sym3 E = matrix_series<2>(M, nm > 0 ? nm : 10);  // exp(M) - I
    float Dn[9];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      Dn[0 * 3 + b] = E.xx * D[0 * 3 + b] + E.xy * D[1 * 3 + b] + E.xz * D[2 * 3 + b];
      Dn[1 * 3 + b] = E.xy * D[0 * 3 + b] + E.yy * D[1 * 3 + b] + E.yz * D[2 * 3 + b];
      Dn[2 * 3 + b] = E.xz * D[0 * 3 + b] + E.yz * D[1 * 3 + b] + E.zz * D[2 * 3 + b];
    }
    D[0] += Dn[0] + E.xx; D[1] += Dn[1] + E.xy; D[2] += Dn[2] + E.xz;
    D[3] += Dn[3] + E.xy; D[4] += Dn[4] + E.yy; D[5] += Dn[5] + E.yz;
    D[6] += Dn[6] + E.xz; D[7] += Dn[7] + E.yz; D[8] += Dn[8] + E.zz;
    out.dT = mt.heat_per_work * 2.449489742783178f * mt.mu * scale * t.len * dep * inv_rho0;
  }
  const float m2s = 2.f * mt.mu * scale;
  const float iso = 2.f * mt.mu * t.tr3 + mt.lam * t.trL;
  out.tau.xx = m2s * dv.xx + iso;
  out.tau.yy = m2s * dv.yy + iso;
  out.tau.zz = m2s * dv.zz + iso;
  out.tau.xy = m2s * dv.xy;
  out.tau.xz = m2s * dv.xz;
  out.tau.yz = m2s * dv.yz;
  out.dep = dep;
  out.Jm1 = t.em1;
  return out;
}

// Constitutive update of one particle after the F update, in place on D (= F - I):
// models 4-7, 10 and 11 run the J2-type radial return (src/three/metal-plasticity.js:20-38,
// src/three/thermal-plasticity.js:22-40; dt is the substep, used by the rate-dependent laws 6,
// 7 and 11) and give the Hencky stress of the returned state
// (src/three/constitutive.js:81-86); models 0 and 1 give the elastic stress of F
// (src/three/math.js:25-32, src/three/constitutive.js:94-100).
// ep is the accumulated plastic strain, T the temperature; rho0 = m / V for the heat term.
// With do_return false the J2 models give the stress of F without a return (the reference's
// updateStress when no cached stress exists, src/three/mpm.js:36).
// Models 2, 3, 8 and 9 also read and update aux with the constants xp (see constitutive_pressure).
// AUX = false compiles their branch out, for kernels that know no such material is in use.
template <bool AUX>
MPM_HD ConstitutiveOut constitutive_update_t(const MaterialDev& mt, float D[9], float ep, float& aux, float T,
                                             float inv_rho0, bool do_return, float dt = 0.f,
                                             const MaterialExt* xp = nullptr) {
  ConstitutiveOut out;
  out.dep = 0.f;
  out.dT = 0.f;
  const Sym3 B = cauchy_green_minus_identity(D);
  // The out-of-line returns work on copies scoped to their branch, so the caller's D (and aux)
  // keep no address: passed directly, they live in local memory on every particle's path (2% of
  // the fused pass).
  if (AUX && aux_model(mt.model)) {
    float Dt[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) Dt[e] = D[e];
    float at = aux;
    const ConstitutiveOut o = constitutive_pressure(mt, xp, B, Dt, ep, at, do_return);
#pragma unroll
    for (int e = 0; e < 9; ++e) D[e] = Dt[e];
    aux = at;
    return o;
  }
  if (mt.model == 1) {  // Neo-Hookean: mu (F F^T - I) + lambda log J I
    const float Jm1 = det_minus_one(D);
    const float J = 1.f + Jm1;
    const float lj = J > 1e-6f ? log1pf(Jm1) : -13.815510558f;
    out.tau.xx = mt.mu * B.xx + mt.lam * lj;
    out.tau.yy = mt.mu * B.yy + mt.lam * lj;
    out.tau.zz = mt.mu * B.zz + mt.lam * lj;
    out.tau.xy = mt.mu * B.xy;
    out.tau.xz = mt.mu * B.xz;
    out.tau.yz = mt.mu * B.yz;
    out.Jm1 = Jm1;
    return out;
  }
  // Small strain (|B| <= 0.15): isotropic matrix functions of B by power series, no eigenvectors.
  // fixed-corotated: V_l = sqrt(I + B), (F - R) F^T = (V_l - I) V_l;  Hencky: L = log(V_l) =
  // log(I + B)/2, |dev e| = |dev L|_F, returned L' = tr L/3 I + scale dev L, and the return
  // F' = U diag(s'/s) U^T F = exp((scale - 1) dev L) F.
  const int nt = series_terms_sq(sym_norm2(B));
  if (nt > 0) {
    if (mt.model == 0) {
      const Sym3 S1 = matrix_series<1>(B, nt);  // sqrt(I + B) - I
      const Sym3 S2 = sym_mul(S1, S1);
      const float Jm1 = det_minus_one(D);
      const float vol = mt.lam * Jm1 * (1.f + Jm1);
      const float m2 = 2.f * mt.mu;
      out.tau.xx = m2 * (S1.xx + S2.xx) + vol;
      out.tau.yy = m2 * (S1.yy + S2.yy) + vol;
      out.tau.zz = m2 * (S1.zz + S2.zz) + vol;
      out.tau.xy = m2 * (S1.xy + S2.xy);
      out.tau.xz = m2 * (S1.xz + S2.xz);
      out.tau.yz = m2 * (S1.yz + S2.yz);
      out.Jm1 = Jm1;
      return out;
    }
    const J2Trial tr = j2_trial_series(mt, B, nt);
    const float dep = do_return ? plastic_increment(mt, tr.q, tr.J, ep, T, dt) : 0.f;
    return j2_finish(mt, tr, D, dep, inv_rho0);
  }
  float Dt[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) Dt[e] = D[e];
  const ConstitutiveOut o = constitutive_eigen(mt, B, Dt, ep, T, inv_rho0, do_return, dt);
#pragma unroll
  for (int e = 0; e < 9; ++e) D[e] = Dt[e];
  return o;
}

MPM_HD ConstitutiveOut constitutive_update_aux(const MaterialDev& mt, const MaterialExt* xp, float D[9], float ep,
                                               float& aux, float T, float inv_rho0, bool do_return, float dt = 0.f) {
  return constitutive_update_t<true>(mt, D, ep, aux, T, inv_rho0, do_return, dt, xp);
}

// Every law with its history scalar at the default (Jp = 1, dilation = 0), not returned; snow,
// sand and the pressure laws give the stress of the stored state only (their constants are not
// passed).
MPM_HD ConstitutiveOut constitutive_update(const MaterialDev& mt, float D[9], float ep, float T, float inv_rho0,
                                           bool do_return, float dt = 0.f) {
  float aux = 0.f;
  return constitutive_update_t<true>(mt, D, ep, aux, T, inv_rho0, do_return, dt);
}

}  // namespace mpm
