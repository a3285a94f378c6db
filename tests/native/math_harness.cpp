// Host build of the device constitutive math (summer-particle-lab_b200/csrc/mpm_math.h) for CPU
// tests against the FP64 oracle. Test infrastructure: compiled by tests/test_host_math.py.
#include "mpm_math.h"

extern "C" void harness_constitutive(int model, double mu, double lam, double A, double B, double Tref,
                                     double Thot, double hot, int n, const double* F, const double* ep,
                                     const double* T, int do_return, double* Fout, double* dep, double* tau) {
  mpm::MaterialDev m{};
  m.model = model;
  m.mu = (float)mu;
  m.lam = (float)lam;
  m.yield_stress = (float)A;
  m.hardening = (float)B;
  m.T_ref = (float)Tref;
  m.inv_T_span = Thot > Tref ? (float)(1.0 / (Thot - Tref)) : 0.f;
  m.hot_ratio = (float)hot;
  for (int i = 0; i < n; ++i) {
    float D[9];
    for (int e = 0; e < 9; ++e) D[e] = (float)(F[i * 9 + e] - (e % 4 == 0 ? 1.0 : 0.0));
    mpm::ConstitutiveOut o = mpm::constitutive_update(m, D, (float)ep[i], (float)T[i], 1.f, do_return != 0);
    for (int e = 0; e < 9; ++e) Fout[i * 9 + e] = (double)D[e] + (e % 4 == 0 ? 1.0 : 0.0);
    dep[i] = o.dep;
    const float t9[9] = {o.tau.xx, o.tau.xy, o.tau.xz, o.tau.xy, o.tau.yy, o.tau.yz, o.tau.xz, o.tau.yz, o.tau.zz};
    for (int e = 0; e < 9; ++e) tau[i * 9 + e] = t9[e];
  }
}

// Every material field (in the order of mpm_material from mu on) and the substep dt, for the
// rate-dependent laws: prm = {mu, lam, A, B, Tref, Thot, hot, jc_n, jc_C, jc_rate0, T_melt, jc_m,
// creep_rate, creep_Q, creep_n, creep_stress, T_offset}.
extern "C" void harness_constitutive_full(int model, const double* prm, double dt, int n, const double* F,
                                          const double* ep, const double* T, double* Fout, double* dep, double* tau) {
  mpm::MaterialDev m{};
  m.model = model;
  m.mu = (float)prm[0];
  m.lam = (float)prm[1];
  m.yield_stress = (float)prm[2];
  m.hardening = (float)prm[3];
  m.T_ref = (float)prm[4];
  m.inv_T_span = prm[5] > prm[4] ? (float)(1.0 / (prm[5] - prm[4])) : 0.f;
  m.hot_ratio = (float)prm[6];
  m.jc_n = (float)prm[7];
  m.jc_C = (float)prm[8];
  m.jc_inv_rate0 = prm[9] > 0 ? (float)(1.0 / prm[9]) : 0.f;
  m.jc_inv_T_span = prm[10] > prm[4] ? (float)(1.0 / (prm[10] - prm[4])) : 0.f;
  m.jc_m = (float)prm[11];
  m.cr_on = prm[12] > 0;
  m.cr_log_rate = prm[12] > 0 ? (float)std::log(prm[12]) : 0.f;
  m.cr_Q_over_R = (float)(prm[13] / 8.314462618);
  m.cr_n = (float)prm[14];
  m.cr_inv_stress = (float)(1.0 / prm[15]);
  m.cr_T_offset = (float)prm[16];
  m.cr_inv_Tref_abs = (float)(1.0 / (prm[4] + prm[16]));
  for (int i = 0; i < n; ++i) {
    float D[9];
    for (int e = 0; e < 9; ++e) D[e] = (float)(F[i * 9 + e] - (e % 4 == 0 ? 1.0 : 0.0));
    mpm::ConstitutiveOut o = mpm::constitutive_update(m, D, (float)ep[i], (float)T[i], 1.f, true, (float)dt);
    for (int e = 0; e < 9; ++e) Fout[i * 9 + e] = (double)D[e] + (e % 4 == 0 ? 1.0 : 0.0);
    dep[i] = o.dep;
    const float t9[9] = {o.tau.xx, o.tau.xy, o.tau.xz, o.tau.xy, o.tau.yy, o.tau.yz, o.tau.xz, o.tau.yz, o.tau.zz};
    for (int e = 0; e < 9; ++e) tau[i * 9 + e] = t9[e];
  }
}

// Snow, sand and the pressure models with their history scalar: prm = {mu, lam, yield_strain,
// friction_deg, cohesion, slope, dilatancy, tension, alpha, plateau, gamma, densify, beta, eps_D}
// (the fields of mpm_material), hist = Jp (models 2, 8, 9) or the dilation (model 3), updated.
extern "C" void harness_constitutive_aux(int model, const double* prm, int n, const double* F, const double* ep,
                                         double* hist, int do_return, double* Fout, double* dep, double* tau) {
  mpm::MaterialDev m{};
  m.model = model;
  m.mu = (float)prm[0];
  m.lam = (float)prm[1];
  m.wave_modulus = (float)(prm[1] + 2 * prm[0]);
  mpm::MaterialExt x{};
  x.snow_lo = (float)(-prm[2]);
  x.snow_hi = (float)(0.3 * prm[2]);
  const double sn = std::sin(prm[3] * 3.14159265358979323846 / 180.0);
  x.sand_k = (float)(std::sqrt(2.0 / 3.0) * 2 * sn / (3 - sn) * (3 * prm[1] + 2 * prm[0]) / (2 * prm[0]));
  x.bulk = (float)(prm[1] + 2 * prm[0] / 3);
  x.dp_c = (float)prm[4];
  x.dp_a = (float)prm[5];
  x.dp_b = (float)prm[6];
  x.dp_T = (float)prm[7];
  x.df_a2 = (float)(prm[8] * prm[8]);
  x.df_B = (float)(1 + prm[8] * prm[8] / 9);
  x.df_plateau = (float)prm[9];
  x.df_gamma = (float)prm[10];
  x.df_densify = (float)prm[11];
  x.df_beta = (float)prm[12];
  x.df_inv_epsd = (float)(1.0 / prm[13]);
  for (int i = 0; i < n; ++i) {
    float D[9];
    for (int e = 0; e < 9; ++e) D[e] = (float)(F[i * 9 + e] - (e % 4 == 0 ? 1.0 : 0.0));
    float aux = model == 3 ? (float)hist[i] : (float)(hist[i] - 1.0);
    mpm::ConstitutiveOut o = mpm::constitutive_update_aux(m, &x, D, (float)ep[i], aux, 0.f, 1.f, do_return != 0, 0.01f);
    for (int e = 0; e < 9; ++e) Fout[i * 9 + e] = (double)D[e] + (e % 4 == 0 ? 1.0 : 0.0);
    dep[i] = o.dep;
    hist[i] = model == 3 ? (double)aux : 1.0 + (double)aux;
    const float t9[9] = {o.tau.xx, o.tau.xy, o.tau.xz, o.tau.xy, o.tau.yy, o.tau.yz, o.tau.xz, o.tau.yz, o.tau.zz};
    for (int e = 0; e < 9; ++e) tau[i * 9 + e] = t9[e];
  }
}

extern "C" void harness_eig(int n, const double* S6, double* lam, double* U) {
  for (int i = 0; i < n; ++i) {
    mpm::Sym3 a{(float)S6[i * 6 + 0], (float)S6[i * 6 + 1], (float)S6[i * 6 + 2],
                (float)S6[i * 6 + 3], (float)S6[i * 6 + 4], (float)S6[i * 6 + 5]};
    float l[3], u[9];
    mpm::sym_eig3(a, l, u);
    for (int k = 0; k < 3; ++k) lam[i * 3 + k] = l[k];
    for (int k = 0; k < 9; ++k) U[i * 9 + k] = u[k];
  }
}

// The learned Johnson-Cook return's refinement and gate (mpm::jc_refine), the exact bisection
// (mpm::jc_bisect) and the network inputs (mpm::jc_features) on trial states (q, J, ep, T, dt):
// prm as harness_constitutive_full. ok[i] = 1 when the gate accepts the refined prediction u_pred[i].
extern "C" void harness_jc_refine(int model, const double* prm, int n, const double* q, const double* J,
                                  const double* ep, const double* T, const double* dt, const double* u_pred,
                                  double tol, int newton, int* ok, double* dep_learned, double* dep_exact,
                                  double* features) {
  mpm::MaterialDev m{};
  m.model = model;
  m.mu = (float)prm[0];
  m.lam = (float)prm[1];
  m.yield_stress = (float)prm[2];
  m.hardening = (float)prm[3];
  m.T_ref = (float)prm[4];
  m.jc_n = (float)prm[7];
  m.jc_C = (float)prm[8];
  m.jc_inv_rate0 = prm[9] > 0 ? (float)(1.0 / prm[9]) : 0.f;
  m.jc_inv_T_span = prm[10] > prm[4] ? (float)(1.0 / (prm[10] - prm[4])) : 0.f;
  m.jc_m = (float)prm[11];
  for (int i = 0; i < n; ++i) {
    const mpm::JcRefined r = mpm::jc_refine(m, (float)q[i], (float)J[i], (float)ep[i], (float)T[i], (float)dt[i],
                                            (float)u_pred[i], (float)tol, newton);
    ok[i] = r.ok ? 1 : 0;
    dep_learned[i] = r.dep;
    dep_exact[i] = mpm::plastic_increment(m, (float)q[i], (float)J[i], (float)ep[i], (float)T[i], (float)dt[i]);
    float x[8];
    mpm::jc_features(m, (float)q[i], (float)J[i], (float)ep[i], (float)T[i], (float)dt[i], x);
    for (int k = 0; k < 8; ++k) features[i * 8 + k] = x[k];
  }
}
