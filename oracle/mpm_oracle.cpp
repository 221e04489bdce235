// mpm_oracle.cpp -- CPU restatement of the reference explicit MPM step.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never the product.
// Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
// load this library.
//
// Every function restates the reference code it cites (paths are relative to
// the geomechanics/mpm source tree).  The reference builds on Eigen (a system
// package, not vendored, no pinned version); here fixed-size arrays replace
// it, sums run left to right, and small inverses are adjugate / determinant
// exactly as Eigen's fixed-size inverse (InverseImpl.h, cofactor form) is
// published.  Compile with -ffp-contract=off so a*b+c is never fused.
#include "mpm_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <set>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int64_t kNone = std::numeric_limits<int64_t>::max();
constexpr double kEps = std::numeric_limits<double>::epsilon();
constexpr double kPi = 3.14159265358979323846;  // M_PI

// ---------------------------------------------------------------- materials
// LinearElastic: include/materials/infinitesimal_strain/linear_elastic.tcc
// MohrCoulomb:   include/materials/infinitesimal_strain/mohr_coulomb.tcc
// Parameter order (LinearElastic): density, youngs_modulus, poisson_ratio
// Parameter order (MohrCoulomb):   density, youngs_modulus, poisson_ratio,
//   friction, dilation, cohesion, residual_friction, residual_dilation,
//   residual_cohesion, peak_pdstrain, residual_pdstrain, tension_cutoff,
//   softening, packing_fraction (initial, default 1),
//   packing_fraction_minimum (default 0), is_wet (default 0)
struct Material {
  int id = 0;
  int type = 0;  // 0 LinearElastic, 1 MohrCoulomb
  double density = 0, E = 0, nu = 0;
  double bulk = 0, shear = 0;
  double de[6][6] = {};
  // MohrCoulomb
  bool softening = false;
  double phi_peak = 0, psi_peak = 0, c_peak = 0;
  double phi_res = 0, psi_res = 0, c_res = 0;
  double pd_peak = 0, pd_res = 0, tension_cutoff = 0;
  double grain_density = 0, min_packing = 0;
};

// linear_elastic.tcc:3-49 (ctor) and :53-69 (compute_elastic_tensor)
// mohr_coulomb.tcc:3-81 (ctor) and :517-533 (compute_elastic_tensor)
bool make_material(int id, int type, const double* p, int np, Material* m,
                   std::string* err) {
  m->id = id;
  m->type = type;
  if (type == 0) {
    if (np < 3) { *err = "LinearElastic needs 3 parameters"; return false; }
    m->density = p[0];
    m->E = p[1];
    m->nu = p[2];
    m->bulk = m->E / (3.0 * (1. - 2. * m->nu));
    const double G = m->E / (2.0 * (1. + m->nu));
    m->shear = G;
    const double a1 = m->bulk + (4.0 / 3.0) * G;
    const double a2 = m->bulk - (2.0 / 3.0) * G;
    std::memset(m->de, 0, sizeof(m->de));
    m->de[0][0] = a1; m->de[0][1] = a2; m->de[0][2] = a2;
    m->de[1][0] = a2; m->de[1][1] = a1; m->de[1][2] = a2;
    m->de[2][0] = a2; m->de[2][1] = a2; m->de[2][2] = a1;
    m->de[3][3] = G; m->de[4][4] = G; m->de[5][5] = G;
    return true;
  }
  if (type == 1) {
    if (np < 13) { *err = "MohrCoulomb needs at least 13 parameters"; return false; }
    m->density = p[0];
    m->E = p[1];
    m->nu = p[2];
    m->phi_peak = p[3] * kPi / 180.;
    m->psi_peak = p[4] * kPi / 180.;
    m->c_peak = p[5];
    m->phi_res = p[6] * kPi / 180.;
    m->psi_res = p[7] * kPi / 180.;
    m->c_res = p[8];
    m->pd_peak = p[9];
    m->pd_res = p[10];
    m->tension_cutoff = p[11];
    m->softening = p[12] != 0.0;
    const double packing = np > 13 ? p[13] : 1.0;
    m->min_packing = np > 14 ? p[14] : 0.0;
    const bool is_wet = np > 15 ? p[15] != 0.0 : false;
    m->grain_density = is_wet ? m->density : m->density / packing;
    m->bulk = m->E / (3.0 * (1. - 2. * m->nu));
    m->shear = m->E / (2.0 * (1 + m->nu));
    const double G = m->shear;
    const double a1 = m->bulk + (4.0 / 3.0) * G;
    const double a2 = m->bulk - (2.0 / 3.0) * G;
    std::memset(m->de, 0, sizeof(m->de));
    m->de[0][0] = a1; m->de[0][1] = a2; m->de[0][2] = a2;
    m->de[1][0] = a2; m->de[1][1] = a1; m->de[1][2] = a2;
    m->de[2][0] = a2; m->de[2][1] = a2; m->de[2][2] = a1;
    m->de[3][3] = G; m->de[4][4] = G; m->de[5][5] = G;
    return true;
  }
  *err = "unknown material type";
  return false;
}

inline double check_low(double val) {  // mohr_coulomb.h:124-126
  return (val > 1.0e-15 ? val : 1.0e-15);
}

// MC state layout (mohr_coulomb.tcc:115-120)
enum { SV_YIELD = 0, SV_PHI, SV_PSI, SV_COH, SV_TC, SV_EPS, SV_RHO, SV_THETA, SV_PD };

// mohr_coulomb.tcc:85-111
void mc_initialise_state(const Material& m, double* sv) {
  sv[SV_YIELD] = 0;
  sv[SV_PHI] = m.phi_peak;
  sv[SV_PSI] = m.psi_peak;
  sv[SV_COH] = m.c_peak;
  sv[SV_TC] = check_low((m.tension_cutoff < m.c_peak / std::tan(m.phi_peak))
                            ? m.tension_cutoff
                            : m.c_peak / std::tan(m.phi_peak));
  sv[SV_EPS] = 0.;
  sv[SV_RHO] = 0.;
  sv[SV_THETA] = 0.;
  sv[SV_PD] = 0.;
}

// ---- stress invariants: include/utilities/material_utility.tcc
double mu_p(const double* s) {  // :2-5
  return (1. / 3. * (s[0] + s[1] + s[2]));
}
void mu_dev(const double* s, double* d) {  // :8-19
  const double p = mu_p(s);
  for (int i = 0; i < 6; ++i) d[i] = s[i];
  for (int i = 0; i < 3; ++i) d[i] -= p;
}
double mu_j2(const double* s) {  // :22-32
  return (std::pow((s[0] - s[1]), 2) + std::pow((s[1] - s[2]), 2) +
          std::pow((s[0] - s[2]), 2)) /
             6.0 +
         std::pow(s[3], 2) + std::pow(s[4], 2) + std::pow(s[5], 2);
}
double mu_j3(const double* s) {  // :35-52
  double d[6];
  mu_dev(s, d);
  return (d[0] * d[1] * d[2]) - (d[2] * std::pow(d[3], 2)) +
         ((2 * d[3] * d[4] * d[5]) - (d[0] * std::pow(d[4], 2)) -
          (d[1] * std::pow(d[5], 2)));
}
double mu_q(const double* s) {  // :55-62
  const double j2 = mu_j2(s);
  return (std::sqrt(3 * j2));
}
double mu_lode_angle(const double* s, double tol = kEps) {  // :65-81
  const double j2 = mu_j2(s);
  const double j3 = mu_j3(s);
  double v = 0.0;
  if (std::abs(j2) > tol) v = (3. * std::sqrt(3.) / 2.) * (j3 / std::pow(j2, 1.5));
  if (v > 1.0) v = 1.0;
  if (v < -1.0) v = -1.0;
  return (1. / 3.) * std::acos(v);
}
void mu_dp_dsigma(double* o) {  // :84-92
  for (int i = 0; i < 6; ++i) o[i] = 0.;
  o[0] = 1. / 3.;
  o[1] = 1. / 3.;
  o[2] = 1. / 3.;
}
void mu_dq_dsigma(const double* s, double* o) {  // :95-117
  const double q = mu_q(s);
  double d[6];
  mu_dev(s, d);
  for (int i = 0; i < 6; ++i) o[i] = 0.;
  if (std::abs(q) > kEps) {
    o[0] = 3. / (2. * q) * d[0];
    o[1] = 3. / (2. * q) * d[1];
    o[2] = 3. / (2. * q) * d[2];
    o[3] = 3. / q * d[3];
    o[4] = 3. / q * d[4];
    o[5] = 3. / q * d[5];
  }
}
void mu_dj2_dsigma(const double* s, double* o) {  // :120-130
  mu_dev(s, o);
  o[3] *= 2.0;
  o[4] *= 2.0;
  o[5] *= 2.0;
}
inline double dot3(const double* a, const double* b) {
  return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}
void mu_dj3_dsigma(const double* s, double* o) {  // :133-163
  const double j2 = mu_j2(s);
  double d[6];
  mu_dev(s, d);
  const double dev1[3] = {d[0], d[3], d[5]};
  const double dev2[3] = {d[3], d[1], d[4]};
  const double dev3[3] = {d[5], d[4], d[2]};
  o[0] = dot3(dev1, dev1) - (2. / 3.) * j2;
  o[1] = dot3(dev2, dev2) - (2. / 3.) * j2;
  o[2] = dot3(dev3, dev3) - (2. / 3.) * j2;
  o[3] = 2.0 * dot3(dev1, dev2);
  o[4] = 2.0 * dot3(dev2, dev3);
  o[5] = 2.0 * dot3(dev1, dev3);
}
void mu_dtheta_dsigma(const double* s, double tol, double* o) {  // :166-200
  const double j2 = mu_j2(s);
  const double j3 = mu_j3(s);
  double dj2[6], dj3[6];
  mu_dj2_dsigma(s, dj2);
  mu_dj3_dsigma(s, dj3);
  double dr_dj2 = -9.0 / 4.0 * std::sqrt(3.0) * j3;
  double dr_dj3 = 3.0 / 2.0 * std::sqrt(3.0);
  double dtheta_dr = -1.0 / 3.0;
  if (std::abs(j2) > tol) {
    const double r = j3 / 2.0 * std::pow(j2 / 3.0, -1.5);
    dr_dj2 *= std::pow(j2, -2.5);
    dr_dj3 *= std::pow(j2, -1.5);
    const double factor = (std::abs(1 - r * r) < tol) ? tol : std::abs(1 - r * r);
    dtheta_dr = -1.0 / (3.0 * std::sqrt(factor));
  }
  for (int i = 0; i < 6; ++i) o[i] = dtheta_dr * ((dr_dj2 * dj2[i]) + (dr_dj3 * dj3[i]));
}

// mohr_coulomb.tcc:124-134
void mc_invariants(const double* s, double* sv) {
  sv[SV_EPS] = mu_p(s) * std::sqrt(3.);
  sv[SV_THETA] = mu_lode_angle(s);
  sv[SV_RHO] = std::sqrt(2. * mu_j2(s));
}

enum FailureState { Elastic = 0, Shear = 1, Tensile = 2, Separated = 3 };

// mohr_coulomb.tcc:139-191
int mc_yield_state(double* yf, const double* sv) {
  const double Tolerance = -1E-1;
  const double epsilon = sv[SV_EPS];
  const double rho = sv[SV_RHO];
  const double theta = sv[SV_THETA];
  const double phi = sv[SV_PHI];
  const double cohesion = sv[SV_COH];
  const double tension_cutoff = sv[SV_TC];
  yf[0] = std::sqrt(2. / 3.) * std::cos(theta) * rho + epsilon / std::sqrt(3.) -
          tension_cutoff;
  yf[1] = std::sqrt(1.5) * rho *
              ((std::sin(theta + kPi / 3.) / (std::sqrt(3.) * std::cos(phi))) +
               (std::cos(theta + kPi / 3.) * std::tan(phi) / 3.)) +
          (epsilon / std::sqrt(3.)) * std::tan(phi) - cohesion;
  int yield_type = Elastic;
  if (yf[0] > Tolerance && yf[1] > Tolerance) {
    const double n_phi = (1. + std::sin(phi)) / (1. - std::sin(phi));
    const double sigma_p = tension_cutoff * n_phi - 2. * cohesion * std::sqrt(n_phi);
    const double alpha_p = std::sqrt(1. + n_phi * n_phi) + n_phi;
    const double h =
        yf[0] + alpha_p * (std::sqrt(2. / 3.) * std::cos(theta - 4. * kPi / 3.) * rho +
                           epsilon / std::sqrt(3.) - sigma_p);
    if (h > kEps)
      yield_type = Tensile;
    else
      yield_type = Shear;
  }
  if (yf[0] < Tolerance && yf[1] > Tolerance) yield_type = Shear;
  if (yf[0] > Tolerance && yf[1] < Tolerance) yield_type = Tensile;
  return yield_type;
}

// mohr_coulomb.tcc:195-344
void mc_df_dp(const Material& m, int yield_type, const double* sv, const double* s,
              double* df, double* dp, double* dp_dq, double* softening) {
  const double rho = sv[SV_RHO];
  const double theta = sv[SV_THETA];
  const double phi = sv[SV_PHI];
  const double psi = sv[SV_PSI];
  const double tension_cutoff = sv[SV_TC];
  const double pdstrain = sv[SV_PD];
  double df_depsilon, df_drho, df_dtheta;
  if (yield_type == Tensile) {
    df_depsilon = 1. / std::sqrt(3.);
    df_drho = std::sqrt(2. / 3.) * std::cos(theta);
    df_dtheta = -std::sqrt(2. / 3.) * rho * std::sin(theta);
  } else {
    df_depsilon = std::tan(phi) / std::sqrt(3.);
    df_drho = std::sqrt(1.5) *
              ((std::sin(theta + kPi / 3.) / (std::sqrt(3.) * std::cos(phi))) +
               (std::cos(theta + kPi / 3.) * std::tan(phi) / 3.));
    df_dtheta = std::sqrt(1.5) * rho *
                ((std::cos(theta + kPi / 3.) / (std::sqrt(3.) * std::cos(phi))) -
                 (std::sin(theta + kPi / 3.) * std::tan(phi) / 3.));
  }
  double depsilon_dsigma[6], drho_dsigma[6], dtheta_dsigma[6];
  mu_dp_dsigma(depsilon_dsigma);
  for (int i = 0; i < 6; ++i) depsilon_dsigma[i] *= std::sqrt(3.);
  mu_dq_dsigma(s, drho_dsigma);
  for (int i = 0; i < 6; ++i) drho_dsigma[i] *= std::sqrt(2. / 3.);
  mu_dtheta_dsigma(s, kEps, dtheta_dsigma);
  for (int i = 0; i < 6; ++i)
    df[i] = ((df_depsilon * depsilon_dsigma[i]) + (df_drho * drho_dsigma[i])) +
            (df_dtheta * dtheta_dsigma[i]);
  if (yield_type == Tensile) {
    const double et_value = 0.6;
    const double xit = 0.1;
    double sqpart = 4. * (1 - et_value * et_value) * std::cos(theta) * std::cos(theta) +
                    5. * et_value * et_value - 4. * et_value;
    if (sqpart < kEps) sqpart = 1.E-5;
    double rt_den = 2. * (1 - et_value * et_value) * std::cos(theta) +
                    (2. * et_value - 1) * std::sqrt(sqpart);
    const double rt_num = 4. * (1 - et_value * et_value) * std::cos(theta) * std::cos(theta) +
                          (2. * et_value - 1) * (2. * et_value - 1);
    if (std::fabs(rt_den) < kEps) rt_den = 1.E-5;
    const double rt = rt_num / (3. * rt_den);
    const double dp_drt =
        1.5 * rho * rho * rt /
        check_low(std::sqrt(xit * xit * tension_cutoff * tension_cutoff + 1.5 * rt * rt * rho * rho));
    const double dp_drho =
        1.5 * rho * rt * rt /
        check_low(std::sqrt(xit * xit * tension_cutoff * tension_cutoff + 1.5 * rt * rt * rho * rho));
    const double dp_depsilon = 1. / std::sqrt(3.);
    const double drtden_dtheta =
        -2. * (1 - et_value * et_value) * std::sin(theta) -
        (2. * et_value - 1) * 4. * (1 - et_value * et_value) * std::cos(theta) * std::sin(theta) /
            std::sqrt(4. * (1 - et_value * et_value) * std::cos(theta) * std::cos(theta) +
                      5. * et_value * et_value - 4. * et_value);
    const double drtnum_dtheta = -8. * (1 - et_value * et_value) * std::cos(theta) * std::sin(theta);
    const double drt_dtheta =
        (drtnum_dtheta * rt_den - drtden_dtheta * rt_num) / (3. * rt_den * rt_den);
    for (int i = 0; i < 6; ++i)
      dp[i] = ((dp_depsilon * depsilon_dsigma[i]) + (dp_drho * drho_dsigma[i])) +
              (dp_drt * drt_dtheta * dtheta_dsigma[i]);
    *dp_dq = dp_drho * std::sqrt(2. / 3.);
  } else {
    const double r_mc = (3. - std::sin(phi)) / (6 * std::cos(phi));
    double e_val = (3. - std::sin(phi)) / (3. + std::sin(phi));
    if (e_val <= 0.5) e_val = 0.5 + 1.E-10;
    if (e_val > 1.) e_val = 1.;
    double sqpart = (4. * (1 - e_val * e_val) * std::pow(std::cos(theta), 2)) +
                    (5 * e_val * e_val) - (4. * e_val);
    if (sqpart < kEps) sqpart = 1.E-5;
    double mm = (2. * (1 - e_val * e_val) * std::cos(theta)) +
                ((2. * e_val - 1) * std::sqrt(sqpart));
    if (std::fabs(mm) < kEps) mm = 1.E-5;
    const double l = (4. * (1. - e_val * e_val) * std::pow(std::cos(theta), 2)) +
                     std::pow((2. * e_val - 1.), 2);
    const double r_mw = (l / mm) * r_mc;
    const double xi = 0.1;
    double omega = std::pow((xi * m.c_peak * std::tan(psi)), 2) +
                   std::pow((r_mw * std::sqrt(1.5) * rho), 2);
    if (omega < kEps) omega = 1.E-5;
    const double dl_dtheta = -8. * (1. - e_val * e_val) * std::cos(theta) * std::sin(theta);
    const double dm_dtheta = (-2. * (1. - e_val * e_val) * std::sin(theta)) +
                             (0.5 * (2. * e_val - 1.) * dl_dtheta) / std::sqrt(sqpart);
    const double drmw_dtheta = ((mm * dl_dtheta) - (l * dm_dtheta)) / (mm * mm);
    const double dp_depsilon = std::tan(psi) / std::sqrt(3.);
    const double dp_drho = 3. * rho * r_mw * r_mw / (2. * std::sqrt(omega));
    const double dp_dtheta =
        (3. * rho * rho * r_mw * r_mc * drmw_dtheta) / (2. * std::sqrt(omega));
    for (int i = 0; i < 6; ++i)
      dp[i] = ((dp_depsilon * depsilon_dsigma[i]) + (dp_drho * drho_dsigma[i])) +
              (dp_dtheta * dtheta_dsigma[i]);
    *dp_dq = dp_drho * std::sqrt(2. / 3.);
  }
  double dphi_dpstrain = 0.;
  double dc_dpstrain = 0.;
  *softening = 0.;
  if (m.softening && pdstrain > m.pd_peak && pdstrain < m.pd_res) {
    dphi_dpstrain = (m.phi_res - m.phi_peak) / (m.pd_res - m.pd_peak);
    dc_dpstrain = (m.c_res - m.c_peak) / (m.pd_res - m.pd_peak);
    const double df_dphi =
        std::sqrt(1.5) * rho *
            ((std::sin(phi) * std::sin(theta + kPi / 3.) /
              (std::sqrt(3.) * std::cos(phi) * std::cos(phi))) +
             (std::cos(theta + kPi / 3.) / (3. * std::cos(phi) * std::cos(phi)))) +
        (mu_p(s) / (std::cos(phi) * std::cos(phi)));
    const double df_dc = -1.;
    *softening = (-1.) * ((df_dphi * dphi_dpstrain) + (df_dc * dc_dpstrain)) * (*dp_dq);
  }
}

// (a^T De) . b, evaluated as the row vector a^T De first, then the dot,
// both left to right (mohr_coulomb.tcc:433,454-455)
double row_de_dot(const double de[6][6], const double* a, const double* b) {
  double r[6];
  for (int j = 0; j < 6; ++j) {
    double s = a[0] * de[0][j];
    for (int i = 1; i < 6; ++i) s = s + a[i] * de[i][j];
    r[j] = s;
  }
  double d = r[0] * b[0];
  for (int j = 1; j < 6; ++j) d = d + r[j] * b[j];
  return d;
}
// De * b (6x6 times 6), sum over k left to right
void de_mul(const double de[6][6], const double* b, double* o) {
  for (int i = 0; i < 6; ++i) {
    double s = de[i][0] * b[0];
    for (int k = 1; k < 6; ++k) s = s + de[i][k] * b[k];
    o[i] = s;
  }
}

// mohr_coulomb.tcc:348-513 (stress_rate None: trial = stress + De dstrain,
// infinitesimal_elasto_plastic.tcc:2-25)
void mc_compute_stress(const Material& m, const double* stress, const double* dstrain,
                       double density, double* sv, double* out) {
  const double current_packing_density = density;
  const double critical_density = m.min_packing * m.grain_density;
  const double pdstrain = sv[SV_PD];
  if (m.softening && pdstrain > m.pd_peak) {
    if (pdstrain < m.pd_res) {
      sv[SV_PHI] = m.phi_res + ((m.phi_peak - m.phi_res) * (pdstrain - m.pd_res) /
                                (m.pd_peak - m.pd_res));
      sv[SV_PSI] = m.psi_res + ((m.psi_peak - m.psi_res) * (pdstrain - m.pd_res) /
                                (m.pd_peak - m.pd_res));
      sv[SV_COH] = m.c_res + ((m.c_peak - m.c_res) * (pdstrain - m.pd_res) /
                              (m.pd_peak - m.pd_res));
    } else {
      sv[SV_PHI] = m.phi_res;
      sv[SV_PSI] = m.psi_res;
      sv[SV_COH] = m.c_res;
    }
    const double apex = sv[SV_COH] / std::tan(sv[SV_PHI]);
    if (sv[SV_TC] > apex) sv[SV_TC] = check_low(apex);
  }
  sv[SV_YIELD] = 0;
  double tmp[6], trial[6];
  de_mul(m.de, dstrain, tmp);
  for (int i = 0; i < 6; ++i) trial[i] = stress[i] + tmp[i];
  if (current_packing_density <= critical_density) {
    sv[SV_PD] += mu_q(trial) / 3.0 / m.shear;
    sv[SV_YIELD] = 3;
    for (int i = 0; i < 6; ++i) out[i] = 0.;
    return;
  }
  mc_invariants(trial, sv);
  double yf_trial[2];
  int yt_trial = mc_yield_state(yf_trial, sv);
  if (yt_trial == Elastic) {
    sv[SV_YIELD] = 0;
    for (int i = 0; i < 6; ++i) out[i] = trial[i];
    return;
  }
  const double Tolerance = 1E-1;
  double softening_trial = 0., dp_dq_trial = 0.;
  double df_trial[6] = {0}, dp_trial[6] = {0};
  mc_df_dp(m, yt_trial, sv, trial, df_trial, dp_trial, &dp_dq_trial, &softening_trial);
  double yield_trial = 0.;
  if (yt_trial == Tensile) {
    sv[SV_YIELD] = 2;
    yield_trial = yf_trial[0];
  }
  if (yt_trial == Shear) {
    sv[SV_YIELD] = 1;
    yield_trial = yf_trial[1];
  }
  double lambda_trial =
      yield_trial / (row_de_dot(m.de, df_trial, dp_trial) + softening_trial);
  mc_invariants(stress, sv);
  double yf[2];
  const int yt = mc_yield_state(yf, sv);
  double yield = std::numeric_limits<double>::max();
  if (yt == Tensile) yield = yf[0];
  if (yt == Shear) yield = yf[1];
  double softening = 0., dp_dq = 0.;
  double df[6] = {0}, dp[6] = {0};
  mc_df_dp(m, yt, sv, stress, df, dp, &dp_dq, &softening);
  const double lambda =
      row_de_dot(m.de, df, dstrain) / (row_de_dot(m.de, df, dp) + softening);
  double upd[6];
  for (int i = 0; i < 6; ++i) upd[i] = trial[i];
  double dpdstrain = 0.;
  // updated_stress += -(lambda * de * dp_dsigma): (lambda*De) * dp, sum over k
  if (std::fabs(yield) < Tolerance) {
    for (int i = 0; i < 6; ++i) {
      double s = (lambda * m.de[i][0]) * dp[0];
      for (int k = 1; k < 6; ++k) s = s + (lambda * m.de[i][k]) * dp[k];
      upd[i] += -s;
    }
    dpdstrain = lambda * dp_dq;
  } else {
    for (int i = 0; i < 6; ++i) {
      double s = (lambda_trial * m.de[i][0]) * dp_trial[0];
      for (int k = 1; k < 6; ++k) s = s + (lambda_trial * m.de[i][k]) * dp_trial[k];
      upd[i] += -s;
    }
    dpdstrain = lambda_trial * dp_dq_trial;
  }
  const int itr_max = 100;
  for (int itr = 0; itr < itr_max; ++itr) {
    mc_invariants(upd, sv);
    yt_trial = mc_yield_state(yf_trial, sv);
    if (yf_trial[0] < Tolerance && yf_trial[1] < Tolerance) break;
    mc_df_dp(m, yt_trial, sv, upd, df_trial, dp_trial, &dp_dq_trial, &softening_trial);
    if (yt_trial == Tensile) yield_trial = yf_trial[0];
    if (yt_trial == Shear) yield_trial = yf_trial[1];
    lambda_trial = yield_trial / (row_de_dot(m.de, df_trial, dp_trial) + softening_trial);
    for (int i = 0; i < 6; ++i) {
      double s = (lambda_trial * m.de[i][0]) * dp_trial[0];
      for (int k = 1; k < 6; ++k) s = s + (lambda_trial * m.de[i][k]) * dp_trial[k];
      upd[i] += -s;
    }
    dpdstrain += lambda_trial * dp_dq_trial;
  }
  mc_invariants(upd, sv);
  sv[SV_PD] += dpdstrain;
  for (int i = 0; i < 6; ++i) out[i] = upd[i];
}

// linear_elastic.tcc:73-94 (stress_rate None)
void le_compute_stress(const Material& m, const double* stress, const double* dstrain,
                       double* out) {
  double tmp[6];
  de_mul(m.de, dstrain, tmp);
  for (int i = 0; i < 6; ++i) out[i] = stress[i] + tmp[i];
}

void material_compute_stress(const Material& m, const double* stress, const double* dstrain,
                             double density, double* sv, double* out) {
  if (m.type == 0)
    le_compute_stress(m, stress, dstrain, out);
  else
    mc_compute_stress(m, stress, dstrain, density, sv, out);
}

// ------------------------------------------------------------------ elements
// Q4: include/elements/2d/quadrilateral_element.tcc:11-43
// H8: include/elements/3d/hexahedron_element.tcc:19-74
void shapefn(int dim, const double* xi, double* N) {
  if (dim == 2) {
    N[0] = 0.25 * (1 - xi[0]) * (1 - xi[1]);
    N[1] = 0.25 * (1 + xi[0]) * (1 - xi[1]);
    N[2] = 0.25 * (1 + xi[0]) * (1 + xi[1]);
    N[3] = 0.25 * (1 - xi[0]) * (1 + xi[1]);
  } else {
    N[0] = 0.125 * (1 - xi[0]) * (1 - xi[1]) * (1 - xi[2]);
    N[1] = 0.125 * (1 + xi[0]) * (1 - xi[1]) * (1 - xi[2]);
    N[2] = 0.125 * (1 + xi[0]) * (1 + xi[1]) * (1 - xi[2]);
    N[3] = 0.125 * (1 - xi[0]) * (1 + xi[1]) * (1 - xi[2]);
    N[4] = 0.125 * (1 - xi[0]) * (1 - xi[1]) * (1 + xi[2]);
    N[5] = 0.125 * (1 + xi[0]) * (1 - xi[1]) * (1 + xi[2]);
    N[6] = 0.125 * (1 + xi[0]) * (1 + xi[1]) * (1 + xi[2]);
    N[7] = 0.125 * (1 - xi[0]) * (1 + xi[1]) * (1 + xi[2]);
  }
}
// G is nv x dim row-major
void grad_shapefn(int dim, const double* xi, double* G) {
  if (dim == 2) {
    G[0 * 2 + 0] = -0.25 * (1 - xi[1]);
    G[1 * 2 + 0] = 0.25 * (1 - xi[1]);
    G[2 * 2 + 0] = 0.25 * (1 + xi[1]);
    G[3 * 2 + 0] = -0.25 * (1 + xi[1]);
    G[0 * 2 + 1] = -0.25 * (1 - xi[0]);
    G[1 * 2 + 1] = -0.25 * (1 + xi[0]);
    G[2 * 2 + 1] = 0.25 * (1 + xi[0]);
    G[3 * 2 + 1] = 0.25 * (1 - xi[0]);
  } else {
    G[0 * 3 + 0] = -0.125 * (1 - xi[1]) * (1 - xi[2]);
    G[1 * 3 + 0] = 0.125 * (1 - xi[1]) * (1 - xi[2]);
    G[2 * 3 + 0] = 0.125 * (1 + xi[1]) * (1 - xi[2]);
    G[3 * 3 + 0] = -0.125 * (1 + xi[1]) * (1 - xi[2]);
    G[4 * 3 + 0] = -0.125 * (1 - xi[1]) * (1 + xi[2]);
    G[5 * 3 + 0] = 0.125 * (1 - xi[1]) * (1 + xi[2]);
    G[6 * 3 + 0] = 0.125 * (1 + xi[1]) * (1 + xi[2]);
    G[7 * 3 + 0] = -0.125 * (1 + xi[1]) * (1 + xi[2]);
    G[0 * 3 + 1] = -0.125 * (1 - xi[0]) * (1 - xi[2]);
    G[1 * 3 + 1] = -0.125 * (1 + xi[0]) * (1 - xi[2]);
    G[2 * 3 + 1] = 0.125 * (1 + xi[0]) * (1 - xi[2]);
    G[3 * 3 + 1] = 0.125 * (1 - xi[0]) * (1 - xi[2]);
    G[4 * 3 + 1] = -0.125 * (1 - xi[0]) * (1 + xi[2]);
    G[5 * 3 + 1] = -0.125 * (1 + xi[0]) * (1 + xi[2]);
    G[6 * 3 + 1] = 0.125 * (1 + xi[0]) * (1 + xi[2]);
    G[7 * 3 + 1] = 0.125 * (1 - xi[0]) * (1 + xi[2]);
    G[0 * 3 + 2] = -0.125 * (1 - xi[0]) * (1 - xi[1]);
    G[1 * 3 + 2] = -0.125 * (1 + xi[0]) * (1 - xi[1]);
    G[2 * 3 + 2] = -0.125 * (1 + xi[0]) * (1 + xi[1]);
    G[3 * 3 + 2] = -0.125 * (1 - xi[0]) * (1 + xi[1]);
    G[4 * 3 + 2] = 0.125 * (1 - xi[0]) * (1 - xi[1]);
    G[5 * 3 + 2] = 0.125 * (1 + xi[0]) * (1 - xi[1]);
    G[6 * 3 + 2] = 0.125 * (1 + xi[0]) * (1 + xi[1]);
    G[7 * 3 + 2] = 0.125 * (1 - xi[0]) * (1 + xi[1]);
  }
}

// Inverse of a dim x dim matrix by adjugate / determinant (Eigen fixed-size
// inverse, cofactor form).
void inverse(int dim, const double* J, double* inv) {
  if (dim == 2) {
    const double det = J[0] * J[3] - J[2] * J[1];
    const double invdet = 1.0 / det;
    inv[0] = J[3] * invdet;
    inv[2] = -J[2] * invdet;
    inv[1] = -J[1] * invdet;
    inv[3] = J[0] * invdet;
  } else {
    auto m = [&](int r, int c) { return J[r * 3 + c]; };
    auto cof = [&](int i, int j) {
      const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
      return m(i1, j1) * m(i2, j2) - m(i1, j2) * m(i2, j1);
    };
    const double c0 = cof(0, 0), c1 = cof(1, 0), c2 = cof(2, 0);
    const double det = (c0 * m(0, 0) + c1 * m(1, 0)) + c2 * m(2, 0);
    const double invdet = 1.0 / det;
    inv[0 * 3 + 0] = c0 * invdet;
    inv[0 * 3 + 1] = c1 * invdet;
    inv[0 * 3 + 2] = c2 * invdet;
    inv[1 * 3 + 0] = cof(0, 1) * invdet;
    inv[1 * 3 + 1] = cof(1, 1) * invdet;
    inv[1 * 3 + 2] = cof(2, 1) * invdet;
    inv[2 * 3 + 0] = cof(0, 2) * invdet;
    inv[2 * 3 + 1] = cof(1, 2) * invdet;
    inv[2 * 3 + 2] = cof(2, 2) * invdet;
  }
}

// dN/dx = grad_sf * inv(J)^T with J = grad_sf^T X
// (quadrilateral_element.tcc:295-309, hexahedron_element.tcc:307-321)
void dn_dx(int dim, const double* xi, const double* X, double* G, double* D) {
  const int nv = dim == 2 ? 4 : 8;
  grad_shapefn(dim, xi, G);
  double J[9], inv[9];
  for (int r = 0; r < dim; ++r)
    for (int c = 0; c < dim; ++c) {
      double s = G[0 * dim + r] * X[0 * dim + c];
      for (int n = 1; n < nv; ++n) s = s + G[n * dim + r] * X[n * dim + c];
      J[r * dim + c] = s;
    }
  inverse(dim, J, inv);
  for (int n = 0; n < nv; ++n)
    for (int c = 0; c < dim; ++c) {
      double s = G[n * dim + 0] * inv[c * dim + 0];
      for (int k = 1; k < dim; ++k) s = s + G[n * dim + k] * inv[c * dim + k];
      D[n * dim + c] = s;
    }
}

double norm(int dim, const double* a) {
  double s = a[0] * a[0];
  for (int i = 1; i < dim; ++i) s = s + a[i] * a[i];
  return std::sqrt(s);
}

// ---------------------------------------------------------------- entities
struct Cell {
  int64_t nodes[8];
  double X[8 * 3];
  double centroid[3];
  double mean_length;
  double volume;
  double dndx_c[8 * 3];
  std::vector<int64_t> neighbours;  // ascending (std::set order)
  std::vector<int64_t> particles;
  double half[3];                   // xlength, ylength, zlength
};

struct Node {
  double coord[3];
  double mass, mom[3], fext[3], fint[3], vel[3], acc[3];
  bool status;
  std::map<unsigned, double> vel_c, acc_c;
  bool friction = false;
  unsigned fdir = 0;
  int fsign = 0;
  double mu = 0;
  bool rotated = false;            // generic_boundary_constraints_
  double R[9] = {}, Ri[9] = {};    // rotation_matrix_ and its inverse (dim x dim)
#ifdef _OPENMP
  omp_lock_t lock;
#endif
};

struct Particle {
  int64_t id;
  double x[3], u[3], v[3], a[3];
  double sig[6], eps[6], deps[6], eps_rate[6];
  double F[9], Finc[9];
  double vol, rho, mass;
  double xi[3];
  int64_t cell;
  double N[8], dndx[8 * 3];
  double dvol;
  int mat;  // index into materials vector
  double sv[9];
  int status;
  std::vector<std::pair<unsigned, double>> pvc;  // particle velocity constraints
  double B[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};      // mapping matrix (row-major dim x dim)
};

struct Oracle {
  mpmo_config cfg;
  int dim = 3, nv = 8;
  std::vector<Node> nodes;
  std::vector<Cell> cells;
  std::vector<Material> materials;
  std::map<int, int> material_index;
  std::vector<Particle> particles;
  int64_t step = 0;
  std::string err;
  // bins for the exhaustive cell search (equivalent to a scan in id order)
  double bmin[3], bsize[3];
  int64_t bn[3];
  std::vector<std::vector<int64_t>> bins;
};

// cell.tcc:33-65, :255-279 (centroid, mean length), :237-250 (volume)
void cell_initialise(Oracle& o, Cell& c) {
  const int dim = o.dim, nv = o.nv;
  for (int i = 0; i < dim; ++i) c.centroid[i] = 0.;
  for (int n = 0; n < nv; ++n)
    for (int i = 0; i < dim; ++i) c.centroid[i] = c.centroid[i] + c.X[n * dim + i];
  for (int i = 0; i < dim; ++i) c.centroid[i] = c.centroid[i] / nv;
  // sides_indices: quadrilateral_element.tcc:375-385, hexahedron_element.tcc:460-480
  static const int q4s[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
  static const int h8s[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                 {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  const int ns = dim == 2 ? 4 : 12;
  c.mean_length = 0.;
  for (int s = 0; s < ns; ++s) {
    const int a = dim == 2 ? q4s[s][0] : h8s[s][0];
    const int b = dim == 2 ? q4s[s][1] : h8s[s][1];
    double d[3];
    for (int i = 0; i < dim; ++i) d[i] = c.X[a * dim + i] - c.X[b * dim + i];
    c.mean_length += norm(dim, d);
  }
  c.mean_length /= ns;
  // lengths used by local_coordinates_point (cell.tcc:458-463, 566-571)
  {
    double d[3];
    for (int i = 0; i < dim; ++i) d[i] = c.X[0 * dim + i] - c.X[1 * dim + i];
    c.half[0] = norm(dim, d);
    for (int i = 0; i < dim; ++i) d[i] = c.X[1 * dim + i] - c.X[2 * dim + i];
    c.half[1] = norm(dim, d);
    if (dim == 3) {
      for (int i = 0; i < dim; ++i) d[i] = c.X[1 * dim + i] - c.X[5 * dim + i];
      c.half[2] = norm(dim, d);
    }
  }
  // volume: quadrilateral_element.tcc:473-496, hexahedron_element.tcc:559-596
  if (dim == 2) {
    auto len = [&](int a, int b) {
      double d[2] = {c.X[a * 2] - c.X[b * 2], c.X[a * 2 + 1] - c.X[b * 2 + 1]};
      return norm(2, d);
    };
    const double a = len(0, 3), b = len(2, 3), cc = len(1, 2), d = len(0, 1);
    const double p = len(0, 2), q = len(1, 3);
    c.volume = 0.25 * std::sqrt(4 * p * p * q * q - std::pow((a * a + cc * cc - b * b - d * d), 2.0));
  } else {
    auto row = [&](int n, double* r) { for (int i = 0; i < 3; ++i) r[i] = c.X[n * 3 + i]; };
    double A[3], B[3], C[3], D[3], E[3], Fv[3], G[3], H[3];
    row(7, A); row(6, B); row(2, C); row(3, D); row(4, E); row(5, Fv); row(1, G); row(0, H);
    auto sub = [](const double* x, const double* y, double* r) { for (int i = 0; i < 3; ++i) r[i] = x[i] - y[i]; };
    auto cross = [](const double* x, const double* y, double* r) {
      r[0] = x[1] * y[2] - x[2] * y[1];
      r[1] = x[2] * y[0] - x[0] * y[2];
      r[2] = x[0] * y[1] - x[1] * y[0];
    };
    auto add = [](const double* x, const double* y, double* r) { for (int i = 0; i < 3; ++i) r[i] = x[i] + y[i]; };
    double t1[3], t2[3], bd[3], ca[3], eb[3], fa[3], de_[3], ha[3];
    sub(B, D, t1); sub(C, A, t2); cross(t1, t2, bd);   // (b-d)x(c-a)
    sub(E, B, t1); sub(Fv, A, t2); cross(t1, t2, eb);  // (e-b)x(f-a)
    sub(D, E, t1); sub(H, A, t2); cross(t1, t2, de_);  // (d-e)x(h-a)
    double s1[3], s2[3], s3[3], s4[3], tmp[3];
    add(bd, eb, tmp); add(tmp, de_, s1);
    sub(C, G, t1); sub(C, Fv, t2); cross(t1, t2, ca); add(bd, ca, s2);
    sub(Fv, G, t1); sub(H, Fv, t2); cross(t1, t2, fa); add(eb, fa, s3);
    sub(H, G, t1); sub(H, C, t2); cross(t1, t2, ha); add(de_, ha, s4);
    double ag[3], bg[3], eg[3], dg[3];
    sub(A, G, ag); sub(B, G, bg); sub(E, G, eg); sub(D, G, dg);
    c.volume = (1.0 / 12) * dot3(ag, s1) + (1.0 / 12) * dot3(bg, s2) +
               (1.0 / 12) * dot3(eg, s3) + (1.0 / 12) * dot3(dg, s4);
  }
  // dn_dx at the centroid (xi = 0)
  double xi0[3] = {0, 0, 0}, G[8 * 3];
  dn_dx(dim, xi0, c.X, G, c.dndx_c);
}

// cell.tcc:423-488 (2D quadrilateral), :492-605 (3D hexahedron)
void local_coordinates_point(const Oracle& o, const Cell& c, const double* p, double* xi) {
  for (int i = 0; i < o.dim; ++i) xi[i] = 2. * (p[i] - c.centroid[i]) / c.half[i];
}

// cell.tcc:324-331
bool approx_point_in_cell(const Oracle& o, const Cell& c, const double* p) {
  double d[3];
  for (int i = 0; i < o.dim; ++i) d[i] = p[i] - c.centroid[i];
  const double length = norm(o.dim, d);
  return length < (c.mean_length * 2.);
}

// cell.tcc:617-826 transform_real_to_unit_cell for quad4 / hex8: the root of
// sum_i N_i(xi) X_i = p.  The reference keeps the best of an analytical (2D) or
// affine guess and Newton iterations with a line search; this restatement runs
// Newton from the cell centre to a step below 1e-12 (quadratic convergence:
// the root to rounding for a convex cell).  False when it does not converge.
bool transform_real_to_unit_cell(const Oracle& o, const Cell& c, const double* p, double* xi) {
  const int dim = o.dim, nv = o.nv;
  for (int d = 0; d < dim; ++d) xi[d] = 0.;
  for (int it = 0; it < 50; ++it) {
    double N[8], G[8 * 3], r[3], Jm[9], Ji[9];
    shapefn(dim, xi, N);
    grad_shapefn(dim, xi, G);
    for (int a = 0; a < dim; ++a) {
      double xa = N[0] * c.X[0 * dim + a];
      for (int i = 1; i < nv; ++i) xa = xa + N[i] * c.X[i * dim + a];
      r[a] = xa - p[a];
      for (int b = 0; b < dim; ++b) {
        double j = c.X[0 * dim + a] * G[0 * dim + b];
        for (int i = 1; i < nv; ++i) j = j + c.X[i * dim + a] * G[i * dim + b];
        Jm[a * dim + b] = j;
      }
    }
    inverse(dim, Jm, Ji);
    double step = 0.;
    for (int b = 0; b < dim; ++b) {
      double dxi = Ji[b * dim + 0] * r[0];
      for (int a = 1; a < dim; ++a) dxi = dxi + Ji[b * dim + a] * r[a];
      xi[b] -= dxi;
      step = std::max(step, std::fabs(dxi));
    }
    if (!(step == step)) return false;
    if (step < 1e-12) return true;  // quadratic convergence: xi now at rounding level
  }
  return false;
}

// cell.tcc:335-384
bool is_point_in_cell(const Oracle& o, const Cell& c, const double* p, double* xi) {
  for (int i = 0; i < o.dim; ++i) xi[i] = std::numeric_limits<double>::max();
  if (!approx_point_in_cell(o, c, p)) return false;
  bool status = true;
  if (o.cfg.isoparametric) {
    if (!transform_real_to_unit_cell(o, c, p, xi)) return false;
  } else {
    local_coordinates_point(o, c, p, xi);
  }
  const double tolerance = kEps;
  for (int i = 0; i < o.dim; ++i) {
    if (xi[i] < -1. || xi[i] > 1. || std::isnan(xi[i]))
      status = false;
    else {
      if (xi[i] < -1. + tolerance) xi[i] = -1. + tolerance;
      if (xi[i] > 1. - tolerance) xi[i] = 1. - tolerance;
    }
  }
  return status;
}

void build_bins(Oracle& o) {
  const int dim = o.dim;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  double maxr = 0;
  for (auto& c : o.cells) {
    const double r = 2. * c.mean_length;
    maxr = std::max(maxr, r);
    for (int i = 0; i < dim; ++i) {
      lo[i] = std::min(lo[i], c.centroid[i] - r);
      hi[i] = std::max(hi[i], c.centroid[i] + r);
    }
  }
  int64_t total = 1;
  for (int i = 0; i < 3; ++i) {
    if (i >= dim) { o.bn[i] = 1; o.bmin[i] = 0; o.bsize[i] = 1; continue; }
    o.bmin[i] = lo[i];
    o.bsize[i] = std::max(maxr, 1e-300);
    o.bn[i] = std::max<int64_t>(1, (int64_t)std::ceil((hi[i] - lo[i]) / o.bsize[i]) + 1);
    total *= o.bn[i];
  }
  o.bins.assign(total, {});
  for (int64_t id = 0; id < (int64_t)o.cells.size(); ++id) {
    const Cell& c = o.cells[id];
    const double r = 2. * c.mean_length;
    int64_t b0[3] = {0, 0, 0}, b1[3] = {0, 0, 0};
    for (int i = 0; i < dim; ++i) {
      b0[i] = std::max<int64_t>(0, (int64_t)std::floor((c.centroid[i] - r - o.bmin[i]) / o.bsize[i]) - 1);
      b1[i] = std::min<int64_t>(o.bn[i] - 1, (int64_t)std::floor((c.centroid[i] + r - o.bmin[i]) / o.bsize[i]) + 1);
    }
    for (int64_t k = b0[2]; k <= b1[2]; ++k)
      for (int64_t j = b0[1]; j <= b1[1]; ++j)
        for (int64_t i = b0[0]; i <= b1[0]; ++i)
          o.bins[(k * o.bn[1] + j) * o.bn[0] + i].push_back(id);
  }
}

// Exhaustive search in cell id order (mesh.tcc:1136-1148 with one thread):
// returns the first cell (smallest id) containing p.  The bins hold every cell
// whose approximate-containment sphere can reach the bin, so the candidates
// include every cell that could pass is_point_in_cell.
int64_t scan_cells(const Oracle& o, const double* p, double* xi_out) {
  int64_t b[3] = {0, 0, 0};
  for (int i = 0; i < o.dim; ++i) {
    const double f = std::floor((p[i] - o.bmin[i]) / o.bsize[i]);
    if (!(f >= 0) || f >= (double)o.bn[i]) return kNone;
    b[i] = (int64_t)f;
  }
  const auto& cand = o.bins[(b[2] * o.bn[1] + b[1]) * o.bn[0] + b[0]];
  for (int64_t id : cand) {  // ascending id (pushed in id order)
    double xi[3];
    if (is_point_in_cell(o, o.cells[id], p, xi)) {
      for (int i = 0; i < o.dim; ++i) xi_out[i] = xi[i];
      return id;
    }
  }
  return kNone;
}

// particle.tcc:420-466 (assign_cell_xi) together with the cell particle list
void assign_cell_xi(Oracle& o, Particle& P, int64_t cell, const double* xi) {
  if (P.cell != kNone && P.cell != cell) {
    auto& lst = o.cells[P.cell].particles;
    lst.erase(std::remove(lst.begin(), lst.end(), P.id), lst.end());
  }
  P.cell = cell;
  for (int i = 0; i < o.dim; ++i) P.xi[i] = xi[i];
  auto& lst = o.cells[cell].particles;
  if (std::find(lst.begin(), lst.end(), P.id) == lst.end()) lst.push_back(P.id);
}

// mesh.tcc:1116-1151 (locate_particle_cells) and particle.tcc:521-533
bool locate_particle(Oracle& o, Particle& P) {
  if (P.cell != kNone) {
    double xi[3];
    if (is_point_in_cell(o, o.cells[P.cell], P.x, xi)) {
      for (int i = 0; i < o.dim; ++i) P.xi[i] = xi[i];
      return true;
    }
    for (int64_t nb : o.cells[P.cell].neighbours) {
      if (is_point_in_cell(o, o.cells[nb], P.x, xi)) {
        assign_cell_xi(o, P, nb, xi);
        return true;
      }
    }
  }
  double xi[3];
  const int64_t c = scan_cells(o, P.x, xi);
  if (c == kNone) return false;
  assign_cell_xi(o, P, c, xi);
  return true;
}

// node.tcc:370-403 (Cartesian constraints)
// y = M x with M dim x dim row-major
void mat_vec(int dim, const double* M, const double* x, double* y) {
  for (int a = 0; a < dim; ++a) {
    double s = M[a * dim + 0] * x[0];
    for (int b = 1; b < dim; ++b) s = s + M[a * dim + b] * x[b];
    y[a] = s;
  }
}

// node.tcc:370-403
void node_apply_velocity_constraints(Oracle& o, Node& n) {
  for (const auto& c : n.vel_c) {
    const unsigned direction = c.first % o.dim;
    if (!n.rotated) {
      n.vel[direction] = c.second;
      n.acc[direction] = 0.;
    } else {
      double lv[3], la[3];
      mat_vec(o.dim, n.Ri, n.vel, lv);
      mat_vec(o.dim, n.Ri, n.acc, la);
      lv[direction] = c.second;
      la[direction] = 0.;
      mat_vec(o.dim, n.R, lv, n.vel);
      mat_vec(o.dim, n.R, la, n.acc);
    }
  }
}
// node.tcc:456-483
void node_apply_acceleration_constraints(Oracle& o, Node& n) {
  for (const auto& c : n.acc_c) {
    const unsigned direction = c.first % o.dim;
    if (!n.rotated) {
      n.acc[direction] = c.second;
    } else {
      double la[3];
      mat_vec(o.dim, n.Ri, n.acc, la);
      la[direction] = c.second;
      mat_vec(o.dim, n.R, la, n.acc);
    }
  }
}
// node.tcc:510-657 (Cartesian)
void node_apply_friction_constraints(Oracle& o, Node& n, double dt) {
  if (!n.friction) return;
  auto sign = [](double value) { return (value > 0.) ? 1. : -1.; };
  const unsigned dir_n = n.fdir;
  const double sign_n = sign(n.fsign);
  const double mu = n.mu;
  // components in the node's frame (the global ones on a Cartesian boundary)
  double lacc[3] = {n.acc[0], n.acc[1], n.acc[2]}, lvel[3] = {n.vel[0], n.vel[1], n.vel[2]};
  if (n.rotated) {
    mat_vec(o.dim, n.Ri, n.acc, lacc);
    mat_vec(o.dim, n.Ri, n.vel, lvel);
  }
  if (o.dim == 2) {
    const unsigned dir_t = (2 - 1) - dir_n;
    const double acc_n = lacc[dir_n];
    double acc_t = lacc[dir_t];
    const double vel_t = lvel[dir_t];
    if ((acc_n * sign_n) > 0.0) {
      if (vel_t != 0.0) {
        const double vel_net = dt * acc_t + vel_t;
        const double vel_frictional = dt * mu * std::abs(acc_n);
        if (std::abs(vel_net) <= vel_frictional)
          acc_t = -vel_t / dt;
        else
          acc_t -= sign(vel_net) * mu * std::abs(acc_n);
      } else {
        if (std::abs(acc_t) <= mu * std::abs(acc_n))
          acc_t = 0.0;
        else
          acc_t -= sign(acc_t) * mu * std::abs(acc_n);
      }
      if (!n.rotated) {
        n.acc[dir_t] = acc_t;
      } else {
        lacc[dir_t] = acc_t;
        mat_vec(o.dim, n.R, lacc, n.acc);
      }
    }
  } else {
    static const int dirs[3][2] = {{1, 2}, {0, 2}, {0, 1}};
    const unsigned t0 = dirs[dir_n][0], t1 = dirs[dir_n][1];
    double acc[3], vel[3];
    for (int i = 0; i < 3; ++i) { acc[i] = lacc[i]; vel[i] = lvel[i]; }
    const double acc_n = acc[dir_n];
    double acc_t = std::sqrt(acc[t0] * acc[t0] + acc[t1] * acc[t1]);
    const double vel_t = std::sqrt(vel[t0] * vel[t0] + vel[t1] * vel[t1]);
    if (acc_n * sign_n > 0.0) {
      if (vel_t != 0.0) {
        double vn0 = vel[t0] + acc[t0] * dt;
        double vn1 = vel[t1] + acc[t1] * dt;
        const double vel_net_t = std::sqrt(vn0 * vn0 + vn1 * vn1);
        const double vel_fricion = mu * std::abs(acc_n) * dt;
        if (vel_net_t <= vel_fricion) {
          acc[t0] = -vel[t0] / dt;
          acc[t1] = -vel[t1] / dt;
        } else {
          acc[t0] -= mu * std::abs(acc_n) * (vn0 / vel_net_t);
          acc[t1] -= mu * std::abs(acc_n) * (vn1 / vel_net_t);
        }
      } else {
        if (acc_t <= mu * std::abs(acc_n)) {
          acc[t0] = 0;
          acc[t1] = 0;
        } else {
          acc_t -= mu * std::abs(acc_n);
          acc[t0] -= mu * std::abs(acc_n) * (acc[t0] / acc_t);
          acc[t1] -= mu * std::abs(acc_n) * (acc[t1] / acc_t);
        }
      }
      if (!n.rotated)
        for (int i = 0; i < 3; ++i) n.acc[i] = acc[i];
      else
        mat_vec(3, n.R, acc, n.acc);
    }
  }
}

// node.tcc:236-252
void node_compute_velocity(Oracle& o, Node& n) {
  const double tolerance = 1.E-16;
  if (n.mass > tolerance) {
    for (int i = 0; i < o.dim; ++i) n.vel[i] = n.mom[i] / n.mass;
    for (int i = 0; i < o.dim; ++i)
      if (std::abs(n.vel[i]) < 1.E-15) n.vel[i] = 0.;
  }
  node_apply_velocity_constraints(o, n);
}

// node.tcc:309-345
void node_compute_acceleration_velocity_cundall(Oracle& o, Node& n, double dt, double damping) {
  const double tolerance = 1.0E-15;
  if (!(n.mass > tolerance)) return;
  const int dim = o.dim;
  double uf[3];
  for (int i = 0; i < dim; ++i) uf[i] = n.fext[i] + n.fint[i];
  const double nrm = norm(dim, uf);
  for (int i = 0; i < dim; ++i) {
    const double s = (n.vel[i] > 0.) ? 1. : ((n.vel[i] < 0.) ? -1. : 0.);
    n.acc[i] = (uf[i] - damping * nrm * s) / n.mass;
  }
  node_apply_friction_constraints(o, n, dt);
  node_apply_acceleration_constraints(o, n);
  for (int i = 0; i < dim; ++i) n.vel[i] += n.acc[i] * dt;
  node_apply_velocity_constraints(o, n);
  for (int i = 0; i < dim; ++i)
    if (std::abs(n.vel[i]) < tolerance) n.vel[i] = 0.;
  for (int i = 0; i < dim; ++i)
    if (std::abs(n.acc[i]) < tolerance) n.acc[i] = 0.;
}

inline void node_add(Node& n, double* dst, const double* val, int cnt, bool threaded) {
#ifdef _OPENMP
  if (threaded) {
    omp_set_lock(&n.lock);
    for (int i = 0; i < cnt; ++i) dst[i] = dst[i] + val[i];
    omp_unset_lock(&n.lock);
    return;
  }
#endif
  (void)n;
  (void)threaded;
  for (int i = 0; i < cnt; ++i) dst[i] = dst[i] + val[i];
}

// particle.tcc:537-553
void particle_compute_shapefn(Oracle& o, Particle& P) {
  const Cell& c = o.cells[P.cell];
  double G[8 * 3];
  shapefn(o.dim, P.xi, P.N);
  dn_dx(o.dim, P.xi, c.X, G, P.dndx);
}

// particle.tcc:819-857
void compute_strain_rate(const Oracle& o, const Particle& P, const double* D, double* sr) {
  for (int i = 0; i < 6; ++i) sr[i] = 0.;
  const Cell& c = o.cells[P.cell];
  if (o.dim == 2) {
    for (int i = 0; i < 4; ++i) {
      const double* vel = o.nodes[c.nodes[i]].vel;
      sr[0] += D[i * 2 + 0] * vel[0];
      sr[1] += D[i * 2 + 1] * vel[1];
      sr[3] += D[i * 2 + 1] * vel[0] + D[i * 2 + 0] * vel[1];
    }
    if (std::fabs(sr[0]) < 1.E-15) sr[0] = 0.;
    if (std::fabs(sr[1]) < 1.E-15) sr[1] = 0.;
    if (std::fabs(sr[3]) < 1.E-15) sr[3] = 0.;
  } else {
    for (int i = 0; i < 8; ++i) {
      const double* vel = o.nodes[c.nodes[i]].vel;
      sr[0] += D[i * 3 + 0] * vel[0];
      sr[1] += D[i * 3 + 1] * vel[1];
      sr[2] += D[i * 3 + 2] * vel[2];
      sr[3] += D[i * 3 + 1] * vel[0] + D[i * 3 + 0] * vel[1];
      sr[4] += D[i * 3 + 2] * vel[1] + D[i * 3 + 1] * vel[2];
      sr[5] += D[i * 3 + 2] * vel[0] + D[i * 3 + 0] * vel[2];
    }
    for (int i = 0; i < 6; ++i)
      if (std::fabs(sr[i]) < 1.E-15) sr[i] = 0.;
  }
}

// particle.tcc:1580-1628, 1643-1649
void update_deformation_gradient_increment(const Oracle& o, Particle& P, double dt) {
  const int dim = o.dim;
  double* Fi = P.Finc;
  for (int i = 0; i < 9; ++i) Fi[i] = 0.;
  Fi[0] = Fi[4] = Fi[8] = 1.;
  const Cell& c = o.cells[P.cell];
  for (int n = 0; n < o.nv; ++n) {
    const double* vel = o.nodes[c.nodes[n]].vel;
    for (int r = 0; r < dim; ++r)
      for (int cc = 0; cc < dim; ++cc)
        Fi[r * 3 + cc] += vel[r] * P.dndx[n * dim + cc] * dt;
  }
  for (int i = 0; i < dim; ++i)
    for (int j = 0; j < dim; ++j) {
      if (i != j && std::fabs(Fi[i * 3 + j]) < 1.E-15) Fi[i * 3 + j] = 0.;
      if (i == j && std::fabs(Fi[i * 3 + j] - 1.) < 1.E-15) Fi[i * 3 + j] = 1.;
    }
}

// particle.tcc:861-876
void compute_strain(const Oracle& o, Particle& P, double dt) {
  compute_strain_rate(o, P, P.dndx, P.eps_rate);
  for (int i = 0; i < 6; ++i) P.deps[i] = P.eps_rate[i] * dt;
  for (int i = 0; i < 6; ++i) P.eps[i] += P.deps[i];
  double src[6];
  compute_strain_rate(o, P, o.cells[P.cell].dndx_c, src);
  double s = src[0];
  for (int i = 1; i < o.dim; ++i) s = s + src[i];
  P.dvol = dt * s;
}

// particle.tcc:598-605
void update_volume(Particle& P) {
  P.vol *= (1. + P.dvol);
  P.rho = P.rho / (1. + P.dvol);
}

// particle.tcc:1654-1658
void update_deformation_gradient(Particle& P) {
  double R[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      R[i * 3 + j] = (P.Finc[i * 3 + 0] * P.F[0 * 3 + j] + P.Finc[i * 3 + 1] * P.F[1 * 3 + j]) +
                     P.Finc[i * 3 + 2] * P.F[2 * 3 + j];
  for (int i = 0; i < 9; ++i) P.F[i] = R[i];
}

// mpm_scheme.tcc:75-103
void compute_stress_strain(Oracle& o, double dt) {
  const int64_t np = (int64_t)o.particles.size();
#pragma omp parallel for schedule(static) if (o.cfg.nthreads > 1)
  for (int64_t p = 0; p < np; ++p) {
    Particle& P = o.particles[p];
    update_deformation_gradient_increment(o, P, dt);
    compute_strain(o, P, dt);
    update_volume(P);
    const Material& m = o.materials[P.mat];
    double out[6];
    material_compute_stress(m, P.sig, P.deps, P.rho, P.sv, out);
    for (int i = 0; i < 6; ++i) P.sig[i] = out[i];
    update_deformation_gradient(P);
  }
}

// mpm_scheme.tcc:19-40 MPMScheme::initialise
void phase_initialise(Oracle& o) {
  const bool thr = o.cfg.nthreads > 1;
  const int64_t np = (int64_t)o.particles.size();
  for (auto& n : o.nodes) {  // node.tcc:26-42
    n.mass = 0;
    for (int i = 0; i < 3; ++i) n.mom[i] = n.fext[i] = n.fint[i] = n.vel[i] = n.acc[i] = 0;
    n.status = false;
  }
  for (auto& c : o.cells)  // cell.tcc:171-177
    if (!c.particles.empty())
      for (int i = 0; i < o.nv; ++i) o.nodes[c.nodes[i]].status = true;
#pragma omp parallel for schedule(static) if (thr)
  for (int64_t p = 0; p < np; ++p) particle_compute_shapefn(o, o.particles[p]);
}

// The matrix M of the affine (APIC, ASFLIP: B D^-1 with the shape tensor
// D = sum_i N_i r_i r_i^T, r_i = x_i - x_p; particle.tcc:661-694) or Taylor
// (TPIC: B; :697-718) mapping velocity v + M r_i.  False for FLIP / PIC.
bool mapping_velocity_matrix(const Oracle& o, const Particle& P, double* M) {
  const int dim = o.dim, vu = o.cfg.velocity_update;
  if (vu != 2 && vu != 3 && vu != 4) return false;
  if (vu == 3) {
    for (int i = 0; i < dim * dim; ++i) M[i] = P.B[i];
    return true;
  }
  const Cell& c = o.cells[P.cell];
  double T[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < o.nv; ++i) {
    const double* X = o.nodes[c.nodes[i]].coord;
    double r[3];
    for (int d = 0; d < dim; ++d) r[d] = X[d] - P.x[d];
    for (int a = 0; a < dim; ++a)
      for (int b = 0; b < dim; ++b) T[a * dim + b] += (P.N[i] * r[a]) * r[b];
  }
  double Ti[9];
  inverse(dim, T, Ti);
  for (int a = 0; a < dim; ++a)
    for (int b = 0; b < dim; ++b) {
      double s = P.B[a * dim + 0] * Ti[0 * dim + b];
      for (int k = 1; k < dim; ++k) s = s + P.B[a * dim + k] * Ti[k * dim + b];
      M[a * dim + b] = s;
    }
  return true;
}

// particle.tcc:630-718 map_mass_momentum_to_nodes (plain, affine, Taylor)
void phase_p2g_mass_momentum(Oracle& o) {
  const int dim = o.dim;
  const bool thr = o.cfg.nthreads > 1;
  const int64_t np = (int64_t)o.particles.size();
#pragma omp parallel for schedule(static) if (thr)
  for (int64_t p = 0; p < np; ++p) {
    Particle& P = o.particles[p];
    const Cell& c = o.cells[P.cell];
    double M[9];
    const bool mapped = mapping_velocity_matrix(o, P, M);
    for (int i = 0; i < o.nv; ++i) {
      Node& n = o.nodes[c.nodes[i]];
      const double mN = P.mass * P.N[i];
      double mv[3];
      for (int d = 0; d < dim; ++d) mv[d] = P.v[d];
      if (mapped) {
        double r[3];
        for (int d = 0; d < dim; ++d) r[d] = n.coord[d] - P.x[d];
        for (int a = 0; a < dim; ++a) {
          double s = M[a * dim + 0] * r[0];
          for (int b = 1; b < dim; ++b) s = s + M[a * dim + b] * r[b];
          mv[a] += s;
        }
      }
      double mom[3];
      for (int d = 0; d < dim; ++d) mom[d] = mN * mv[d];
      node_add(n, &n.mass, &mN, 1, thr);
      node_add(n, n.mom, mom, dim, thr);
    }
  }
}

// mpm_scheme.tcc:66-70 compute_velocity on active nodes
void phase_compute_velocity(Oracle& o) {
  const int64_t nn = (int64_t)o.nodes.size();
#pragma omp parallel for schedule(static) if (o.cfg.nthreads > 1)
  for (int64_t i = 0; i < nn; ++i)
    if (o.nodes[i].status) node_compute_velocity(o, o.nodes[i]);
}

// particle.tcc:893-898 map_body_force
void phase_body_force(Oracle& o, const double* g) {
  const int dim = o.dim;
  const bool thr = o.cfg.nthreads > 1;
  const int64_t np = (int64_t)o.particles.size();
#pragma omp parallel for schedule(static) if (thr)
  for (int64_t p = 0; p < np; ++p) {
    Particle& P = o.particles[p];
    const Cell& c = o.cells[P.cell];
    for (int i = 0; i < o.nv; ++i) {
      Node& n = o.nodes[c.nodes[i]];
      double fb[3];
      for (int d = 0; d < dim; ++d) fb[d] = (g[d] * P.mass) * P.N[i];
      node_add(n, n.fext, fb, dim, thr);
    }
  }
}

// particle.tcc:915-949 map_internal_force
void phase_internal_force(Oracle& o) {
  const int dim = o.dim;
  const bool thr = o.cfg.nthreads > 1;
  const int64_t np = (int64_t)o.particles.size();
#pragma omp parallel for schedule(static) if (thr)
  for (int64_t p = 0; p < np; ++p) {
    Particle& P = o.particles[p];
    const Cell& c = o.cells[P.cell];
    const double* s = P.sig;
    for (int i = 0; i < o.nv; ++i) {
      Node& n = o.nodes[c.nodes[i]];
      const double* D = &P.dndx[i * dim];
      double f[3];
      if (dim == 2) {
        f[0] = D[0] * s[0] + D[1] * s[3];
        f[1] = D[1] * s[1] + D[0] * s[3];
      } else {
        f[0] = D[0] * s[0] + D[1] * s[3] + D[2] * s[5];
        f[1] = D[1] * s[1] + D[0] * s[3] + D[2] * s[4];
        f[2] = D[2] * s[2] + D[1] * s[4] + D[0] * s[5];
      }
      const double sc = -1. * P.vol;
      for (int d = 0; d < dim; ++d) f[d] *= sc;
      node_add(n, n.fint, f, dim, thr);
    }
  }
}

// mpm_scheme.tcc:222-233 node update on active nodes
void phase_node_update(Oracle& o, double dt) {
  const int64_t nn = (int64_t)o.nodes.size();
#pragma omp parallel for schedule(static) if (o.cfg.nthreads > 1)
  for (int64_t i = 0; i < nn; ++i)
    if (o.nodes[i].status)
      node_compute_acceleration_velocity_cundall(o, o.nodes[i], dt, o.cfg.damping_factor);
}

// |B_ij| < 1e-15 set to 0 (particle.tcc:1671-1676, 1700-1704)
void clean_small(int dim, double* B) {
  for (int i = 0; i < dim * dim; ++i)
    if (std::fabs(B[i]) < 1.E-15) B[i] = 0.;
}

// particle.tcc:1711-1730 ASFLIP beta: 0 next to a velocity-constrained node
// or when the deformation gradient increment compresses (det < 1)
double asflip_beta(const Oracle& o, const Particle& P, double dt) {
  const Cell& c = o.cells[P.cell];
  for (int i = 0; i < o.nv; ++i)
    if (!o.nodes[c.nodes[i]].vel_c.empty()) return 0.0;
  Particle Q = P;
  update_deformation_gradient_increment(o, Q, dt);
  const double* F = Q.Finc;
  const double J = F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
                   F[2] * (F[3] * F[7] - F[4] * F[6]);
  return J < 1.0 ? 0.0 : 1.0;
}

// particle.tcc:994-1139 FLIP / PIC / ASFLIP / APIC / TPIC position and
// velocity update, mesh.tcc:1454-1467 velocity constraints
void phase_g2p(Oracle& o, double dt) {
  const int dim = o.dim, vu = o.cfg.velocity_update;
  const int64_t np = (int64_t)o.particles.size();
  const double beta = o.cfg.blending_ratio;
#pragma omp parallel for schedule(static) if (o.cfg.nthreads > 1)
  for (int64_t p = 0; p < np; ++p) {
    Particle& P = o.particles[p];
    const Cell& c = o.cells[P.cell];
    double nvel[3] = {0, 0, 0}, nacc[3] = {0, 0, 0};
    const bool with_acc = vu == 0 || vu == 2;
    for (int i = 0; i < o.nv; ++i) {
      const Node& n = o.nodes[c.nodes[i]];
      for (int d = 0; d < dim; ++d) nvel[d] += P.N[i] * n.vel[d];
      if (with_acc)
        for (int d = 0; d < dim; ++d) nacc[d] += P.N[i] * n.acc[d];
    }
    if (vu == 2 || vu == 4) {  // compute_affine_mapping_matrix, at the step-start position
      double B[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int i = 0; i < o.nv; ++i) {
        const Node& n = o.nodes[c.nodes[i]];
        for (int a = 0; a < dim; ++a)
          for (int b = 0; b < dim; ++b) B[a * dim + b] += (P.N[i] * n.vel[a]) * (n.coord[b] - P.x[b]);
      }
      clean_small(dim, B);
      for (int i = 0; i < 9; ++i) P.B[i] = B[i];
    }
    if (vu == 3) {  // compute_velocity_gradient
      double B[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int i = 0; i < o.nv; ++i) {
        const Node& n = o.nodes[c.nodes[i]];
        for (int a = 0; a < dim; ++a)
          for (int b = 0; b < dim; ++b) B[a * dim + b] += n.vel[a] * P.dndx[i * dim + b];
      }
      clean_small(dim, B);
      for (int i = 0; i < 9; ++i) P.B[i] = B[i];
    }
    if (vu == 2) {
      const double bp = asflip_beta(o, P, dt);
      double flip[3], sep[3];
      for (int d = 0; d < dim; ++d) flip[d] = P.v[d] + nacc[d] * dt;
      for (int d = 0; d < dim; ++d) P.v[d] = beta * flip[d] + (1.0 - beta) * nvel[d];
      for (int d = 0; d < dim; ++d) sep[d] = bp * beta * flip[d] + (1.0 - bp * beta) * nvel[d];
      for (int d = 0; d < dim; ++d) P.x[d] += sep[d] * dt;
      for (int d = 0; d < dim; ++d) P.u[d] += sep[d] * dt;
    } else {
      if (vu == 0) {
        for (int d = 0; d < dim; ++d) P.v[d] += nacc[d] * dt;
        for (int d = 0; d < dim; ++d) P.v[d] = beta * P.v[d] + (1.0 - beta) * nvel[d];
      } else {
        for (int d = 0; d < dim; ++d) P.v[d] = nvel[d];
      }
      for (int d = 0; d < dim; ++d) P.x[d] += nvel[d] * dt;
      for (int d = 0; d < dim; ++d) P.u[d] += nvel[d] * dt;
    }
    for (const auto& pc : P.pvc) P.v[pc.first] = pc.second;
  }
}

void current_gravity(const Oracle& o, double* g) {  // mpm_explicit.tcc:145-153
  double gmul = 1.0;
  if (o.cfg.gravity_ramping_time > 0.0)
    gmul = std::min(1.0, static_cast<double>(o.step) * o.cfg.dt / o.cfg.gravity_ramping_time);
  for (int i = 0; i < 3; ++i) g[i] = i < o.dim ? gmul * o.cfg.gravity[i] : 0.;
}

// mpm_explicit.tcc:128-179 one step (USF / USL)
void one_step(Oracle& o) {
  const double dt = o.cfg.dt;
  phase_initialise(o);
  phase_p2g_mass_momentum(o);
  phase_compute_velocity(o);
  if (o.cfg.scheme == 0) compute_stress_strain(o, dt);  // mpm_scheme_usf.tcc:9-12
  double g[3];
  current_gravity(o, g);
  phase_body_force(o, g);
  phase_internal_force(o);
  phase_node_update(o, dt);
  phase_g2p(o, dt);
  if (o.cfg.scheme == 1) compute_stress_strain(o, dt);  // mpm_scheme_usl.tcc:14-17
  if (o.cfg.scheme == 2) {
    // mpm_scheme_musl.tcc:20-35: mass and momentum of the active nodes set to
    // zero and mapped again with the updated particle velocities (the
    // particles keep the shape functions of the step start), nodal velocity,
    // then the stress update on it (mpm_scheme_musl.tcc:13-17)
    for (auto& n : o.nodes)
      if (n.status) {
        n.mass = 0;
        for (int d = 0; d < 3; ++d) n.mom[d] = 0;
      }
    phase_p2g_mass_momentum(o);
    phase_compute_velocity(o);
    compute_stress_strain(o, dt);
  }
}

}  // namespace

extern "C" {

void* mpmo_create(const mpmo_config* cfg) {
  if (!cfg || (cfg->dim != 2 && cfg->dim != 3)) return nullptr;
  Oracle* o = new Oracle();
  o->cfg = *cfg;
  o->dim = cfg->dim;
  o->nv = cfg->dim == 2 ? 4 : 8;
#ifdef _OPENMP
  if (cfg->nthreads > 0) omp_set_num_threads(cfg->nthreads);
#endif
  return o;
}

void mpmo_destroy(void* h) {
  Oracle* o = (Oracle*)h;
  if (!o) return;
#ifdef _OPENMP
  for (auto& n : o->nodes) omp_destroy_lock(&n.lock);
#endif
  delete o;
}

const char* mpmo_last_error(void* h) { return h ? ((Oracle*)h)->err.c_str() : "null handle"; }

// mesh.tcc:17-48 (create_nodes), :211-256 (create_cells), :287-306 (neighbours)
int mpmo_set_mesh(void* h, int64_t nnodes, const double* coords, int64_t ncells,
                  int32_t nv, const int64_t* cell_nodes) {
  Oracle& o = *(Oracle*)h;
  if (nv != o.nv) { o.err = "nodes_per_cell does not match dimension"; return -1; }
  o.nodes.assign(nnodes, Node());
  for (int64_t i = 0; i < nnodes; ++i) {
    Node& n = o.nodes[i];
    for (int d = 0; d < 3; ++d) n.coord[d] = d < o.dim ? coords[i * o.dim + d] : 0.;
#ifdef _OPENMP
    omp_init_lock(&n.lock);
#endif
  }
  o.cells.assign(ncells, Cell());
  std::vector<std::set<int64_t>> node_cells(nnodes);
  for (int64_t c = 0; c < ncells; ++c) {
    Cell& cc = o.cells[c];
    for (int i = 0; i < nv; ++i) {
      const int64_t nid = cell_nodes[c * nv + i];
      if (nid < 0 || nid >= nnodes) { o.err = "cell node id out of range"; return -1; }
      cc.nodes[i] = nid;
      for (int d = 0; d < o.dim; ++d) cc.X[i * o.dim + d] = coords[nid * o.dim + d];
      node_cells[nid].insert(c);
    }
    cell_initialise(o, cc);
  }
  for (int64_t c = 0; c < ncells; ++c) {
    std::set<int64_t> nb;
    for (int i = 0; i < nv; ++i)
      for (int64_t other : node_cells[o.cells[c].nodes[i]])
        if (other != c) nb.insert(other);
    o.cells[c].neighbours.assign(nb.begin(), nb.end());
  }
  build_bins(o);
  return 0;
}

int mpmo_add_material(void* h, int32_t id, int32_t type, const double* params, int32_t np) {
  Oracle& o = *(Oracle*)h;
  Material m;
  if (!make_material(id, type, params, np, &m, &o.err)) return -1;
  o.material_index[id] = (int)o.materials.size();
  o.materials.push_back(m);
  return 0;
}

// node.tcc:349-366: a direction already constrained keeps its first value
int mpmo_add_velocity_constraints(void* h, int64_t n, const int64_t* nid,
                                  const int32_t* dir, const double* val) {
  Oracle& o = *(Oracle*)h;
  for (int64_t i = 0; i < n; ++i) {
    if (nid[i] < 0 || nid[i] >= (int64_t)o.nodes.size() || dir[i] < 0 || dir[i] >= o.dim) {
      o.err = "bad velocity constraint";
      return -1;
    }
    o.nodes[nid[i]].vel_c.insert(std::make_pair((unsigned)dir[i], val[i]));
  }
  return 0;
}

int mpmo_add_acceleration_constraints(void* h, int64_t n, const int64_t* nid,
                                      const int32_t* dir, const double* val) {
  Oracle& o = *(Oracle*)h;
  for (int64_t i = 0; i < n; ++i) {
    if (nid[i] < 0 || nid[i] >= (int64_t)o.nodes.size() || dir[i] < 0 || dir[i] >= o.dim) {
      o.err = "bad acceleration constraint";
      return -1;
    }
    o.nodes[nid[i]].acc_c.insert(std::make_pair((unsigned)dir[i], val[i]));
  }
  return 0;
}

// node.tcc:489-505: the last friction constraint assigned to a node wins
int mpmo_add_friction_constraints(void* h, int64_t n, const int64_t* nid, const int32_t* dir,
                                  const int32_t* sign_n, const double* mu) {
  Oracle& o = *(Oracle*)h;
  for (int64_t i = 0; i < n; ++i) {
    if (nid[i] < 0 || nid[i] >= (int64_t)o.nodes.size() || dir[i] < 0 || dir[i] >= o.dim) {
      o.err = "bad friction constraint";
      return -1;
    }
    Node& nd = o.nodes[nid[i]];
    nd.friction = true;
    nd.fdir = (unsigned)dir[i];
    nd.fsign = sign_n[i];
    nd.mu = mu[i];
  }
  return 0;
}

int mpmo_set_nodal_euler_angles(void* h, int64_t n, const int64_t* nid, const double* angles) {
  Oracle& o = *(Oracle*)h;
  const int dim = o.dim;
  for (int64_t i = 0; i < n; ++i) {
    if (nid[i] < 0 || nid[i] >= (int64_t)o.nodes.size()) return -1;
    Node& nd = o.nodes[nid[i]];
    const double* a = angles + i * dim;
    // mesh.tcc:1318-1345 rotation_matrix: 2D the rotation by a0 + a1 written
    // through the angle products, 3D Rz(a0) Rx(a2) Rz(a1)
    const double c0 = std::cos(a[0]), s0 = std::sin(a[0]), c1 = std::cos(a[1]), s1 = std::sin(a[1]);
    double R[9];
    if (dim == 2) {
      R[0] = c0 * c1 - s0 * s1;
      R[1] = -(c0 * s1) - s0 * c1;
      R[2] = s0 * c1 + c0 * s1;
      R[3] = -(s0 * s1) + c0 * c1;
    } else {
      const double c2 = std::cos(a[2]), s2 = std::sin(a[2]);
      R[0] = c0 * c1 - (s0 * s1) * c2;
      R[1] = -(c0 * s1) - (s0 * c1) * c2;
      R[2] = s0 * s2;
      R[3] = s0 * c1 + (c0 * s1) * c2;
      R[4] = -(s0 * s1) + (c0 * c1) * c2;
      R[5] = -(c0 * s2);
      R[6] = s1 * s2;
      R[7] = c1 * s2;
      R[8] = c2;
    }
    for (int k = 0; k < dim * dim; ++k) nd.R[k] = R[k];
    inverse(dim, nd.R, nd.Ri);
    nd.rotated = true;
  }
  return 0;
}

int mpmo_add_particle_velocity_constraint(void* h, int64_t n, const int64_t* pids,
                                          int32_t dir, double velocity) {
  Oracle& o = *(Oracle*)h;
  if (dir < 0 || dir >= o.dim) { o.err = "bad particle velocity constraint"; return -1; }
  if (n < 0) {
    for (auto& P : o.particles) P.pvc.emplace_back((unsigned)dir, velocity);
    return 0;
  }
  for (int64_t i = 0; i < n; ++i) {
    if (pids[i] < 0 || pids[i] >= (int64_t)o.particles.size()) {
      o.err = "bad particle id";
      return -1;
    }
    o.particles[pids[i]].pvc.emplace_back((unsigned)dir, velocity);
  }
  return 0;
}

// mesh.tcc:2114-2148 read_particles_file -> create_particles; particle.cc ctor
int mpmo_add_particles(void* h, int64_t n, const double* coords, int32_t material_id) {
  Oracle& o = *(Oracle*)h;
  auto it = o.material_index.find(material_id);
  if (it == o.material_index.end()) { o.err = "unknown material id"; return -1; }
  const Material& m = o.materials[it->second];
  for (int64_t i = 0; i < n; ++i) {
    Particle P{};
    P.id = (int64_t)o.particles.size();
    for (int d = 0; d < o.dim; ++d) P.x[d] = coords[i * o.dim + d];
    P.F[0] = P.F[4] = P.F[8] = 1.;
    P.Finc[0] = P.Finc[4] = P.Finc[8] = 1.;
    P.cell = kNone;
    P.mat = it->second;
    P.status = 1;
    if (m.type == 1) mc_initialise_state(m, P.sv);
    o.particles.push_back(P);
  }
  return 0;
}

// mpm_base.tcc:347-473 (locate, compute_volume), particle.tcc:557-626,
// mpm_explicit.tcc:94-95 (compute_mass), mpm_base.tcc:834-836 (acceleration)
int mpmo_initialise(void* h) {
  Oracle& o = *(Oracle*)h;
  for (auto& P : o.particles) {
    if (!locate_particle(o, P)) {
      o.err = "Particle outside the mesh domain";
      return -2;
    }
  }
  for (auto& P : o.particles) {
    const Cell& c = o.cells[P.cell];
    P.vol = c.volume / (double)c.particles.size();
    const Material& m = o.materials[P.mat];
    P.rho = m.density;
    P.mass = P.vol * P.rho;
    double gmul = 1.0;
    if (o.cfg.gravity_ramping_time > 0.0)
      gmul = std::min(1.0, 0.0 * o.cfg.dt / o.cfg.gravity_ramping_time);
    for (int d = 0; d < o.dim; ++d) P.a[d] = gmul * o.cfg.gravity[d];
  }
  return 0;
}

int mpmo_set_particles(void* h, const mpmo_particles* in) {
  Oracle& o = *(Oracle*)h;
  const int dim = o.dim;
  for (auto& c : o.cells) c.particles.clear();
  for (size_t p = 0; p < o.particles.size(); ++p) {
    Particle& P = o.particles[p];
    for (int d = 0; d < dim; ++d) {
      if (in->x) P.x[d] = in->x[p * 3 + d];
      if (in->u) P.u[d] = in->u[p * 3 + d];
      if (in->v) P.v[d] = in->v[p * 3 + d];
      if (in->a) P.a[d] = in->a[p * 3 + d];
      if (in->xi) P.xi[d] = in->xi[p * 3 + d];
    }
    for (int i = 0; i < 6; ++i) {
      if (in->stress) P.sig[i] = in->stress[p * 6 + i];
      if (in->strain) P.eps[i] = in->strain[p * 6 + i];
    }
    if (in->F)
      for (int i = 0; i < 9; ++i) P.F[i] = in->F[p * 9 + i];
    if (in->volume) P.vol = in->volume[p];
    if (in->mass) P.mass = in->mass[p];
    if (in->density) P.rho = in->density[p];
    if (in->svars)
      for (int i = 0; i < 9; ++i) P.sv[i] = in->svars[p * 9 + i];
    if (in->mapping)
      for (int a = 0; a < dim; ++a)
        for (int b = 0; b < dim; ++b) P.B[a * dim + b] = in->mapping[p * 9 + a * 3 + b];
    if (in->cell) P.cell = in->cell[p];
    if (P.cell != kNone) o.cells[P.cell].particles.push_back(P.id);
  }
  return 0;
}

int64_t mpmo_nparticles(void* h) { return (int64_t)((Oracle*)h)->particles.size(); }

int mpmo_get_particles(void* h, mpmo_particles* out) {
  Oracle& o = *(Oracle*)h;
  for (size_t p = 0; p < o.particles.size(); ++p) {
    const Particle& P = o.particles[p];
    for (int d = 0; d < 3; ++d) {
      const bool in = d < o.dim;
      if (out->x) out->x[p * 3 + d] = in ? P.x[d] : 0.;
      if (out->u) out->u[p * 3 + d] = in ? P.u[d] : 0.;
      if (out->v) out->v[p * 3 + d] = in ? P.v[d] : 0.;
      if (out->a) out->a[p * 3 + d] = in ? P.a[d] : 0.;
      if (out->xi) out->xi[p * 3 + d] = in ? P.xi[d] : 0.;
    }
    for (int i = 0; i < 6; ++i) {
      if (out->stress) out->stress[p * 6 + i] = P.sig[i];
      if (out->strain) out->strain[p * 6 + i] = P.eps[i];
      if (out->dstrain) out->dstrain[p * 6 + i] = P.deps[i];
      if (out->strain_rate) out->strain_rate[p * 6 + i] = P.eps_rate[i];
    }
    if (out->F)
      for (int i = 0; i < 9; ++i) out->F[p * 9 + i] = P.F[i];
    if (out->volume) out->volume[p] = P.vol;
    if (out->mass) out->mass[p] = P.mass;
    if (out->density) out->density[p] = P.rho;
    if (out->cell) out->cell[p] = P.cell == kNone ? -1 : P.cell;
    if (out->material) out->material[p] = o.materials[P.mat].id;
    if (out->svars)
      for (int i = 0; i < 9; ++i) out->svars[p * 9 + i] = P.sv[i];
    if (out->status) out->status[p] = P.status;
    if (out->mapping)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
          out->mapping[p * 9 + a * 3 + b] = (a < o.dim && b < o.dim) ? P.B[a * o.dim + b] : 0.;
  }
  return 0;
}

// mpm_explicit.tcc:112-190 step loop; mpm_scheme.tcc:245-261 locate
int mpmo_step(void* h, int64_t nsteps) {
  Oracle& o = *(Oracle*)h;
  for (int64_t s = 0; s < nsteps; ++s) {
    one_step(o);
    std::vector<int64_t> lost;
    for (auto& P : o.particles)
      if (!locate_particle(o, P)) lost.push_back(P.id);
    if (!lost.empty()) {
      if (o.cfg.locate_particles) {
        o.err = "Particle(s) outside the mesh domain: " + std::to_string(lost.size());
        return -2;
      }
      // mpm_scheme.tcc:258-260 remove_particle
      std::vector<Particle> keep;
      std::set<int64_t> drop(lost.begin(), lost.end());
      for (auto& P : o.particles)
        if (!drop.count(P.id)) keep.push_back(P);
      for (auto& c : o.cells) {
        auto& lst = c.particles;
        lst.erase(std::remove_if(lst.begin(), lst.end(), [&](int64_t id) { return drop.count(id) > 0; }),
                  lst.end());
      }
      o.particles.swap(keep);
    }
    ++o.step;
  }
  return 0;
}

int mpmo_get_nodes(void* h, double* out) {
  Oracle& o = *(Oracle*)h;
  for (size_t i = 0; i < o.nodes.size(); ++i) {
    const Node& n = o.nodes[i];
    double* r = out + i * 17;
    r[0] = n.mass;
    for (int d = 0; d < 3; ++d) {
      r[1 + d] = n.mom[d];
      r[4 + d] = n.fext[d];
      r[7 + d] = n.fint[d];
      r[10 + d] = n.vel[d];
      r[13 + d] = n.acc[d];
    }
    r[16] = n.status ? 1. : 0.;
  }
  return 0;
}

int mpmo_set_nodes(void* h, const double* in) {
  Oracle& o = *(Oracle*)h;
  for (size_t i = 0; i < o.nodes.size(); ++i) {
    Node& n = o.nodes[i];
    const double* r = in + i * 17;
    n.mass = r[0];
    for (int d = 0; d < 3; ++d) {
      n.mom[d] = r[1 + d];
      n.fext[d] = r[4 + d];
      n.fint[d] = r[7 + d];
      n.vel[d] = r[10 + d];
      n.acc[d] = r[13 + d];
    }
    n.status = r[16] != 0.;
  }
  return 0;
}

int mpmo_phase(void* h, int32_t phase, double dt, const double* gravity) {
  Oracle& o = *(Oracle*)h;
  switch (phase) {
    case 0: phase_initialise(o); break;
    case 1: phase_p2g_mass_momentum(o); break;
    case 2: phase_compute_velocity(o); break;
    case 3: compute_stress_strain(o, dt); break;
    case 4: phase_body_force(o, gravity); break;
    case 5: phase_internal_force(o); break;
    case 6: phase_node_update(o, dt); break;
    case 7: phase_g2p(o, dt); break;
    case 8:
      for (auto& P : o.particles)
        if (!locate_particle(o, P)) return -2;
      break;
    default: o.err = "unknown phase"; return -1;
  }
  return 0;
}

int mpmo_element_dn_dx(int32_t dim, const double* xi, const double* X, double* N,
                       double* grad, double* dndx) {
  if (dim != 2 && dim != 3) return -1;
  shapefn(dim, xi, N);
  double G[8 * 3];
  dn_dx(dim, xi, X, G, dndx);
  if (grad) std::memcpy(grad, G, sizeof(double) * (dim == 2 ? 8 : 24));
  return 0;
}

int mpmo_material_stress(int32_t dim, int32_t type, const double* params, int32_t np,
                         const double* stress, const double* dstrain, double density,
                         double* state, double* out) {
  (void)dim;
  Material m;
  std::string err;
  if (!make_material(0, type, params, np, &m, &err)) return -1;
  material_compute_stress(m, stress, dstrain, density, state, out);
  return 0;
}

int mpmo_mc_diagnostics(int32_t dim, const double* params, int32_t np, const double* stress,
                        double* state, double* out) {
  (void)dim;
  Material m;
  std::string err;
  if (!make_material(0, 1, params, np, &m, &err)) return -1;
  mc_invariants(stress, state);
  double yf[2];
  const int yt = mc_yield_state(yf, state);
  double df[6], dp[6], dp_dq = 0, soft = 0;
  mc_df_dp(m, yt, state, stress, df, dp, &dp_dq, &soft);
  out[0] = state[SV_EPS];
  out[1] = state[SV_RHO];
  out[2] = state[SV_THETA];
  out[3] = yf[0];
  out[4] = yf[1];
  out[5] = yt;
  for (int i = 0; i < 6; ++i) {
    out[6 + i] = df[i];
    out[12 + i] = dp[i];
  }
  out[18] = dp_dq;
  out[19] = soft;
  return 0;
}

}  // extern "C"
