// mpm_math.cuh -- per-particle and per-node arithmetic of the explicit MPM
// step, written for the device (and usable on the host for set-up).
//
// The arithmetic follows the reference solver (geomechanics/mpm) operation by
// operation so that the FP64 path agrees with it to rounding: sums run in the
// reference's loop order, 2x2/3x3 inverses are adjugate / determinant as in
// Eigen's fixed-size inverse, and the FP64 translation unit is compiled with
// --fmad=false so no multiply-add is fused.  File:line citations are relative
// to the reference source tree.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define MPM_HD __host__ __device__ __forceinline__
#define MPM_HD_OUTLINE __host__ __device__ __noinline__
#else
#define MPM_HD inline
#define MPM_HD_OUTLINE inline
#endif

namespace mpm_b200 {

constexpr double kDblEps = 2.220446049250313080847e-16;  // numeric_limits<double>::epsilon
constexpr double kPiD = 3.14159265358979323846;           // M_PI

template <int DIM>
struct Elem;
template <>
struct Elem<2> {
  static constexpr int NV = 4;
};
template <>
struct Elem<3> {
  static constexpr int NV = 8;
};

// ------------------------------------------------------------ shape functions
// quadrilateral_element.tcc:11-22, hexahedron_element.tcc:19-34
template <int DIM, typename R>
MPM_HD void shapefn(const R* xi, R* N) {
  if constexpr (DIM == 2) {
    N[0] = R(0.25) * (1 - xi[0]) * (1 - xi[1]);
    N[1] = R(0.25) * (1 + xi[0]) * (1 - xi[1]);
    N[2] = R(0.25) * (1 + xi[0]) * (1 + xi[1]);
    N[3] = R(0.25) * (1 - xi[0]) * (1 + xi[1]);
  } else {
    N[0] = R(0.125) * (1 - xi[0]) * (1 - xi[1]) * (1 - xi[2]);
    N[1] = R(0.125) * (1 + xi[0]) * (1 - xi[1]) * (1 - xi[2]);
    N[2] = R(0.125) * (1 + xi[0]) * (1 + xi[1]) * (1 - xi[2]);
    N[3] = R(0.125) * (1 - xi[0]) * (1 + xi[1]) * (1 - xi[2]);
    N[4] = R(0.125) * (1 - xi[0]) * (1 - xi[1]) * (1 + xi[2]);
    N[5] = R(0.125) * (1 + xi[0]) * (1 - xi[1]) * (1 + xi[2]);
    N[6] = R(0.125) * (1 + xi[0]) * (1 + xi[1]) * (1 + xi[2]);
    N[7] = R(0.125) * (1 - xi[0]) * (1 + xi[1]) * (1 + xi[2]);
  }
}

// Gradient in natural coordinates, G[n*DIM + k] = dN_n / dxi_k
// quadrilateral_element.tcc:26-43, hexahedron_element.tcc:38-74
template <int DIM, typename R>
MPM_HD void grad_shapefn(const R* xi, R* G) {
  if constexpr (DIM == 2) {
    G[0] = R(-0.25) * (1 - xi[1]);
    G[2] = R(0.25) * (1 - xi[1]);
    G[4] = R(0.25) * (1 + xi[1]);
    G[6] = R(-0.25) * (1 + xi[1]);
    G[1] = R(-0.25) * (1 - xi[0]);
    G[3] = R(-0.25) * (1 + xi[0]);
    G[5] = R(0.25) * (1 + xi[0]);
    G[7] = R(0.25) * (1 - xi[0]);
  } else {
    G[0 * 3 + 0] = R(-0.125) * (1 - xi[1]) * (1 - xi[2]);
    G[1 * 3 + 0] = R(0.125) * (1 - xi[1]) * (1 - xi[2]);
    G[2 * 3 + 0] = R(0.125) * (1 + xi[1]) * (1 - xi[2]);
    G[3 * 3 + 0] = R(-0.125) * (1 + xi[1]) * (1 - xi[2]);
    G[4 * 3 + 0] = R(-0.125) * (1 - xi[1]) * (1 + xi[2]);
    G[5 * 3 + 0] = R(0.125) * (1 - xi[1]) * (1 + xi[2]);
    G[6 * 3 + 0] = R(0.125) * (1 + xi[1]) * (1 + xi[2]);
    G[7 * 3 + 0] = R(-0.125) * (1 + xi[1]) * (1 + xi[2]);
    G[0 * 3 + 1] = R(-0.125) * (1 - xi[0]) * (1 - xi[2]);
    G[1 * 3 + 1] = R(-0.125) * (1 + xi[0]) * (1 - xi[2]);
    G[2 * 3 + 1] = R(0.125) * (1 + xi[0]) * (1 - xi[2]);
    G[3 * 3 + 1] = R(0.125) * (1 - xi[0]) * (1 - xi[2]);
    G[4 * 3 + 1] = R(-0.125) * (1 - xi[0]) * (1 + xi[2]);
    G[5 * 3 + 1] = R(-0.125) * (1 + xi[0]) * (1 + xi[2]);
    G[6 * 3 + 1] = R(0.125) * (1 + xi[0]) * (1 + xi[2]);
    G[7 * 3 + 1] = R(0.125) * (1 - xi[0]) * (1 + xi[2]);
    G[0 * 3 + 2] = R(-0.125) * (1 - xi[0]) * (1 - xi[1]);
    G[1 * 3 + 2] = R(-0.125) * (1 + xi[0]) * (1 - xi[1]);
    G[2 * 3 + 2] = R(-0.125) * (1 + xi[0]) * (1 + xi[1]);
    G[3 * 3 + 2] = R(-0.125) * (1 - xi[0]) * (1 + xi[1]);
    G[4 * 3 + 2] = R(0.125) * (1 - xi[0]) * (1 - xi[1]);
    G[5 * 3 + 2] = R(0.125) * (1 + xi[0]) * (1 - xi[1]);
    G[6 * 3 + 2] = R(0.125) * (1 + xi[0]) * (1 + xi[1]);
    G[7 * 3 + 2] = R(0.125) * (1 - xi[0]) * (1 + xi[1]);
  }
}

// inverse by adjugate / determinant (Eigen fixed-size 2x2 / 3x3 inverse)
template <int DIM, typename R>
MPM_HD void inverse(const R* J, R* inv) {
  if constexpr (DIM == 2) {
    const R det = J[0] * J[3] - J[2] * J[1];
    const R invdet = R(1) / det;
    inv[0] = J[3] * invdet;
    inv[2] = -J[2] * invdet;
    inv[1] = -J[1] * invdet;
    inv[3] = J[0] * invdet;
  } else {
#define MPM_COF(i, j)                                                    \
  (J[(((i) + 1) % 3) * 3 + (((j) + 1) % 3)] * J[(((i) + 2) % 3) * 3 + (((j) + 2) % 3)] - \
   J[(((i) + 1) % 3) * 3 + (((j) + 2) % 3)] * J[(((i) + 2) % 3) * 3 + (((j) + 1) % 3)])
    const R c0 = MPM_COF(0, 0), c1 = MPM_COF(1, 0), c2 = MPM_COF(2, 0);
    const R det = (c0 * J[0] + c1 * J[3]) + c2 * J[6];
    const R invdet = R(1) / det;
    inv[0] = c0 * invdet;
    inv[1] = c1 * invdet;
    inv[2] = c2 * invdet;
    inv[3] = MPM_COF(0, 1) * invdet;
    inv[4] = MPM_COF(1, 1) * invdet;
    inv[5] = MPM_COF(2, 1) * invdet;
    inv[6] = MPM_COF(0, 2) * invdet;
    inv[7] = MPM_COF(1, 2) * invdet;
    inv[8] = MPM_COF(2, 2) * invdet;
#undef MPM_COF
  }
}

// dN/dx = G inv(J)^T with J = G^T X (quadrilateral_element.tcc:295-309,
// hexahedron_element.tcc:307-321).  X[n*DIM + c] nodal coordinates.
template <int DIM, typename R>
MPM_HD void dn_dx(const R* xi, const R* X, R* D) {
  constexpr int NV = Elem<DIM>::NV;
  R G[NV * DIM];
  grad_shapefn<DIM>(xi, G);
  R J[DIM * DIM], inv[DIM * DIM];
#pragma unroll
  for (int r = 0; r < DIM; ++r)
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      R s = G[0 * DIM + r] * X[0 * DIM + c];
#pragma unroll
      for (int n = 1; n < NV; ++n) s = s + G[n * DIM + r] * X[n * DIM + c];
      J[r * DIM + c] = s;
    }
  inverse<DIM>(J, inv);
#pragma unroll
  for (int n = 0; n < NV; ++n)
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      R s = G[n * DIM + 0] * inv[c * DIM + 0];
#pragma unroll
      for (int k = 1; k < DIM; ++k) s = s + G[n * DIM + k] * inv[c * DIM + k];
      D[n * DIM + c] = s;
    }
}

// ------------------------------------------------------------------- location
// Per-cell geometry (cell.tcc:255-279 centroid and mean length; local
// coordinate lengths cell.tcc:458-463, 566-571), computed once on the host.
struct CellGeom {
  double centroid[3];
  double len[3];
  double mean_length;
};

// cell.tcc:324-384 with local_coordinates_point (isoparametric false).
// Returns true when the point is inside; xi is clamped to +-(1 - eps).
template <int DIM>
MPM_HD bool point_in_cell(const double* p, const double* centroid, const double* len,
                          double mean_length, double* xi) {
  double d[DIM];
#pragma unroll
  for (int i = 0; i < DIM; ++i) d[i] = p[i] - centroid[i];
  double s = d[0] * d[0];
#pragma unroll
  for (int i = 1; i < DIM; ++i) s = s + d[i] * d[i];
  const double length = sqrt(s);
  if (!(length < (mean_length * 2.))) return false;
  bool status = true;
#pragma unroll
  for (int i = 0; i < DIM; ++i) {
    double x = 2. * (p[i] - centroid[i]) / len[i];
    if (x < -1. || x > 1. || x != x) {
      status = false;
    } else {
      if (x < -1. + kDblEps) x = -1. + kDblEps;
      if (x > 1. - kDblEps) x = 1. - kDblEps;
    }
    xi[i] = x;
  }
  return status;
}

// Isoparametric local coordinates (cell.tcc:617-826 transform_real_to_unit_cell
// for quad4 / hex8): the xi with sum_i N_i(xi) X_i = p, by Newton iterations on
// the bilinear / trilinear map from the cell centre until the step is below
// 1e-12 (the next error is at rounding level; at most 50 iterations).  The
// reference tries an analytical (2D) or affine guess and Newton with a line
// search and keeps the smallest residual; every accepted solution is the same
// root to rounding for a convex cell.  False when the iteration did not
// converge or the point maps to a non-finite xi.
template <int DIM>
MPM_HD bool iso_local_xi(const double* p, const double* X, double* xi) {
  constexpr int NV = DIM == 2 ? 4 : 8;
#pragma unroll
  for (int d = 0; d < DIM; ++d) xi[d] = 0.;
  for (int it = 0; it < 50; ++it) {
    double N[NV], G[NV * DIM], r[DIM], Jm[DIM * DIM], Ji[DIM * DIM];
    shapefn<DIM>(xi, N);
    grad_shapefn<DIM>(xi, G);
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      double xa = N[0] * X[0 * DIM + a];
      for (int i = 1; i < NV; ++i) xa = xa + N[i] * X[i * DIM + a];
      r[a] = xa - p[a];
#pragma unroll
      for (int b = 0; b < DIM; ++b) {  // dx_a / dxi_b
        double j = X[0 * DIM + a] * G[0 * DIM + b];
        for (int i = 1; i < NV; ++i) j = j + X[i * DIM + a] * G[i * DIM + b];
        Jm[a * DIM + b] = j;
      }
    }
    inverse<DIM>(Jm, Ji);
    double step = 0.;
#pragma unroll
    for (int b = 0; b < DIM; ++b) {
      double dxi = Ji[b * DIM + 0] * r[0];
#pragma unroll
      for (int a = 1; a < DIM; ++a) dxi = dxi + Ji[b * DIM + a] * r[a];
      xi[b] -= dxi;
      step = step > fabs(dxi) ? step : fabs(dxi);
    }
    if (!(step == step)) return false;
    if (step < 1e-12) return true;  // quadratic convergence: xi now at rounding level
  }
  return false;
}

// cell.tcc:335-384 with transform_real_to_unit_cell (isoparametric true);
// X: the cell's nodal coordinates.
template <int DIM>
MPM_HD bool point_in_cell_iso(const double* p, const double* X, const double* centroid,
                              double mean_length, double* xi) {
  double d[DIM];
#pragma unroll
  for (int i = 0; i < DIM; ++i) d[i] = p[i] - centroid[i];
  double s = d[0] * d[0];
#pragma unroll
  for (int i = 1; i < DIM; ++i) s = s + d[i] * d[i];
  if (!(sqrt(s) < (mean_length * 2.))) return false;
  if (!iso_local_xi<DIM>(p, X, xi)) return false;
  bool status = true;
#pragma unroll
  for (int i = 0; i < DIM; ++i) {
    double x = xi[i];
    if (x < -1. || x > 1. || x != x) {
      status = false;
    } else {
      if (x < -1. + kDblEps) x = -1. + kDblEps;
      if (x > 1. - kDblEps) x = 1. - kDblEps;
    }
    xi[i] = x;
  }
  return status;
}

// xi of a particle in the cell it was last located in (bit-identical to the
// value the locate step stored: same formula, same inputs).
template <int DIM>
MPM_HD void local_xi(const double* p, const double* centroid, const double* len, double* xi) {
#pragma unroll
  for (int i = 0; i < DIM; ++i) {
    double x = 2. * (p[i] - centroid[i]) / len[i];
    if (x < -1. + kDblEps) x = -1. + kDblEps;
    if (x > 1. - kDblEps) x = 1. - kDblEps;
    xi[i] = x;
  }
}

// Index of the axis interval [a[i], a[i+1]] holding v (largest i with
// a[i] <= v, clamped to [0, ncell-1]); a has ncell+1 ascending entries.
MPM_HD int axis_interval(const double* a, int ncell, double v) {
  int lo = 0, hi = ncell;  // a[lo] <= v < a[hi] invariant on the clamped range
  if (!(v >= a[0])) return 0;
  if (v >= a[ncell]) return ncell - 1;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] <= v)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// The first cell in id order containing p on a tensor-product grid: the
// same answer as scanning every cell (a containing cell's box holds p up to
// rounding, so only the intervals around p's interval can contain it).
template <int DIM>
MPM_HD int structured_scan(const double* p, const int32_t* ncell, const double* const* axis,
                           const CellGeom* geom) {
  int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  for (int d = 0; d < DIM; ++d) {
    if (!(p[d] == p[d])) return -1;
    const int i = axis_interval(axis[d], ncell[d], p[d]);
    lo[d] = i > 0 ? i - 1 : 0;
    hi[d] = i + 1 < ncell[d] ? i + 1 : ncell[d] - 1;
  }
  for (int k = lo[2]; k <= hi[2]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[0]; i <= hi[0]; ++i) {
        const int c = DIM == 2 ? i + ncell[0] * j : i + ncell[0] * (j + ncell[1] * k);
        double xi[DIM];
        const CellGeom& g = geom[c];
        if (point_in_cell<DIM>(p, g.centroid, g.len, g.mean_length, xi)) return c;
      }
  return -1;
}

// ------------------------------------------------------------------ materials
// Material parameters in the working precision R (double on the FP64 path;
// float on the mixed path, converted once per material).
template <typename R>
struct MaterialT {
  int type;  // 0 LinearElastic, 1 MohrCoulomb
  int softening;
  R density, E, nu;
  R bulk, shear, a1, a2;  // elastic tensor entries (a1 diag, a2 off-diag, G shear)
  R phi_peak, psi_peak, c_peak, phi_res, psi_res, c_res;
  R pd_peak, pd_res, tension_cutoff;
  R grain_density, min_packing;
  R tc_init;  // initial tension cutoff state (mohr_coulomb.tcc:97-100)
  // sin, cos, tan of the peak friction angle and tan of the peak dilation
  // angle, computed once on the host (they enter every yield-function
  // evaluation; softening replaces them per point)
  R sin_phi, cos_phi, tan_phi, tan_psi;
};
using MaterialParams = MaterialT<double>;

template <typename R>
MPM_HD MaterialT<R> material_cast(const MaterialParams& m) {
  MaterialT<R> r;
  r.type = m.type;
  r.softening = m.softening;
  r.density = R(m.density);
  r.E = R(m.E);
  r.nu = R(m.nu);
  r.bulk = R(m.bulk);
  r.shear = R(m.shear);
  r.a1 = R(m.a1);
  r.a2 = R(m.a2);
  r.phi_peak = R(m.phi_peak);
  r.psi_peak = R(m.psi_peak);
  r.c_peak = R(m.c_peak);
  r.phi_res = R(m.phi_res);
  r.psi_res = R(m.psi_res);
  r.c_res = R(m.c_res);
  r.pd_peak = R(m.pd_peak);
  r.pd_res = R(m.pd_res);
  r.tension_cutoff = R(m.tension_cutoff);
  r.grain_density = R(m.grain_density);
  r.min_packing = R(m.min_packing);
  r.tc_init = R(m.tc_init);
  r.sin_phi = R(m.sin_phi);
  r.cos_phi = R(m.cos_phi);
  r.tan_phi = R(m.tan_phi);
  r.tan_psi = R(m.tan_psi);
  return r;
}

enum { SV_YIELD = 0, SV_PHI, SV_PSI, SV_COH, SV_TC, SV_EPS, SV_RHO, SV_THETA, SV_PD, SV_N };

template <typename R>
MPM_HD R check_low(R v) {  // mohr_coulomb.h:124
  return v > R(1.0e-15) ? v : R(1.0e-15);
}
template <typename R>
MPM_HD R dbl_eps() {  // numeric_limits<double>::epsilon, the reference's threshold
  return R(kDblEps);
}

// De * b for the isotropic elastic tensor, summed over k = 0..5 in order with
// the zero entries of the dense 6x6 skipped (they add exact zeros).
template <typename R>
MPM_HD void de_mul(const MaterialT<R>& m, const R* b, R* o) {
  const R a1 = m.a1, a2 = m.a2, G = m.shear;
  o[0] = (a1 * b[0] + a2 * b[1]) + a2 * b[2];
  o[1] = (a2 * b[0] + a1 * b[1]) + a2 * b[2];
  o[2] = (a2 * b[0] + a2 * b[1]) + a1 * b[2];
  o[3] = G * b[3];
  o[4] = G * b[4];
  o[5] = G * b[5];
}

// (a^T De) . b (mohr_coulomb.tcc:433,454-455)
template <typename R>
MPM_HD R row_de_dot(const MaterialT<R>& m, const R* a, const R* b) {
  const R a1 = m.a1, a2 = m.a2, G = m.shear;
  const R r0 = (a[0] * a1 + a[1] * a2) + a[2] * a2;
  const R r1 = (a[0] * a2 + a[1] * a1) + a[2] * a2;
  const R r2 = (a[0] * a2 + a[1] * a2) + a[2] * a1;
  const R r3 = a[3] * G, r4 = a[4] * G, r5 = a[5] * G;
  return ((((r0 * b[0] + r1 * b[1]) + r2 * b[2]) + r3 * b[3]) + r4 * b[4]) + r5 * b[5];
}

// updated += -((lambda * De) * v)  (mohr_coulomb.tcc:463,468,502)
template <typename R>
MPM_HD void sub_lambda_de(const MaterialT<R>& m, R lambda, const R* v, R* u) {
  const R l1 = lambda * m.a1, l2 = lambda * m.a2, lg = lambda * m.shear;
  u[0] += -((l1 * v[0] + l2 * v[1]) + l2 * v[2]);
  u[1] += -((l2 * v[0] + l1 * v[1]) + l2 * v[2]);
  u[2] += -((l2 * v[0] + l2 * v[1]) + l1 * v[2]);
  u[3] += -(lg * v[3]);
  u[4] += -(lg * v[4]);
  u[5] += -(lg * v[5]);
}

// material_utility.tcc:2-200
template <typename R>
MPM_HD R mu_p(const R* s) {
  return (R(1) / R(3) * (s[0] + s[1] + s[2]));
}
template <typename R>
MPM_HD R sq(R x) {
  return x * x;
}
template <typename R>
MPM_HD R mu_j2(const R* s) {
  return (sq(s[0] - s[1]) + sq(s[1] - s[2]) + sq(s[0] - s[2])) / R(6) + sq(s[3]) + sq(s[4]) +
         sq(s[5]);
}
template <typename R>
MPM_HD R mu_j3(const R* s) {
  const R p = mu_p(s);
  const R d0 = s[0] - p, d1 = s[1] - p, d2 = s[2] - p;
  return (d0 * d1 * d2) - (d2 * sq(s[3])) +
         ((R(2) * s[3] * s[4] * s[5]) - (d0 * sq(s[4])) - (d1 * sq(s[5])));
}

// The type the stress invariants are evaluated in for a working type R: FP64
// for FP32 and FP64 (see mc_invariants), the tangent type itself for tangents.
template <typename R>
struct HighPrecision {
  using T = double;
};

// Value-preserving hook for the tangent type: the identity for plain numbers.
// For tangents (mpm_dual.cuh) it drops the derivative of a Lode-angle quantity
// within a small distance of a triaxial corner of the yield surface, where
// the derivative of theta(sigma) is unbounded.
template <typename T>
MPM_HD T lode_corner(const T& x, double /*dist_to_corner*/) {
  return x;
}
MPM_HD double value(double x) { return x; }
MPM_HD float value(float x) { return x; }

// sin and cos of an FP64 angle in one evaluation
MPM_HD void sin_cos(double x, double* sn, double* cs) {
#ifdef __CUDA_ARCH__
  sincos(x, sn, cs);
#else
  *sn = std::sin(x);
  *cs = std::cos(x);
#endif
}

// Trigonometric values of the Lode angle theta of one invariant evaluation:
// cos, sin of theta, theta + pi/3 and theta - 4 pi/3 all follow from one
// sin/cos evaluation of theta by the angle-addition formulas.
template <typename R>
struct LodeTrig {
  R ct, st;    // cos theta, sin theta
  R sp3, cp3;  // sin (theta + pi/3), cos (theta + pi/3)
  R cm43;      // cos (theta - 4 pi/3)
};
// Friction and dilation angle functions of one return (fixed during a
// return: softening moves phi and psi only before the predictor).
template <typename R>
struct FrictionTrig {
  R sphi, cphi, tphi, tpsi;
};

template <typename R>
MPM_HD FrictionTrig<R> friction_trig(const MaterialT<R>& m, const R* sv) {
  FrictionTrig<R> t;
  if (sv[SV_PHI] == m.phi_peak && sv[SV_PSI] == m.psi_peak) {
    t.sphi = m.sin_phi;
    t.cphi = m.cos_phi;
    t.tphi = m.tan_phi;
    t.tpsi = m.tan_psi;
  } else {
    t.sphi = sin(sv[SV_PHI]);
    t.cphi = cos(sv[SV_PHI]);
    t.tphi = tan(sv[SV_PHI]);
    t.tpsi = tan(sv[SV_PSI]);
  }
  return t;
}

// mohr_coulomb.tcc:124-134 with lode_angle (material_utility.tcc:65-81).
// Evaluated in FP64 for every working precision R: the Lode angle is acos of
// a ratio that reaches +-1 on triaxial stress paths (a geostatic K0 state is
// one), where acos turns a rounding error e of the ratio into an angle error
// of about sqrt(2e) -- 5e-4 rad from FP32 rounding, which moves the returned
// stress by 1e-4 of its magnitude.
template <typename R>
MPM_HD void mc_invariants(const R* s, R* sv, LodeTrig<R>& lt) {
  using H = typename HighPrecision<R>::T;
  const H d[6] = {H(s[0]), H(s[1]), H(s[2]), H(s[3]), H(s[4]), H(s[5])};
  const H j2 = mu_j2(d);
  const H j3 = mu_j3(d);
  sv[SV_EPS] = R(mu_p(d) * sqrt(3.0));
  H v = H(0.0);
  if (fabs(j2) > kDblEps) v = (3.0 * sqrt(3.0) / 2.0) * (j3 / (j2 * sqrt(j2)));
  if (v > 1.0) v = H(1.0);
  if (v < -1.0) v = H(-1.0);
  const H theta = lode_corner((1.0 / 3.0) * acos(v), value(1.0 - v * v));
  sv[SV_THETA] = R(theta);
  sv[SV_RHO] = R(sqrt(2.0 * j2));
  H sn, cs;
  sin_cos(theta, &sn, &cs);
  const double h = 0.5, r3 = 0.86602540378443864676;  // cos, sin of pi/3
  lt.ct = R(cs);
  lt.st = R(sn);
  lt.sp3 = R(sn * h + cs * r3);
  lt.cp3 = R(cs * h - sn * r3);
  lt.cm43 = R(-(cs * h) - sn * r3);
}

enum { MC_ELASTIC = 0, MC_SHEAR = 1, MC_TENSILE = 2, MC_SEPARATED = 3 };

// mohr_coulomb.tcc:139-191
template <typename R>
MPM_HD int mc_yield_state(R* yf, const R* sv, const LodeTrig<R>& lt, const FrictionTrig<R>& ft) {
  const R Tolerance = R(-1E-1);
  const R epsilon = sv[SV_EPS], rho = sv[SV_RHO];
  const R cohesion = sv[SV_COH], tension_cutoff = sv[SV_TC];
  yf[0] = sqrt(R(2) / R(3)) * lt.ct * rho + epsilon / sqrt(R(3)) - tension_cutoff;
  yf[1] = sqrt(R(1.5)) * rho * ((lt.sp3 / (sqrt(R(3)) * ft.cphi)) + (lt.cp3 * ft.tphi / R(3))) +
          (epsilon / sqrt(R(3))) * ft.tphi - cohesion;
  int yield_type = MC_ELASTIC;
  if (yf[0] > Tolerance && yf[1] > Tolerance) {
    const R n_phi = (R(1) + ft.sphi) / (R(1) - ft.sphi);
    const R sigma_p = tension_cutoff * n_phi - R(2) * cohesion * sqrt(n_phi);
    const R alpha_p = sqrt(R(1) + n_phi * n_phi) + n_phi;
    const R h = yf[0] + alpha_p * (sqrt(R(2) / R(3)) * lt.cm43 * rho + epsilon / sqrt(R(3)) - sigma_p);
    yield_type = (h > dbl_eps<R>()) ? MC_TENSILE : MC_SHEAR;
  }
  if (yf[0] < Tolerance && yf[1] > Tolerance) yield_type = MC_SHEAR;
  if (yf[0] > Tolerance && yf[1] < Tolerance) yield_type = MC_TENSILE;
  return yield_type;
}

// mohr_coulomb.tcc:195-344 (dF/dsigma, dP/dsigma, dP/dq, softening).  pdstrain
// is passed separately (it is kept in FP64 on every path).
template <typename R>
MPM_HD void mc_df_dp(const MaterialT<R>& m, int yield_type, const R* sv, const LodeTrig<R>& lt,
                     const FrictionTrig<R>& ft, R pdstrain, const R* s, R* df, R* dp, R* dp_dq,
                     R* softening) {
  const R eps = dbl_eps<R>();
  const R rho = sv[SV_RHO];
  const R phi = sv[SV_PHI], tension_cutoff = sv[SV_TC];
  const R ct = lt.ct, st = lt.st;
  R df_depsilon, df_drho, df_dtheta;
  if (yield_type == MC_TENSILE) {
    df_depsilon = R(1) / sqrt(R(3));
    df_drho = sqrt(R(2) / R(3)) * ct;
    df_dtheta = -sqrt(R(2) / R(3)) * rho * st;
  } else {
    df_depsilon = ft.tphi / sqrt(R(3));
    df_drho = sqrt(R(1.5)) * ((lt.sp3 / (sqrt(R(3)) * ft.cphi)) + (lt.cp3 * ft.tphi / R(3)));
    df_dtheta = sqrt(R(1.5)) * rho * ((lt.cp3 / (sqrt(R(3)) * ft.cphi)) - (lt.sp3 * ft.tphi / R(3)));
  }
  // dEpsilon/dsigma = dp/dsigma * sqrt(3); dRho/dsigma = dq/dsigma * sqrt(2/3)
  const R deps_ds = R(1) / R(3) * sqrt(R(3));
  const R j2 = mu_j2(s);
  const R q = sqrt(R(3) * j2);
  const R pm = mu_p(s);
  const R dev[6] = {s[0] - pm, s[1] - pm, s[2] - pm, s[3], s[4], s[5]};
  R drho_ds[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
  if (fabs(q) > eps) {
    drho_ds[0] = R(3) / (R(2) * q) * dev[0];
    drho_ds[1] = R(3) / (R(2) * q) * dev[1];
    drho_ds[2] = R(3) / (R(2) * q) * dev[2];
    drho_ds[3] = R(3) / q * dev[3];
    drho_ds[4] = R(3) / q * dev[4];
    drho_ds[5] = R(3) / q * dev[5];
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) drho_ds[i] *= sqrt(R(2) / R(3));
  // dtheta/dsigma (material_utility.tcc:166-200), in FP64 for every R for
  // the reason given at mc_invariants (1 - r^2 vanishes on triaxial paths)
  R dtheta_ds[6];
  {
    using H = typename HighPrecision<R>::T;
    const H sd[6] = {H(s[0]), H(s[1]), H(s[2]), H(s[3]), H(s[4]), H(s[5])};
    const H j2d = mu_j2(sd);
    const H pmd = mu_p(sd);
    const H dv[6] = {sd[0] - pmd, sd[1] - pmd, sd[2] - pmd, sd[3], sd[4], sd[5]};
    const H j3 = mu_j3(sd);
    const H dj2[6] = {dv[0], dv[1], dv[2], dv[3] * 2.0, dv[4] * 2.0, dv[5] * 2.0};
    const H dev1[3] = {dv[0], dv[3], dv[5]};
    const H dev2[3] = {dv[3], dv[1], dv[4]};
    const H dev3[3] = {dv[5], dv[4], dv[2]};
    auto dot3 = [](const H* a, const H* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; };
    const H dj3[6] = {dot3(dev1, dev1) - (2.0 / 3.0) * j2d,
                      dot3(dev2, dev2) - (2.0 / 3.0) * j2d,
                      dot3(dev3, dev3) - (2.0 / 3.0) * j2d,
                      2.0 * dot3(dev1, dev2),
                      2.0 * dot3(dev2, dev3),
                      2.0 * dot3(dev1, dev3)};
    H dr_dj2 = -9.0 / 4.0 * sqrt(3.0) * j3;
    H dr_dj3 = H(3.0 / 2.0 * sqrt(3.0));
    H dtheta_dr = H(-1.0 / 3.0);
    if (fabs(j2d) > kDblEps) {
      // j2^-1.5 and j2^-2.5 from one square root
      const H p15 = 1.0 / (j2d * sqrt(j2d));
      const H r = j3 / 2.0 * (3.0 * sqrt(3.0)) * p15;
      dr_dj2 *= p15 / j2d;
      dr_dj3 *= p15;
      const H factor = lode_corner((fabs(1.0 - r * r) < kDblEps) ? H(kDblEps) : fabs(1.0 - r * r),
                                   value(fabs(1.0 - r * r)));
      dtheta_dr = -1.0 / (3.0 * sqrt(factor));
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) dtheta_ds[i] = R(dtheta_dr * ((dr_dj2 * dj2[i]) + (dr_dj3 * dj3[i])));
  }
#pragma unroll
  for (int i = 0; i < 6; ++i)
    df[i] = ((df_depsilon * (i < 3 ? deps_ds : R(0))) + (df_drho * drho_ds[i])) +
            (df_dtheta * dtheta_ds[i]);
  if (yield_type == MC_TENSILE) {
    const R et_value = R(0.6);
    const R xit = R(0.1);
    R sqpart = R(4) * (R(1) - et_value * et_value) * ct * ct + R(5) * et_value * et_value -
               R(4) * et_value;
    if (sqpart < eps) sqpart = R(1.E-5);
    R rt_den = R(2) * (R(1) - et_value * et_value) * ct + (R(2) * et_value - R(1)) * sqrt(sqpart);
    const R rt_num = R(4) * (R(1) - et_value * et_value) * ct * ct +
                     (R(2) * et_value - R(1)) * (R(2) * et_value - R(1));
    if (fabs(rt_den) < eps) rt_den = R(1.E-5);
    const R rt = rt_num / (R(3) * rt_den);
    const R den = check_low(
        sqrt(xit * xit * tension_cutoff * tension_cutoff + R(1.5) * rt * rt * rho * rho));
    const R dp_drt = R(1.5) * rho * rho * rt / den;
    const R dp_drho = R(1.5) * rho * rt * rt / den;
    const R dp_depsilon = R(1) / sqrt(R(3));
    const R drtden_dtheta =
        R(-2) * (R(1) - et_value * et_value) * st -
        (R(2) * et_value - R(1)) * R(4) * (R(1) - et_value * et_value) * ct * st /
            sqrt(R(4) * (R(1) - et_value * et_value) * ct * ct + R(5) * et_value * et_value -
                 R(4) * et_value);
    const R drtnum_dtheta = R(-8) * (R(1) - et_value * et_value) * ct * st;
    const R drt_dtheta =
        (drtnum_dtheta * rt_den - drtden_dtheta * rt_num) / (R(3) * rt_den * rt_den);
#pragma unroll
    for (int i = 0; i < 6; ++i)
      dp[i] = ((dp_depsilon * (i < 3 ? deps_ds : R(0))) + (dp_drho * drho_ds[i])) +
              (dp_drt * drt_dtheta * dtheta_ds[i]);
    *dp_dq = dp_drho * sqrt(R(2) / R(3));
  } else {
    const R sphi = ft.sphi, cphi = ft.cphi;
    const R r_mc = (R(3) - sphi) / (R(6) * cphi);
    R e_val = (R(3) - sphi) / (R(3) + sphi);
    if (e_val <= R(0.5)) e_val = R(0.5) + R(1.E-10);
    if (e_val > R(1)) e_val = R(1);
    R sqpart = (R(4) * (R(1) - e_val * e_val) * sq(ct)) + (R(5) * e_val * e_val) - (R(4) * e_val);
    if (sqpart < eps) sqpart = R(1.E-5);
    R mm = (R(2) * (R(1) - e_val * e_val) * ct) + ((R(2) * e_val - R(1)) * sqrt(sqpart));
    if (fabs(mm) < eps) mm = R(1.E-5);
    const R l = (R(4) * (R(1) - e_val * e_val) * sq(ct)) + sq(R(2) * e_val - R(1));
    const R r_mw = (l / mm) * r_mc;
    const R xi = R(0.1);
    R omega = sq(xi * m.c_peak * ft.tpsi) + sq(r_mw * sqrt(R(1.5)) * rho);
    if (omega < eps) omega = R(1.E-5);
    const R dl_dtheta = R(-8) * (R(1) - e_val * e_val) * ct * st;
    const R dm_dtheta = (R(-2) * (R(1) - e_val * e_val) * st) +
                        (R(0.5) * (R(2) * e_val - R(1)) * dl_dtheta) / sqrt(sqpart);
    const R drmw_dtheta = ((mm * dl_dtheta) - (l * dm_dtheta)) / (mm * mm);
    const R dp_depsilon = ft.tpsi / sqrt(R(3));
    const R dp_drho = R(3) * rho * r_mw * r_mw / (R(2) * sqrt(omega));
    const R dp_dtheta = (R(3) * rho * rho * r_mw * r_mc * drmw_dtheta) / (R(2) * sqrt(omega));
#pragma unroll
    for (int i = 0; i < 6; ++i)
      dp[i] = ((dp_depsilon * (i < 3 ? deps_ds : R(0))) + (dp_drho * drho_ds[i])) +
              (dp_dtheta * dtheta_ds[i]);
    *dp_dq = dp_drho * sqrt(R(2) / R(3));
  }
  *softening = R(0);
  if (m.softening && pdstrain > m.pd_peak && pdstrain < m.pd_res) {
    const R dphi_dpstrain = (m.phi_res - m.phi_peak) / (m.pd_res - m.pd_peak);
    const R dc_dpstrain = (m.c_res - m.c_peak) / (m.pd_res - m.pd_peak);
    const R df_dphi =
        sqrt(R(1.5)) * rho *
            ((ft.sphi * lt.sp3 / (sqrt(R(3)) * ft.cphi * ft.cphi)) +
             (lt.cp3 / (R(3) * ft.cphi * ft.cphi))) +
        (mu_p(s) / (ft.cphi * ft.cphi));
    const R df_dc = R(-1);
    *softening = R(-1) * ((df_dphi * dphi_dpstrain) + (df_dc * dc_dpstrain)) * (*dp_dq);
  }
  (void)phi;
}

// Out-of-line copies of the three heavy pieces of the return map, for the
// full (non-deferred) update: it evaluates each at up to four places (trial
// stress, old stress, every correction, the final stress), and one shared body
// keeps the kernels that run it -- the dense plastic-return kernels -- small
// enough for the instruction cache (inlined, their warps stalled mostly on
// instruction fetch).  Same arithmetic, so the same results.
template <typename R>
MPM_HD_OUTLINE void mc_invariants_o(const R* s, R* sv, LodeTrig<R>& lt) {
  mc_invariants(s, sv, lt);
}
template <typename R>
MPM_HD_OUTLINE int mc_yield_state_o(R* yf, const R* sv, const LodeTrig<R>& lt,
                                    const FrictionTrig<R>& ft) {
  return mc_yield_state(yf, sv, lt, ft);
}
template <typename R>
MPM_HD_OUTLINE void mc_df_dp_o(const MaterialT<R>& m, int yield_type, const R* sv,
                               const LodeTrig<R>& lt, const FrictionTrig<R>& ft, R pdstrain,
                               const R* s, R* df, R* dp, R* dp_dq, R* softening) {
  mc_df_dp(m, yield_type, sv, lt, ft, pdstrain, s, df, dp, dp_dq, softening);
}

template <typename R>
MPM_HD R huge_value() {
  return R(1.7976931348623157e308);
}
template <>
MPM_HD float huge_value<float>() {
  return 3.402823466e38f;
}

// Outcome of mc_stress: the stress is in out (MC_OK), a return iteration left
// it non-finite (MC_NONFINITE), or the trial stress is plastic and DEFER asked
// to stop there (MC_DEFERRED: out, sv and pdstrain hold nothing to keep; the
// caller redoes the whole update later, with the same inputs).
enum { MC_OK = 0, MC_NONFINITE = 1, MC_DEFERRED = 2 };

// MohrCoulomb<Tdim>::compute_stress (mohr_coulomb.tcc:348-513), stress_rate
// None (infinitesimal_elasto_plastic.tcc:2-25).  sv holds the state variables
// in the reference order; the plastic deviatoric strain (slot SV_PD) is kept in
// PD (double on every path).  With DEFER the elastic predictor and the yield
// check run, and a plastic point returns MC_DEFERRED before the corrector: the
// step kernels finish elastic points in place and hand plastic ones to a
// dense kernel, so that the few plastic lanes of a warp do not hold the
// elastic ones through the return iterations.
template <typename R, typename PD, bool DEFER>
MPM_HD int mc_stress(const MaterialT<R>& m, const R* stress, const R* dstrain, R density, R* sv,
                     PD& pdstrain_io, R* out, int* corrections = nullptr) {
  const R critical_density = m.min_packing * m.grain_density;
  const R pdstrain = R(pdstrain_io);
  if (m.softening && pdstrain > m.pd_peak) {
    if (pdstrain < m.pd_res) {
      sv[SV_PHI] = m.phi_res + ((m.phi_peak - m.phi_res) * (pdstrain - m.pd_res) /
                                (m.pd_peak - m.pd_res));
      sv[SV_PSI] = m.psi_res + ((m.psi_peak - m.psi_res) * (pdstrain - m.pd_res) /
                                (m.pd_peak - m.pd_res));
      sv[SV_COH] = m.c_res + ((m.c_peak - m.c_res) * (pdstrain - m.pd_res) / (m.pd_peak - m.pd_res));
    } else {
      sv[SV_PHI] = m.phi_res;
      sv[SV_PSI] = m.psi_res;
      sv[SV_COH] = m.c_res;
    }
    const R apex = sv[SV_COH] / tan(sv[SV_PHI]);
    if (sv[SV_TC] > apex) sv[SV_TC] = check_low(apex);
  }
  sv[SV_YIELD] = R(0);
  R trial[6];
  {
    R t[6];
    de_mul(m, dstrain, t);
#pragma unroll
    for (int i = 0; i < 6; ++i) trial[i] = stress[i] + t[i];
  }
  if (density <= critical_density) {
    pdstrain_io += PD(sqrt(R(3) * mu_j2(trial)) / R(3) / m.shear);
    sv[SV_YIELD] = R(3);
#pragma unroll
    for (int i = 0; i < 6; ++i) out[i] = R(0);
    return MC_OK;
  }
  const FrictionTrig<R> ft = friction_trig(m, sv);
  LodeTrig<R> lt;
  mc_invariants(trial, sv, lt);
  R yf_trial[2];
  int yt_trial = mc_yield_state(yf_trial, sv, lt, ft);
  if (yt_trial == MC_ELASTIC) {
    sv[SV_YIELD] = R(0);
#pragma unroll
    for (int i = 0; i < 6; ++i) out[i] = trial[i];
    return MC_OK;
  }
  if constexpr (DEFER) return MC_DEFERRED;
  const R Tolerance = R(1E-1);
  R softening_trial = R(0), dp_dq_trial = R(0);
  R df_trial[6], dp_trial[6];
  R yield_trial = R(0);
  if (yt_trial == MC_TENSILE) {
    sv[SV_YIELD] = R(2);
    yield_trial = yf_trial[0];
  }
  if (yt_trial == MC_SHEAR) {
    sv[SV_YIELD] = R(1);
    yield_trial = yf_trial[1];
  }
  // the trial stress's invariants, for its dF/dsigma and dP/dsigma below: the
  // reference evaluates them here, but only the branch of an old stress off
  // the yield surface uses them, so they are evaluated there (same inputs)
  const LodeTrig<R> lt_trial = lt;
  const R sv_trial[3] = {sv[SV_EPS], sv[SV_RHO], sv[SV_THETA]};
  mc_invariants_o(stress, sv, lt);
  R yf[2];
  const int yt = mc_yield_state_o(yf, sv, lt, ft);
  R yield = huge_value<R>();
  if (yt == MC_TENSILE) yield = yf[0];
  if (yt == MC_SHEAR) yield = yf[1];
  R softening = R(0), dp_dq = R(0);
  R df[6], dp[6];
  mc_df_dp_o(m, yt, sv, lt, ft, pdstrain, stress, df, dp, &dp_dq, &softening);
  const R lambda = row_de_dot(m, df, dstrain) / (row_de_dot(m, df, dp) + softening);
  R upd[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) upd[i] = trial[i];
  R dpdstrain;
  if (fabs(yield) < Tolerance) {
    sub_lambda_de(m, lambda, dp, upd);
    dpdstrain = lambda * dp_dq;
  } else {
    R svt[SV_N];
#pragma unroll
    for (int k = 0; k < SV_N; ++k) svt[k] = sv[k];
    svt[SV_EPS] = sv_trial[0];
    svt[SV_RHO] = sv_trial[1];
    svt[SV_THETA] = sv_trial[2];
    mc_df_dp_o(m, yt_trial, svt, lt_trial, ft, pdstrain, trial, df_trial, dp_trial, &dp_dq_trial,
               &softening_trial);
    const R lambda_trial = yield_trial / (row_de_dot(m, df_trial, dp_trial) + softening_trial);
    sub_lambda_de(m, lambda_trial, dp_trial, upd);
    dpdstrain = lambda_trial * dp_dq_trial;
  }
  int itr = 0;
  for (; itr < 100; ++itr) {
    mc_invariants_o(upd, sv, lt);
    yt_trial = mc_yield_state_o(yf_trial, sv, lt, ft);
    if (yf_trial[0] < Tolerance && yf_trial[1] < Tolerance) break;
    mc_df_dp_o(m, yt_trial, sv, lt, ft, pdstrain, upd, df_trial, dp_trial, &dp_dq_trial,
               &softening_trial);
    if (yt_trial == MC_TENSILE) yield_trial = yf_trial[0];
    if (yt_trial == MC_SHEAR) yield_trial = yf_trial[1];
    const R lambda_trial = yield_trial / (row_de_dot(m, df_trial, dp_trial) + softening_trial);
    sub_lambda_de(m, lambda_trial, dp_trial, upd);
    dpdstrain += lambda_trial * dp_dq_trial;
  }
  if (corrections) *corrections = itr;
  mc_invariants_o(upd, sv, lt);
  pdstrain_io += PD(dpdstrain);
  bool finite = true;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    out[i] = upd[i];
    finite = finite && (upd[i] - upd[i] == R(0));
  }
  return finite ? MC_OK : MC_NONFINITE;
}

// The full update; false when the return left the stress non-finite.
template <typename R, typename PD>
MPM_HD bool mc_compute_stress(const MaterialT<R>& m, const R* stress, const R* dstrain, R density,
                              R* sv, PD& pdstrain_io, R* out, int* corrections = nullptr) {
  return mc_stress<R, PD, false>(m, stress, dstrain, density, sv, pdstrain_io, out, corrections) ==
         MC_OK;
}

// Material<Tdim>::compute_stress dispatch (material.h:97-106)
template <typename R, typename PD>
MPM_HD bool material_compute_stress(const MaterialT<R>& m, const R* stress, const R* dstrain,
                                    R density, R* sv, PD& pdstrain, R* out) {
  if (m.type == 0) {
    R t[6];
    de_mul(m, dstrain, t);  // linear_elastic.tcc:73-94
#pragma unroll
    for (int i = 0; i < 6; ++i) out[i] = stress[i] + t[i];
    return true;
  }
  return mc_compute_stress(m, stress, dstrain, density, sv, pdstrain, out);
}

// FP64 form used by the FP64 kernels: the state array holds pdstrain in SV_PD.
MPM_HD void material_compute_stress(const MaterialParams& m, const double* stress,
                                    const double* dstrain, double density, double* sv,
                                    double* out, int* corrections = nullptr) {
  if (m.type == 0) {
    double pd = 0.;
    material_compute_stress<double, double>(m, stress, dstrain, density, sv, pd, out);
    return;
  }
  mc_compute_stress<double, double>(m, stress, dstrain, density, sv, sv[SV_PD], out, corrections);
}

// ---------------------------------------------------------------- node update
struct NodeBC {
  // velocity constraints (node.tcc:370-403); mask bit d = direction d
  uint8_t vel_mask, acc_mask, friction, fric_dir;
  int32_t fric_sign;
  double vel[3];
  double acc[3];
  double mu;
  // general boundaries (node.h assign_rotation_matrix): the constraint
  // directions are those of the node's local frame, rot maps local to global
  // components, irot = rot^-1 (both row-major, leading DIM x DIM block)
  int32_t rotated;
  double rot[9], irot[9];
};

// Rotation of a node's local frame from its Euler angles (radians): in 2D
// the rotation by alpha + beta; in 3D Rz(alpha) Rx(gamma) Rz(beta) (angles
// alpha, beta, gamma as mesh.tcc:1318-1345 reads them).  Row-major into R.
MPM_HD void euler_rotation(int dim, const double* angles, double* R) {
  const double ca = cos(angles[0]), sa = sin(angles[0]);
  const double cb = cos(angles[1]), sb = sin(angles[1]);
  const double cacb = ca * cb, casb = ca * sb, sacb = sa * cb, sasb = sa * sb;
  if (dim == 2) {
    R[0] = cacb - sasb;
    R[1] = -casb - sacb;
    R[3] = sacb + casb;
    R[4] = -sasb + cacb;
    return;
  }
  const double cg = cos(angles[2]), sg = sin(angles[2]);
  R[0] = cacb - sasb * cg;
  R[1] = -casb - sacb * cg;
  R[2] = sa * sg;
  R[3] = sacb + casb * cg;
  R[4] = -sasb + cacb * cg;
  R[5] = -ca * sg;
  R[6] = sb * sg;
  R[7] = cb * sg;
  R[8] = cg;
}

// out = M v for the leading DIM x DIM block of a row-major 3 x 3 M
template <int DIM, typename R>
MPM_HD void rot_apply(const double* M, const R* v, R* out) {
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    R s = M[a * 3 + 0] * v[0];
#pragma unroll
    for (int b = 1; b < DIM; ++b) s = s + M[a * 3 + b] * v[b];
    out[a] = s;
  }
}

template <int DIM, typename R>
MPM_HD void apply_velocity_constraints(const NodeBC& bc, R* v, R* a) {
#pragma unroll
  for (int d = 0; d < DIM; ++d)
    if (bc.vel_mask & (1u << d)) {
      if (!bc.rotated) {
        v[d] = R(bc.vel[d]);
        a[d] = R(0.);
      } else {  // node.tcc:385-401: in the local frame, one direction at a time
        R lv[DIM], la[DIM];
        rot_apply<DIM>(bc.irot, v, lv);
        rot_apply<DIM>(bc.irot, a, la);
        lv[d] = R(bc.vel[d]);
        la[d] = R(0.);
        rot_apply<DIM>(bc.rot, lv, v);
        rot_apply<DIM>(bc.rot, la, a);
      }
    }
}

// node.tcc:456-483
template <int DIM, typename R>
MPM_HD void apply_acceleration_constraints(const NodeBC& bc, R* a) {
#pragma unroll
  for (int d = 0; d < DIM; ++d)
    if (bc.acc_mask & (1u << d)) {
      if (!bc.rotated) {
        a[d] = R(bc.acc[d]);
      } else {
        R la[DIM];
        rot_apply<DIM>(bc.irot, a, la);
        la[d] = R(bc.acc[d]);
        rot_apply<DIM>(bc.rot, la, a);
      }
    }
}

// node.tcc:510-657; on a general boundary in the node's local frame
template <int DIM, typename R>
MPM_HD void apply_friction_constraints(const NodeBC& bc, const R* vel_g, R* acc_g, double dt) {
  auto sign = [](const R& value) { return (value > 0.) ? 1. : -1.; };
  const unsigned dir_n = bc.fric_dir;
  const double sign_n = bc.fric_sign > 0 ? 1. : -1.;
  const double mu = bc.mu;
  R vel_l[DIM], acc_l[DIM];
  if (bc.rotated) {
    rot_apply<DIM>(bc.irot, vel_g, vel_l);
    rot_apply<DIM>(bc.irot, acc_g, acc_l);
  } else {
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      vel_l[d] = vel_g[d];
      acc_l[d] = acc_g[d];
    }
  }
  const R* vel = vel_l;
  R* acc = acc_l;
  if constexpr (DIM == 2) {
    const unsigned dir_t = 1 - dir_n;
    const R acc_n = acc[dir_n];
    R acc_t = acc[dir_t];
    const R vel_t = vel[dir_t];
    if ((acc_n * sign_n) > 0.0) {
      if (vel_t != 0.0) {
        const R vel_net = dt * acc_t + vel_t;
        const R vel_frictional = dt * mu * fabs(acc_n);
        if (fabs(vel_net) <= vel_frictional)
          acc_t = -vel_t / dt;
        else
          acc_t -= sign(vel_net) * mu * fabs(acc_n);
      } else {
        if (fabs(acc_t) <= mu * fabs(acc_n))
          acc_t = R(0.0);
        else
          acc_t -= sign(acc_t) * mu * fabs(acc_n);
      }
      acc[dir_t] = acc_t;
      if (bc.rotated)
        rot_apply<DIM>(bc.rot, acc, acc_g);
      else
        acc_g[dir_t] = acc_t;
    }
  } else {
    const unsigned t0 = dir_n == 0 ? 1 : 0;
    const unsigned t1 = dir_n == 2 ? 1 : 2;
    const R acc_n = acc[dir_n];
    R acc_t = sqrt(acc[t0] * acc[t0] + acc[t1] * acc[t1]);
    const R vel_t = sqrt(vel[t0] * vel[t0] + vel[t1] * vel[t1]);
    if (acc_n * sign_n > 0.0) {
      if (vel_t != 0.0) {
        const R vn0 = vel[t0] + acc[t0] * dt;
        const R vn1 = vel[t1] + acc[t1] * dt;
        const R vel_net_t = sqrt(vn0 * vn0 + vn1 * vn1);
        const R vel_fricion = mu * fabs(acc_n) * dt;
        if (vel_net_t <= vel_fricion) {
          acc[t0] = -vel[t0] / dt;
          acc[t1] = -vel[t1] / dt;
        } else {
          acc[t0] -= mu * fabs(acc_n) * (vn0 / vel_net_t);
          acc[t1] -= mu * fabs(acc_n) * (vn1 / vel_net_t);
        }
      } else {
        if (acc_t <= mu * fabs(acc_n)) {
          acc[t0] = R(0.);
          acc[t1] = R(0.);
        } else {
          acc_t -= mu * fabs(acc_n);
          acc[t0] -= mu * fabs(acc_n) * (acc[t0] / acc_t);
          acc[t1] -= mu * fabs(acc_n) * (acc[t1] / acc_t);
        }
      }
      if (bc.rotated) {
        rot_apply<DIM>(bc.rot, acc, acc_g);
      } else {
#pragma unroll
        for (int d = 0; d < DIM; ++d) acc_g[d] = acc[d];
      }
    }
  }
}

}  // namespace mpm_b200
