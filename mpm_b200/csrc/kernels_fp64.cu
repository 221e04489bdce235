// kernels_fp64.cu -- FP64 kernels of the explicit MPM step (USF and USL).
//
// Compiled with --fmad=false: every product and sum rounds on its own, as in
// the reference's scalar C++ arithmetic, so the only differences from the
// reference arithmetic are the order of the nodal sums and the device libm.
//
// One step (USL):   p2g(mass, momentum, forces) -> node update -> g2p(+stress,
//                   locate) -> locate fallback
// One step (USF):   p2g(mass, momentum) -> node velocity -> stress + force p2g
//                   -> node update -> g2p(locate) -> locate fallback
#include <cuda_runtime.h>

#include "mpm_kernels.h"
#include "mpm_state.cuh"

namespace mpm_b200 {

namespace {

template <int DIM>
struct CellCtx {
  static constexpr int NV = Elem<DIM>::NV;
  int nid[NV];
  double X[NV * DIM];
};

template <int DIM>
__device__ __forceinline__ void load_cell(const DevState& s, int c, CellCtx<DIM>& cc) {
  constexpr int NV = Elem<DIM>::NV;
#pragma unroll
  for (int i = 0; i < NV; ++i) cc.nid[i] = __ldg(&s.cell_nodes[(int64_t)c * NV + i]);
#pragma unroll
  for (int i = 0; i < NV; ++i)
#pragma unroll
    for (int d = 0; d < DIM; ++d) cc.X[i * DIM + d] = __ldg(&s.ncoord[(int64_t)d * s.nn + cc.nid[i]]);
}

template <int DIM>
__device__ __forceinline__ void load_x(const DevState& s, int64_t p, double* x) {
#pragma unroll
  for (int d = 0; d < DIM; ++d) x[d] = s.pf[(int64_t)(PF<DIM>::X + d) * s.np + p];
}

template <int DIM>
__device__ __forceinline__ void particle_xi(const DevState& s, int c, const double* x, double* xi) {
  const CellGeom& g = s.geom[c];
  local_xi<DIM>(x, g.centroid, g.len, xi);
}

__device__ __forceinline__ void raise_err(const DevState& s, unsigned bits) { atomicOr(s.err, bits); }

// ------------------------------------------------------------------------ P2G
// particle.tcc:630-657 (mass, momentum), :893-898 (body force),
// :915-949 (internal force)
template <int DIM, bool FORCES>
__global__ void __launch_bounds__(256) k_p2g(DevState s, double g0, double g1, double g2) {
  constexpr int NV = Elem<DIM>::NV;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0) return;
  if (c >= s.ncells) {
    raise_err(s, ERR_BADCELL);
    return;
  }
  double x[DIM], xi[DIM], N[NV];
  load_x<DIM>(s, p, x);
  particle_xi<DIM>(s, c, x, xi);
  shapefn<DIM>(xi, N);
  CellCtx<DIM> cc;
  load_cell<DIM>(s, c, cc);
  const int64_t np = s.np, nn = s.nn;
  const double m = s.pf[(int64_t)PF<DIM>::MASS * np + p];
  double v[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) v[d] = s.pf[(int64_t)(PF<DIM>::V + d) * np + p];
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const int n = cc.nid[i];
    const double mN = m * N[i];
    atomicAdd(&s.nf[(int64_t)NF<DIM>::MASS * nn + n], mN);
#pragma unroll
    for (int d = 0; d < DIM; ++d) atomicAdd(&s.nf[(int64_t)(NF<DIM>::MOM + d) * nn + n], mN * v[d]);
    s.active[n] = 1;
  }
  if constexpr (FORCES) {
    const double g[3] = {g0, g1, g2};
    double D[NV * DIM];
    dn_dx<DIM>(xi, cc.X, D);
    const double vol = s.pf[(int64_t)PF<DIM>::VOL * np + p];
    double sig[6];
#pragma unroll
    for (int k = 0; k < PF<DIM>::NS; ++k) sig[k] = s.pf[(int64_t)(PF<DIM>::S + k) * np + p];
    const double sc = -1. * vol;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      const int n = cc.nid[i];
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        atomicAdd(&s.nf[(int64_t)(NF<DIM>::FEXT + d) * nn + n], (g[d] * m) * N[i]);
      const double* Dn = &D[i * DIM];
      double f[DIM];
      if constexpr (DIM == 2) {
        f[0] = Dn[0] * sig[0] + Dn[1] * sig[3];
        f[1] = Dn[1] * sig[1] + Dn[0] * sig[3];
      } else {
        f[0] = Dn[0] * sig[0] + Dn[1] * sig[3] + Dn[2] * sig[5];
        f[1] = Dn[1] * sig[1] + Dn[0] * sig[3] + Dn[2] * sig[4];
        f[2] = Dn[2] * sig[2] + Dn[1] * sig[4] + Dn[0] * sig[5];
      }
#pragma unroll
      for (int d = 0; d < DIM; ++d) atomicAdd(&s.nf[(int64_t)(NF<DIM>::FINT + d) * nn + n], f[d] * sc);
    }
  }
}

// ---------------------------------------------------------------- node update
// node.tcc:236-252 compute_velocity; node.tcc:309-345 Cundall update
template <int DIM>
__device__ __forceinline__ void node_accel_update(const DevState& s, int64_t n, double m,
                                                  double* vel, double* acc, int bci, double dt,
                                                  double damping) {
  const int64_t nn = s.nn;
  if (!(m > 1.0E-15)) return;
  double uf[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d)
    uf[d] = s.nf[(int64_t)(NF<DIM>::FEXT + d) * nn + n] + s.nf[(int64_t)(NF<DIM>::FINT + d) * nn + n];
  double ss = uf[0] * uf[0];
#pragma unroll
  for (int d = 1; d < DIM; ++d) ss = ss + uf[d] * uf[d];
  const double nrm = sqrt(ss);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const double sg = (vel[d] > 0.) ? 1. : ((vel[d] < 0.) ? -1. : 0.);
    acc[d] = (uf[d] - damping * nrm * sg) / m;
  }
  if (bci >= 0) {
    const NodeBC& bc = s.bcs[bci];
    if (bc.friction) apply_friction_constraints<DIM>(bc, vel, acc, dt);
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      if (bc.acc_mask & (1u << d)) acc[d] = bc.acc[d];
  }
#pragma unroll
  for (int d = 0; d < DIM; ++d) vel[d] += acc[d] * dt;
  if (bci >= 0) apply_velocity_constraints<DIM>(s.bcs[bci], vel, acc);
#pragma unroll
  for (int d = 0; d < DIM; ++d)
    if (fabs(vel[d]) < 1.0E-15) vel[d] = 0.;
#pragma unroll
  for (int d = 0; d < DIM; ++d)
    if (fabs(acc[d]) < 1.0E-15) acc[d] = 0.;
}

// MODE 0: velocity only (USF first pass); 1: velocity + acceleration (USL);
// 2: acceleration only, velocity from the first pass (USF second pass)
template <int DIM, int MODE>
__global__ void __launch_bounds__(256) k_nodes(DevState s, double dt, double damping) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= s.nn) return;
  if (!s.active[n]) return;
  const int64_t nn = s.nn;
  const double m = s.nf[(int64_t)NF<DIM>::MASS * nn + n];
  const int bci = s.bc_index[n];
  double vel[DIM], acc[DIM];
  if constexpr (MODE == 2) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      vel[d] = s.nf[(int64_t)(NF<DIM>::VEL + d) * nn + n];
      acc[d] = s.nf[(int64_t)(NF<DIM>::ACC + d) * nn + n];
    }
  } else {
#pragma unroll
    for (int d = 0; d < DIM; ++d) vel[d] = acc[d] = 0.;
    if (m > 1.E-16) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) vel[d] = s.nf[(int64_t)(NF<DIM>::MOM + d) * nn + n] / m;
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        if (fabs(vel[d]) < 1.E-15) vel[d] = 0.;
    }
    if (bci >= 0) apply_velocity_constraints<DIM>(s.bcs[bci], vel, acc);
  }
  if constexpr (MODE != 0) node_accel_update<DIM>(s, n, m, vel, acc, bci, dt, damping);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    s.nf[(int64_t)(NF<DIM>::VEL + d) * nn + n] = vel[d];
    s.nf[(int64_t)(NF<DIM>::ACC + d) * nn + n] = acc[d];
  }
}

// ------------------------------------------------------- stress and strain
// mpm_scheme.tcc:75-103: F increment (particle.tcc:1580-1628), strain
// (:819-876), volume (:598-605), material stress (:880-889), F (:1654-1658)
template <int DIM>
__device__ __forceinline__ void stress_update(const DevState& s, int64_t p, const CellCtx<DIM>& cc,
                                              const double* D, double dt) {
  constexpr int NV = Elem<DIM>::NV;
  const int64_t np = s.np, nn = s.nn;
  double vel[NV][DIM];
#pragma unroll
  for (int i = 0; i < NV; ++i)
#pragma unroll
    for (int d = 0; d < DIM; ++d) vel[i][d] = s.nf[(int64_t)(NF<DIM>::VEL + d) * nn + cc.nid[i]];
  // deformation gradient increment
  double Fi[DIM * DIM];
#pragma unroll
  for (int r = 0; r < DIM; ++r)
#pragma unroll
    for (int c = 0; c < DIM; ++c) Fi[r * DIM + c] = (r == c) ? 1. : 0.;
#pragma unroll
  for (int i = 0; i < NV; ++i)
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
      for (int c = 0; c < DIM; ++c) Fi[r * DIM + c] += vel[i][r] * D[i * DIM + c] * dt;
#pragma unroll
  for (int r = 0; r < DIM; ++r)
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      if (r != c && fabs(Fi[r * DIM + c]) < 1.E-15) Fi[r * DIM + c] = 0.;
      if (r == c && fabs(Fi[r * DIM + c] - 1.) < 1.E-15) Fi[r * DIM + c] = 1.;
    }
  // strain rate at the particle and at the cell centroid
  double sr[6] = {0, 0, 0, 0, 0, 0};
  double src[3] = {0, 0, 0};
  double Dc[NV * DIM];
  {
    double xi0[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) xi0[d] = 0.;
    dn_dx<DIM>(xi0, cc.X, Dc);
  }
  if constexpr (DIM == 2) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      sr[0] += D[i * 2 + 0] * vel[i][0];
      sr[1] += D[i * 2 + 1] * vel[i][1];
      sr[3] += D[i * 2 + 1] * vel[i][0] + D[i * 2 + 0] * vel[i][1];
      src[0] += Dc[i * 2 + 0] * vel[i][0];
      src[1] += Dc[i * 2 + 1] * vel[i][1];
    }
  } else {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      sr[0] += D[i * 3 + 0] * vel[i][0];
      sr[1] += D[i * 3 + 1] * vel[i][1];
      sr[2] += D[i * 3 + 2] * vel[i][2];
      sr[3] += D[i * 3 + 1] * vel[i][0] + D[i * 3 + 0] * vel[i][1];
      sr[4] += D[i * 3 + 2] * vel[i][1] + D[i * 3 + 1] * vel[i][2];
      sr[5] += D[i * 3 + 2] * vel[i][0] + D[i * 3 + 0] * vel[i][2];
      src[0] += Dc[i * 3 + 0] * vel[i][0];
      src[1] += Dc[i * 3 + 1] * vel[i][1];
      src[2] += Dc[i * 3 + 2] * vel[i][2];
    }
  }
#pragma unroll
  for (int k = 0; k < 6; ++k)
    if (fabs(sr[k]) < 1.E-15) sr[k] = 0.;
#pragma unroll
  for (int k = 0; k < DIM; ++k)
    if (fabs(src[k]) < 1.E-15) src[k] = 0.;
  double dstrain[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) dstrain[k] = sr[k] * dt;
  double ssum = src[0];
#pragma unroll
  for (int k = 1; k < DIM; ++k) ssum = ssum + src[k];
  const double dvol = dt * ssum;
  // strain += dstrain
  if constexpr (DIM == 2) {
    const int map[3] = {0, 1, 3};
#pragma unroll
    for (int k = 0; k < 3; ++k) s.pf[(int64_t)(PF<2>::E + k) * np + p] += dstrain[map[k]];
  } else {
#pragma unroll
    for (int k = 0; k < 6; ++k) s.pf[(int64_t)(PF<3>::E + k) * np + p] += dstrain[k];
  }
  // volume and density
  double* volp = &s.pf[(int64_t)PF<DIM>::VOL * np + p];
  double* rhop = &s.pf[(int64_t)PF<DIM>::RHO * np + p];
  const double vol = *volp * (1. + dvol);
  const double rho = *rhop / (1. + dvol);
  *volp = vol;
  *rhop = rho;
  // stress
  double sig[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < PF<DIM>::NS; ++k) sig[k] = s.pf[(int64_t)(PF<DIM>::S + k) * np + p];
  const MaterialParams& mp = s.mats[s.mat[p]];
  double out[6];
  if (mp.type == 0) {
    material_compute_stress(mp, sig, dstrain, rho, nullptr, out);
  } else {
    double sv[SV_N];
#pragma unroll
    for (int k = 0; k < SV_N; ++k) sv[k] = s.sv[(int64_t)k * np + p];
    material_compute_stress(mp, sig, dstrain, rho, sv, out);
#pragma unroll
    for (int k = 0; k < SV_N; ++k) s.sv[(int64_t)k * np + p] = sv[k];
  }
#pragma unroll
  for (int k = 0; k < PF<DIM>::NS; ++k) s.pf[(int64_t)(PF<DIM>::S + k) * np + p] = out[k];
  // F = F_inc * F
  if constexpr (DIM == 2) {
    double F[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) F[k] = s.pf[(int64_t)(PF<2>::F + k) * np + p];
    // 3x3 product with F_inc(2,:) = (0,0,1) and F(2,:) = (0,0,1): the zero
    // terms are exact and dropped
    const double r00 = Fi[0] * F[0] + Fi[1] * F[2];
    const double r01 = Fi[0] * F[1] + Fi[1] * F[3];
    const double r10 = Fi[2] * F[0] + Fi[3] * F[2];
    const double r11 = Fi[2] * F[1] + Fi[3] * F[3];
    s.pf[(int64_t)(PF<2>::F + 0) * np + p] = r00;
    s.pf[(int64_t)(PF<2>::F + 1) * np + p] = r01;
    s.pf[(int64_t)(PF<2>::F + 2) * np + p] = r10;
    s.pf[(int64_t)(PF<2>::F + 3) * np + p] = r11;
  } else {
    double F[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) F[k] = s.pf[(int64_t)(PF<3>::F + k) * np + p];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        s.pf[(int64_t)(PF<3>::F + r * 3 + c) * np + p] =
            (Fi[r * 3 + 0] * F[0 * 3 + c] + Fi[r * 3 + 1] * F[1 * 3 + c]) + Fi[r * 3 + 2] * F[2 * 3 + c];
  }
}

// USF: stress update with the velocities of compute_velocity, then the force
// P2G with the updated stress and volume (mpm_scheme.tcc:131-190)
template <int DIM>
__global__ void __launch_bounds__(128) k_stress_forces(DevState s, double dt, double g0, double g1,
                                                       double g2) {
  constexpr int NV = Elem<DIM>::NV;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0) return;
  double x[DIM], xi[DIM], N[NV], D[NV * DIM];
  load_x<DIM>(s, p, x);
  particle_xi<DIM>(s, c, x, xi);
  shapefn<DIM>(xi, N);
  CellCtx<DIM> cc;
  load_cell<DIM>(s, c, cc);
  dn_dx<DIM>(xi, cc.X, D);
  stress_update<DIM>(s, p, cc, D, dt);
  const int64_t np = s.np, nn = s.nn;
  const double m = s.pf[(int64_t)PF<DIM>::MASS * np + p];
  const double vol = s.pf[(int64_t)PF<DIM>::VOL * np + p];
  double sig[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < PF<DIM>::NS; ++k) sig[k] = s.pf[(int64_t)(PF<DIM>::S + k) * np + p];
  const double g[3] = {g0, g1, g2};
  const double sc = -1. * vol;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const int n = cc.nid[i];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      atomicAdd(&s.nf[(int64_t)(NF<DIM>::FEXT + d) * nn + n], (g[d] * m) * N[i]);
    const double* Dn = &D[i * DIM];
    double f[DIM];
    if constexpr (DIM == 2) {
      f[0] = Dn[0] * sig[0] + Dn[1] * sig[3];
      f[1] = Dn[1] * sig[1] + Dn[0] * sig[3];
    } else {
      f[0] = Dn[0] * sig[0] + Dn[1] * sig[3] + Dn[2] * sig[5];
      f[1] = Dn[1] * sig[1] + Dn[0] * sig[3] + Dn[2] * sig[4];
      f[2] = Dn[2] * sig[2] + Dn[1] * sig[4] + Dn[0] * sig[5];
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) atomicAdd(&s.nf[(int64_t)(NF<DIM>::FINT + d) * nn + n], f[d] * sc);
  }
}

// ------------------------------------------------------------------ locate
// mesh.tcc:1116-1151: the current cell, then neighbours in ascending id
template <int DIM>
__device__ __forceinline__ int locate_near(const DevState& s, const double* x, int c) {
  double xi[DIM];
  {
    const CellGeom& g = s.geom[c];
    if (point_in_cell<DIM>(x, g.centroid, g.len, g.mean_length, xi)) return c;
  }
  const int b = s.nb_off[c], e = s.nb_off[c + 1];
  for (int k = b; k < e; ++k) {
    const int nc = s.nb[k];
    const CellGeom& g = s.geom[nc];
    if (point_in_cell<DIM>(x, g.centroid, g.len, g.mean_length, xi)) return nc;
  }
  return -1;
}

// --------------------------------------------------------------------- G2P
// particle.tcc:994-1067 FLIP / PIC; mesh.tcc:1454-1467 particle velocity
// constraints; USL stress update (mpm_scheme_usl.tcc:14-17); locate.
template <int DIM, bool STRESS, bool FLIP>
__global__ void __launch_bounds__(128) k_g2p(DevState s, double dt, double beta) {
  constexpr int NV = Elem<DIM>::NV;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0) return;
  const int64_t np = s.np, nn = s.nn;
  double x[DIM], xi[DIM], N[NV];
  load_x<DIM>(s, p, x);
  particle_xi<DIM>(s, c, x, xi);
  shapefn<DIM>(xi, N);
  CellCtx<DIM> cc;
  load_cell<DIM>(s, c, cc);
  double nvel[DIM], nacc[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) nvel[d] = nacc[d] = 0.;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const int n = cc.nid[i];
#pragma unroll
    for (int d = 0; d < DIM; ++d) nvel[d] += N[i] * s.nf[(int64_t)(NF<DIM>::VEL + d) * nn + n];
    if constexpr (FLIP) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) nacc[d] += N[i] * s.nf[(int64_t)(NF<DIM>::ACC + d) * nn + n];
    }
  }
  double v[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) v[d] = s.pf[(int64_t)(PF<DIM>::V + d) * np + p];
  if constexpr (FLIP) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] += nacc[d] * dt;
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] = beta * v[d] + (1.0 - beta) * nvel[d];
  } else {
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] = nvel[d];
  }
  double xn[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    xn[d] = x[d] + nvel[d] * dt;
    s.pf[(int64_t)(PF<DIM>::X + d) * np + p] = xn[d];
    s.pf[(int64_t)(PF<DIM>::U + d) * np + p] += nvel[d] * dt;
  }
  const int pv = s.pvc[p];
  if (pv >= 0) {
    const ParticleVC& r = s.pvcs[pv];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      if (r.mask & (1u << d)) v[d] = r.value[d];
  }
#pragma unroll
  for (int d = 0; d < DIM; ++d) s.pf[(int64_t)(PF<DIM>::V + d) * np + p] = v[d];
  if constexpr (STRESS) {
    double D[NV * DIM];
    dn_dx<DIM>(xi, cc.X, D);
    stress_update<DIM>(s, p, cc, D, dt);
  }
  bool finite = true;
#pragma unroll
  for (int d = 0; d < DIM; ++d) finite = finite && isfinite(xn[d]);
  if (!finite) {
    raise_err(s, ERR_NONFINITE);
    s.lost[atomicAdd(s.nlost, 1u)] = (int32_t)p;
    return;
  }
  const int nc = locate_near<DIM>(s, xn, c);
  if (nc >= 0) {
    if (nc != c) s.cell[p] = nc;
  } else {
    s.lost[atomicAdd(s.nlost, 1u)] = (int32_t)p;
  }
}

// Exhaustive search for particles not in their cell or its neighbours
// (mesh.tcc:1136-1148, one thread: the first cell in id order that contains
// the point).  Grid-stride over the lost list; usually empty.
template <int DIM>
__global__ void k_locate_fallback(DevState s, int remove_lost) {
  const unsigned count = *s.nlost;
  for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    const int64_t p = s.lost[k];
    double x[DIM];
    load_x<DIM>(s, p, x);
    int found = -1;
    if (s.structured) {
      found = structured_scan<DIM>(x, s.gcells, s.axis, s.geom);
    } else {
      bool inside = true;
      int b[3] = {0, 0, 0};
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        const double f = floor((x[d] - s.bmin[d]) / s.bsize[d]);
        if (!(f >= 0.) || f >= (double)s.bn[d]) inside = false;
        else b[d] = (int)f;
      }
      if (inside) {
        const int64_t bi = ((int64_t)b[2] * s.bn[1] + b[1]) * s.bn[0] + b[0];
        for (int j = s.bin_off[bi]; j < s.bin_off[bi + 1]; ++j) {
          const int cid = s.bin_cells[j];
          const CellGeom& g = s.geom[cid];
          double xi[DIM];
          if (point_in_cell<DIM>(x, g.centroid, g.len, g.mean_length, xi)) {
            found = cid;
            break;
          }
        }
      }
    }
    if (found >= 0) {
      s.cell[p] = found;
    } else if (remove_lost) {
      s.cell[p] = -1;
    } else {
      raise_err(s, ERR_OUTSIDE);
    }
  }
}

inline unsigned nblocks(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

template <int DIM>
void step_impl(const DevState& s, const StepArgs& a, cudaStream_t st, Profiler& pr) {
  const int64_t np = s.np, nn = s.nn;
  if (np == 0) return;
  // Node::initialise (node.tcc:26-42): zero the accumulated fields and flags
  cudaMemsetAsync(s.nf, 0, sizeof(double) * NF<DIM>::NACC_FIELDS * nn, st);
  cudaMemsetAsync(s.active, 0, nn, st);
  cudaMemsetAsync(s.nlost, 0, sizeof(unsigned), st);
  const unsigned pb256 = nblocks(np, 256), pb128 = nblocks(np, 128), nb = nblocks(nn, 256);
  if (a.scheme == 1) {  // USL
    pr.begin(K_P2G, st);
    k_p2g<DIM, true><<<pb256, 256, 0, st>>>(s, a.g[0], a.g[1], a.g[2]);
    pr.end(K_P2G, st);
    pr.begin(K_NODES_VEL, st);
    k_nodes<DIM, 1><<<nb, 256, 0, st>>>(s, a.dt, a.damping);
    pr.end(K_NODES_VEL, st);
    pr.begin(K_G2P, st);
    if (a.flip)
      k_g2p<DIM, true, true><<<pb128, 128, 0, st>>>(s, a.dt, a.beta);
    else
      k_g2p<DIM, true, false><<<pb128, 128, 0, st>>>(s, a.dt, a.beta);
    pr.end(K_G2P, st);
  } else {  // USF
    pr.begin(K_P2G, st);
    k_p2g<DIM, false><<<pb256, 256, 0, st>>>(s, a.g[0], a.g[1], a.g[2]);
    pr.end(K_P2G, st);
    pr.begin(K_NODES_VEL, st);
    k_nodes<DIM, 0><<<nb, 256, 0, st>>>(s, a.dt, a.damping);
    pr.end(K_NODES_VEL, st);
    pr.begin(K_STRESS_FORCES, st);
    k_stress_forces<DIM><<<pb128, 128, 0, st>>>(s, a.dt, a.g[0], a.g[1], a.g[2]);
    pr.end(K_STRESS_FORCES, st);
    pr.begin(K_NODES_ACC, st);
    k_nodes<DIM, 2><<<nb, 256, 0, st>>>(s, a.dt, a.damping);
    pr.end(K_NODES_ACC, st);
    pr.begin(K_G2P, st);
    if (a.flip)
      k_g2p<DIM, false, true><<<pb128, 128, 0, st>>>(s, a.dt, a.beta);
    else
      k_g2p<DIM, false, false><<<pb128, 128, 0, st>>>(s, a.dt, a.beta);
    pr.end(K_G2P, st);
  }
  pr.begin(K_LOCATE, st);
  k_locate_fallback<DIM><<<148, 128, 0, st>>>(s, a.remove_lost);
  pr.end(K_LOCATE, st);
}

template <int DIM>
__global__ void k_material_batch(int64_t n, MaterialParams m, const double* stress,
                                 const double* dstrain, const double* density, double* state,
                                 double* out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double sg[6], de[6], sv[SV_N], o[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    sg[k] = stress[i * 6 + k];
    de[k] = dstrain[i * 6 + k];
  }
#pragma unroll
  for (int k = 0; k < SV_N; ++k) sv[k] = state[i * SV_N + k];
  material_compute_stress(m, sg, de, density[i], sv, o);
#pragma unroll
  for (int k = 0; k < 6; ++k) out[i * 6 + k] = o[k];
  if (m.type != 0)
#pragma unroll
    for (int k = 0; k < SV_N; ++k) state[i * SV_N + k] = sv[k];
}

}  // namespace

void launch_step_fp64(int dim, const DevState& s, const StepArgs& a, cudaStream_t st,
                      Profiler& prof) {
  if (dim == 2)
    step_impl<2>(s, a, st, prof);
  else
    step_impl<3>(s, a, st, prof);
}

void launch_material_batch_fp64(int dim, int64_t n, const MaterialParams& m, const double* stress,
                                const double* dstrain, const double* density, double* state,
                                double* out, cudaStream_t st) {
  if (n <= 0) return;
  if (dim == 2)
    k_material_batch<2><<<nblocks(n, 128), 128, 0, st>>>(n, m, stress, dstrain, density, state, out);
  else
    k_material_batch<3><<<nblocks(n, 128), 128, 0, st>>>(n, m, stress, dstrain, density, state, out);
}

}  // namespace mpm_b200
