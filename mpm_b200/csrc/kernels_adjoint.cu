// kernels_adjoint.cu -- reverse sweep of the FP64 USL step (discrete adjoint).
//
// Given the cotangents of the particle state after a step, the kernels here
// produce the cotangents of the state before it and add the step's
// contribution to the gradient of the material parameters.  Only four
// particle fields influence later positions and velocities on the USL
// FLIP/PIC path: the position x (through the shape functions), the velocity v
// (through the momentum map and the FLIP update), the stress sigma (through
// the internal force and the next return map) and the volume V (through the
// internal force).  Strain, F, displacement, density and the MohrCoulomb
// invariant state are outputs only; cells and yield branches are discrete.
// So the adjoint state is (x~, v~, sigma~, V~) per particle.
//
// One reversed step, in order (the forward kernels of the step -- sort, P2G,
// node update -- are first recomputed from the stored step-start state):
//   k_adj_material     elastic points: sigma~ = sigma~', deps~ = De sigma~',
//                      the parameters' share; plastic points listed
//   k_adj_return       plastic points: the return map's local Jacobian by
//                      forward-mode passes (two directions each) over the
//                      templated return map, contracted with sigma~'
//   k_adj_kinematics   G2P reverse: x~, v~, V~ of the step start and the
//                      per-particle coefficients of the node scatter
//   k_adj_scatter      the node cotangents (v~, a~) as cell-slot sums in
//                      particle id order (deterministic: no atomics)
//   k_adj_nodes        node update reverse: the node's (m, p, f_ext, f_int)
//                      cotangents by forward-mode passes over its inputs
//   k_adj_p2g          P2G reverse as a gather: each particle reads the
//                      cotangents of its cell's nodes
// Box cells of a tensor-product grid only (the second derivatives of the
// trilinear / bilinear shape functions are taken in closed form).
//
// Compiled with --fmad=false: the recomputed values are the FP64 step's bit
// for bit, so every branch follows the forward run.
#include <cuda_runtime.h>

#include <algorithm>

#include "mpm_device.cuh"
#include "mpm_dual.cuh"
#include "mpm_kernels.h"
#include "mpm_return.cuh"
#include "mpm_state.cuh"

namespace mpm_b200 {
namespace {

using D = Dual;
using MatD = MaterialT<Dual>;

inline unsigned nblk(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

template <int DIM>
struct AdjAt {  // offsets in AdjointArgs::adj (units of np); 2 DIM + NS + 1 fields
  static constexpr int X = 0, V = DIM, S = 2 * DIM, VOL = 2 * DIM + PF<DIM>::NS;
};
template <int DIM>
struct CoefAt {  // offsets in AdjointArgs::coef
  static constexpr int WV = 0, WA = DIM, SR = 2 * DIM, SRC = 2 * DIM + 6, N = 3 * DIM + 6;
};

__device__ __forceinline__ double& at(double* a, int f, int64_t np, int64_t p) {
  return a[(int64_t)f * np + p];
}

// The particle's box-cell geometry: local coordinates (and which axes sit on
// the clamp of local_xi, where they pass no derivative), node ids, 2 / len.
template <int DIM>
struct BoxPoint {
  double xi[DIM];
  bool free[DIM];  // xi_d not clamped
  double ihl[DIM];
  double dxi_dx[DIM];
  int nid[Elem<DIM>::NV];
};

template <int DIM>
__device__ __forceinline__ void box_point(const DevState& s, int c, const double* x, BoxPoint<DIM>& b) {
  const CellGeom& g = s.geom[c];
  local_xi<DIM>(x, g.centroid, g.len, b.xi);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const double r = 2. * (x[d] - g.centroid[d]) / g.len[d];
    b.free[d] = !(r < -1. + kDblEps) && !(r > 1. - kDblEps);
    b.dxi_dx[d] = 2. / g.len[d];
  }
  int ijk[3] = {0, 0, 0};
  cell_ijk<DIM>(s, c, ijk);
#pragma unroll
  for (int d = 0; d < DIM; ++d) b.ihl[d] = s.axis_ihl[d][ijk[d]];
  grid_cell_nodes<DIM>(s, c, b.nid);
}

// xi~ += N~ dN/dxi + sum_d G~_d dG_d/dxi for local node n (node_shape's
// polynomial: G_d is linear in every other coordinate and free of its own).
template <int DIM>
__device__ __forceinline__ void shape_reverse(const double* xi, int n, double Nbar, const double* G,
                                              const double* Gbar, double* xibar) {
  const double sx = off_i(n) ? 1. : -1., sy = off_j(n) ? 1. : -1.;
  const double a = 1. + sx * xi[0], b = 1. + sy * xi[1];
  if constexpr (DIM == 2) {
    const double e = 0.25;
    xibar[0] += Nbar * G[0] + Gbar[1] * (sx * sy * e);
    xibar[1] += Nbar * G[1] + Gbar[0] * (sx * sy * e);
  } else {
    const double sz = off_k(n) ? 1. : -1.;
    const double z = 1. + sz * xi[2];
    const double e = 0.125;
    xibar[0] += Nbar * G[0] + Gbar[1] * (sx * sy * e * z) + Gbar[2] * (sx * sz * e * b);
    xibar[1] += Nbar * G[1] + Gbar[0] * (sx * sy * e * z) + Gbar[2] * (sy * sz * e * a);
    xibar[2] += Nbar * G[2] + Gbar[0] * (sx * sz * e * b) + Gbar[1] * (sy * sz * e * a);
  }
}

// strain rate and centroid divergence of the USL stress update
// (stress_update's sums and 1e-15 snapping): sr (Voigt 6), src (DIM), and
// which entries survived the snapping
template <int DIM>
__device__ __forceinline__ void strain_rates(const DevState& s, int c, const BoxPoint<DIM>& b,
                                             double* sr, bool* sr_live, double* src, bool* src_live) {
  constexpr int NV = Elem<DIM>::NV;
  const int64_t nn = s.nn;
  const double* Dc = s.dndx_c + (int64_t)c * NV * DIM;
#pragma unroll
  for (int k = 0; k < 6; ++k) sr[k] = 0.;
#pragma unroll
  for (int k = 0; k < DIM; ++k) src[k] = 0.;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double vel[DIM], N, G[DIM], Dn[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) vel[d] = s.nf[(int64_t)(NF<DIM>::VEL + d) * nn + b.nid[i]];
    node_shape<DIM>(b.xi, i, N, G);
#pragma unroll
    for (int d = 0; d < DIM; ++d) Dn[d] = G[d] * b.ihl[d];
    double dc[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) dc[d] = Dc[i * DIM + d];
    if constexpr (DIM == 2) {
      sr[0] += Dn[0] * vel[0];
      sr[1] += Dn[1] * vel[1];
      sr[3] += Dn[1] * vel[0] + Dn[0] * vel[1];
      src[0] += dc[0] * vel[0];
      src[1] += dc[1] * vel[1];
    } else {
      sr[0] += Dn[0] * vel[0];
      sr[1] += Dn[1] * vel[1];
      sr[2] += Dn[2] * vel[2];
      sr[3] += Dn[1] * vel[0] + Dn[0] * vel[1];
      sr[4] += Dn[2] * vel[1] + Dn[1] * vel[2];
      sr[5] += Dn[2] * vel[0] + Dn[0] * vel[2];
      src[0] += dc[0] * vel[0];
      src[1] += dc[1] * vel[1];
      src[2] += dc[2] * vel[2];
    }
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    sr_live[k] = !(fabs(sr[k]) < 1.E-15);
    if (!sr_live[k]) sr[k] = 0.;
  }
#pragma unroll
  for (int k = 0; k < DIM; ++k) {
    src_live[k] = !(fabs(src[k]) < 1.E-15);
    if (!src_live[k]) src[k] = 0.;
  }
}

// ------------------------------------------------------------ material reverse
// Elastic points (LinearElastic, or a MohrCoulomb trial stress inside the
// yield surface): sigma' = sigma + De deps, so sigma~ = sigma~', deps~ =
// De sigma~' (De is symmetric) and the parameters receive sigma~' . dDe/dtheta
// deps.  A separated point (sigma' = 0) passes nothing.  Plastic points are
// listed with their inputs for k_adj_return.
template <int DIM>
__global__ void __launch_bounds__(128) k_adj_material(DevState s, AdjointArgs A, double dt) {
  constexpr int NS = PF<DIM>::NS;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0) return;
  const int64_t np = s.np;
  double x[DIM];
  load_x<DIM>(s, p, x);
  BoxPoint<DIM> b;
  box_point<DIM>(s, c, x, b);
  double sr[6], src[3];
  bool srl[6], srcl[3];
  strain_rates<DIM>(s, c, b, sr, srl, src, srcl);
  double dstrain[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) dstrain[k] = sr[k] * dt;
  double ssum = src[0];
#pragma unroll
  for (int k = 1; k < DIM; ++k) ssum = ssum + src[k];
  const double dvol = dt * ssum;
  const double rho = s.pf[(int64_t)PF<DIM>::RHO * np + p] / (1. + dvol);
  double sig[6] = {0, 0, 0, 0, 0, 0}, sbar[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    sig[k] = s.pf[(int64_t)(PF<DIM>::S + k) * np + p];
    sbar[k] = at(A.adj, AdjAt<DIM>::S + k, np, p);
  }
  const int slot = s.mat[p];
  const MaterialParams& mp = s.mats[slot];
  bool separated = false;
  if (mp.type != 0) {
    double sv[SV_N], out[6];
#pragma unroll
    for (int k = 0; k < SV_N; ++k) sv[k] = s.sv[(int64_t)k * np + p];
    if (mc_stress<double, double, true>(mp, sig, dstrain, rho, sv, sv[SV_PD], out) == MC_DEFERRED) {
      const unsigned i = defer_slot_by_cost(s, p);
      s.plist[i] = (int32_t)p;
#pragma unroll
      for (int k = 0; k < 6; ++k) s.pbuf[(int64_t)k * np + i] = dstrain[k];
      s.pbuf[(int64_t)6 * np + i] = rho;
#pragma unroll
      for (int k = 0; k < NS; ++k) A.dsbar[(int64_t)k * np + i] = sbar[k];
#pragma unroll
      for (int k = 0; k < 6; ++k) at(A.deps, k, np, p) = 0.;  // the return passes fill the rest
      return;
    }
    separated = sv[SV_YIELD] == 3.;
  }
  double deb[6] = {0, 0, 0, 0, 0, 0};
  if (separated) {
#pragma unroll
    for (int k = 0; k < NS; ++k) at(A.adj, AdjAt<DIM>::S + k, np, p) = 0.;
  } else {
    de_mul(mp, sbar, deb);
    // the parameters: d(De deps)/dtheta from the parameter-seeded material
    const MatD& mq = static_cast<const MatD*>(A.mats_param)[slot];
    D ded[6], o[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) ded[k] = D(dstrain[k]);
    de_mul(mq, ded, o);
#pragma unroll
    for (int q = 0; q < NT; ++q) {
      if (q >= A.nparams) break;
      double t = 0.;
#pragma unroll
      for (int k = 0; k < 6; ++k) t += sbar[k] * o[k].d[q];
      at(A.theta, q, np, p) += t;
    }
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) at(A.deps, k, np, p) = deb[k];
}

// Plastic points: the Jacobian of the return map (mc_compute_stress on Dual
// values, the function the forward step evaluated) with respect to the stress
// and strain-increment entries that vary, two columns per pass, contracted
// with sigma~'; one more pass with the parameter-seeded material and state.
// The passes of a point are independent, so each runs on its own thread (one
// thread per point and pass): the plastic points of a step are far fewer than
// the threads the GPU holds.  A pass writes only its own entries of sigma~,
// deps~ and theta; sigma~' comes from the copy taken when the point was listed.
template <int DIM>
struct ReturnPasses {
  static constexpr int NS = PF<DIM>::NS;
  static constexpr int NE = DIM == 2 ? 3 : 6;  // deps entries that vary (2D: xx, yy, xy)
  static constexpr int NIN = NS + NE;
  static constexpr int N = (NIN + 1) / 2 + 1;  // Jacobian passes + the parameter pass
};

template <int DIM>
__global__ void __launch_bounds__(128) k_adj_return(DevState s, AdjointArgs A) {
  using RP = ReturnPasses<DIM>;
  constexpr int NS = RP::NS, NIN = RP::NIN, NPASS = RP::N;
  constexpr int EIDX[6] = {0, 1, DIM == 2 ? 3 : 2, 3, 4, 5};
  const unsigned nl = *s.nplastic, n = nl + *s.nplastic_heavy;
  const int64_t np = s.np;
  const int64_t work = (int64_t)n * NPASS;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < work;
       w += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = list_slot(s, (unsigned)(w / NPASS), nl);
    const int pass = (int)(w % NPASS);
    const int64_t p = s.plist[i];
    const int slot = s.mat[p];
    const bool param = pass == NPASS - 1;
    if (param && A.nparams == 0) continue;
    D sg[6], dd[6], sv[SV_N], out[6];
    double sbar[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      sg[k] = D(k < NS ? s.pf[(int64_t)(PF<DIM>::S + k) * np + p] : 0.);
      dd[k] = D(s.pbuf[(int64_t)k * np + i]);
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) sbar[k] = A.dsbar[(int64_t)k * np + i];
#pragma unroll
    for (int k = 0; k < SV_N; ++k) sv[k] = D(s.sv[(int64_t)k * np + p]);
    const double rho = s.pbuf[(int64_t)6 * np + i];
    const MatD* mats = static_cast<const MatD*>(param ? A.mats_param : A.mats_zero);
    if (param) {
      const double* seed = A.sv_seed + (size_t)slot * SV_N * NT;
#pragma unroll
      for (int k = 0; k < SV_N; ++k)
#pragma unroll
        for (int q = 0; q < NT; ++q) sv[k].d[q] = seed[k * NT + q];
    } else {
      for (int l = 0; l < 2; ++l) {
        const int j = 2 * pass + l;
        if (j >= NIN) break;
        if (j < NS)
          sg[j].d[l] = 1.;
        else
          dd[EIDX[j - NS]].d[l] = 1.;
      }
    }
    int nc = 0;
    mc_return<D>(mats[slot], sg, dd, D(rho), sv, out, &nc);
    for (int l = 0; l < 2; ++l) {
      double t = 0.;
#pragma unroll
      for (int k = 0; k < NS; ++k) t += sbar[k] * out[k].d[l];
      if (param) {
        if (l < A.nparams) at(A.theta, l, np, p) += t;
        continue;
      }
      const int j = 2 * pass + l;
      if (j >= NIN) break;
      if (j < NS)
        at(A.adj, AdjAt<DIM>::S + j, np, p) = t;
      else
        at(A.deps, EIDX[j - NS], np, p) = t;
    }
  }
}

// --------------------------------------------------------- G2P kinematics
// x' = x + dt sum_i N_i v_i;  v' = beta (v + dt sum_i N_i a_i) + (1 - beta)
// sum_i N_i v_i (FLIP; PIC: v' = sum_i N_i v_i), constrained components set;
// V' = V (1 + dvol); deps from the strain rate at the step-start position.
template <int DIM, bool FLIP>
__global__ void __launch_bounds__(128) k_adj_kinematics(DevState s, AdjointArgs A, double dt,
                                                        double beta) {
  constexpr int NV = Elem<DIM>::NV;
  using AA = AdjAt<DIM>;
  using CC = CoefAt<DIM>;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0) return;
  const int64_t np = s.np, nn = s.nn;
  double x[DIM];
  load_x<DIM>(s, p, x);
  BoxPoint<DIM> b;
  box_point<DIM>(s, c, x, b);
  double sr[6], src[3];
  bool srl[6], srcl[3];
  strain_rates<DIM>(s, c, b, sr, srl, src, srcl);
  double ssum = src[0];
#pragma unroll
  for (int k = 1; k < DIM; ++k) ssum = ssum + src[k];
  const double dvol = dt * ssum;
  double xb[DIM], vb[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    xb[d] = at(A.adj, AA::X + d, np, p);
    vb[d] = at(A.adj, AA::V + d, np, p);
  }
  const int pv = s.pvc[p];
  if (pv >= 0) {
    const ParticleVC& r = s.pvcs[pv];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      if (r.mask & (1u << d)) vb[d] = 0.;
  }
  const double Vb = at(A.adj, AA::VOL, np, p);
  const double V = s.pf[(int64_t)PF<DIM>::VOL * np + p];
  double wv[DIM], wa[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    wv[d] = dt * xb[d] + (FLIP ? (1.0 - beta) * vb[d] : vb[d]);
    wa[d] = FLIP ? beta * dt * vb[d] : 0.;
  }
  double srb[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) srb[k] = srl[k] ? dt * at(A.deps, k, np, p) : 0.;
  const double dvolb = Vb * V;
  double srcb[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) srcb[d] = srcl[d] ? dt * dvolb : 0.;
  // x~ through the shape functions and their gradients
  double xib[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) xib[d] = 0.;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double vel[DIM], acc[DIM], N, G[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      vel[d] = s.nf[(int64_t)(NF<DIM>::VEL + d) * nn + b.nid[i]];
      acc[d] = FLIP ? s.nf[(int64_t)(NF<DIM>::ACC + d) * nn + b.nid[i]] : 0.;
    }
    node_shape<DIM>(b.xi, i, N, G);
    double Nb = 0.;
#pragma unroll
    for (int d = 0; d < DIM; ++d) Nb += wv[d] * vel[d] + wa[d] * acc[d];
    double Dnb[DIM], Gb[DIM];
    if constexpr (DIM == 2) {
      Dnb[0] = srb[0] * vel[0] + srb[3] * vel[1];
      Dnb[1] = srb[1] * vel[1] + srb[3] * vel[0];
    } else {
      Dnb[0] = srb[0] * vel[0] + srb[3] * vel[1] + srb[5] * vel[2];
      Dnb[1] = srb[1] * vel[1] + srb[3] * vel[0] + srb[4] * vel[2];
      Dnb[2] = srb[2] * vel[2] + srb[4] * vel[1] + srb[5] * vel[0];
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) Gb[d] = Dnb[d] * b.ihl[d];
    shape_reverse<DIM>(b.xi, i, Nb, G, Gb, xib);
  }
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    at(A.adj, AA::X + d, np, p) = xb[d] + (b.free[d] ? xib[d] * b.dxi_dx[d] : 0.);
    at(A.adj, AA::V + d, np, p) = FLIP ? beta * vb[d] : 0.;
    at(A.coef, CC::WV + d, np, p) = wv[d];
    at(A.coef, CC::WA + d, np, p) = wa[d];
    at(A.coef, CC::SRC + d, np, p) = srcb[d];
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) at(A.coef, CC::SR + k, np, p) = srb[k];
  at(A.adj, AA::VOL, np, p) = Vb * (1. + dvol);
}

// --------------------------------------------------- node cotangent scatter
// Cell-slot sums of the particles' contributions to the cotangents of the
// nodal velocity and acceleration: for slot k of cell c, over the cell's
// particles in id order (the order P2G sorted them into),
//   v~_k += N_k wv + (dN_k/dx)^T sr~ + dN_k/dx(centroid) src~,   a~_k += N_k wa.
// Tiles of 256 / NV cells, particle rows staged in shared memory as in P2G.
template <int DIM>
__global__ void __launch_bounds__(256) k_adj_scatter(DevState s, AdjointArgs A) {
  constexpr int NV = Elem<DIM>::NV;
  constexpr int T = 256;
  constexpr int CB = T / NV;
  using CC = CoefAt<DIM>;
  constexpr int XI = 0, CO = DIM, NR = DIM + CC::N;
  __shared__ double rows[NR][T];
  const int t = threadIdx.x;
  const int64_t c0 = (int64_t)blockIdx.x * CB;
  if (c0 >= s.ncells) return;
  const int64_t c1 = c0 + CB < s.ncells ? c0 + CB : s.ncells;
  const int64_t q_begin = s.start[c0], q_end = s.start[c1 - 1] + s.cnt[c1 - 1];
  if (q_begin == q_end) return;
  const int64_t c = c0 + t / NV;
  const int k = t % NV;
  const bool mine = c < c1;
  const int64_t a0 = mine ? s.start[c] : 0;
  const int64_t a1 = mine ? a0 + s.cnt[c] : 0;
  double ihl[DIM], dc[DIM];
  if (a1 > a0) {
    int ijk[3] = {0, 0, 0};
    cell_ijk<DIM>(s, (int)c, ijk);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      ihl[d] = s.axis_ihl[d][ijk[d]];
      dc[d] = s.dndx_c[((int64_t)c * NV + k) * DIM + d];
    }
  }
  const int64_t np = s.np;
  double vb[DIM], ab[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) vb[d] = ab[d] = 0.;
  for (int64_t q0 = q_begin; q0 < q_end; q0 += T) {
    if (q0 != q_begin) __syncthreads();
    if (q0 + t < q_end) {
      const int64_t p = s.order[q0 + t];
      const int pc = s.cell[p];
      double x[DIM], xi[DIM];
      load_x<DIM>(s, p, x);
      const CellGeom& g = s.geom[pc];
      local_xi<DIM>(x, g.centroid, g.len, xi);
#pragma unroll
      for (int d = 0; d < DIM; ++d) rows[XI + d][t] = xi[d];
#pragma unroll
      for (int f = 0; f < CC::N; ++f) rows[CO + f][t] = at(A.coef, f, np, p);
    }
    __syncthreads();
    const int64_t j0 = a0 > q0 ? a0 : q0;
    const int64_t j1 = a1 < q0 + T ? a1 : q0 + T;
    for (int64_t j = j0; j < j1; ++j) {
      const int r = (int)(j - q0);
      double xi[DIM], N, G[DIM], Dn[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) xi[d] = rows[XI + d][r];
      node_shape<DIM>(xi, k, N, G);
#pragma unroll
      for (int d = 0; d < DIM; ++d) Dn[d] = G[d] * ihl[d];
      const double* sb = &rows[CO + CC::SR][0];
      const auto SB = [&](int q) { return sb[q * T + r]; };
      double g[DIM];
      if constexpr (DIM == 2) {
        g[0] = Dn[0] * SB(0) + Dn[1] * SB(3);
        g[1] = Dn[1] * SB(1) + Dn[0] * SB(3);
      } else {
        g[0] = Dn[0] * SB(0) + Dn[1] * SB(3) + Dn[2] * SB(5);
        g[1] = Dn[1] * SB(1) + Dn[0] * SB(3) + Dn[2] * SB(4);
        g[2] = Dn[2] * SB(2) + Dn[1] * SB(4) + Dn[0] * SB(5);
      }
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        vb[d] += N * rows[CO + CC::WV + d][r] + g[d] + dc[d] * rows[CO + CC::SRC + d][r];
        ab[d] += N * rows[CO + CC::WA + d][r];
      }
    }
  }
  if (!mine || a1 == a0) return;
  double* out = A.apart + ((int64_t)c * NV + k) * (2 * DIM);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    out[d] = vb[d];
    out[DIM + d] = ab[d];
  }
}

// ------------------------------------------------------------- node reverse
// The USL node update (k_nodes<DIM, 1>: node.tcc:236-252 then :309-345) on
// Dual values, from the node's gathered (m, p, f_ext, f_int).
template <int DIM>
__device__ __forceinline__ void node_update_dual(const DevState& s, int bci, const D* sum, double dt,
                                                 double damping, D* vel, D* acc) {
  const D m = sum[0];
  if (m > 1.E-16) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) vel[d] = sum[1 + d] / m;
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      if (fabs(vel[d]) < 1.E-15) vel[d] = D(0.);
  }
  if (bci >= 0) apply_velocity_constraints<DIM>(s.bcs[bci], vel, acc);
  if (m > 1.0E-15) {
    D uf[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) uf[d] = sum[1 + DIM + d] + sum[1 + 2 * DIM + d];
    D ss = uf[0] * uf[0];
#pragma unroll
    for (int d = 1; d < DIM; ++d) ss = ss + uf[d] * uf[d];
    const D nrm = sqrt(ss);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const double sg = (vel[d] > 0.) ? 1. : ((vel[d] < 0.) ? -1. : 0.);
      acc[d] = (uf[d] - damping * nrm * sg) / m;
    }
    if (bci >= 0) {
      const NodeBC& bc = s.bcs[bci];
      if (bc.friction) apply_friction_constraints<DIM>(bc, vel, acc, dt);
      apply_acceleration_constraints<DIM>(bc, acc);
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) vel[d] += acc[d] * dt;
    if (bci >= 0) apply_velocity_constraints<DIM>(s.bcs[bci], vel, acc);
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      if (fabs(vel[d]) < 1.0E-15) vel[d] = D(0.);
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      if (fabs(acc[d]) < 1.0E-15) acc[d] = D(0.);
  }
}

// Sums of the cell-slot values of node n's cells in ascending cell id (the
// node kernel's order), from `src` with `nval` values per slot; false when no
// cell of the node holds particles.
template <int DIM>
__device__ __forceinline__ bool gather_slots(const DevState& s, const double* src, int nval, int64_t n,
                                             double* sum) {
  constexpr int NC = DIM == 2 ? 4 : 8;
  constexpr int NV = Elem<DIM>::NV;
  int cid[NC], slot[NC], count[NC];
  grid_node_cells<DIM>(s, (int)n, cid, slot, count);
  bool active = false;
#pragma unroll
  for (int q = 0; q < NC; ++q) {
    if (count[q] <= 0) continue;
    const double* v = src + ((int64_t)cid[q] * NV + slot[q]) * nval;
    for (int j = 0; j < nval; ++j) sum[j] = active ? sum[j] + v[j] : v[j];
    active = true;
  }
  return active;
}

template <int DIM>
__global__ void __launch_bounds__(128) k_adj_nodes(DevState s, AdjointArgs A, double dt, double damping) {
  constexpr int NVAL = PV<DIM>::N;
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= s.nn) return;
  const int64_t nn = s.nn;
  double vin[NVAL], ob[2 * DIM];
  if (!gather_slots<DIM>(s, s.partials, NVAL, n, vin)) return;
  gather_slots<DIM>(s, A.apart, 2 * DIM, n, ob);
  double ib[NVAL];
#pragma unroll
  for (int j = 0; j < NVAL; ++j) ib[j] = 0.;
  // nodes a particle only grazes pass no derivatives (as the tangent step)
  if (!(vin[0] < A.mass_floor)) {
    const int bci = s.bc_index[n];
    for (int j0 = 0; j0 < NVAL; j0 += 2) {
      D in[NVAL], vel[DIM], acc[DIM];
#pragma unroll
      for (int j = 0; j < NVAL; ++j) in[j] = D(vin[j]);
      in[j0].d[0] = 1.;
      if (j0 + 1 < NVAL) in[j0 + 1].d[1] = 1.;
      node_update_dual<DIM>(s, bci, in, dt, damping, vel, acc);
#pragma unroll
      for (int l = 0; l < 2; ++l) {
        if (j0 + l >= NVAL) break;
        double t = 0.;
#pragma unroll
        for (int d = 0; d < DIM; ++d) t += ob[d] * vel[d].d[l] + ob[DIM + d] * acc[d].d[l];
        ib[j0 + l] = t;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < NVAL; ++j) A.nbar[(int64_t)j * nn + n] = ib[j];
}

// ------------------------------------------------------------- P2G reverse
// Each particle gathers the cotangents of its cell's nodes (the reverse of
// P2G's scatter): m_i += m N_i, p_i += (m N_i) v, f_ext,i += (g m) N_i,
// f_int,i += -V (dN_i/dx . sigma) (particle.tcc:630-657, 893-949).
template <int DIM>
__global__ void __launch_bounds__(128) k_adj_p2g(DevState s, AdjointArgs A, double g0, double g1,
                                                 double g2) {
  constexpr int NV = Elem<DIM>::NV;
  constexpr int NS = PF<DIM>::NS;
  using AA = AdjAt<DIM>;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0) return;
  const int64_t np = s.np, nn = s.nn;
  const double gv[3] = {g0, g1, g2};
  double x[DIM];
  load_x<DIM>(s, p, x);
  BoxPoint<DIM> b;
  box_point<DIM>(s, c, x, b);
  const double m = s.pf[(int64_t)PF<DIM>::MASS * np + p];
  const double V = s.pf[(int64_t)PF<DIM>::VOL * np + p];
  double v[DIM], sig[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int d = 0; d < DIM; ++d) v[d] = s.pf[(int64_t)(PF<DIM>::V + d) * np + p];
#pragma unroll
  for (int k = 0; k < NS; ++k) sig[k] = s.pf[(int64_t)(PF<DIM>::S + k) * np + p];
  double vb[DIM], sb[6] = {0, 0, 0, 0, 0, 0}, Vb = 0., xib[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) vb[d] = xib[d] = 0.;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const int nd = b.nid[i];
    double mb = A.nbar[(int64_t)PV<DIM>::MASS * nn + nd];
    double pb[DIM], feb[DIM], fib[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      pb[d] = A.nbar[(int64_t)(PV<DIM>::MOM + d) * nn + nd];
      feb[d] = A.nbar[(int64_t)(PV<DIM>::FEXT + d) * nn + nd];
      fib[d] = A.nbar[(int64_t)(PV<DIM>::FINT + d) * nn + nd];
    }
    double N, G[DIM], Dn[DIM];
    node_shape<DIM>(b.xi, i, N, G);
#pragma unroll
    for (int d = 0; d < DIM; ++d) Dn[d] = G[d] * b.ihl[d];
    double Nb = m * mb;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      Nb += m * (pb[d] * v[d]) + m * (gv[d] * feb[d]);
      vb[d] += m * N * pb[d];
    }
    double f[DIM], Dnb[DIM];
    if constexpr (DIM == 2) {
      f[0] = Dn[0] * sig[0] + Dn[1] * sig[3];
      f[1] = Dn[1] * sig[1] + Dn[0] * sig[3];
      sb[0] += -V * (fib[0] * Dn[0]);
      sb[1] += -V * (fib[1] * Dn[1]);
      sb[3] += -V * (fib[0] * Dn[1] + fib[1] * Dn[0]);
      Dnb[0] = -V * (fib[0] * sig[0] + fib[1] * sig[3]);
      Dnb[1] = -V * (fib[0] * sig[3] + fib[1] * sig[1]);
    } else {
      f[0] = Dn[0] * sig[0] + Dn[1] * sig[3] + Dn[2] * sig[5];
      f[1] = Dn[1] * sig[1] + Dn[0] * sig[3] + Dn[2] * sig[4];
      f[2] = Dn[2] * sig[2] + Dn[1] * sig[4] + Dn[0] * sig[5];
      sb[0] += -V * (fib[0] * Dn[0]);
      sb[1] += -V * (fib[1] * Dn[1]);
      sb[2] += -V * (fib[2] * Dn[2]);
      sb[3] += -V * (fib[0] * Dn[1] + fib[1] * Dn[0]);
      sb[4] += -V * (fib[1] * Dn[2] + fib[2] * Dn[1]);
      sb[5] += -V * (fib[0] * Dn[2] + fib[2] * Dn[0]);
      Dnb[0] = -V * (fib[0] * sig[0] + fib[1] * sig[3] + fib[2] * sig[5]);
      Dnb[1] = -V * (fib[0] * sig[3] + fib[1] * sig[1] + fib[2] * sig[4]);
      Dnb[2] = -V * (fib[0] * sig[5] + fib[1] * sig[4] + fib[2] * sig[2]);
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) Vb += -(fib[d] * f[d]);
    double Gb[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) Gb[d] = Dnb[d] * b.ihl[d];
    shape_reverse<DIM>(b.xi, i, Nb, G, Gb, xib);
  }
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    if (b.free[d]) at(A.adj, AA::X + d, np, p) += xib[d] * b.dxi_dx[d];
    at(A.adj, AA::V + d, np, p) += vb[d];
  }
#pragma unroll
  for (int k = 0; k < NS; ++k) at(A.adj, AA::S + k, np, p) += sb[k];
  at(A.adj, AA::VOL, np, p) += Vb;
}

template <int DIM>
void adjoint_step(const DevState& s, const AdjointArgs& A, const StepArgs& a, cudaStream_t st,
                  Profiler& pr) {
  constexpr int NV = Elem<DIM>::NV;
  if (s.np == 0) return;
  const unsigned pb = nblk(s.np, 128);
  if (s.sv) cudaMemsetAsync(s.nplastic, 0, 2 * sizeof(unsigned), st);  // and nplastic_heavy
  pr.begin(K_ADJ_MATERIAL, st);
  k_adj_material<DIM><<<pb, 128, 0, st>>>(s, A, a.dt);
  pr.end(K_ADJ_MATERIAL, st);
  if (s.sv) {
    pr.begin(K_ADJ_RETURN, st);
    const unsigned mcb =
        (unsigned)std::min<int64_t>(nblk(s.np * ReturnPasses<DIM>::N, 128), 148 * 16);
    k_adj_return<DIM><<<mcb, 128, 0, st>>>(s, A);
    pr.end(K_ADJ_RETURN, st);
  }
  pr.begin(K_ADJ_KINEMATICS, st);
  if (a.flip)
    k_adj_kinematics<DIM, true><<<pb, 128, 0, st>>>(s, A, a.dt, a.beta);
  else
    k_adj_kinematics<DIM, false><<<pb, 128, 0, st>>>(s, A, a.dt, a.beta);
  pr.end(K_ADJ_KINEMATICS, st);
  pr.begin(K_ADJ_SCATTER, st);
  k_adj_scatter<DIM><<<nblk(s.ncells, 256 / NV), 256, 0, st>>>(s, A);
  pr.end(K_ADJ_SCATTER, st);
  pr.begin(K_ADJ_NODES, st);
  k_adj_nodes<DIM><<<nblk(s.nn, 128), 128, 0, st>>>(s, A, a.dt, a.damping);
  pr.end(K_ADJ_NODES, st);
  pr.begin(K_ADJ_P2G, st);
  k_adj_p2g<DIM><<<pb, 128, 0, st>>>(s, A, a.g[0], a.g[1], a.g[2]);
  pr.end(K_ADJ_P2G, st);
}

}  // namespace

void launch_adjoint_step(int dim, const DevState& s, const AdjointArgs& A, const StepArgs& a,
                         cudaStream_t st, Profiler& prof) {
  if (dim == 2)
    adjoint_step<2>(s, A, a, st, prof);
  else
    adjoint_step<3>(s, A, a, st, prof);
}

}  // namespace mpm_b200
