// kernels_tangent.cu -- the FP64 USL step carrying tangents: every particle,
// node and cell-slot quantity is a Dual (value + derivatives with respect to
// NT material parameters), so a run yields, besides its state, the exact
// derivatives of that state with respect to the parameters (forward-mode
// differentiation of the whole step: P2G, node update with its boundary
// conditions, G2P, strain, volume, MohrCoulomb return).  Values are computed
// with the operations of the FP64 step (kernels_fp64.cu), derivatives by the
// chain rule; discrete decisions (cell, yield state, boundary branches) follow
// the values.
//
// Value arrays keep the FP64 layout (DevState::pf, sv, nf, partials); the
// derivative k of each lives in the same layout in pft[k], svt[k], nft[k],
// partt[k].  P2G runs by cell tiles, one thread per cell slot holding 1 + 3 DIM
// Dual sums.
#include <cuda_runtime.h>

#include <algorithm>

#include "mpm_device.cuh"
#include "mpm_dual.cuh"
#include "mpm_kernels.h"
#include "mpm_return.cuh"
#include "mpm_state.cuh"

#ifndef MPM_TANGENT_G2P_MIN_BLOCKS
#define MPM_TANGENT_G2P_MIN_BLOCKS 1  // the stress part
#endif
#ifndef MPM_TANGENT_NODES_MIN_BLOCKS
#define MPM_TANGENT_NODES_MIN_BLOCKS 4  // 128 registers: 0.054 -> 0.045 ms at 256k particles
#endif
#ifndef MPM_TANGENT_RETURN_MIN_BLOCKS
#define MPM_TANGENT_RETURN_MIN_BLOCKS 1
#endif
#ifndef MPM_TANGENT_KIN_MIN_BLOCKS
#define MPM_TANGENT_KIN_MIN_BLOCKS 5  // the kinematics part (6 spills and is slower)
#endif
#ifndef MPM_TANGENT_P2G_MIN_BLOCKS
#define MPM_TANGENT_P2G_MIN_BLOCKS 4  // 128 registers on a grid, no spills
#endif

namespace mpm_b200 {
namespace {

using D = Dual;
using MatD = MaterialT<Dual>;

__device__ __forceinline__ D ld(const double* v, double* const* t, int64_t i) {
  D r;
  r.v = v[i];
#pragma unroll
  for (int k = 0; k < NT; ++k) r.d[k] = t[k][i];
  return r;
}
__device__ __forceinline__ void st(double* v, double* const* t, int64_t i, const D& x) {
  v[i] = x.v;
#pragma unroll
  for (int k = 0; k < NT; ++k) t[k][i] = x.d[k];
}
template <int DIM>
__device__ __forceinline__ D pfield(const DevState& s, int f, int64_t p) {
  return ld(s.pf, s.pft, (int64_t)f * s.np + p);
}
template <int DIM>
__device__ __forceinline__ void set_pfield(const DevState& s, int f, int64_t p, const D& x) {
  st(s.pf, const_cast<double* const*>(s.pft), (int64_t)f * s.np + p, x);
}

// local coordinate (local_xi's arithmetic on the value)
template <int DIM>
__device__ __forceinline__ void xi_dual(const CellGeom& g, const D* x, D* xi) {
#pragma unroll
  for (int i = 0; i < DIM; ++i) {
    D v = 2. * (x[i] - g.centroid[i]) / g.len[i];
    if (v < -1. + kDblEps) v = D(-1. + kDblEps);
    if (v > 1. - kDblEps) v = D(1. - kDblEps);
    xi[i] = v;
  }
}

// J^-1 at xi for constant nodal coordinates (jacobian_inverse's sums)
template <int DIM>
__device__ __forceinline__ void jinv_dual(const D* xi, const double* X, D* inv) {
  constexpr int NV = Elem<DIM>::NV;
  D G[NV * DIM];
  grad_shapefn<DIM>(xi, G);
  D J[DIM * DIM];
#pragma unroll
  for (int r = 0; r < DIM; ++r)
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      D a = G[0 * DIM + r] * X[0 * DIM + c];
#pragma unroll
      for (int n = 1; n < NV; ++n) a = a + G[n * DIM + r] * X[n * DIM + c];
      J[r * DIM + c] = a;
    }
  inverse<DIM>(J, inv);
}

// dN/dx of one local node from its natural gradient G at the particle, with
// the FP64 step's operations: box cells of a tensor-product grid take
// dN/dxi * (2 / len) per axis (CellMap<DIM, true>: ihl), other cells
// J^-1 at xi (inv).
template <int DIM, bool BOX>
__device__ __forceinline__ void grad_dual(const D* G, const double* ihl, const D* inv, D* Dn) {
#pragma unroll
  for (int q = 0; q < DIM; ++q) {
    if constexpr (BOX) {
      Dn[q] = G[q] * ihl[q];
    } else {
      D a = G[0] * inv[q * DIM + 0];
#pragma unroll
      for (int e = 1; e < DIM; ++e) a = a + G[e] * inv[q * DIM + e];
      Dn[q] = a;
    }
  }
}

// ---------------------------------------------------------------- P2G tiles
// k_p2g_tiles on Dual values: a block takes tangent_tile_t / NV consecutive
// cells, stages their particles (local coordinates, velocity, -V, stress and,
// off a tensor-product grid, J^-1, each a Dual of 1 + NT doubles, and the
// mass) in shared memory, and thread (cell, slot k) adds its slot's
// contributions in particle id order.  N and dN/dx of slot k come from
// node_shape with the FP64 tiles' operations, so the values are the FP64
// step's bit for bit.
template <bool BOX>
constexpr int tangent_tile_t() { return BOX ? 128 : 64; }

template <int DIM, bool BOX>
__global__ void __launch_bounds__(tangent_tile_t<BOX>(), MPM_TANGENT_P2G_MIN_BLOCKS)
    k_p2g_tiles_tangent(DevState s, double g0, double g1, double g2) {
  constexpr int NV = Elem<DIM>::NV;
  constexpr int T = tangent_tile_t<BOX>();
  constexpr int CB = T / NV;
  constexpr int NVAL = 1 + 3 * DIM;
  constexpr int MASS = 0, MOM = 1, FEXT = 1 + DIM, FINT = 1 + 2 * DIM;
  constexpr int NS = PF<DIM>::NS;
  constexpr int W = 1 + NT;  // doubles per staged Dual
  constexpr int R_XI = 0, R_V = DIM, R_SC = 2 * DIM, R_S = 2 * DIM + 1, R_INV = R_S + NS;
  constexpr int NDUAL = R_INV + (BOX ? 0 : DIM * DIM);
  __shared__ double rows[NDUAL * W + 1][T];  // the last row: mass
  auto put = [&](int f, int t, const D& x) {
    rows[f * W][t] = x.v;
#pragma unroll
    for (int q = 0; q < NT; ++q) rows[f * W + 1 + q][t] = x.d[q];
  };
  auto get = [&](int f, int r) {
    D x;
    x.v = rows[f * W][r];
#pragma unroll
    for (int q = 0; q < NT; ++q) x.d[q] = rows[f * W + 1 + q][r];
    return x;
  };
  const int t = threadIdx.x;
  const int64_t c0 = (int64_t)blockIdx.x * CB;
  if (c0 >= s.ncells) return;
  const int64_t c1 = c0 + CB < s.ncells ? c0 + CB : s.ncells;
  const int64_t q_begin = s.start[c0], q_end = s.start[c1 - 1] + s.cnt[c1 - 1];
  if (q_begin == q_end) return;  // no particles in the tile (the whole block)
  const int64_t c = c0 + t / NV;
  const int k = t % NV;
  const bool mine = c < c1;
  const int64_t a0 = mine ? s.start[c] : 0;
  const int64_t a1 = mine ? a0 + s.cnt[c] : 0;
  sort_cell_ids<NV>(s.order + a0, (int)(a1 - a0), k);  // ascending particle ids
  double ihl[DIM];  // J^-1 of a box cell
  if constexpr (BOX) {
    int ijk[3] = {0, 0, 0};
    if (a1 > a0) cell_ijk<DIM>(s, (int)c, ijk);
#pragma unroll
    for (int d = 0; d < DIM; ++d) ihl[d] = a1 > a0 ? s.axis_ihl[d][ijk[d]] : 0.;
  }
  const double gv[3] = {g0, g1, g2};
  const int64_t np = s.np;
  D acc[NVAL];
  for (int64_t q0 = q_begin; q0 < q_end; q0 += T) {
    if (q0 != q_begin) __syncthreads();  // the previous chunk is consumed
    if (q0 + t < q_end) {
      const int64_t p = s.order[q0 + t];
      const int pc = s.cell[p];
      D x[DIM], xi[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) x[d] = pfield<DIM>(s, PF<DIM>::X + d, p);
      xi_dual<DIM>(s.geom[pc], x, xi);
#pragma unroll
      for (int d = 0; d < DIM; ++d) put(R_XI + d, t, xi[d]);
#pragma unroll
      for (int d = 0; d < DIM; ++d) put(R_V + d, t, pfield<DIM>(s, PF<DIM>::V + d, p));
      put(R_SC, t, -1. * pfield<DIM>(s, PF<DIM>::VOL, p));
#pragma unroll
      for (int q = 0; q < NS; ++q) put(R_S + q, t, pfield<DIM>(s, PF<DIM>::S + q, p));
      rows[NDUAL * W][t] = s.pf[(int64_t)PF<DIM>::MASS * np + p];  // the mass carries no tangent
      if constexpr (!BOX) {
        int nid[NV];
        double X[NV * DIM];
        D inv[DIM * DIM];
        cell_nodes_coords<DIM>(s, pc, nid, X);
        jinv_dual<DIM>(xi, X, inv);
#pragma unroll
        for (int q = 0; q < DIM * DIM; ++q) put(R_INV + q, t, inv[q]);
      }
    }
    __syncthreads();
    const int64_t j0 = a0 > q0 ? a0 : q0;
    const int64_t j1 = a1 < q0 + T ? a1 : q0 + T;
    for (int64_t j = j0; j < j1; ++j) {
      const int r = (int)(j - q0);
      D xi[DIM], Nk, G[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) xi[d] = get(R_XI + d, r);
      node_shape<DIM>(xi, k, Nk, G);
      const double m = rows[NDUAL * W][r];
      const D mN = m * Nk;
      acc[MASS] += mN;
#pragma unroll
      for (int d = 0; d < DIM; ++d) acc[MOM + d] += mN * get(R_V + d, r);
#pragma unroll
      for (int d = 0; d < DIM; ++d) acc[FEXT + d] += (gv[d] * m) * Nk;
      D Dn[DIM];
      if constexpr (BOX) {
#pragma unroll
        for (int q = 0; q < DIM; ++q) Dn[q] = G[q] * ihl[q];
      } else {
#pragma unroll
        for (int q = 0; q < DIM; ++q) {
          D a = G[0] * get(R_INV + q * DIM + 0, r);
#pragma unroll
          for (int e = 1; e < DIM; ++e) a = a + G[e] * get(R_INV + q * DIM + e, r);
          Dn[q] = a;
        }
      }
      D sig[6];
#pragma unroll
      for (int q = 0; q < NS; ++q) sig[q] = get(R_S + q, r);
      const D sc = get(R_SC, r);
      D f[DIM];
      if constexpr (DIM == 2) {
        f[0] = Dn[0] * sig[0] + Dn[1] * sig[3];
        f[1] = Dn[1] * sig[1] + Dn[0] * sig[3];
      } else {
        f[0] = Dn[0] * sig[0] + Dn[1] * sig[3] + Dn[2] * sig[5];
        f[1] = Dn[1] * sig[1] + Dn[0] * sig[3] + Dn[2] * sig[4];
        f[2] = Dn[2] * sig[2] + Dn[1] * sig[4] + Dn[0] * sig[5];
      }
#pragma unroll
      for (int d = 0; d < DIM; ++d) acc[FINT + d] += f[d] * sc;
    }
  }
  if (!mine || a1 == a0) return;  // empty cells keep no partials
  const int64_t o = ((int64_t)c * NV + k) * NVAL;
#pragma unroll
  for (int v = 0; v < NVAL; ++v) st(s.partials, const_cast<double* const*>(s.partt), o + v, acc[v]);
}

// ---------------------------------------------------------------- node update
template <int DIM>
__device__ __forceinline__ bool gather_node_tangent(const DevState& s, int64_t node, D* sum) {
  constexpr int NV = Elem<DIM>::NV;
  constexpr int NVAL = 1 + 3 * DIM;
  bool active = false;
  auto add = [&](int c, int slot) {
    const int64_t o = ((int64_t)c * NV + slot) * NVAL;
    // the row of values and of each derivative, loaded in pairs where aligned
    double val[NVAL], der[NT][NVAL];
    load_partial_row<double, NVAL, 0, NVAL>(s.partials + o, val);
#pragma unroll
    for (int k = 0; k < NT; ++k) load_partial_row<double, NVAL, 0, NVAL>(s.partt[k] + o, der[k]);
#pragma unroll
    for (int v = 0; v < NVAL; ++v) {
      D x;
      x.v = val[v];
#pragma unroll
      for (int k = 0; k < NT; ++k) x.d[k] = der[k][v];
      sum[v] = active ? sum[v] + x : x;
    }
    active = true;
  };
  if (s.structured) {
    constexpr int NC = DIM == 2 ? 4 : 8;
    int cid[NC], slot[NC], count[NC];
    grid_node_cells<DIM>(s, (int)node, cid, slot, count);
#pragma unroll
    for (int q = 0; q < NC; ++q)
      if (count[q] > 0) add(cid[q], slot[q]);
  } else {
    for (int e = s.nc_off[node]; e < s.nc_off[node + 1]; ++e)
      if (s.cnt[s.nc_cell[e]] > 0) add(s.nc_cell[e], s.nc_slot[e]);
  }
  return active;
}

// USL node update (node.tcc:236-252 then :309-345) on Dual values
template <int DIM>
__global__ void __launch_bounds__(128, MPM_TANGENT_NODES_MIN_BLOCKS) k_nodes_tangent(DevState s, double dt, double damping) {
  constexpr int NVAL = 1 + 3 * DIM;
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= s.nn) return;
  const int64_t nn = s.nn;
  D sum[NVAL];
  if (!gather_node_tangent<DIM>(s, n, sum)) return;
  const int bci = s.bc_index[n];
  const D m = sum[0];
  D vel[DIM], acc[DIM];
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
  // A node that a particle only grazes (it just entered the node's cells) has
  // a mass many orders below a particle's; the quotient rule for momentum /
  // mass then subtracts two nearly equal derivatives and divides by that mass,
  // and the rounding error, amplified by 1 / mass, reaches the particles
  // through dN/dx (which is not small there).  Such nodes keep their values
  // and pass no derivatives.
  if (m.v < s.tangent_mass_floor) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      vel[d] = D(vel[d].v);
      acc[d] = D(acc[d].v);
    }
  }
  double* const* t = const_cast<double* const*>(s.nft);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    st(s.nf, t, (int64_t)(NF<DIM>::VEL + d) * nn + n, vel[d]);
    st(s.nf, t, (int64_t)(NF<DIM>::ACC + d) * nn + n, acc[d]);
  }
}

// --------------------------------------------------------------------- G2P
// stress_update of the FP64 step on Dual values (strain, F, volume, density,
// material; plastic MohrCoulomb points deferred to k_mc_return_tangent), then
// k_g2p<DIM, true, FLIP>'s kinematics and locate: two kernels, so that the
// register-heavy Dual material update does not hold the kinematics to its
// occupancy.  The stress kernel runs first: both work at the step-start
// position.
template <int DIM, bool BOX>
__global__ void __launch_bounds__(128, MPM_TANGENT_G2P_MIN_BLOCKS) k_stress_tangent(DevState s, double dt) {
  constexpr int NV = Elem<DIM>::NV;
  constexpr int NS = PF<DIM>::NS;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0) return;
  const int64_t nn = s.nn;
  double* const* nt = s.nft;
  const int64_t np = s.np;
  D x[DIM], xi[DIM];
  int nid[NV];
  double X[NV * DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) x[d] = pfield<DIM>(s, PF<DIM>::X + d, p);
  xi_dual<DIM>(s.geom[c], x, xi);  // at the step-start position
  cell_nodes_coords<DIM>(s, c, nid, X);
  // stress update (mpm_scheme.tcc:75-103) with dN/dx at the particle, one
  // node at a time
  double ihl[DIM];
  D inv[DIM * DIM];
  if constexpr (BOX) {
    int ijk[3] = {0, 0, 0};
    cell_ijk<DIM>(s, c, ijk);
#pragma unroll
    for (int d = 0; d < DIM; ++d) ihl[d] = s.axis_ihl[d][ijk[d]];
  } else {
    jinv_dual<DIM>(xi, X, inv);
  }
  const double* Dc = s.dndx_c + (int64_t)c * NV * DIM;
  D Fi[DIM * DIM];
#pragma unroll
  for (int r = 0; r < DIM; ++r) Fi[r * DIM + r] = D(1.);
  D sr[6], src[3];
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    D vel[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) vel[d] = ld(s.nf, nt, (int64_t)(NF<DIM>::VEL + d) * nn + nid[i]);
    D Ni, G[DIM], Dn[DIM];
    node_shape<DIM>(xi, i, Ni, G);
    grad_dual<DIM, BOX>(G, ihl, inv, Dn);
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
      for (int q = 0; q < DIM; ++q) Fi[r * DIM + q] += vel[r] * Dn[q] * dt;
    if constexpr (DIM == 2) {
      sr[0] += Dn[0] * vel[0];
      sr[1] += Dn[1] * vel[1];
      sr[3] += Dn[1] * vel[0] + Dn[0] * vel[1];
      src[0] += Dc[i * DIM + 0] * vel[0];
      src[1] += Dc[i * DIM + 1] * vel[1];
    } else {
      sr[0] += Dn[0] * vel[0];
      sr[1] += Dn[1] * vel[1];
      sr[2] += Dn[2] * vel[2];
      sr[3] += Dn[1] * vel[0] + Dn[0] * vel[1];
      sr[4] += Dn[2] * vel[1] + Dn[1] * vel[2];
      sr[5] += Dn[2] * vel[0] + Dn[0] * vel[2];
      src[0] += Dc[i * DIM + 0] * vel[0];
      src[1] += Dc[i * DIM + 1] * vel[1];
      src[2] += Dc[i * DIM + 2] * vel[2];
    }
  }
#pragma unroll
  for (int r = 0; r < DIM; ++r)
#pragma unroll
    for (int q = 0; q < DIM; ++q) {
      if (r != q && fabs(Fi[r * DIM + q]) < 1.E-15) Fi[r * DIM + q] = D(0.);
      if (r == q && fabs(Fi[r * DIM + q] - 1.) < 1.E-15) Fi[r * DIM + q] = D(1.);
    }
#pragma unroll
  for (int k = 0; k < 6; ++k)
    if (fabs(sr[k]) < 1.E-15) sr[k] = D(0.);
#pragma unroll
  for (int k = 0; k < DIM; ++k)
    if (fabs(src[k]) < 1.E-15) src[k] = D(0.);
  D dstrain[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) dstrain[k] = sr[k] * dt;
  D ssum = src[0];
#pragma unroll
  for (int k = 1; k < DIM; ++k) ssum = ssum + src[k];
  const D dvol = dt * ssum;
  if constexpr (DIM == 2) {
    const int map[3] = {0, 1, 3};
#pragma unroll
    for (int k = 0; k < 3; ++k)
      set_pfield<DIM>(s, PF<2>::E + k, p, pfield<DIM>(s, PF<2>::E + k, p) + dstrain[map[k]]);
  } else {
#pragma unroll
    for (int k = 0; k < 6; ++k)
      set_pfield<DIM>(s, PF<3>::E + k, p, pfield<DIM>(s, PF<3>::E + k, p) + dstrain[k]);
  }
  const D vol = pfield<DIM>(s, PF<DIM>::VOL, p) * (1. + dvol);
  const D rho = pfield<DIM>(s, PF<DIM>::RHO, p) / (1. + dvol);
  set_pfield<DIM>(s, PF<DIM>::VOL, p, vol);
  set_pfield<DIM>(s, PF<DIM>::RHO, p, rho);
  // F update (independent of the stress; done first so that Fi is not live
  // through the material update)
  if constexpr (DIM == 2) {
    D F[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) F[k] = pfield<DIM>(s, PF<2>::F + k, p);
    set_pfield<DIM>(s, PF<2>::F + 0, p, Fi[0] * F[0] + Fi[1] * F[2]);
    set_pfield<DIM>(s, PF<2>::F + 1, p, Fi[0] * F[1] + Fi[1] * F[3]);
    set_pfield<DIM>(s, PF<2>::F + 2, p, Fi[2] * F[0] + Fi[3] * F[2]);
    set_pfield<DIM>(s, PF<2>::F + 3, p, Fi[2] * F[1] + Fi[3] * F[3]);
  } else {
    D F[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) F[k] = pfield<DIM>(s, PF<3>::F + k, p);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int q = 0; q < 3; ++q)
        set_pfield<DIM>(s, PF<3>::F + a * 3 + q, p,
                        (Fi[a * 3 + 0] * F[0 * 3 + q] + Fi[a * 3 + 1] * F[1 * 3 + q]) +
                            Fi[a * 3 + 2] * F[2 * 3 + q]);
  }
  D sig[6];
#pragma unroll
  for (int k = 0; k < NS; ++k) sig[k] = pfield<DIM>(s, PF<DIM>::S + k, p);
  const MatD& mp = static_cast<const MatD*>(s.mats_t)[s.mat[p]];
  D out[6];
  bool deferred = false;
  if (mp.type == 0) {
    D tt[6];
    de_mul(mp, dstrain, tt);
#pragma unroll
    for (int i = 0; i < 6; ++i) out[i] = sig[i] + tt[i];
  } else {
    D sv[SV_N];
#pragma unroll
    for (int k = 0; k < SV_N; ++k) sv[k] = ld(s.sv, s.svt, (int64_t)k * np + p);
    if (mc_stress<D, D, true>(mp, sig, dstrain, rho, sv, sv[SV_PD], out) == MC_DEFERRED) {
      // plastic: k_mc_return_tangent runs the update from the unchanged state
      deferred = true;
      const unsigned i = defer_slot(s);
      s.plist[i] = (int32_t)p;
      for (int k = 0; k < 7; ++k) {
        const D v = k < 6 ? dstrain[k] : rho;
        s.tpbuf[(int64_t)(k * (1 + NT)) * np + i] = v.v;
#pragma unroll
        for (int q = 0; q < NT; ++q) s.tpbuf[(int64_t)(k * (1 + NT) + 1 + q) * np + i] = v.d[q];
      }
    } else {
#pragma unroll
      for (int k = 0; k < SV_N; ++k) st(s.sv, const_cast<double* const*>(s.svt), (int64_t)k * np + p, sv[k]);
    }
  }
  if (!deferred) {
#pragma unroll
    for (int k = 0; k < NS; ++k) set_pfield<DIM>(s, PF<DIM>::S + k, p, out[k]);
  }
}

template <int DIM, bool FLIP>
__global__ void __launch_bounds__(128, MPM_TANGENT_KIN_MIN_BLOCKS) k_g2p_tangent(DevState s, double dt, double beta) {
  constexpr int NV = Elem<DIM>::NV;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0) return;
  const int64_t nn = s.nn;
  double* const* nt = s.nft;
  D x[DIM], xi[DIM], N[NV];
  int nid[NV];
#pragma unroll
  for (int d = 0; d < DIM; ++d) x[d] = pfield<DIM>(s, PF<DIM>::X + d, p);
  xi_dual<DIM>(s.geom[c], x, xi);  // at the step-start position
  shapefn<DIM>(xi, N);
  if (s.structured) {
    grid_cell_nodes<DIM>(s, c, nid);
  } else {
#pragma unroll
    for (int n = 0; n < NV; ++n) nid[n] = s.cell_nodes[(int64_t)c * NV + n];
  }
  D nvel[DIM], nacc[DIM];
#pragma unroll
  for (int i = 0; i < NV; ++i) {
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      nvel[d] += N[i] * ld(s.nf, nt, (int64_t)(NF<DIM>::VEL + d) * nn + nid[i]);
    if constexpr (FLIP) {
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        nacc[d] += N[i] * ld(s.nf, nt, (int64_t)(NF<DIM>::ACC + d) * nn + nid[i]);
    }
  }
  D v[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) v[d] = pfield<DIM>(s, PF<DIM>::V + d, p);
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
    const D xd = x[d] + nvel[d] * dt;
    xn[d] = xd.v;
    set_pfield<DIM>(s, PF<DIM>::X + d, p, xd);
    set_pfield<DIM>(s, PF<DIM>::U + d, p, pfield<DIM>(s, PF<DIM>::U + d, p) + nvel[d] * dt);
  }
  const int pv = s.pvc[p];
  if (pv >= 0) {
    const ParticleVC& r = s.pvcs[pv];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      if (r.mask & (1u << d)) v[d] = D(r.value[d]);
  }
#pragma unroll
  for (int d = 0; d < DIM; ++d) set_pfield<DIM>(s, PF<DIM>::V + d, p, v[d]);

  // locate on the values
  bool finite = true;
#pragma unroll
  for (int d = 0; d < DIM; ++d) finite = finite && (xn[d] - xn[d] == 0.0);
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

// the MohrCoulomb returns deferred by k_stress_tangent (dense, grid-stride)
template <int DIM>
__global__ void __launch_bounds__(128, MPM_TANGENT_RETURN_MIN_BLOCKS) k_mc_return_tangent(DevState s) {
  const unsigned n = *s.nplastic;
  const int64_t np = s.np;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int64_t p = s.plist[i];
    D sig[6], de[6], sv[SV_N], out[6], rho;
#pragma unroll
    for (int k = 0; k < PF<DIM>::NS; ++k) sig[k] = pfield<DIM>(s, PF<DIM>::S + k, p);
    for (int k = 0; k < 7; ++k) {
      D v;
      v.v = s.tpbuf[(int64_t)(k * (1 + NT)) * np + i];
#pragma unroll
      for (int q = 0; q < NT; ++q) v.d[q] = s.tpbuf[(int64_t)(k * (1 + NT) + 1 + q) * np + i];
      if (k < 6)
        de[k] = v;
      else
        rho = v;
    }
#pragma unroll
    for (int k = 0; k < SV_N; ++k) sv[k] = ld(s.sv, s.svt, (int64_t)k * np + p);
    const MatD& mp = static_cast<const MatD*>(s.mats_t)[s.mat[p]];
    int nc = 0;
    mc_return<D>(mp, sig, de, rho, sv, out, &nc);
#pragma unroll
    for (int k = 0; k < SV_N; ++k) st(s.sv, const_cast<double* const*>(s.svt), (int64_t)k * np + p, sv[k]);
#pragma unroll
    for (int k = 0; k < PF<DIM>::NS; ++k) set_pfield<DIM>(s, PF<DIM>::S + k, p, out[k]);
  }
}

inline unsigned nblk(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

template <int DIM>
void step_tangent(const DevState& s, const StepArgs& a, cudaStream_t st, Profiler& pr) {
  constexpr int NV = Elem<DIM>::NV;
  if (s.np == 0) return;
  cudaMemsetAsync(s.nlost, 0, sizeof(unsigned), st);
  if (s.sv) cudaMemsetAsync(s.nplastic, 0, sizeof(unsigned), st);
  pr.begin(K_SORT, st, SORT_KERNELS);
  counting_sort(s, st);
  pr.end(K_SORT, st);
  pr.begin(K_P2G, st);
  if (s.structured)
    k_p2g_tiles_tangent<DIM, true><<<nblk(s.ncells, tangent_tile_t<true>() / NV),
                                     tangent_tile_t<true>(), 0, st>>>(s, a.g[0], a.g[1], a.g[2]);
  else
    k_p2g_tiles_tangent<DIM, false><<<nblk(s.ncells, tangent_tile_t<false>() / NV),
                                      tangent_tile_t<false>(), 0, st>>>(s, a.g[0], a.g[1], a.g[2]);
  pr.end(K_P2G, st);
  pr.begin(K_NODES_VEL, st);
  k_nodes_tangent<DIM><<<nblk(s.nn, 128), 128, 0, st>>>(s, a.dt, a.damping);
  pr.end(K_NODES_VEL, st);
  pr.begin(K_G2P, st, 2);
  if (s.structured)
    k_stress_tangent<DIM, true><<<nblk(s.np, 128), 128, 0, st>>>(s, a.dt);
  else
    k_stress_tangent<DIM, false><<<nblk(s.np, 128), 128, 0, st>>>(s, a.dt);
  if (a.flip)
    k_g2p_tangent<DIM, true><<<nblk(s.np, 128), 128, 0, st>>>(s, a.dt, a.beta);
  else
    k_g2p_tangent<DIM, false><<<nblk(s.np, 128), 128, 0, st>>>(s, a.dt, a.beta);
  pr.end(K_G2P, st);
  if (s.sv) {
    pr.begin(K_MC_RETURN, st);
    const unsigned mcb = (unsigned)std::min<int64_t>(nblk(s.np, 128), 148 * 8);
    k_mc_return_tangent<DIM><<<mcb, 128, 0, st>>>(s);
    pr.end(K_MC_RETURN, st);
  }
  pr.begin(K_LOCATE, st);
  launch_locate_fallback(DIM, s, a.remove_lost, st);
  pr.end(K_LOCATE, st);
}

}  // namespace

size_t tangent_material_bytes() { return sizeof(MatD); }

// MaterialT<Dual> of each material slot: the value of every entry is the
// FP64 material's (make_material's formulas), its derivative k is that with
// respect to parameter k (Young's modulus in Pa; friction, dilation in
// degrees and cohesion in Pa, each moving its peak and residual value).
void make_tangent_materials(const MaterialParams* mats, int nmats, const TangentParam* params,
                            int nparams, void* out_v, double* sv_seed) {
  MatD* out = static_cast<MatD*>(out_v);
  const double deg = kPiD / 180.;
  for (int mi = 0; mi < nmats; ++mi) {
    const MaterialParams& m = mats[mi];
    auto seeded = [&](double v, int kind, double scale) {
      D r(v);
      for (int k = 0; k < nparams && k < NT; ++k)
        if (params[k].material_slot == mi && params[k].kind == kind) r.d[k] = scale;
      return r;
    };
    MatD r;
    r.type = m.type;
    r.softening = m.softening;
    r.density = D(m.density);
    r.nu = D(m.nu);
    const D E = seeded(m.E, TP_YOUNGS_MODULUS, 1.0);
    r.E = E;
    r.bulk = E / (3.0 * (1. - 2. * m.nu));
    r.shear = E / (2.0 * (1. + m.nu));
    r.a1 = r.bulk + (4.0 / 3.0) * r.shear;
    r.a2 = r.bulk - (2.0 / 3.0) * r.shear;
    r.phi_peak = seeded(m.phi_peak, TP_FRICTION, deg);
    r.phi_res = seeded(m.phi_res, TP_FRICTION, deg);
    r.psi_peak = seeded(m.psi_peak, TP_DILATION, deg);
    r.psi_res = seeded(m.psi_res, TP_DILATION, deg);
    r.c_peak = seeded(m.c_peak, TP_COHESION, 1.0);
    r.c_res = seeded(m.c_res, TP_COHESION, 1.0);
    r.pd_peak = D(m.pd_peak);
    r.pd_res = D(m.pd_res);
    r.tension_cutoff = D(m.tension_cutoff);
    r.grain_density = D(m.grain_density);
    r.min_packing = D(m.min_packing);
    if (m.type == 1) {
      const D apex = r.c_peak / tan(r.phi_peak);
      r.tc_init = check_low(r.tension_cutoff < apex ? r.tension_cutoff : apex);
      r.sin_phi = sin(r.phi_peak);
      r.cos_phi = cos(r.phi_peak);
      r.tan_phi = tan(r.phi_peak);
      r.tan_psi = tan(r.psi_peak);
      // the values must be the FP64 material's
      r.tc_init.v = m.tc_init;
      r.sin_phi.v = m.sin_phi;
      r.cos_phi.v = m.cos_phi;
      r.tan_phi.v = m.tan_phi;
      r.tan_psi.v = m.tan_psi;
    }
    r.bulk.v = m.bulk;
    r.shear.v = m.shear;
    r.a1.v = m.a1;
    r.a2.v = m.a2;
    out[mi] = r;
    // derivatives of the initial state variables (mohr_coulomb.tcc:85-111)
    double* sd = sv_seed + (size_t)mi * SV_N * NT;
    for (int i = 0; i < SV_N * NT; ++i) sd[i] = 0.0;
    if (m.type == 1)
      for (int k = 0; k < NT; ++k) {
        sd[SV_PHI * NT + k] = r.phi_peak.d[k];
        sd[SV_PSI * NT + k] = r.psi_peak.d[k];
        sd[SV_COH * NT + k] = r.c_peak.d[k];
        sd[SV_TC * NT + k] = r.tc_init.d[k];
      }
  }
}

void launch_step_tangent(int dim, const DevState& s, const StepArgs& a, cudaStream_t st,
                         Profiler& prof) {
  if (dim == 2)
    step_tangent<2>(s, a, st, prof);
  else
    step_tangent<3>(s, a, st, prof);
}

}  // namespace mpm_b200
