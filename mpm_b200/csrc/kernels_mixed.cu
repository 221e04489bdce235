// kernels_mixed.cu -- mixed-precision kernels of the explicit MPM step.
//
// Arithmetic in FP32 with FP64 where it carries the result:
//   * positions and displacements are stored and advanced in FP64;
//   * the shape functions use a local coordinate computed in FP64 (x and the
//     cell centroid are FP64) and then rounded;
//   * P2G forms each particle's contributions in FP32 and sums them per cell
//     slot in FP64 (one FP64 add per value costs less than a compensated FP32
//     sum), the node adds its (at most eight) cell partials in FP64 and divides
//     momentum by mass in FP64;
//   * the MohrCoulomb elastic predictor and yield check run in FP32 (stress
//     invariants in FP64, see mc_invariants); plastic returns, points at the
//     apex and separated points run in FP64 in a dense second kernel (an FP32
//     return cancels when it removes most of the trial stress and near the
//     apex, and plastic points are few and scattered, so batching them keeps
//     the elastic lanes of a warp from waiting on the return iterations);
//     the plastic deviatoric strain is kept in FP64;
//   * F, volume and density are stored as deviations (H = F - I,
//     P = V / V0 - 1) so that FP32 keeps the 1e-9 per-step increments.
// Same step structure as the FP64 path (kernels_fp64.cu): counting sort,
// per-cell P2G, node gather and update, G2P + stress + locate.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "mpm_bulk.cuh"
#include "mpm_device.cuh"
#include "mpm_grid.cuh"
#include "mpm_kernels.h"
#include "mpm_return.cuh"
#include "mpm_state.cuh"

#ifndef MPM_MIXED_G2P_MIN_BLOCKS
// 80 registers: 0.478 -> 0.374 ms (4M, 3D).  7 and 8 blocks (72 / 64 registers, more
// spills): early steps g2p 0.389 -> 0.377 / 0.379 ms, step at 2000 0.542 -> 0.545 /
// 0.547 ms (1M column): no net gain over a run.
#define MPM_MIXED_G2P_MIN_BLOCKS 6
#endif
#ifndef MPM_MIXED_AFFINE_G2P_MIN_BLOCKS
#define MPM_MIXED_AFFINE_G2P_MIN_BLOCKS 4  // the nodal velocities stay in registers for B
#endif
#ifndef MPM_MC_RETURN_MIN_BLOCKS
#define MPM_MC_RETURN_MIN_BLOCKS 4  // pass-loop return, 1M column at step 2000: 2 / 3 / 4 / 6 blocks -> FP64 0.362 / 0.320 / 0.323 / 0.403 ms, mixed 0.370 / 0.318 / 0.311 / 0.384 ms
#endif
// Blocks per SM of the persistent step kernel (3D, 2D).  Measured with 20
// steps per launch, ms per step on the 4M-particle column / the 512-slope
// ensemble: 4 blocks 1.303 / 3.018, 6 blocks 1.128 / 2.382, 8 blocks 1.161 /
// 2.047 (per-pass launches: 0.748 / 1.555).
#ifndef MPM_MIXED_NODES_MIN_BLOCKS
// 256-thread blocks, 32 registers; 6 and 4 blocks (40 / 64 registers), 4M column:
// 0.048 / 0.054 ms against 0.049 ms
#define MPM_MIXED_NODES_MIN_BLOCKS 8
#endif
#ifndef MPM_PERSISTENT_MIN_BLOCKS_3D
#define MPM_PERSISTENT_MIN_BLOCKS_3D 6
#endif
#ifndef MPM_PERSISTENT_MIN_BLOCKS_2D
#define MPM_PERSISTENT_MIN_BLOCKS_2D 8
#endif
#ifndef MPM_MIXED_P2G_TILE_MIN_BLOCKS
// 48 registers, small spills: 0.32 -> 0.26 ms (4M, 3D); against 4 and 6 (64 / 40
// registers) with the body force at the node: 128-thread tiles 0.193 vs 0.206 / 0.203
// ms, 256-thread tiles 0.216 vs 0.237 / 0.227 ms.
#define MPM_MIXED_P2G_TILE_MIN_BLOCKS 5
#endif

namespace mpm_b200 {
namespace {

template <int DIM>
__device__ __forceinline__ float pmf(const DevState& s, int f, int64_t p) {
  return s.pm[(int64_t)f * s.np + p];
}
template <int DIM>
__device__ __forceinline__ void set_pmf(const DevState& s, int f, int64_t p, float v) {
  s.pm[(int64_t)f * s.np + p] = v;
}

// The nodal velocity (and, with ACC, acceleration) of node n from its
// nfv record (nfv_stride floats: 3D v0 v1 v2 a0 | a1 a2 - -, 2D v0 v1 a0 a1).
template <int DIM, bool ACC>
__device__ __forceinline__ void load_nfv(const float* nfv, int64_t n, float* v, float* a) {
  const float4* q = reinterpret_cast<const float4*>(nfv + n * nfv_stride(DIM));
  const float4 h0 = q[0];
  v[0] = h0.x;
  v[1] = h0.y;
  if constexpr (DIM == 3) {
    v[2] = h0.z;
    if constexpr (ACC) {
      const float4 h1 = q[1];
      a[0] = h0.w;
      a[1] = h1.x;
      a[2] = h1.y;
    }
  } else if constexpr (ACC) {
    a[0] = h0.z;
    a[1] = h0.w;
  }
}
template <int DIM>
__device__ __forceinline__ void store_nfv(float* nfv, int64_t n, const float* v, const float* a) {
  float4* q = reinterpret_cast<float4*>(nfv + n * nfv_stride(DIM));
  if constexpr (DIM == 3) {
    q[0] = make_float4(v[0], v[1], v[2], a[0]);
    q[1] = make_float4(a[1], a[2], 0.f, 0.f);
  } else {
    q[0] = make_float4(v[0], v[1], a[0], a[1]);
  }
}

// local coordinate in FP64, rounded to FP32 for the shape functions
template <int DIM, bool BOX>
__device__ __forceinline__ void xi_f32(const DevState& s, int c, const double* x, float* xf) {
  double xi[DIM];
  particle_xi<DIM, BOX>(s, c, x, xi);
#pragma unroll
  for (int d = 0; d < DIM; ++d) xf[d] = (float)xi[d];
}

// node ids and nodal coordinates relative to node 0 of the cell (FP32); the
// coordinates are not needed (nor set) for the box cells of a tensor-product
// grid
template <int DIM, bool BOX>
__device__ __forceinline__ void cell_nodes_rel(const DevState& s, int c, int* nid, float* Xr) {
  constexpr int NV = Elem<DIM>::NV;
  if constexpr (BOX) {
    grid_cell_nodes<DIM>(s, c, nid);
    return;
  }
  double X[NV * DIM];
  cell_nodes_coords<DIM>(s, c, nid, X);
#pragma unroll
  for (int n = 0; n < NV; ++n)
#pragma unroll
    for (int d = 0; d < DIM; ++d) Xr[n * DIM + d] = (float)(X[n * DIM + d] - X[d]);
}

// ---------------------------------------------------------------- P2G tiles
// The FP64 path's cell tiles (k_p2g_tiles) in FP32: staged local coordinates
// (the FP64 local coordinate rounded), mass, velocity, the stress times the
// particle's -V0 (1 + P)
// and, off a tensor-product grid, J^-1; per (cell, slot) thread 1 + 2 DIM
// FP64 sums (mass, momentum, internal force; the body force is formed by the
// node update) of the FP32 contributions of the cell's particles in id order,
// stored as FP32 partials.  AFF: the mass-momentum mapping velocity v + M r of
// the affine (1: M = B D^-1) or Taylor (2: M = B) updates, with M formed in
// FP64 by the staging thread and the branch vectors r taken from FP64
// positions relative to the cell's first node, both rounded to FP32.
template <int DIM, int MODE, bool BOX, int AFF = 0>
struct MTileRows {
  static constexpr bool MM = MODE != 1, FORCES = MODE != 0;
  static constexpr int XI = 0, M = DIM;  // the mass row only with mass and momentum
  static constexpr int V = M + (MM ? 1 : 0);
  static constexpr int S = V + (MM ? DIM : 0);  // stress times -V0 (1 + P)
  static constexpr int INV = S + (FORCES ? PF<DIM>::NS : 0);
  static constexpr int XP = INV + (FORCES && !BOX ? DIM * DIM : 0);  // x - node 0
  static constexpr int MV = XP + (MM && AFF ? DIM : 0);              // mapping matrix
  static constexpr int N = MV + (MM && AFF ? DIM * DIM : 0);
};

// On box cells the tile may also take 128 threads (a launch-shape choice);
// the blocks per SM scale so that the registers per thread stay the same.
// The mapping-velocity tiles (128 threads) form the FP64 matrix when they
// stage a row and take up to 128 registers.
template <bool BOX, int T, int AFF = 0>
constexpr int mixed_tile_min_blocks() {
  return AFF ? 4 : BOX ? MPM_MIXED_P2G_TILE_MIN_BLOCKS * 256 / T : MPM_MIXED_P2G_TILE_MIN_BLOCKS;
}

// One tile (block-sized group of cells, tile index bx) of the P2G pass; the
// block's threads are the tile's (cell, slot) pairs.
template <int DIM, int MODE, bool BOX, int T, int AFF = 0>
__device__ __forceinline__ void p2g_tile_mixed(const DevState& s, int64_t bx) {
  constexpr int NV = Elem<DIM>::NV;
  constexpr int CB = T / NV;
  constexpr int NVAL = mixed_nval(DIM);
  constexpr int MASS = 0, MOM = 1, FINT = 1 + DIM;
  using RW = MTileRows<DIM, MODE, BOX, AFF>;
  constexpr bool MM = RW::MM, FORCES = RW::FORCES;
  __shared__ float rows[RW::N][T];
  const int t = threadIdx.x;
  const int64_t c0 = bx * CB;
  if (c0 >= s.ncells) return;
  const int64_t c1 = c0 + CB < s.ncells ? c0 + CB : s.ncells;
  const int64_t q_begin = s.start[c0], q_end = s.start[c1 - 1] + s.cnt[c1 - 1];
  if (q_begin == q_end) return;  // no particles in the tile (the whole block)
  const int64_t c = c0 + t / NV;
  const int k = t % NV;
  const bool mine = c < c1;
  const int64_t a0 = mine ? s.start[c] : 0;
  const int64_t a1 = mine ? a0 + s.cnt[c] : 0;
  // One staged particle row (one particle per thread, coalesced reads).
  auto stage = [&](int r, int64_t p) {
    const int pc = s.cell[p];
    double x[DIM];
    load_x<DIM>(s, p, x);
    float xi[DIM];
    xi_f32<DIM, BOX>(s, pc, x, xi);
#pragma unroll
    for (int d = 0; d < DIM; ++d) rows[RW::XI + d][r] = xi[d];
    if constexpr (MM) rows[RW::M][r] = pmf<DIM>(s, PM<DIM>::MASS, p);
    if constexpr (MM) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) rows[RW::V + d][r] = pmf<DIM>(s, PM<DIM>::V + d, p);
    }
    if constexpr (MM && AFF) {
      int nid[NV];
      double X[NV * DIM], xid[DIM], Mv[DIM * DIM];
      cell_nodes_coords<DIM>(s, pc, nid, X);
      particle_xi<DIM, BOX>(s, pc, x, xid);
      mapping_velocity_matrix<DIM, AFF>(s, p, pc, x, xid, Mv);
#pragma unroll
      for (int d = 0; d < DIM; ++d) rows[RW::XP + d][r] = (float)(x[d] - X[d]);
#pragma unroll
      for (int q = 0; q < DIM * DIM; ++q) rows[RW::MV + q][r] = (float)Mv[q];
    }
    if constexpr (FORCES) {
      const float sc = -(pmf<DIM>(s, PM<DIM>::V0, p) * (1.f + pmf<DIM>(s, PM<DIM>::JP, p)));
#pragma unroll
      for (int q = 0; q < PF<DIM>::NS; ++q) rows[RW::S + q][r] = sc * pmf<DIM>(s, PM<DIM>::S + q, p);
      if constexpr (!BOX) {
        int nid[NV];
        float Xr[NV * DIM];
        cell_nodes_rel<DIM, false>(s, pc, nid, Xr);
        const CellMap<DIM, false, float> m = cell_map<DIM, false>(s, pc, xi, Xr);
#pragma unroll
        for (int q = 0; q < DIM * DIM; ++q) rows[RW::INV + q][r] = m.inv[q];
      }
    }
  };
  CellMap<DIM, BOX, float> box_map;
  if constexpr (BOX && FORCES) {
    if (a1 > a0) box_map = cell_map<DIM, true, float>(s, (int)c, nullptr, nullptr);
  }
  float xkr[DIM];  // this slot's node relative to the cell's first node (AFF)
  if constexpr (MM && AFF) {
    int nid[NV];
    double X[NV * DIM];
    if (a1 > a0) cell_nodes_coords<DIM>(s, (int)c, nid, X);
#pragma unroll
    for (int d = 0; d < DIM; ++d) xkr[d] = a1 > a0 ? (float)(X[k * DIM + d] - X[d]) : 0.f;
  }
  double acc[NVAL];
#pragma unroll
  for (int v = 0; v < NVAL; ++v) acc[v] = 0.;
  // this slot's contributions of staged row r
  auto add = [&](int r) {
    float xi[DIM], N, G[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) xi[d] = rows[RW::XI + d][r];
    node_shape<DIM>(xi, k, N, G);
    if constexpr (MM) {
      const float mN = rows[RW::M][r] * N;
      acc[MASS] += (double)mN;
      float mv[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) mv[d] = rows[RW::V + d][r];
      if constexpr (AFF) {
        float br[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) br[d] = xkr[d] - rows[RW::XP + d][r];
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          float sum = rows[RW::MV + a * DIM + 0][r] * br[0];
#pragma unroll
          for (int b = 1; b < DIM; ++b) sum = sum + rows[RW::MV + a * DIM + b][r] * br[b];
          mv[a] += sum;
        }
      }
#pragma unroll
      for (int d = 0; d < DIM; ++d) acc[MOM + d] += (double)(mN * mv[d]);
    }
    if constexpr (FORCES) {
      float sig[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int q = 0; q < PF<DIM>::NS; ++q) sig[q] = rows[RW::S + q][r];
      float Dn[DIM];
      if constexpr (BOX) {
        box_map.grad(G, Dn);
      } else {
        CellMap<DIM, false, float> m2;
#pragma unroll
        for (int q = 0; q < DIM * DIM; ++q) m2.inv[q] = rows[RW::INV + q][r];
        m2.grad(G, Dn);
      }
      float f[DIM];
      if constexpr (DIM == 2) {
        f[0] = Dn[0] * sig[0] + Dn[1] * sig[3];
        f[1] = Dn[1] * sig[1] + Dn[0] * sig[3];
      } else {
        f[0] = Dn[0] * sig[0] + Dn[1] * sig[3] + Dn[2] * sig[5];
        f[1] = Dn[1] * sig[1] + Dn[0] * sig[3] + Dn[2] * sig[4];
        f[2] = Dn[2] * sig[2] + Dn[1] * sig[4] + Dn[0] * sig[5];
      }
#pragma unroll
      for (int d = 0; d < DIM; ++d) acc[FINT + d] += (double)f[d];
    }
  };
  // each cell's particle ids in ascending order in the first mapping of a step
  if constexpr (MODE != 1) sort_cell_ids<NV>(s.order + a0, (int)(a1 - a0), k);
  for (int64_t q0 = q_begin; q0 < q_end; q0 += T) {
    if (q0 != q_begin) __syncthreads();  // the previous chunk is consumed
    if (q0 + t < q_end) stage(t, s.order[q0 + t]);
    __syncthreads();
    const int64_t j0 = a0 > q0 ? a0 : q0;
    const int64_t j1 = a1 < q0 + T ? a1 : q0 + T;
    for (int64_t j = j0; j < j1; ++j) add((int)(j - q0));
  }
  if (!mine || a1 == a0) return;  // empty cells keep no partials
  float* out = s.partials_f + ((int64_t)c * NV + k) * NVAL;
  float row[NVAL];  // the padding stays zero
#pragma unroll
  for (int v = 0; v < NVAL; ++v) row[v] = (float)acc[v];
  if constexpr (MM && FORCES)
    store_partial_row<NVAL, 0, NVAL>(out, row);
  else if constexpr (MM)
    store_partial_row<NVAL, MASS, FINT>(out, row);
  else
    store_partial_row<NVAL, FINT, NVAL - FINT>(out, row + FINT);
}

template <int DIM, int MODE, bool BOX, int T = p2g_tile_t<BOX>(), int AFF = 0>
__global__ void __launch_bounds__(T, (mixed_tile_min_blocks<BOX, T, AFF>()))
    k_p2g_tiles_mixed(DevState s) {
  p2g_tile_mixed<DIM, MODE, BOX, T, AFF>(s, blockIdx.x);
}

// ---------------------------------------------------------------- node update
// The cell partials of a node (ascending cell id) added in FP64.
template <int DIM, int V0, int NVS>
__device__ __forceinline__ bool gather_node_mixed(const DevState& s, int64_t node, double* sum) {
  constexpr int NV = Elem<DIM>::NV;
  constexpr int NVAL = mixed_nval(DIM);
#pragma unroll
  for (int v = 0; v < NVS; ++v) sum[v] = 0.;
  bool active = false;
  auto add = [&](int c, int slot) {
    float src[NVS];
    load_partial_row<float, NVAL, V0, NVS>(s.partials_f + ((int64_t)c * NV + slot) * NVAL, src);
#pragma unroll
    for (int v = 0; v < NVS; ++v) sum[v] += (double)src[v];
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

// node.tcc:309-345 in FP64 on the gathered sums
template <int DIM>
__device__ __forceinline__ void node_accel_update_d(const DevState& s, double m, const double* fe,
                                                    const double* fi, double* vel, double* acc,
                                                    int bci, double dt, double damping) {
  if (!(m > 1.0E-15)) return;
  double uf[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) uf[d] = fe[d] + fi[d];
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
    apply_acceleration_constraints<DIM>(bc, acc);
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

// 8 blocks per SM: 0.111 -> 0.108 ms per 1M-node launch (more warps in flight
// on the scattered partial loads, despite small spills)
// The body force of a node is gravity times its mass (particle.tcc:893-898
// summed over the node's particles: sum_p g m_p N_p = g sum_p m_p N_p), formed
// here in FP64 from the gathered mass instead of carried in the partials.
template <int DIM, int MODE>
__device__ __forceinline__ void node_update_mixed(const DevState& s, double dt, double damping,
                                                  const double* g, int64_t n) {
  if (n >= s.nn) return;
  constexpr int NVAL = mixed_nval(DIM);
  double sum[NVAL];
  constexpr int V0 = MODE == 2 ? 1 + DIM : 0;  // MODE 2: the internal force and the padding
  constexpr int NVS = MODE == 0 ? 1 + DIM : (MODE == 1 ? NVAL : NVAL - (1 + DIM));
  if (!gather_node_mixed<DIM, V0, NVS>(s, n, sum)) return;
  const int bci = s.bc_index[n];
  double vel[DIM], acc[DIM];
  if constexpr (MODE == 2) {
    double mm[1];
    gather_node_mixed<DIM, 0, 1>(s, n, mm);
    float vf[DIM], af[DIM];
    load_nfv<DIM, true>(s.nfv, n, vf, af);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      vel[d] = (double)vf[d];
      acc[d] = (double)af[d];
    }
    double fe[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) fe[d] = g[d] * mm[0];
    node_accel_update_d<DIM>(s, mm[0], fe, &sum[0], vel, acc, bci, dt, damping);
  } else {
    const double m = sum[0];
#pragma unroll
    for (int d = 0; d < DIM; ++d) vel[d] = acc[d] = 0.;
    if (m > 1.E-16) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) vel[d] = sum[1 + d] / m;  // FP64 mass division
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        if (fabs(vel[d]) < 1.E-15) vel[d] = 0.;
    }
    if (bci >= 0) apply_velocity_constraints<DIM>(s.bcs[bci], vel, acc);
    if constexpr (MODE == 1) {
      double fe[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) fe[d] = g[d] * m;
      node_accel_update_d<DIM>(s, m, fe, &sum[1 + DIM], vel, acc, bci, dt, damping);
    }
  }
  float vf[DIM], af[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    vf[d] = (float)vel[d];
    af[d] = (float)acc[d];
  }
  store_nfv<DIM>(s.nfv, n, vf, af);
}

template <int DIM, int MODE>
__global__ void __launch_bounds__(256, MPM_MIXED_NODES_MIN_BLOCKS) k_nodes_mixed(DevState s, double dt, double damping, double g0,
                                                        double g1, double g2) {
  const double g[3] = {g0, g1, g2};
  node_update_mixed<DIM, MODE>(s, dt, damping, g, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// ------------------------------------------------------- stress and strain
// MohrCoulomb elastic predictor and yield check in FP32 (invariants in FP64):
// true with out and svf updated when the trial stress is elastic and away
// from the apex of the yield surface (deviatoric trial stress above 1e-2 of
// the stress magnitude); false for every other point (plastic, apex,
// separated), which the caller defers to the FP64 return of
// k_mc_return_mixed with its inputs unchanged.
__device__ __forceinline__ bool mc_elastic_mixed(const MaterialT<float>& mf, const float* sig,
                                                 const float* de, float rho, float* svf, float* out) {
  float trial[6];
  {
    float t[6];
    de_mul(mf, de, t);
#pragma unroll
    for (int i = 0; i < 6; ++i) trial[i] = sig[i] + t[i];
  }
  float smax = 0.f;
#pragma unroll
  for (int i = 0; i < 6; ++i) smax = fmaxf(smax, fabsf(trial[i]));
  const float rho_dev = sqrtf(2.f * mu_j2(trial));
  if (rho_dev <= 1e-2f * smax) return false;
  float sv[SV_N];
#pragma unroll
  for (int k = 0; k < SVF_N; ++k) sv[k] = svf[k];
  sv[SV_PD] = 0.f;
  double pd_unused = 0.0;
  if (mc_stress<float, double, true>(mf, sig, de, rho, sv, pd_unused, out) != MC_OK ||
      sv[SV_YIELD] != 0.f)
    return false;
#pragma unroll
  for (int k = 0; k < SVF_N; ++k) svf[k] = sv[k];
  return true;
}

// One particle's mixed-precision fields in global memory (MGlobalRow) or in
// the block's shared-memory staging (MSmemRow, MSTAGE_T particles per row):
// m(f) the FP32 field f of PM, svf(k) the FP32 MohrCoulomb state, pd() the
// FP64 plastic deviatoric strain (read only by the deferred returns, which
// work in global memory).
template <int DIM>
struct MGlobalRow {
  const DevState& s;
  int64_t p;
  __device__ __forceinline__ int64_t index() const { return p; }
  __device__ __forceinline__ float& m(int f) const { return s.pm[(int64_t)f * s.np + p]; }
  __device__ __forceinline__ float& svf(int k) const { return s.svf[(int64_t)k * s.np + p]; }
  __device__ __forceinline__ double& pd() const { return s.pf[(int64_t)PDX<DIM>::PDS * s.np + p]; }
  __device__ __forceinline__ int mat() const { return s.mat[p]; }
};
constexpr int MSTAGE_T = 128;  // particles per staged block (= PAD_PARTICLES)
struct MSmemRow {
  float* mrows;  // [PM field][MSTAGE_T]
  float* svr;    // [SVF_N][MSTAGE_T]
  int t;
  int mi;
  int64_t p;
  __device__ __forceinline__ int64_t index() const { return p; }
  __device__ __forceinline__ float& m(int f) const { return mrows[f * MSTAGE_T + t]; }
  __device__ __forceinline__ float& svf(int k) const { return svr[k * MSTAGE_T + t]; }
  __device__ __forceinline__ int mat() const { return mi; }
};

// mpm_scheme.tcc:75-103 in FP32 on the deviation variables (H, P).
template <int DIM, class Row>
__device__ __forceinline__ void stress_update_mixed(const DevState& s, const Row& r, int c,
                                                    const int* nid, const float* D, float dt) {
  constexpr int NV = Elem<DIM>::NV;
  constexpr int NS = PF<DIM>::NS;
  const float* Dc = s.dndx_cf + (int64_t)c * NV * DIM;
  float Hi[DIM * DIM];
#pragma unroll
  for (int a = 0; a < DIM * DIM; ++a) Hi[a] = 0.f;
  float sr[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float src[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    float vel[DIM];
    load_nfv<DIM, false>(s.nfv, nid[i], vel, nullptr);
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
      for (int q = 0; q < DIM; ++q) Hi[a * DIM + q] += vel[a] * D[i * DIM + q] * dt;
    const float* Dn = &D[i * DIM];
    float dc[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) dc[d] = __ldg(&Dc[i * DIM + d]);
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
  // F_inc = I + Hi with the reference's 1e-15 snapping (particle.tcc:1619-1626)
#pragma unroll
  for (int a = 0; a < DIM * DIM; ++a)
    if (fabsf(Hi[a]) < 1.E-15f) Hi[a] = 0.f;
#pragma unroll
  for (int k = 0; k < 6; ++k)
    if (fabsf(sr[k]) < 1.E-15f) sr[k] = 0.f;
#pragma unroll
  for (int k = 0; k < DIM; ++k)
    if (fabsf(src[k]) < 1.E-15f) src[k] = 0.f;
  float dstrain[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) dstrain[k] = sr[k] * dt;
  float ssum = src[0];
#pragma unroll
  for (int k = 1; k < DIM; ++k) ssum += src[k];
  const float dvol = dt * ssum;
  if constexpr (DIM == 2) {
    const int map[3] = {0, 1, 3};
#pragma unroll
    for (int k = 0; k < 3; ++k) r.m(PM<2>::E + k) += dstrain[map[k]];
  } else {
#pragma unroll
    for (int k = 0; k < 6; ++k) r.m(PM<3>::E + k) += dstrain[k];
  }
  // V *= (1 + dvol), rho /= (1 + dvol) as P = V / V0 - 1 (particle.tcc:598-605)
  const float P = r.m(PM<DIM>::JP);
  const float Pn = P + dvol + P * dvol;
  r.m(PM<DIM>::JP) = Pn;
  const float rho = r.m(PM<DIM>::RHO0) / (1.f + Pn);
  float sig[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int k = 0; k < NS; ++k) sig[k] = r.m(PM<DIM>::S + k);
  const int mi = r.mat();
  float out[6];
  bool deferred = false;
  if (s.mats_f[mi].type == 0) {
    float t[6];
    de_mul(s.mats_f[mi], dstrain, t);
#pragma unroll
    for (int i = 0; i < 6; ++i) out[i] = sig[i] + t[i];
  } else {
    float svf[SVF_N];
#pragma unroll
    for (int k = 0; k < SVF_N; ++k) svf[k] = r.svf(k);
    if (mc_elastic_mixed(s.mats_f[mi], sig, dstrain, rho, svf, out)) {
      const int first = s.mats_f[mi].softening ? 0 : SV_EPS;  // phi..tc change only with softening
      r.svf(SV_YIELD) = svf[SV_YIELD];
#pragma unroll
      for (int k = 1; k < SVF_N; ++k)
        if (k >= first) r.svf(k) = svf[k];
    } else {
      // plastic, apex or separated: the FP64 update of k_mc_return_mixed
      deferred = true;
      const unsigned i = defer_slot_by_cost(s, r.index());
      s.plist[i] = (int32_t)r.index();
#pragma unroll
      for (int k = 0; k < 6; ++k) s.pbuf_f[(int64_t)k * s.np + i] = dstrain[k];
      s.pbuf_f[(int64_t)6 * s.np + i] = rho;
    }
  }
  if (!deferred) {
#pragma unroll
    for (int k = 0; k < NS; ++k) r.m(PM<DIM>::S + k) = out[k];
  }
  // F = F_inc F as H = H + Hi + Hi H
  if constexpr (DIM == 2) {
    float H[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) H[k] = r.m(PM<2>::H + k);
    const float n00 = H[0] + Hi[0] + (Hi[0] * H[0] + Hi[1] * H[2]);
    const float n01 = H[1] + Hi[1] + (Hi[0] * H[1] + Hi[1] * H[3]);
    const float n10 = H[2] + Hi[2] + (Hi[2] * H[0] + Hi[3] * H[2]);
    const float n11 = H[3] + Hi[3] + (Hi[2] * H[1] + Hi[3] * H[3]);
    r.m(PM<2>::H + 0) = n00;
    r.m(PM<2>::H + 1) = n01;
    r.m(PM<2>::H + 2) = n10;
    r.m(PM<2>::H + 3) = n11;
  } else {
    float H[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) H[k] = r.m(PM<3>::H + k);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int q = 0; q < 3; ++q)
        r.m(PM<3>::H + a * 3 + q) =
            H[a * 3 + q] + Hi[a * 3 + q] +
            ((Hi[a * 3 + 0] * H[0 * 3 + q] + Hi[a * 3 + 1] * H[1 * 3 + q]) + Hi[a * 3 + 2] * H[2 * 3 + q]);
  }
}

template <int DIM, bool BOX>
__device__ __forceinline__ void dn_dx_all_f(const DevState& s, int c, const float* xi,
                                            const float* Xr, float* D) {
  constexpr int NV = Elem<DIM>::NV;
  const CellMap<DIM, BOX, float> map = cell_map<DIM, BOX>(s, c, xi, Xr);
  float G[NV * DIM];
  grad_shapefn<DIM>(xi, G);
#pragma unroll
  for (int n = 0; n < NV; ++n) map.grad(&G[n * DIM], &D[n * DIM]);
}

template <int DIM, bool BOX>
__global__ void __launch_bounds__(128) k_stress_mixed(DevState s, float dt) {
  constexpr int NV = Elem<DIM>::NV;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0) return;
  double x[DIM];
  load_x<DIM>(s, p, x);
  float xi[DIM], D[NV * DIM], Xr[NV * DIM];
  int nid[NV];
  xi_f32<DIM, BOX>(s, c, x, xi);
  cell_nodes_rel<DIM, BOX>(s, c, nid, Xr);
  dn_dx_all_f<DIM, BOX>(s, c, xi, Xr, D);
  stress_update_mixed<DIM>(s, MGlobalRow<DIM>{s, p}, c, nid, D, dt);
}

// --------------------------------------------------------------------- G2P
// MUSL (mpm_scheme_musl.tcc:20-35): the kinematics without committing the
// positions -- the updated ones go to xnext (k_commit_locate_mixed commits them
// after the second mapping and the stress update), no locate here.
template <int DIM, bool STRESS, bool FLIP, bool BOX, bool MUSL = false>
__global__ void __launch_bounds__(128, MPM_MIXED_G2P_MIN_BLOCKS)
    k_g2p_mixed(DevState s, double dt, float beta) {
  static_assert(!(MUSL && STRESS), "MUSL updates the stress after its second mapping");
  constexpr int NV = Elem<DIM>::NV;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0) return;
  const int64_t np = s.np;
  double x[DIM];
  load_x<DIM>(s, p, x);
  float xi[DIM], N[NV], Xr[NV * DIM];
  int nid[NV];
  xi_f32<DIM, BOX>(s, c, x, xi);
  shapefn<DIM>(xi, N);
  cell_nodes_rel<DIM, BOX>(s, c, nid, Xr);
  float nvel[DIM], nacc[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) nvel[d] = nacc[d] = 0.f;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    float vn[DIM], an[DIM];
    load_nfv<DIM, FLIP>(s.nfv, nid[i], vn, an);
#pragma unroll
    for (int d = 0; d < DIM; ++d) nvel[d] += N[i] * vn[d];
    if constexpr (FLIP) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) nacc[d] += N[i] * an[d];
    }
  }
  const float dtf = (float)dt;
  float v[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) v[d] = pmf<DIM>(s, PM<DIM>::V + d, p);
  if constexpr (FLIP) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] += nacc[d] * dtf;
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] = beta * v[d] + (1.f - beta) * nvel[d];
  } else {
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] = nvel[d];
  }
  double xn[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const double dx = (double)nvel[d] * dt;  // FP64 position / displacement update
    xn[d] = x[d] + dx;
    if constexpr (MUSL)
      s.xnext[(int64_t)d * np + p] = xn[d];
    else
      s.pf[(int64_t)(PDX<DIM>::X + d) * np + p] = xn[d];
    s.pf[(int64_t)(PDX<DIM>::U + d) * np + p] += dx;
  }
  const int pv = s.pvc[p];
  if (pv >= 0) {
    const ParticleVC& r = s.pvcs[pv];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      if (r.mask & (1u << d)) v[d] = (float)r.value[d];
  }
#pragma unroll
  for (int d = 0; d < DIM; ++d) set_pmf<DIM>(s, PM<DIM>::V + d, p, v[d]);
  if constexpr (MUSL) return;
  if constexpr (STRESS) {
    float D[NV * DIM];
    dn_dx_all_f<DIM, BOX>(s, c, xi, Xr, D);
    stress_update_mixed<DIM>(s, MGlobalRow<DIM>{s, p}, c, nid, D, dtf);
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

// G2P of the velocity updates that carry a mapping matrix (particle.tcc:
// 1071-1139, 1663-1730), k_g2p<DIM, STRESS, VU, BOX> of the FP64 path with the
// nodal values in FP32: the matrix B at the step-start position -- affine
// sum_i N_i v_i r_i^T (APIC, ASFLIP; r_i = node i - x from FP64 positions) or
// the velocity gradient sum_i v_i dN_i/dx^T (TPIC), entries below 1e-15 set to
// zero, kept in FP64 -- then APIC and TPIC take the PIC update and ASFLIP the
// FLIP/PIC blend for the velocity and the separable blend for the position.
template <int DIM, bool STRESS, int VU, bool BOX>
__global__ void __launch_bounds__(128, MPM_MIXED_AFFINE_G2P_MIN_BLOCKS)
    k_g2p_mixed_affine(DevState s, double dt, float beta) {
  static_assert(VU >= 2, "the mapping-matrix updates");
  constexpr int NV = Elem<DIM>::NV;
  constexpr bool ASFLIP = VU == 2, TPIC = VU == 3;  // 4 APIC
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0) return;
  const int64_t np = s.np;
  const float dtf = (float)dt;
  double x[DIM];
  load_x<DIM>(s, p, x);
  float xi[DIM], N[NV], Xr[NV * DIM], xr[DIM];
  int nid[NV];
  xi_f32<DIM, BOX>(s, c, x, xi);
  shapefn<DIM>(xi, N);
  {
    // the branch vectors r_i = X_i - x as (X_i - X_0) - (x - X_0) in FP32
    double X[NV * DIM];
    cell_nodes_coords<DIM>(s, c, nid, X);
#pragma unroll
    for (int n = 0; n < NV; ++n)
#pragma unroll
      for (int d = 0; d < DIM; ++d) Xr[n * DIM + d] = (float)(X[n * DIM + d] - X[d]);
#pragma unroll
    for (int d = 0; d < DIM; ++d) xr[d] = (float)(x[d] - X[d]);
  }
  float nvel[DIM], nacc[DIM], vn[NV][DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) nvel[d] = nacc[d] = 0.f;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    float an[DIM];
    load_nfv<DIM, ASFLIP>(s.nfv, nid[i], vn[i], an);
#pragma unroll
    for (int d = 0; d < DIM; ++d) nvel[d] += N[i] * vn[i][d];
    if constexpr (ASFLIP) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) nacc[d] += N[i] * an[d];
    }
  }
  float D[NV * DIM];
  if constexpr (TPIC || ASFLIP || STRESS) dn_dx_all_f<DIM, BOX>(s, c, xi, Xr, D);
  float B[DIM * DIM];
#pragma unroll
  for (int q = 0; q < DIM * DIM; ++q) B[q] = 0.f;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    float r[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) r[d] = Xr[i * DIM + d] - xr[d];
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
      for (int b = 0; b < DIM; ++b) {
        if constexpr (TPIC)
          B[a * DIM + b] += vn[i][a] * D[i * DIM + b];
        else
          B[a * DIM + b] += (N[i] * vn[i][a]) * r[b];
      }
  }
#pragma unroll
  for (int q = 0; q < DIM * DIM; ++q) {
    if (fabsf(B[q]) < 1.E-15f) B[q] = 0.f;
    s.mapb[(int64_t)q * np + p] = (double)B[q];
  }
  float v[DIM], sep[DIM];  // sep: the velocity that moves the particle
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    v[d] = pmf<DIM>(s, PM<DIM>::V + d, p);
    sep[d] = nvel[d];
  }
  if constexpr (ASFLIP) {
    // beta (particle.tcc:1711-1730): 0 next to a velocity-constrained node or
    // when the deformation gradient increment compresses
    float bp = 1.f;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      const int bci = s.bc_index[nid[i]];
      if (bci >= 0 && s.bcs[bci].vel_mask != 0) bp = 0.f;
    }
    // det(I + A) < 1 with A = sum_i v_i dN_i/dx^T dt: the test is on
    // det(I + A) - 1 = tr A + (sum of A's principal 2x2 minors) + det A, which
    // FP32 resolves down to A's own rounding (1 + A in FP32 would lose every
    // increment below 6e-8 and flip the sign of J - 1 against the FP64 run)
    float A[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int i = 0; i < NV; ++i)
#pragma unroll
      for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int b = 0; b < DIM; ++b) A[a * 3 + b] += vn[i][a] * D[i * DIM + b] * dtf;
#pragma unroll
    for (int q = 0; q < 9; ++q)
      if (fabsf(A[q]) < 1.E-15f) A[q] = 0.f;  // the snaps of F's entries at 1e-15
    const float tr = A[0] + A[4] + A[8];
    const float m2 = (A[0] * A[4] - A[1] * A[3]) + (A[0] * A[8] - A[2] * A[6]) + (A[4] * A[8] - A[5] * A[7]);
    const float d3 = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
                     A[2] * (A[3] * A[7] - A[4] * A[6]);
    if (tr + m2 + d3 < 0.f) bp = 0.f;
    // particle.tcc:1096-1110: FLIP/PIC blend for the velocity, the separable
    // blend for the position
    float flip[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) flip[d] = v[d] + nacc[d] * dtf;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      sep[d] = bp * beta * flip[d] + (1.f - bp * beta) * nvel[d];
      v[d] = beta * flip[d] + (1.f - beta) * nvel[d];
    }
  } else {
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] = nvel[d];
  }
  double xn[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const double dx = (double)sep[d] * dt;  // FP64 position / displacement update
    xn[d] = x[d] + dx;
    s.pf[(int64_t)(PDX<DIM>::X + d) * np + p] = xn[d];
    s.pf[(int64_t)(PDX<DIM>::U + d) * np + p] += dx;
  }
  const int pv = s.pvc[p];
  if (pv >= 0) {
    const ParticleVC& r = s.pvcs[pv];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      if (r.mask & (1u << d)) v[d] = (float)r.value[d];
  }
#pragma unroll
  for (int d = 0; d < DIM; ++d) set_pmf<DIM>(s, PM<DIM>::V + d, p, v[d]);
  if constexpr (STRESS) stress_update_mixed<DIM>(s, MGlobalRow<DIM>{s, p}, c, nid, D, dtf);
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

// MUSL end of step: the new positions (FP64) replace the old, then locate
template <int DIM>
__global__ void __launch_bounds__(128) k_commit_locate_mixed(DevState s) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0) return;
  const int64_t np = s.np;
  double xn[DIM];
  bool finite = true;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    xn[d] = s.xnext[(int64_t)d * np + p];
    s.pf[(int64_t)(PDX<DIM>::X + d) * np + p] = xn[d];
    finite = finite && isfinite(xn[d]);
  }
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

// USL G2P + stress update + locate with the block's particle slices staged in
// shared memory by the bulk-copy engine (as k_g2p_staged of the FP64 path):
// phase A x, u (FP64), v (FP32), cell, material, velocity-constraint slot;
// phase B stress .. P (FP32), MohrCoulomb state (FP32).  The arithmetic is
// k_g2p_mixed<DIM, true, FLIP, BOX>'s.
static_assert(MSTAGE_T == PAD_PARTICLES, "staged slices are whole padded blocks");
template <int DIM>
constexpr size_t mixed_staged_smem_bytes(bool mc) {
  return (size_t)2 * DIM * MSTAGE_T * 8 + (size_t)(PM<DIM>::MASS + (mc ? SVF_N : 0)) * MSTAGE_T * 4 +
         MSTAGE_T * (4 + 2 + 2);
}

// One block of MSTAGE_T particles (block index bx) with the staging buffers
// smem, the two initialised copy barriers bar in the phase of the given
// parity, and the block's timed-out flag.
// WRITES_DONE: wait for the block's stores to complete (a later pass of the
// same launch reads them), else only until they have read shared memory.
template <int DIM, bool FLIP, bool BOX, bool WRITES_DONE = false>
__device__ __forceinline__ void g2p_staged_block_mixed(const DevState& s, double dt, float beta,
                                                       int64_t bx, unsigned char* smem, uint64_t* bar,
                                                       unsigned parity, int& timed_out) {
  constexpr int NV = Elem<DIM>::NV;
  constexpr int T = MSTAGE_T;
  constexpr int XROWS = 2 * DIM;       // x, u
  constexpr int MROWS = PM<DIM>::MASS;  // v .. P
  const bool mc = s.svf != nullptr;
  double* xr = reinterpret_cast<double*>(smem);
  float* mr = reinterpret_cast<float*>(xr + XROWS * T);
  float* svr = mr + MROWS * T;
  int32_t* scell = reinterpret_cast<int32_t*>(svr + (mc ? SVF_N * T : 0));
  uint16_t* smat = reinterpret_cast<uint16_t*>(scell + T);
  int16_t* spvc = reinterpret_cast<int16_t*>(smat + T);
  const int t = threadIdx.x;
  const int64_t p0 = bx * T;
  const int64_t np = s.np;
  if (t == 0) timed_out = 0;
  __syncthreads();
  if (t == 0) {
    bulk::mbar_arrive_expect_tx(&bar[0], 2 * DIM * T * 8 + DIM * T * 4 + T * (4 + 2 + 2));
    for (int f = 0; f < XROWS; ++f) bulk::load(xr + f * T, s.pf + f * np + p0, T * 8, &bar[0]);
    for (int f = PM<DIM>::V; f < PM<DIM>::V + DIM; ++f)
      bulk::load(mr + f * T, s.pm + f * np + p0, T * 4, &bar[0]);
    bulk::load(scell, s.cell + p0, T * 4, &bar[0]);
    bulk::load(smat, s.mat + p0, T * 2, &bar[0]);
    bulk::load(spvc, s.pvc + p0, T * 2, &bar[0]);
    bulk::mbar_arrive_expect_tx(&bar[1], (MROWS - DIM + (mc ? SVF_N : 0)) * T * 4);
    for (int f = PM<DIM>::V + DIM; f < MROWS; ++f)
      bulk::load(mr + f * T, s.pm + f * np + p0, T * 4, &bar[1]);
    if (mc)
      for (int k = 0; k < SVF_N; ++k) bulk::load(svr + k * T, s.svf + k * np + p0, T * 4, &bar[1]);
  }
  // the test hook waits for the next phase, which no copy completes
  const bool okA = bulk::mbar_wait(&bar[0], parity) &&
                   !(s.test_wait_timeout && !bulk::mbar_wait(&bar[0], parity ^ 1u, 16));
  const int c = okA ? scell[t] : -1;
  const int64_t p = p0 + t;
  const MSmemRow r{mr, svr, t, okA ? (int)smat[t] : 0, p0 + t};
  double xn[DIM];
  const bool active = c >= 0;
  float xi[DIM];
  if (active) {
    double x[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) x[d] = xr[(PDX<DIM>::X + d) * T + t];
    float N[NV], Xr[NV * DIM];
    int nid[NV];
    xi_f32<DIM, BOX>(s, c, x, xi);
    shapefn<DIM>(xi, N);
    cell_nodes_rel<DIM, BOX>(s, c, nid, Xr);
    float nvel[DIM], nacc[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) nvel[d] = nacc[d] = 0.f;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      float vn[DIM], an[DIM];
      load_nfv<DIM, FLIP>(s.nfv, nid[i], vn, an);
#pragma unroll
      for (int d = 0; d < DIM; ++d) nvel[d] += N[i] * vn[d];
      if constexpr (FLIP) {
#pragma unroll
        for (int d = 0; d < DIM; ++d) nacc[d] += N[i] * an[d];
      }
    }
    const float dtf = (float)dt;
    float v[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] = r.m(PM<DIM>::V + d);
    if constexpr (FLIP) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) v[d] += nacc[d] * dtf;
#pragma unroll
      for (int d = 0; d < DIM; ++d) v[d] = beta * v[d] + (1.f - beta) * nvel[d];
    } else {
#pragma unroll
      for (int d = 0; d < DIM; ++d) v[d] = nvel[d];
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const double dx = (double)nvel[d] * dt;  // FP64 position / displacement update
      xn[d] = x[d] + dx;
      xr[(PDX<DIM>::X + d) * T + t] = xn[d];
      xr[(PDX<DIM>::U + d) * T + t] += dx;
    }
    const int pv = spvc[t];
    if (pv >= 0) {
      const ParticleVC& vc = s.pvcs[pv];
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        if (vc.mask & (1u << d)) v[d] = (float)vc.value[d];
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) r.m(PM<DIM>::V + d) = v[d];
  }
  const bool okB = okA && bulk::mbar_wait(&bar[1], parity);
  if (!okA || !okB) timed_out = 1;
  if (active && okB) {
    // node ids and coordinates again rather than kept live across the wait
    float Xr[NV * DIM], D[NV * DIM];
    int nid[NV];
    cell_nodes_rel<DIM, BOX>(s, c, nid, Xr);
    dn_dx_all_f<DIM, BOX>(s, c, xi, Xr, D);
    stress_update_mixed<DIM>(s, r, c, nid, D, (float)dt);
  }
  bulk::fence_shared_to_async();
  __syncthreads();
  if (timed_out) {
    if (t == 0) {
      raise_err(s, ERR_TIMEOUT);
      bulk::mbar_wait(&bar[0], parity);
      bulk::mbar_wait(&bar[1], parity);
    }
    return;
  }
  if (t == 0) {
    for (int f = 0; f < XROWS; ++f) bulk::store(s.pf + f * np + p0, xr + f * T, T * 8);
    for (int f = 0; f < MROWS; ++f)  // the initial volume and density never change
      if (f != PM<DIM>::V0 && f != PM<DIM>::RHO0) bulk::store(s.pm + f * np + p0, mr + f * T, T * 4);
    if (mc)  // phi, psi, cohesion and tension cutoff change only with softening
      for (int k = 0; k < SVF_N; ++k)
        if (s.any_softening || k == SV_YIELD || k >= SV_EPS)
          bulk::store(s.svf + k * np + p0, svr + k * T, T * 4);
    bulk::store_commit();
  }
  if (active) {
    bool finite = true;
#pragma unroll
    for (int d = 0; d < DIM; ++d) finite = finite && isfinite(xn[d]);
    if (!finite) {
      raise_err(s, ERR_NONFINITE);
      s.lost[atomicAdd(s.nlost, 1u)] = (int32_t)p;
    } else {
      const int nc = locate_near<DIM>(s, xn, c);
      if (nc >= 0) {
        if (nc != c) s.cell[p] = nc;
      } else {
        s.lost[atomicAdd(s.nlost, 1u)] = (int32_t)p;
      }
    }
  }
  if (t == 0) {
    if constexpr (WRITES_DONE)
      bulk::store_wait_all();
    else
      bulk::store_wait_read();
  }
}

template <int DIM, bool FLIP, bool BOX>
__global__ void __launch_bounds__(MSTAGE_T, MPM_MIXED_G2P_MIN_BLOCKS)
    k_g2p_mixed_staged(DevState s, double dt, float beta) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar[2];
  __shared__ int timed_out;
  if (threadIdx.x == 0) {
    bulk::mbar_init(&bar[0], 1);
    bulk::mbar_init(&bar[1], 1);
    bulk::fence_barrier_init();
  }
  g2p_staged_block_mixed<DIM, FLIP, BOX>(s, dt, beta, blockIdx.x, smem, bar, 0u, timed_out);
}

template <auto Kernel>
void prefer_shared_memory() {
  static unsigned done = 0;  // one bit per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 32 && !(done & (1u << dev))) {
    cudaFuncSetAttribute(Kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    done |= 1u << dev;
  }
}

// The MohrCoulomb updates deferred by stress_update_mixed, one thread per
// listed particle (the light entries, then the heavy ones): the full FP64
// update (mohr_coulomb.tcc:348-513, as mc_return's passes) from the FP32
// stress and state before the step's update, rounded back to FP32; the number
// of corrections is kept for the next step's grouping.
// The FP64 returns of listed entries begin, begin + stride, ...
template <int DIM>
__device__ __forceinline__ void mc_return_mixed_range(const DevState& s, unsigned begin, unsigned stride) {
  const unsigned nl = *s.nplastic, n = nl + *s.nplastic_heavy;
  const int64_t np = s.np;
  for (unsigned t = begin; t < n; t += stride) {
    const unsigned i = list_slot(s, t, nl);
    const int64_t p = s.plist[i];
    const MGlobalRow<DIM> r{s, p};
    const int mi = s.mat[p];
    float sig[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, de[6], svf[SVF_N], out[6];
#pragma unroll
    for (int k = 0; k < PF<DIM>::NS; ++k) sig[k] = r.m(PM<DIM>::S + k);
#pragma unroll
    for (int k = 0; k < 6; ++k) de[k] = s.pbuf_f[(int64_t)k * np + i];
    const float rho = s.pbuf_f[(int64_t)6 * np + i];
#pragma unroll
    for (int k = 0; k < SVF_N; ++k) svf[k] = r.svf(k);
    double sd[6], ded[6], svd[SV_N], od[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      sd[k] = (double)sig[k];
      ded[k] = (double)de[k];
    }
#pragma unroll
    for (int k = 0; k < SVF_N; ++k) svd[k] = (double)svf[k];
    svd[SV_PD] = r.pd();
    int nc = 0;
    mc_return<double>(s.mats[mi], sd, ded, (double)rho, svd, od, &nc);
    s.rpass[p] = (uint8_t)(nc < 255 ? nc : 255);
#pragma unroll
    for (int k = 0; k < 6; ++k) out[k] = (float)od[k];
#pragma unroll
    for (int k = 0; k < SVF_N; ++k) svf[k] = (float)svd[k];
    r.pd() = svd[SV_PD];
    const int first = s.mats_f[mi].softening ? 0 : SV_EPS;  // phi..tc change only with softening
    r.svf(SV_YIELD) = svf[SV_YIELD];
#pragma unroll
    for (int k = 1; k < SVF_N; ++k)
      if (k >= first) r.svf(k) = svf[k];
#pragma unroll
    for (int k = 0; k < PF<DIM>::NS; ++k) r.m(PM<DIM>::S + k) = out[k];
  }
}

template <int DIM>
__global__ void __launch_bounds__(128, MPM_MC_RETURN_MIN_BLOCKS) k_mc_return_mixed(DevState s) {
  mc_return_mixed_range<DIM>(s, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

inline unsigned nblk(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// ------------------------------------------------------ persistent steps
// The exclusive scan of the counts of chunk `chunk` (SCAN_BLOCK cells; T
// threads, SCAN_BLOCK / T consecutive cells each) into start, and the chunk's
// total into bsum[chunk].
template <int T>
__device__ __forceinline__ void scan_chunk(const int32_t* cnt, int32_t* start, int32_t* bsum,
                                           int64_t n, int64_t chunk, int32_t* red) {
  constexpr int PER = SCAN_BLOCK / T;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int64_t base = chunk * SCAN_BLOCK + (int64_t)t * PER;
  int32_t v[PER], run = 0;
#pragma unroll
  for (int i = 0; i < PER; ++i) v[i] = base + i < n ? cnt[base + i] : 0;
#pragma unroll
  for (int i = 0; i < PER; ++i) run += v[i];
  int32_t x = run;  // inclusive scan of the thread totals within the warp
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int32_t y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) red[w] = x;
  __syncthreads();
  int32_t prefix = x - run;
  for (int k = 0; k < w; ++k) prefix += red[k];
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    if (base + i < n) start[base + i] = prefix;
    prefix += v[i];
  }
  if (t == T - 1) bsum[chunk] = prefix;
  __syncthreads();  // red is reused by the next chunk
}

// The total of bsum[0, count) by the block's T threads (every thread gets it).
template <int T>
__device__ __forceinline__ int32_t block_total(const int32_t* bsum, int64_t count, int32_t* red) {
  int32_t x = 0;
  for (int64_t j = threadIdx.x; j < count; j += T) x += bsum[j];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
  __syncthreads();
  int32_t total = 0;
#pragma unroll
  for (int k = 0; k < T / 32; ++k) total += red[k];
  __syncthreads();
  return total;
}

// K whole mixed USL steps on a tensor-product grid in one cooperative launch.
// Each pass is the body of the corresponding one-pass kernel of step_mixed,
// over block-sized pieces (cell tiles, particle blocks, node blocks) taken
// grid-stride, so the results are bit for bit those of the per-pass launches
// (the P2G tiles have 128 threads; each cell's particle ids are sorted before
// they are added, so the slot order the counting sort leaves does not matter):
//   count | scan chunks | chunk prefixes | fill | P2G | nodes |
//   G2P + stress (and the next step's counts zeroed) | returns [| locate]
template <int DIM, bool FLIP>
__global__ void __launch_bounds__(MSTAGE_T, DIM == 2 ? MPM_PERSISTENT_MIN_BLOCKS_2D : MPM_PERSISTENT_MIN_BLOCKS_3D)
    k_steps_persistent_mixed(DevState s, StepArgs a, PersistentArgs q) {
  constexpr int T = MSTAGE_T;
  constexpr int NV = Elem<DIM>::NV;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar[2];
  __shared__ int timed_out, go;
  __shared__ int32_t red[T / 32];
  const int t = threadIdx.x;
  const unsigned G = gridDim.x;
  const int64_t np = s.np, nc = s.ncells;
  const int64_t pblocks = (np + T - 1) / T, tiles = (nc + T / NV - 1) / (T / NV);
  const int64_t nodeblocks = (s.nn + T - 1) / T, chunks = (nc + SCAN_BLOCK - 1) / SCAN_BLOCK;
  const unsigned gi = blockIdx.x * T + t, gs = G * T;  // grid-stride start and stride
  __shared__ long long step0;
  unsigned gen = 0;
  if (t == 0) {
    bulk::mbar_init(&bar[0], 1);
    bulk::mbar_init(&bar[1], 1);
    bulk::fence_barrier_init();
    gen = ld_acquire_gpu(&q.barrier[1]);
    step0 = *q.step;  // block 0 advances it only after the last barrier
  }
  for (int64_t i = gi; i < nc; i += gs) s.cnt[i] = 0;
  if (!grid_barrier(s, q.barrier, G, gen, go)) return;
  unsigned parity = 0;
  for (int64_t k = 0; k < q.nsteps; ++k) {
    double gm = 1.0;  // the host's ramp, the same operations
    if (q.ramp > 0.0) gm = fmin(1.0, static_cast<double>(step0 + k) * a.dt / q.ramp);
    const double g[3] = {gm * q.gravity[0], gm * q.gravity[1], gm * q.gravity[2]};
    // counting sort
    if (blockIdx.x == 0 && t == 0) {
      *s.nlost = 0;
      if (s.svf) *s.nplastic = *s.nplastic_heavy = 0;
    }
    for (int64_t b = blockIdx.x; b < pblocks; b += G) count_particle(s, b * T + t);
    if (!grid_barrier(s, q.barrier, G, gen, go)) return;
    for (int64_t b = blockIdx.x; b < chunks; b += G) scan_chunk<T>(s.cnt, s.start, s.bsum, nc, b, red);
    if (!grid_barrier(s, q.barrier, G, gen, go)) return;
    for (int64_t b = blockIdx.x; b < chunks; b += G) {
      const int32_t prefix = block_total<T>(s.bsum, b, red);
      for (int64_t i = b * SCAN_BLOCK + t; i < nc && i < (b + 1) * SCAN_BLOCK; i += T) s.start[i] += prefix;
      if (b == chunks - 1 && t == 0) s.start[nc] = prefix + s.bsum[b];
    }
    if (!grid_barrier(s, q.barrier, G, gen, go)) return;
    for (int64_t b = blockIdx.x; b < pblocks; b += G) fill_particle(s, b * T + t);
    if (!grid_barrier(s, q.barrier, G, gen, go)) return;
    // P2G of mass, momentum and forces
    for (int64_t b = blockIdx.x; b < tiles; b += G) {
      p2g_tile_mixed<DIM, 2, true, T>(s, b);
      __syncthreads();  // the tile's staged rows are consumed
    }
    if (!grid_barrier(s, q.barrier, G, gen, go)) return;
    for (int64_t b = blockIdx.x; b < nodeblocks; b += G) node_update_mixed<DIM, 1>(s, a.dt, a.damping, g, b * T + t);
    if (!grid_barrier(s, q.barrier, G, gen, go)) return;
    // G2P with the stress update; the counts are free once the nodes are done
    for (int64_t b = blockIdx.x; b < pblocks; b += G) {
      g2p_staged_block_mixed<DIM, FLIP, true, true>(s, a.dt, (float)a.beta, b, smem, bar, parity,
                                                    timed_out);
      parity ^= 1u;
      __syncthreads();  // the block's staging buffers are free again
    }
    for (int64_t i = gi; i < nc; i += gs) s.cnt[i] = 0;
    if (!grid_barrier(s, q.barrier, G, gen, go)) return;
    if (s.svf) {
      mc_return_mixed_range<DIM>(s, gi, gs);
      if (!grid_barrier(s, q.barrier, G, gen, go)) return;
    }
    if (ld_acquire_gpu(s.nlost) != 0) {  // the same value in every block
      locate_lost<DIM>(s, a.remove_lost, gi, gs);
      if (!grid_barrier(s, q.barrier, G, gen, go)) return;
    }
  }
  if (blockIdx.x == 0 && t == 0) *q.step = step0 + q.nsteps;
}

template <int DIM, bool FLIP>
cudaError_t launch_persistent(const DevState& s, const StepArgs& a, const PersistentArgs& q,
                              cudaStream_t st) {
  auto kernel = k_steps_persistent_mixed<DIM, FLIP>;
  const size_t sm = mixed_staged_smem_bytes<DIM>(s.svf != nullptr);
  prefer_shared_memory<k_steps_persistent_mixed<DIM, FLIP>>();
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, MSTAGE_T, sm);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
  e = cudaMemsetAsync(q.barrier, 0, 2 * sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  DevState sv = s;
  StepArgs av = a;
  PersistentArgs qv = q;
  void* args[] = {&sv, &av, &qv};
  return cudaLaunchCooperativeKernel((const void*)kernel, dim3((unsigned)(per_sm * sms)), dim3(MSTAGE_T),
                                     args, sm, st);
}

template <int DIM, bool BOX>
void step_mixed(const DevState& s, const StepArgs& a, cudaStream_t st, Profiler& pr) {
  const int64_t np = s.np, nn = s.nn;
  if (np == 0) return;
  cudaMemsetAsync(s.nlost, 0, sizeof(unsigned), st);
  if (s.svf) cudaMemsetAsync(s.nplastic, 0, 2 * sizeof(unsigned), st);  // and nplastic_heavy
  const unsigned nt = (unsigned)node_block(a);
  const unsigned pb = nblk(np, 128), nb = nblk(nn, nt);
  const unsigned mcap = 148u * (unsigned)return_blocks(a);
  const unsigned mcb = pb < mcap ? pb : mcap;
  // P2G cell tiles of the step's launch shape
  auto p2g = [&](auto mode) {
    constexpr int MODE = decltype(mode)::value;
    constexpr int NV = Elem<DIM>::NV;
    if constexpr (MODE != 1) {  // the mass-momentum mapping velocity (128-thread tiles)
      if (a.vupd == 2 || a.vupd == 4) {
        k_p2g_tiles_mixed<DIM, MODE, BOX, 128, 1><<<nblk(s.ncells, 128 / NV), 128, 0, st>>>(s);
        return;
      }
      if (a.vupd == 3) {
        k_p2g_tiles_mixed<DIM, MODE, BOX, 128, 2><<<nblk(s.ncells, 128 / NV), 128, 0, st>>>(s);
        return;
      }
    }
    if (BOX && tile_threads(a, BOX) == 128)
      k_p2g_tiles_mixed<DIM, MODE, BOX, 128><<<nblk(s.ncells, 128 / NV), 128, 0, st>>>(s);
    else
      k_p2g_tiles_mixed<DIM, MODE, BOX><<<nblk(s.ncells, p2g_tile_t<BOX>() / NV), p2g_tile_t<BOX>(),
                                          0, st>>>(s);
  };
  // G2P of the mapping-matrix updates (ASFLIP 2, TPIC 3, APIC 4)
  auto g2p_affine = [&](auto stress) {
    constexpr bool STRESS = decltype(stress)::value;
    const float b = (float)a.beta;
    if (a.vupd == 2)
      k_g2p_mixed_affine<DIM, STRESS, 2, BOX><<<pb, 128, 0, st>>>(s, a.dt, b);
    else if (a.vupd == 3)
      k_g2p_mixed_affine<DIM, STRESS, 3, BOX><<<pb, 128, 0, st>>>(s, a.dt, b);
    else
      k_g2p_mixed_affine<DIM, STRESS, 4, BOX><<<pb, 128, 0, st>>>(s, a.dt, b);
  };
  auto mc_returns = [&]() {
    if (!s.svf) return;
    pr.begin(K_MC_RETURN, st);
    k_mc_return_mixed<DIM><<<mcb, 128, 0, st>>>(s);
    pr.end(K_MC_RETURN, st);
  };
  if (a.scheme == 1 && a.phase == 2) goto usl_second_half;
  pr.begin(K_SORT, st, SORT_KERNELS);
  counting_sort(s, st);
  pr.end(K_SORT, st);
  if (a.scheme == 2) {  // MUSL (mpm_scheme_musl.tcc:20-35)
    pr.begin(K_P2G, st);
    p2g(std::integral_constant<int, 2>{});
    pr.end(K_P2G, st);
    pr.begin(K_NODES_VEL, st);
    k_nodes_mixed<DIM, 1><<<nb, nt, 0, st>>>(s, a.dt, a.damping, a.g[0], a.g[1], a.g[2]);
    pr.end(K_NODES_VEL, st);
    pr.begin(K_G2P, st);
    if (a.flip)
      k_g2p_mixed<DIM, false, true, BOX, true><<<pb, 128, 0, st>>>(s, a.dt, (float)a.beta);
    else
      k_g2p_mixed<DIM, false, false, BOX, true><<<pb, 128, 0, st>>>(s, a.dt, (float)a.beta);
    pr.end(K_G2P, st);
    // mass and momentum again with the updated velocities, nodal velocity,
    // then the stress update at the step's positions
    pr.begin(K_P2G_FORCES, st);
    p2g(std::integral_constant<int, 0>{});
    pr.end(K_P2G_FORCES, st);
    pr.begin(K_NODES_ACC, st);
    k_nodes_mixed<DIM, 0><<<nb, nt, 0, st>>>(s, a.dt, a.damping, a.g[0], a.g[1], a.g[2]);
    pr.end(K_NODES_ACC, st);
    pr.begin(K_STRESS, st);
    k_stress_mixed<DIM, BOX><<<pb, 128, 0, st>>>(s, (float)a.dt);
    pr.end(K_STRESS, st);
    mc_returns();
    pr.begin(K_LOCATE, st);
    k_commit_locate_mixed<DIM><<<pb, 128, 0, st>>>(s);
    pr.end(K_LOCATE, st);
  } else if (a.scheme == 1) {  // USL
    pr.begin(K_P2G, st);
    p2g(std::integral_constant<int, 2>{});
    pr.end(K_P2G, st);
    if (a.phase == 1) return;
  usl_second_half:
    pr.begin(K_NODES_VEL, st);
    k_nodes_mixed<DIM, 1><<<nb, nt, 0, st>>>(s, a.dt, a.damping, a.g[0], a.g[1], a.g[2]);
    pr.end(K_NODES_VEL, st);
    pr.begin(K_G2P, st);
    const size_t sm = mixed_staged_smem_bytes<DIM>(s.svf != nullptr);
    if (a.vupd >= 2) {
      g2p_affine(std::true_type{});
    } else if (a.flip) {
      prefer_shared_memory<k_g2p_mixed_staged<DIM, true, BOX>>();
      k_g2p_mixed_staged<DIM, true, BOX><<<pb, MSTAGE_T, sm, st>>>(s, a.dt, (float)a.beta);
    } else {
      prefer_shared_memory<k_g2p_mixed_staged<DIM, false, BOX>>();
      k_g2p_mixed_staged<DIM, false, BOX><<<pb, MSTAGE_T, sm, st>>>(s, a.dt, (float)a.beta);
    }
    pr.end(K_G2P, st);
    mc_returns();
  } else {  // USF
    pr.begin(K_P2G, st);
    p2g(std::integral_constant<int, 0>{});
    pr.end(K_P2G, st);
    pr.begin(K_NODES_VEL, st);
    k_nodes_mixed<DIM, 0><<<nb, nt, 0, st>>>(s, a.dt, a.damping, a.g[0], a.g[1], a.g[2]);
    pr.end(K_NODES_VEL, st);
    pr.begin(K_STRESS, st);
    k_stress_mixed<DIM, BOX><<<pb, 128, 0, st>>>(s, (float)a.dt);
    pr.end(K_STRESS, st);
    mc_returns();
    pr.begin(K_P2G_FORCES, st);
    p2g(std::integral_constant<int, 1>{});
    pr.end(K_P2G_FORCES, st);
    pr.begin(K_NODES_ACC, st);
    k_nodes_mixed<DIM, 2><<<nb, nt, 0, st>>>(s, a.dt, a.damping, a.g[0], a.g[1], a.g[2]);
    pr.end(K_NODES_ACC, st);
    pr.begin(K_G2P, st);
    if (a.vupd >= 2)
      g2p_affine(std::false_type{});
    else if (a.flip)
      k_g2p_mixed<DIM, false, true, BOX><<<pb, 128, 0, st>>>(s, a.dt, (float)a.beta);
    else
      k_g2p_mixed<DIM, false, false, BOX><<<pb, 128, 0, st>>>(s, a.dt, (float)a.beta);
    pr.end(K_G2P, st);
  }
  pr.begin(K_LOCATE, st);
  launch_locate_fallback(DIM, s, a.remove_lost, st);
  pr.end(K_LOCATE, st);
}

}  // namespace

cudaError_t launch_steps_persistent_mixed(int dim, const DevState& s, const StepArgs& a,
                                          const PersistentArgs& q, cudaStream_t st) {
  if (s.np == 0 || q.nsteps <= 0) return cudaSuccess;
  if (dim == 2)
    return a.flip ? launch_persistent<2, true>(s, a, q, st) : launch_persistent<2, false>(s, a, q, st);
  return a.flip ? launch_persistent<3, true>(s, a, q, st) : launch_persistent<3, false>(s, a, q, st);
}

void launch_step_mixed(int dim, const DevState& s, const StepArgs& a, cudaStream_t st,
                       Profiler& prof) {
  // the particle kernels are compiled for tensor-product grids (box cells)
  // and for general meshes
  if (dim == 2)
    s.structured ? step_mixed<2, true>(s, a, st, prof) : step_mixed<2, false>(s, a, st, prof);
  else
    s.structured ? step_mixed<3, true>(s, a, st, prof) : step_mixed<3, false>(s, a, st, prof);
}

}  // namespace mpm_b200
