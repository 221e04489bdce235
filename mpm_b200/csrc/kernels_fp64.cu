// kernels_fp64.cu -- FP64 kernels of the explicit MPM step (USF and USL).
//
// Compiled with --fmad=false: every product and sum rounds on its own, as in
// the reference's scalar C++ arithmetic.  The nodal sums are deterministic:
// no floating-point atomics.  Each step sorts the particles by cell (counting
// sort); lanes that own a cell add its particles' contributions slot by slot
// in particle-id order; each node then adds the partial sums of its cells in
// ascending cell id.  The per-particle arithmetic is the reference's; only the
// order of the nodal sums differs (the reference adds in particle order).
//
// One step (USL):  sort -> p2g -> node update -> g2p(+stress, locate)
// One step (USF):  sort -> p2g(mass, momentum) -> node velocity -> stress
//                  -> p2g(forces) -> node update -> g2p(locate)
// followed by the exhaustive locate of particles that left their
// neighbourhood (usually none).
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "mpm_bulk.cuh"
#include "mpm_device.cuh"
#include "mpm_kernels.h"
#include "mpm_return.cuh"
#include "mpm_state.cuh"

// Minimum resident blocks per SM requested from the register allocator for
// the two particle kernels (occupancy versus spills, tuned on the B200).
#ifndef MPM_G2P_MIN_BLOCKS
#define MPM_G2P_MIN_BLOCKS 4  // 1.41 -> 1.01 ms per 4M-particle step despite spills
#endif
#ifndef MPM_MC_RETURN_MIN_BLOCKS
#define MPM_MC_RETURN_MIN_BLOCKS 4  // pass-loop return, 1M column at step 2000: 2 / 3 / 4 / 6 blocks -> FP64 0.362 / 0.320 / 0.323 / 0.403 ms, mixed 0.370 / 0.318 / 0.311 / 0.384 ms
#endif
#ifndef MPM_P2G_TILE_MIN_BLOCKS
#define MPM_P2G_TILE_MIN_BLOCKS 4  // 64 registers on a grid: 0.39 -> 0.345 ms (4M, 3D); 5, 6 spill
#endif

namespace mpm_b200 {

namespace {

// ------------------------------------------------------------ counting sort
__global__ void __launch_bounds__(256) k_count(DevState s) {
  count_particle(s, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// exclusive scan of n ints, SCAN_BLOCK per block (1024 threads x 4)
__global__ void __launch_bounds__(1024) k_scan_local(const int32_t* in, int32_t* out,
                                                     int32_t* bsum, int64_t n) {
  __shared__ int32_t warp_tot[32];
  const int64_t base = (int64_t)blockIdx.x * SCAN_BLOCK + threadIdx.x * 4;
  int32_t v[4], e[4], t = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    v[i] = (base + i < n) ? in[base + i] : 0;
    e[i] = t;
    t += v[i];
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int32_t x = t;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int32_t y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    int32_t z = warp_tot[lane];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, z, off);
      if (lane >= off) z += y;
    }
    warp_tot[lane] = z;
  }
  __syncthreads();
  const int32_t prefix = (w > 0 ? warp_tot[w - 1] : 0) + x - t;
#pragma unroll
  for (int i = 0; i < 4; ++i)
    if (base + i < n) out[base + i] = prefix + e[i];
  if (threadIdx.x == 1023 && bsum) bsum[blockIdx.x] = prefix + t;
}

// add the scanned block totals; start[n] = total
__global__ void __launch_bounds__(256) k_scan_add(int32_t* out, const int32_t* bscan,
                                                  const int32_t* bsum, int64_t n, int64_t nb) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += bscan[i / SCAN_BLOCK];
  if (i == 0) out[n] = bscan[nb - 1] + bsum[nb - 1];
}

__global__ void __launch_bounds__(256) k_fill(DevState s) {
  fill_particle(s, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------- P2G tiles
// Cell-slot partials: for slot k of cell c (its local node k), the sums over
// the cell's particles, in particle id order, of
//   mass m N (particle.tcc:643-655), momentum (m N) v, body force (g m) N
//   (:893-898), internal force -V (dN . sigma) (:915-949).
// MODE 0: mass and momentum; 1: forces; 2: all.
//
// Computed by cell tiles: a block takes p2g_tile_t / NV consecutive cells,
// whose particles are one contiguous range of the sorted order.  The block
// stages that range in chunks of p2g_tile_t particles (one particle per
// thread: local coordinates, mass, velocity, volume, stress and, off a
// tensor-product grid, J^-1) in shared memory; then thread (cell, slot) adds
// its slot's contributions of the cell's particles to 1 + 3 DIM accumulators:
// few registers per thread, coalesced particle reads, no atomics.
// AFF: the mass-momentum mapping velocity of the velocity update
// (particle.tcc:630-718): 0 the particle velocity (FLIP, PIC); 1 the affine
// v + B D^-1 r_i (APIC, ASFLIP; D the shape tensor sum_i N_i r_i r_i^T,
// r_i = x_i - x_p); 2 the Taylor v + B r_i (TPIC).  B is the particle's
// mapping matrix.
template <int DIM, int MODE, bool BOX, int AFF>
struct TileRows {
  static constexpr bool MM = MODE != 1, FORCES = MODE != 0;
  static constexpr int XI = 0, M = DIM, V = DIM + 1;
  static constexpr int SC = V + (MM ? DIM : 0);  // -volume
  static constexpr int S = SC + 1;
  static constexpr int INV = S + (FORCES ? PF<DIM>::NS : 0);
  static constexpr int XP = INV + (FORCES && !BOX ? DIM * DIM : 0);  // particle position
  static constexpr int MV = XP + (MM && AFF ? DIM : 0);              // velocity map matrix
  static constexpr int N = MV + (MM && AFF ? DIM * DIM : 0);
};

// On box cells without the affine rows the tile may also take 128 threads (a
// launch-shape choice); the blocks per SM scale so that the registers per
// thread stay the same.
template <bool BOX, int AFF, int T>
constexpr int tile_min_blocks() {
  return BOX && !AFF ? MPM_P2G_TILE_MIN_BLOCKS * 256 / T : MPM_P2G_TILE_MIN_BLOCKS;
}

template <int DIM, int MODE, bool BOX, int AFF, int T = p2g_tile_t<BOX, AFF>()>
__global__ void __launch_bounds__(T, (tile_min_blocks<BOX, AFF, T>()))
    k_p2g_tiles(DevState s, double g0, double g1, double g2) {
  constexpr int NV = Elem<DIM>::NV;
  constexpr int CB = T / NV;
  constexpr int NVAL = PV<DIM>::N;
  using RW = TileRows<DIM, MODE, BOX, AFF>;
  constexpr bool MM = RW::MM, FORCES = RW::FORCES;
  __shared__ double rows[RW::N][T];
  const int t = threadIdx.x;
  const int64_t c0 = (int64_t)blockIdx.x * CB;
  if (c0 >= s.ncells) return;
  const int64_t c1 = c0 + CB < s.ncells ? c0 + CB : s.ncells;
  const int64_t q_begin = s.start[c0], q_end = s.start[c1 - 1] + s.cnt[c1 - 1];
  if (q_begin == q_end) return;  // no particles in the tile (the whole block)
  // this thread's cell and slot
  const int64_t c = c0 + t / NV;
  const int k = t % NV;
  const bool mine = c < c1;
  const int64_t a0 = mine ? s.start[c] : 0;
  const int64_t a1 = mine ? a0 + s.cnt[c] : 0;
  // each cell's particle ids in ascending order in the first mapping of a step
  if constexpr (MODE != 1) sort_cell_ids<NV>(s.order + a0, (int)(a1 - a0), k);
  CellMap<DIM, BOX, double> box_map;
  if constexpr (BOX && FORCES) {
    if (a1 > a0) box_map = cell_map<DIM, true, double>(s, (int)c, nullptr, nullptr);
  }
  double xk[DIM];  // this slot's node, for the branch vectors of the mapping velocity
  if constexpr (MM && AFF) {
    int nid[NV];
    double X[NV * DIM];
    if (a1 > a0) cell_nodes_coords<DIM>(s, (int)c, nid, X);
#pragma unroll
    for (int d = 0; d < DIM; ++d) xk[d] = a1 > a0 ? X[k * DIM + d] : 0.;
  }
  const int64_t np = s.np;
  const double gv[3] = {g0, g1, g2};
  double acc[NVAL];
#pragma unroll
  for (int v = 0; v < NVAL; ++v) acc[v] = 0.;
  for (int64_t q0 = q_begin; q0 < q_end; q0 += T) {
    if (q0 != q_begin) __syncthreads();  // the previous chunk is consumed
    if (q0 + t < q_end) {
      const int64_t p = s.order[q0 + t];
      const int pc = s.cell[p];
      double x[DIM], xi[DIM];
      load_x<DIM>(s, p, x);
      particle_xi<DIM, BOX>(s, pc, x, xi);
#pragma unroll
      for (int d = 0; d < DIM; ++d) rows[RW::XI + d][t] = xi[d];
      if constexpr (MM && AFF) {
        double Mv[DIM * DIM];
        mapping_velocity_matrix<DIM, AFF>(s, p, pc, x, xi, Mv);
#pragma unroll
        for (int d = 0; d < DIM; ++d) rows[RW::XP + d][t] = x[d];
#pragma unroll
        for (int q = 0; q < DIM * DIM; ++q) rows[RW::MV + q][t] = Mv[q];
      }
      rows[RW::M][t] = s.pf[(int64_t)PF<DIM>::MASS * np + p];
      if constexpr (MM) {
#pragma unroll
        for (int d = 0; d < DIM; ++d) rows[RW::V + d][t] = s.pf[(int64_t)(PF<DIM>::V + d) * np + p];
      }
      if constexpr (FORCES) {
        rows[RW::SC][t] = -1. * s.pf[(int64_t)PF<DIM>::VOL * np + p];
#pragma unroll
        for (int q = 0; q < PF<DIM>::NS; ++q) rows[RW::S + q][t] = s.pf[(int64_t)(PF<DIM>::S + q) * np + p];
        if constexpr (!BOX) {
          int nid[NV];
          double X[NV * DIM];
          cell_nodes_coords<DIM>(s, pc, nid, X);
          const CellMap<DIM, false, double> m = cell_map<DIM, false>(s, pc, xi, X);
#pragma unroll
          for (int q = 0; q < DIM * DIM; ++q) rows[RW::INV + q][t] = m.inv[q];
        }
      }
    }
    __syncthreads();
    const int64_t j0 = a0 > q0 ? a0 : q0;
    const int64_t j1 = a1 < q0 + T ? a1 : q0 + T;
    for (int64_t j = j0; j < j1; ++j) {
      const int r = (int)(j - q0);
      double xi[DIM], N, G[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) xi[d] = rows[RW::XI + d][r];
      node_shape<DIM>(xi, k, N, G);
      const double m = rows[RW::M][r];
      if constexpr (MM) {
        const double mN = m * N;
        acc[PV<DIM>::MASS] += mN;
        double mv[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) mv[d] = rows[RW::V + d][r];
        if constexpr (AFF) {
          double br[DIM];
#pragma unroll
          for (int d = 0; d < DIM; ++d) br[d] = xk[d] - rows[RW::XP + d][r];
#pragma unroll
          for (int a = 0; a < DIM; ++a) {
            double sum = rows[RW::MV + a * DIM + 0][r] * br[0];
#pragma unroll
            for (int b = 1; b < DIM; ++b) sum = sum + rows[RW::MV + a * DIM + b][r] * br[b];
            mv[a] += sum;
          }
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) acc[PV<DIM>::MOM + d] += mN * mv[d];
      }
      if constexpr (FORCES) {
        const double sc = rows[RW::SC][r];
        double sig[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int q = 0; q < PF<DIM>::NS; ++q) sig[q] = rows[RW::S + q][r];
#pragma unroll
        for (int d = 0; d < DIM; ++d) acc[PV<DIM>::FEXT + d] += (gv[d] * m) * N;
        double Dn[DIM];
        if constexpr (BOX) {
          box_map.grad(G, Dn);
        } else {
          CellMap<DIM, false, double> m2;
#pragma unroll
          for (int q = 0; q < DIM * DIM; ++q) m2.inv[q] = rows[RW::INV + q][r];
          m2.grad(G, Dn);
        }
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
        for (int d = 0; d < DIM; ++d) acc[PV<DIM>::FINT + d] += f[d] * sc;
      }
    }
  }
  if (!mine || a1 == a0) return;  // empty cells keep no partials
  double* out = s.partials + ((int64_t)c * NV + k) * NVAL;
  if constexpr (MM) {
    out[PV<DIM>::MASS] = acc[PV<DIM>::MASS];
#pragma unroll
    for (int d = 0; d < DIM; ++d) out[PV<DIM>::MOM + d] = acc[PV<DIM>::MOM + d];
  }
  if constexpr (FORCES) {
#pragma unroll
    for (int d = 0; d < 2 * DIM; ++d) out[PV<DIM>::FEXT + d] = acc[PV<DIM>::FEXT + d];
  }
}

// ---------------------------------------------------------------- node update
// Adds the partial sums of the node's cells (ascending cell id) for the value
// range [v0, v0 + nv); returns false when no cell of the node holds particles
// (the node is inactive, cell.tcc:171-177).
template <int DIM, int V0, int NVS>
__device__ __forceinline__ bool gather_node(const DevState& s, int64_t node, double* sum) {
  constexpr int NV = Elem<DIM>::NV;
  constexpr int NVAL = PV<DIM>::N;
#pragma unroll
  for (int v = 0; v < NVS; ++v) sum[v] = 0.;
  bool active = false;
  auto add = [&](int c, int slot) {
    double src[NVS];
    load_partial_row<double, NVAL, V0, NVS>(s.partials + ((int64_t)c * NV + slot) * NVAL, src);
    if (!active) {
#pragma unroll
      for (int v = 0; v < NVS; ++v) sum[v] = src[v];
      active = true;
    } else {
#pragma unroll
      for (int v = 0; v < NVS; ++v) sum[v] = sum[v] + src[v];
    }
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

// node.tcc:309-345 (Cundall form of the nodal update, always taken:
// mpm_explicit.tcc:168-170)
template <int DIM>
__device__ __forceinline__ void node_accel_update(const DevState& s, double m, const double* fe,
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

// MODE 0: velocity from momentum (node.tcc:236-252, USF first pass);
// 1: velocity and then the acceleration update (USL);
// 2: acceleration update on the velocity of the first pass (USF)
template <int DIM, int MODE>
__global__ void __launch_bounds__(256) k_nodes(DevState s, double dt, double damping) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= s.nn) return;
  const int64_t nn = s.nn;
  double sum[PV<DIM>::N];
  constexpr int V0 = MODE == 2 ? PV<DIM>::FEXT : 0;
  constexpr int NVS = MODE == 0 ? 1 + DIM : (MODE == 1 ? PV<DIM>::N : 2 * DIM);
  if (!gather_node<DIM, V0, NVS>(s, n, sum)) return;
  const int bci = s.bc_index[n];
  double vel[DIM], acc[DIM];
  if constexpr (MODE == 2) {
    double mm[1];
    gather_node<DIM, PV<DIM>::MASS, 1>(s, n, mm);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      vel[d] = s.nf[(int64_t)(NF<DIM>::VEL + d) * nn + n];
      acc[d] = s.nf[(int64_t)(NF<DIM>::ACC + d) * nn + n];
    }
    node_accel_update<DIM>(s, mm[0], &sum[0], &sum[DIM], vel, acc, bci, dt, damping);
  } else {
    const double m = sum[PV<DIM>::MASS];
#pragma unroll
    for (int d = 0; d < DIM; ++d) vel[d] = acc[d] = 0.;
    if (m > 1.E-16) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) vel[d] = sum[PV<DIM>::MOM + d] / m;
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        if (fabs(vel[d]) < 1.E-15) vel[d] = 0.;
    }
    if (bci >= 0) apply_velocity_constraints<DIM>(s.bcs[bci], vel, acc);
    if constexpr (MODE == 1)
      node_accel_update<DIM>(s, m, &sum[PV<DIM>::FEXT], &sum[PV<DIM>::FINT], vel, acc, bci, dt,
                             damping);
  }
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    s.nf[(int64_t)(NF<DIM>::VEL + d) * nn + n] = vel[d];
    s.nf[(int64_t)(NF<DIM>::ACC + d) * nn + n] = acc[d];
  }
}

// One particle's fields, read and written in global memory (GlobalRow) or in
// the block's shared-memory staging (SmemRow, STAGE_T particles per row).
struct GlobalRow {
  const DevState& s;
  int64_t p;
  __device__ __forceinline__ int64_t index() const { return p; }
  __device__ __forceinline__ double& f(int field) const { return s.pf[(int64_t)field * s.np + p]; }
  __device__ __forceinline__ double& sv(int k) const { return s.sv[(int64_t)k * s.np + p]; }
  __device__ __forceinline__ int mat() const { return s.mat[p]; }
};
constexpr int STAGE_T = 128;  // particles per staged block (= PAD_PARTICLES)
struct SmemRow {
  double* rows;  // [field][STAGE_T]
  double* svr;   // [SV_N][STAGE_T]
  int t;
  int m;
  int64_t p;
  __device__ __forceinline__ int64_t index() const { return p; }
  __device__ __forceinline__ double& f(int field) const { return rows[field * STAGE_T + t]; }
  __device__ __forceinline__ double& sv(int k) const { return svr[k * STAGE_T + t]; }
  __device__ __forceinline__ int mat() const { return m; }
};

// ------------------------------------------------------- stress and strain
// mpm_scheme.tcc:75-103: F increment (particle.tcc:1580-1628), strain
// (:819-876), volume (:598-605), material stress (:880-889), F (:1654-1658).
// D: dN/dx at the particle (start of step); the cell's centroid gradients
// come from the per-cell table computed once from the mesh.
template <int DIM, class Row>
__device__ __forceinline__ void stress_update(const DevState& s, const Row& r, int c,
                                              const int* nid, const double* D, double dt) {
  constexpr int NV = Elem<DIM>::NV;
  const int64_t nn = s.nn;
  const double* Dc = s.dndx_c + (int64_t)c * NV * DIM;
  double Fi[DIM * DIM];
#pragma unroll
  for (int r = 0; r < DIM; ++r)
#pragma unroll
    for (int q = 0; q < DIM; ++q) Fi[r * DIM + q] = (r == q) ? 1. : 0.;
  double sr[6] = {0, 0, 0, 0, 0, 0};
  double src[3] = {0, 0, 0};
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double vel[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) vel[d] = s.nf[(int64_t)(NF<DIM>::VEL + d) * nn + nid[i]];
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
      for (int q = 0; q < DIM; ++q) Fi[r * DIM + q] += vel[r] * D[i * DIM + q] * dt;
    const double* Dn = &D[i * DIM];
    double dc[DIM];
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
#pragma unroll
  for (int r = 0; r < DIM; ++r)
#pragma unroll
    for (int q = 0; q < DIM; ++q) {
      if (r != q && fabs(Fi[r * DIM + q]) < 1.E-15) Fi[r * DIM + q] = 0.;
      if (r == q && fabs(Fi[r * DIM + q] - 1.) < 1.E-15) Fi[r * DIM + q] = 1.;
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
  if constexpr (DIM == 2) {
    const int map[3] = {0, 1, 3};
#pragma unroll
    for (int k = 0; k < 3; ++k) r.f(PF<2>::E + k) += dstrain[map[k]];
  } else {
#pragma unroll
    for (int k = 0; k < 6; ++k) r.f(PF<3>::E + k) += dstrain[k];
  }
  double* volp = &r.f(PF<DIM>::VOL);
  double* rhop = &r.f(PF<DIM>::RHO);
  const double vol = *volp * (1. + dvol);
  const double rho = *rhop / (1. + dvol);
  *volp = vol;
  *rhop = rho;
  double sig[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < PF<DIM>::NS; ++k) sig[k] = r.f(PF<DIM>::S + k);
  const MaterialParams& mp = s.mats[r.mat()];
  double out[6];
  bool deferred = false;
  if (mp.type == 0) {
    material_compute_stress(mp, sig, dstrain, rho, nullptr, out);
  } else {
    double sv[SV_N];
#pragma unroll
    for (int k = 0; k < SV_N; ++k) sv[k] = r.sv(k);
    if (mc_stress<double, double, true>(mp, sig, dstrain, rho, sv, sv[SV_PD], out) == MC_DEFERRED) {
      // plastic: the return runs in k_mc_return from the unchanged stress and state
      deferred = true;
      const unsigned i = defer_slot_by_cost(s, r.index());
      s.plist[i] = (int32_t)r.index();
#pragma unroll
      for (int k = 0; k < 6; ++k) s.pbuf[(int64_t)k * s.np + i] = dstrain[k];
      s.pbuf[(int64_t)6 * s.np + i] = rho;
    } else {
#pragma unroll
      for (int k = 0; k < SV_N; ++k) r.sv(k) = sv[k];
    }
  }
  if (!deferred) {
#pragma unroll
    for (int k = 0; k < PF<DIM>::NS; ++k) r.f(PF<DIM>::S + k) = out[k];
  }
  if constexpr (DIM == 2) {
    double F[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) F[k] = r.f(PF<2>::F + k);
    // 3x3 product with F_inc and F both (0,0,1) in the third row and column:
    // the dropped terms are exact zeros
    const double r00 = Fi[0] * F[0] + Fi[1] * F[2];
    const double r01 = Fi[0] * F[1] + Fi[1] * F[3];
    const double r10 = Fi[2] * F[0] + Fi[3] * F[2];
    const double r11 = Fi[2] * F[1] + Fi[3] * F[3];
    r.f(PF<2>::F + 0) = r00;
    r.f(PF<2>::F + 1) = r01;
    r.f(PF<2>::F + 2) = r10;
    r.f(PF<2>::F + 3) = r11;
  } else {
    double F[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) F[k] = r.f(PF<3>::F + k);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int q = 0; q < 3; ++q)
        r.f(PF<3>::F + a * 3 + q) =
            (Fi[a * 3 + 0] * F[0 * 3 + q] + Fi[a * 3 + 1] * F[1 * 3 + q]) + Fi[a * 3 + 2] * F[2 * 3 + q];
  }
}

// dN/dx of all local nodes at xi
template <int DIM, bool BOX>
__device__ __forceinline__ void dn_dx_all(const DevState& s, int c, const double* xi,
                                          const double* X, double* D) {
  constexpr int NV = Elem<DIM>::NV;
  const CellMap<DIM, BOX, double> map = cell_map<DIM, BOX>(s, c, xi, X);
#pragma unroll
  for (int n = 0; n < NV; ++n) dn_dx_node<DIM>(xi, map, n, &D[n * DIM]);
}

// USF: the stress update with the velocities of compute_velocity
template <int DIM, bool BOX>
__global__ void __launch_bounds__(128) k_stress(DevState s, double dt) {
  constexpr int NV = Elem<DIM>::NV;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0) return;
  double x[DIM], xi[DIM], D[NV * DIM], X[NV * DIM];
  int nid[NV];
  load_x<DIM>(s, p, x);
  particle_xi<DIM, BOX>(s, c, x, xi);
  cell_nodes_for<DIM, BOX>(s, c, nid, X);
  dn_dx_all<DIM, BOX>(s, c, xi, X, D);
  stress_update<DIM>(s, GlobalRow{s, p}, c, nid, D, dt);
}

// --------------------------------------------------------------------- G2P
// particle.tcc:994-1067 FLIP / PIC; mesh.tcc:1454-1467 particle velocity
// constraints; USL stress update (mpm_scheme_usl.tcc:14-17); locate.
template <int DIM, bool STRESS, int VU, bool BOX>
__global__ void __launch_bounds__(128, MPM_G2P_MIN_BLOCKS) k_g2p(DevState s, double dt,
                                                                 double beta) {
  constexpr int NV = Elem<DIM>::NV;
  constexpr bool FLIP = VU == 0, ASFLIP = VU == 2, TPIC = VU == 3;  // 1 PIC, 4 APIC
  constexpr bool ACC = FLIP || ASFLIP;  // nodal acceleration interpolated
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0) return;
  const int64_t np = s.np, nn = s.nn;
  double x[DIM], xi[DIM], N[NV], X[NV * DIM];
  int nid[NV];
  load_x<DIM>(s, p, x);
  particle_xi<DIM, BOX>(s, c, x, xi);
  shapefn<DIM>(xi, N);
  if constexpr (VU >= 2)
    cell_nodes_coords<DIM>(s, c, nid, X);  // the branch vectors need the nodes
  else
    cell_nodes_for<DIM, BOX>(s, c, nid, X);
  double nvel[DIM], nacc[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) nvel[d] = nacc[d] = 0.;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const int n = nid[i];
#pragma unroll
    for (int d = 0; d < DIM; ++d) nvel[d] += N[i] * s.nf[(int64_t)(NF<DIM>::VEL + d) * nn + n];
    if constexpr (ACC) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) nacc[d] += N[i] * s.nf[(int64_t)(NF<DIM>::ACC + d) * nn + n];
    }
  }
  double sep[DIM];  // the velocity that moves the particle
#pragma unroll
  for (int d = 0; d < DIM; ++d) sep[d] = nvel[d];
  if constexpr (VU >= 2) {
    // mapping matrix at the step-start position (particle.tcc:1663-1704):
    // affine B = sum_i N_i v_i r_i^T (APIC, ASFLIP) or the velocity
    // gradient sum_i v_i dN_i/dx^T (TPIC); entries below 1e-15 set to 0
    double B[DIM * DIM], D[NV * DIM];
#pragma unroll
    for (int q = 0; q < DIM * DIM; ++q) B[q] = 0.;
    if constexpr (TPIC || ASFLIP) dn_dx_all<DIM, BOX>(s, c, xi, X, D);
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double vel[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) vel[d] = s.nf[(int64_t)(NF<DIM>::VEL + d) * nn + nid[i]];
#pragma unroll
      for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int b = 0; b < DIM; ++b) {
          if constexpr (TPIC)
            B[a * DIM + b] += vel[a] * D[i * DIM + b];
          else
            B[a * DIM + b] += (N[i] * vel[a]) * (X[i * DIM + b] - x[b]);
        }
    }
#pragma unroll
    for (int q = 0; q < DIM * DIM; ++q) {
      if (fabs(B[q]) < 1.E-15) B[q] = 0.;
      s.mapb[(int64_t)q * np + p] = B[q];
    }
    if constexpr (ASFLIP) {
      // beta (particle.tcc:1711-1730): 0 next to a velocity-constrained node
      // or when the deformation gradient increment compresses
      double bp = 1.0;
#pragma unroll
      for (int i = 0; i < NV; ++i) {
        const int bci = s.bc_index[nid[i]];
        if (bci >= 0 && s.bcs[bci].vel_mask != 0) bp = 0.0;
      }
      double Fi[9] = {1., 0., 0., 0., 1., 0., 0., 0., 1.};
#pragma unroll
      for (int i = 0; i < NV; ++i) {
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          const double va = s.nf[(int64_t)(NF<DIM>::VEL + a) * nn + nid[i]];
#pragma unroll
          for (int b = 0; b < DIM; ++b) Fi[a * 3 + b] += va * D[i * DIM + b] * dt;
        }
      }
#pragma unroll
      for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int b = 0; b < DIM; ++b) {
          if (a != b && fabs(Fi[a * 3 + b]) < 1.E-15) Fi[a * 3 + b] = 0.;
          if (a == b && fabs(Fi[a * 3 + b] - 1.) < 1.E-15) Fi[a * 3 + b] = 1.;
        }
      const double J = Fi[0] * (Fi[4] * Fi[8] - Fi[5] * Fi[7]) -
                       Fi[1] * (Fi[3] * Fi[8] - Fi[5] * Fi[6]) +
                       Fi[2] * (Fi[3] * Fi[7] - Fi[4] * Fi[6]);
      if (J < 1.0) bp = 0.0;
      // particle.tcc:1096-1110: FLIP/PIC blend for the velocity, the
      // separable blend for the position
      double flip[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        flip[d] = s.pf[(int64_t)(PF<DIM>::V + d) * np + p] + nacc[d] * dt;
#pragma unroll
      for (int d = 0; d < DIM; ++d) nacc[d] = flip[d];  // keeps the FLIP velocity
#pragma unroll
      for (int d = 0; d < DIM; ++d) sep[d] = bp * beta * flip[d] + (1.0 - bp * beta) * nvel[d];
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
  } else if constexpr (ASFLIP) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] = beta * nacc[d] + (1.0 - beta) * nvel[d];
  } else {
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] = nvel[d];
  }
  double xn[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    xn[d] = x[d] + sep[d] * dt;
    s.pf[(int64_t)(PF<DIM>::X + d) * np + p] = xn[d];
    s.pf[(int64_t)(PF<DIM>::U + d) * np + p] += sep[d] * dt;
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
    dn_dx_all<DIM, BOX>(s, c, xi, X, D);
    stress_update<DIM>(s, GlobalRow{s, p}, c, nid, D, dt);
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

// USL G2P + stress update + locate with the block's particle slices staged in
// shared memory by the bulk-copy engine.  One thread issues the copies of
// every field slice (1 KB each) at block start: phase A (x, u, v, cell,
// material, velocity-constraint slot) and phase B (stress, strain, F,
// volume, density, MohrCoulomb state).  The threads gather nodal values while
// phase B is in flight, update the staged rows in place and one thread stores
// the rows back with bulk copies.  The arithmetic is k_g2p<DIM, true, FLIP ? 0 : 1, BOX>'s.
static_assert(STAGE_T == PAD_PARTICLES, "staged slices are whole padded blocks");
template <int DIM>
constexpr int staged_rows() { return PF<DIM>::MASS; }  // fields X .. RHO
template <int DIM>
constexpr size_t staged_smem_bytes(bool mc) {
  return (size_t)(staged_rows<DIM>() + (mc ? SV_N : 0)) * STAGE_T * 8 + STAGE_T * (4 + 2 + 2);
}

template <int DIM, bool FLIP, bool BOX>
__global__ void __launch_bounds__(STAGE_T, MPM_G2P_MIN_BLOCKS)
    k_g2p_staged(DevState s, double dt, double beta) {
  constexpr int NV = Elem<DIM>::NV;
  constexpr int T = STAGE_T;
  constexpr int ROWS = staged_rows<DIM>();
  constexpr int ROWS_A = PF<DIM>::S;  // x, u, v
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar[2];
  __shared__ int timed_out;
  const bool mc = s.sv != nullptr;
  double* rows = reinterpret_cast<double*>(smem);
  double* svr = rows + ROWS * T;
  int32_t* scell = reinterpret_cast<int32_t*>(svr + (mc ? SV_N * T : 0));
  uint16_t* smat = reinterpret_cast<uint16_t*>(scell + T);
  int16_t* spvc = reinterpret_cast<int16_t*>(smat + T);
  const int t = threadIdx.x;
  const int64_t p0 = (int64_t)blockIdx.x * T;
  const int64_t np = s.np, nn = s.nn;
  if (t == 0) {
    timed_out = 0;
    bulk::mbar_init(&bar[0], 1);
    bulk::mbar_init(&bar[1], 1);
    bulk::fence_barrier_init();
  }
  __syncthreads();
  if (t == 0) {
    bulk::mbar_arrive_expect_tx(&bar[0], ROWS_A * T * 8 + T * (4 + 2 + 2));
    for (int f = 0; f < ROWS_A; ++f) bulk::load(rows + f * T, s.pf + f * np + p0, T * 8, &bar[0]);
    bulk::load(scell, s.cell + p0, T * 4, &bar[0]);
    bulk::load(smat, s.mat + p0, T * 2, &bar[0]);
    bulk::load(spvc, s.pvc + p0, T * 2, &bar[0]);
    bulk::mbar_arrive_expect_tx(&bar[1], (ROWS - ROWS_A + (mc ? SV_N : 0)) * T * 8);
    for (int f = ROWS_A; f < ROWS; ++f) bulk::load(rows + f * T, s.pf + f * np + p0, T * 8, &bar[1]);
    if (mc)
      for (int k = 0; k < SV_N; ++k) bulk::load(svr + k * T, s.sv + k * np + p0, T * 8, &bar[1]);
  }
  const bool okA = bulk::mbar_wait(&bar[0], 0) && !(s.test_wait_timeout && !bulk::mbar_wait_never(&bar[0]));
  const int c = okA ? scell[t] : -1;
  const int64_t p = p0 + t;
  const SmemRow r{rows, svr, t, okA ? (int)smat[t] : 0, p0 + t};
  double xn[DIM];
  const bool active = c >= 0;
  double xi[DIM];
  if (active) {
    double x[DIM], N[NV], X[NV * DIM];
    int nid[NV];
#pragma unroll
    for (int d = 0; d < DIM; ++d) x[d] = r.f(PF<DIM>::X + d);
    particle_xi<DIM, BOX>(s, c, x, xi);
    shapefn<DIM>(xi, N);
    cell_nodes_for<DIM, BOX>(s, c, nid, X);
    double nvel[DIM], nacc[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) nvel[d] = nacc[d] = 0.;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      const int n = nid[i];
#pragma unroll
      for (int d = 0; d < DIM; ++d) nvel[d] += N[i] * s.nf[(int64_t)(NF<DIM>::VEL + d) * nn + n];
      if constexpr (FLIP) {
#pragma unroll
        for (int d = 0; d < DIM; ++d) nacc[d] += N[i] * s.nf[(int64_t)(NF<DIM>::ACC + d) * nn + n];
      }
    }
    double v[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] = r.f(PF<DIM>::V + d);
    if constexpr (FLIP) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) v[d] += nacc[d] * dt;
#pragma unroll
      for (int d = 0; d < DIM; ++d) v[d] = beta * v[d] + (1.0 - beta) * nvel[d];
    } else {
#pragma unroll
      for (int d = 0; d < DIM; ++d) v[d] = nvel[d];
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      xn[d] = x[d] + nvel[d] * dt;
      r.f(PF<DIM>::X + d) = xn[d];
      r.f(PF<DIM>::U + d) += nvel[d] * dt;
    }
    const int pv = spvc[t];
    if (pv >= 0) {
      const ParticleVC& vc = s.pvcs[pv];
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        if (vc.mask & (1u << d)) v[d] = vc.value[d];
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) r.f(PF<DIM>::V + d) = v[d];
  }
  const bool okB = okA && bulk::mbar_wait(&bar[1], 0);
  if (!okA || !okB) timed_out = 1;
  if (active && okB) {
    // node ids and coordinates again rather than kept live across the wait
    double X[NV * DIM], D[NV * DIM];
    int nid[NV];
    cell_nodes_for<DIM, BOX>(s, c, nid, X);
    dn_dx_all<DIM, BOX>(s, c, xi, X, D);
    stress_update<DIM>(s, r, c, nid, D, dt);
  }
  bulk::fence_shared_to_async();
  __syncthreads();
  if (timed_out) {
    // copies that never completed: report, give in-flight copies a last
    // bounded wait, store nothing
    if (t == 0) {
      raise_err(s, ERR_TIMEOUT);
      bulk::mbar_wait(&bar[0], 0);
      bulk::mbar_wait(&bar[1], 0);
    }
    return;
  }
  if (t == 0) {
    for (int f = 0; f < ROWS; ++f) bulk::store(s.pf + f * np + p0, rows + f * T, T * 8);
    if (mc)  // phi, psi, cohesion and tension cutoff change only with softening
      for (int k = 0; k < SV_N; ++k)
        if (s.any_softening || k == SV_YIELD || k >= SV_EPS)
          bulk::store(s.sv + k * np + p0, svr + k * T, T * 8);
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
  if (t == 0) bulk::store_wait_read();
}

// MUSL particle kinematics (particle.tcc:994-1067 as in k_g2p): the new
// positions go to xnext, so that the second mapping of mass and momentum and
// the stress update of the step still see the step-start positions (the
// reference keeps each particle's shape functions until the next step).
template <int DIM, bool FLIP, bool BOX>
__global__ void __launch_bounds__(128, MPM_G2P_MIN_BLOCKS) k_g2p_musl(DevState s, double dt,
                                                                      double beta) {
  constexpr int NV = Elem<DIM>::NV;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0) return;
  const int64_t np = s.np, nn = s.nn;
  double x[DIM], xi[DIM], N[NV], X[NV * DIM];
  int nid[NV];
  load_x<DIM>(s, p, x);
  particle_xi<DIM, BOX>(s, c, x, xi);
  shapefn<DIM>(xi, N);
  cell_nodes_for<DIM, BOX>(s, c, nid, X);
  double nvel[DIM], nacc[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) nvel[d] = nacc[d] = 0.;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const int n = nid[i];
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
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    s.xnext[(int64_t)d * np + p] = x[d] + nvel[d] * dt;
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
}

// MUSL end of step: the new positions replace the old, then locate
template <int DIM>
__global__ void __launch_bounds__(128) k_commit_locate(DevState s) {
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
    s.pf[(int64_t)(PF<DIM>::X + d) * np + p] = xn[d];
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

// The MohrCoulomb returns deferred by stress_update, one thread per listed
// particle (grid-stride over the light entries, then the heavy ones), from the
// particle's stress and state before the step's update: the evaluations of
// the undeferred update with the same inputs, run as mc_return's passes, so
// the same results.  Records the return's number of corrections for the next
// step's grouping.
template <int DIM>
__global__ void __launch_bounds__(128, MPM_MC_RETURN_MIN_BLOCKS) k_mc_return(DevState s) {
  const unsigned nl = *s.nplastic, n = nl + *s.nplastic_heavy;
  const int64_t np = s.np;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const unsigned i = list_slot(s, t, nl);
    const int64_t p = s.plist[i];
    double sig[6] = {0, 0, 0, 0, 0, 0}, de[6], sv[SV_N], out[6];
#pragma unroll
    for (int k = 0; k < PF<DIM>::NS; ++k) sig[k] = s.pf[(int64_t)(PF<DIM>::S + k) * np + p];
#pragma unroll
    for (int k = 0; k < 6; ++k) de[k] = s.pbuf[(int64_t)k * np + i];
    const double rho = s.pbuf[(int64_t)6 * np + i];
#pragma unroll
    for (int k = 0; k < SV_N; ++k) sv[k] = s.sv[(int64_t)k * np + p];
    int nc = 0;
    mc_return(s.mats[s.mat[p]], sig, de, rho, sv, out, &nc);  // a MohrCoulomb point
    s.rpass[p] = (uint8_t)(nc < 255 ? nc : 255);
#pragma unroll
    for (int k = 0; k < SV_N; ++k) s.sv[(int64_t)k * np + p] = sv[k];
#pragma unroll
    for (int k = 0; k < PF<DIM>::NS; ++k) s.pf[(int64_t)(PF<DIM>::S + k) * np + p] = out[k];
  }
}

// Exhaustive search for particles not in their cell or its neighbours
// (mesh.tcc:1136-1148 with one thread: the first cell in id order that
// contains the point).  Grid-stride over the lost list; usually empty.
template <int DIM>
__global__ void k_locate_fallback(DevState s, int remove_lost) {
  locate_lost<DIM>(s, remove_lost, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

inline unsigned nblocks(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

void counting_sort_impl(const DevState& s, cudaStream_t st) {
  const int64_t nc = s.ncells;
  cudaMemsetAsync(s.cnt, 0, sizeof(int32_t) * nc, st);
  k_count<<<nblocks(s.np, 256), 256, 0, st>>>(s);
  const int64_t nb = (nc + SCAN_BLOCK - 1) / SCAN_BLOCK;
  k_scan_local<<<(unsigned)nb, 1024, 0, st>>>(s.cnt, s.start, s.bsum, nc);
  // block totals (nb <= SCAN_BLOCK is checked at set-up) scanned by one block
  k_scan_local<<<1, 1024, 0, st>>>(s.bsum, s.bsum + nb, nullptr, nb);
  k_scan_add<<<nblocks(nc, 256), 256, 0, st>>>(s.start, s.bsum + nb, s.bsum, nc, nb);
  k_fill<<<nblocks(s.np, 256), 256, 0, st>>>(s);
}

// Ask for the shared-memory carveout that lets MIN_BLOCKS staged blocks share
// an SM (set once per kernel and device).
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

template <int DIM, bool BOX>
void step_impl(const DevState& s, const StepArgs& a, cudaStream_t st, Profiler& pr) {
  const int64_t np = s.np, nn = s.nn;
  if (np == 0) return;
  cudaMemsetAsync(s.nlost, 0, sizeof(unsigned), st);
  if (s.sv) cudaMemsetAsync(s.nplastic, 0, 2 * sizeof(unsigned), st);  // and nplastic_heavy
  const unsigned nt = (unsigned)node_block(a);
  const unsigned pb128 = nblocks(np, 128), nb = nblocks(nn, nt);
  const unsigned mcb = (unsigned)std::min<int64_t>(nblocks(np, 128), 148 * return_blocks(a));
  auto mc_returns = [&]() {
    if (!s.sv) return;
    pr.begin(K_MC_RETURN, st);
    k_mc_return<DIM><<<mcb, 128, 0, st>>>(s);
    pr.end(K_MC_RETURN, st);
  };
  auto p2g = [&](auto mode) {
    constexpr int MODE = decltype(mode)::value;
    auto launch = [&](auto aff) {
      constexpr int AFF = decltype(aff)::value;
      constexpr int TT = p2g_tile_t<BOX, AFF>();
      if (BOX && !AFF && tile_threads(a, BOX) == 128)
        k_p2g_tiles<DIM, MODE, BOX, AFF, 128><<<nblocks(s.ncells, 128 / Elem<DIM>::NV), 128, 0, st>>>(
            s, a.g[0], a.g[1], a.g[2]);
      else
        k_p2g_tiles<DIM, MODE, BOX, AFF><<<nblocks(s.ncells, TT / Elem<DIM>::NV), TT, 0, st>>>(
            s, a.g[0], a.g[1], a.g[2]);
    };
    if constexpr (MODE != 1) {  // the mass-momentum mapping velocity
      if (a.vupd == 2 || a.vupd == 4) return launch(std::integral_constant<int, 1>{});
      if (a.vupd == 3) return launch(std::integral_constant<int, 2>{});
    }
    launch(std::integral_constant<int, 0>{});
  };
  // unstaged G2P (USF kinematics, or USL with its stress update) for the
  // velocity update of the run
  auto g2p = [&](auto stress) {
    constexpr bool STRESS = decltype(stress)::value;
    switch (a.vupd) {
      case 0: k_g2p<DIM, STRESS, 0, BOX><<<pb128, 128, 0, st>>>(s, a.dt, a.beta); break;
      case 1: k_g2p<DIM, STRESS, 1, BOX><<<pb128, 128, 0, st>>>(s, a.dt, a.beta); break;
      case 2: k_g2p<DIM, STRESS, 2, BOX><<<pb128, 128, 0, st>>>(s, a.dt, a.beta); break;
      case 3: k_g2p<DIM, STRESS, 3, BOX><<<pb128, 128, 0, st>>>(s, a.dt, a.beta); break;
      default: k_g2p<DIM, STRESS, 4, BOX><<<pb128, 128, 0, st>>>(s, a.dt, a.beta); break;
    }
  };
  if (a.scheme == 1 && a.phase == 2) goto usl_second_half;
  pr.begin(K_SORT, st, SORT_KERNELS);
  counting_sort_impl(s, st);
  pr.end(K_SORT, st);
  if (a.scheme == 2) {  // MUSL (mpm_scheme_musl.tcc)
    pr.begin(K_P2G, st);
    p2g(std::integral_constant<int, 2>{});
    pr.end(K_P2G, st);
    pr.begin(K_NODES_VEL, st);
    k_nodes<DIM, 1><<<nb, nt, 0, st>>>(s, a.dt, a.damping);
    pr.end(K_NODES_VEL, st);
    pr.begin(K_G2P, st);
    if (a.flip)
      k_g2p_musl<DIM, true, BOX><<<pb128, 128, 0, st>>>(s, a.dt, a.beta);
    else
      k_g2p_musl<DIM, false, BOX><<<pb128, 128, 0, st>>>(s, a.dt, a.beta);
    pr.end(K_G2P, st);
    // mass and momentum again with the updated velocities, nodal velocity,
    // then the stress update (mpm_scheme_musl.tcc:13-35)
    pr.begin(K_P2G_FORCES, st);
    p2g(std::integral_constant<int, 0>{});
    pr.end(K_P2G_FORCES, st);
    pr.begin(K_NODES_ACC, st);
    k_nodes<DIM, 0><<<nb, nt, 0, st>>>(s, a.dt, a.damping);
    pr.end(K_NODES_ACC, st);
    pr.begin(K_STRESS, st);
    k_stress<DIM, BOX><<<pb128, 128, 0, st>>>(s, a.dt);
    pr.end(K_STRESS, st);
    mc_returns();
    pr.begin(K_LOCATE, st);
    k_commit_locate<DIM><<<pb128, 128, 0, st>>>(s);
    pr.end(K_LOCATE, st);
  } else if (a.scheme == 1) {  // USL
    pr.begin(K_P2G, st);
    p2g(std::integral_constant<int, 2>{});
    pr.end(K_P2G, st);
    if (a.phase == 1) return;
  usl_second_half:
    pr.begin(K_NODES_VEL, st);
    k_nodes<DIM, 1><<<nb, nt, 0, st>>>(s, a.dt, a.damping);
    pr.end(K_NODES_VEL, st);
    pr.begin(K_G2P, st);
    const size_t sm = staged_smem_bytes<DIM>(s.sv != nullptr);
    if (a.vupd >= 2) {  // the mapping-matrix updates: G2P and stress unstaged
      g2p(std::true_type{});
    } else if (a.flip) {
      prefer_shared_memory<k_g2p_staged<DIM, true, BOX>>();
      k_g2p_staged<DIM, true, BOX><<<pb128, STAGE_T, sm, st>>>(s, a.dt, a.beta);
    } else {
      prefer_shared_memory<k_g2p_staged<DIM, false, BOX>>();
      k_g2p_staged<DIM, false, BOX><<<pb128, STAGE_T, sm, st>>>(s, a.dt, a.beta);
    }
    pr.end(K_G2P, st);
    mc_returns();
  } else {  // USF
    pr.begin(K_P2G, st);
    p2g(std::integral_constant<int, 0>{});
    pr.end(K_P2G, st);
    pr.begin(K_NODES_VEL, st);
    k_nodes<DIM, 0><<<nb, nt, 0, st>>>(s, a.dt, a.damping);
    pr.end(K_NODES_VEL, st);
    pr.begin(K_STRESS, st);
    k_stress<DIM, BOX><<<pb128, 128, 0, st>>>(s, a.dt);
    pr.end(K_STRESS, st);
    mc_returns();
    pr.begin(K_P2G_FORCES, st);
    p2g(std::integral_constant<int, 1>{});
    pr.end(K_P2G_FORCES, st);
    pr.begin(K_NODES_ACC, st);
    k_nodes<DIM, 2><<<nb, nt, 0, st>>>(s, a.dt, a.damping);
    pr.end(K_NODES_ACC, st);
    pr.begin(K_G2P, st);
    g2p(std::false_type{});
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
  // the particle kernels are compiled for tensor-product grids (box cells)
  // and for general meshes
  if (dim == 2)
    s.structured ? step_impl<2, true>(s, a, st, prof) : step_impl<2, false>(s, a, st, prof);
  else
    s.structured ? step_impl<3, true>(s, a, st, prof) : step_impl<3, false>(s, a, st, prof);
}

void counting_sort(const DevState& s, cudaStream_t st) { counting_sort_impl(s, st); }

// The first half of a USL step: sort, P2G of mass, momentum and forces, and the
// node update (FLIP / PIC mapping velocity), leaving the cell-slot partials and
// the nodal velocity and acceleration of the step.  The reverse sweep of the
// adjoint recomputes these from a stored step-start state.
void launch_p2g_nodes_fp64(int dim, const DevState& s, const StepArgs& a, cudaStream_t st) {
  if (s.np == 0) return;
  counting_sort_impl(s, st);
  auto run = [&](auto dimc, auto boxc) {
    constexpr int DIM = decltype(dimc)::value;
    constexpr bool BOX = decltype(boxc)::value;
    constexpr int TT = p2g_tile_t<BOX, 0>();
    k_p2g_tiles<DIM, 2, BOX, 0><<<nblocks(s.ncells, TT / Elem<DIM>::NV), TT, 0, st>>>(
        s, a.g[0], a.g[1], a.g[2]);
    k_nodes<DIM, 1><<<nblocks(s.nn, 256), 256, 0, st>>>(s, a.dt, a.damping);
  };
  if (dim == 2)
    s.structured ? run(std::integral_constant<int, 2>{}, std::true_type{})
                 : run(std::integral_constant<int, 2>{}, std::false_type{});
  else
    s.structured ? run(std::integral_constant<int, 3>{}, std::true_type{})
                 : run(std::integral_constant<int, 3>{}, std::false_type{});
}

void launch_locate_fallback(int dim, const DevState& s, int remove_lost, cudaStream_t st) {
  if (dim == 2)
    k_locate_fallback<2><<<148, 128, 0, st>>>(s, remove_lost);
  else
    k_locate_fallback<3><<<148, 128, 0, st>>>(s, remove_lost);
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
