// mpm_device.cuh -- device helpers shared by the FP64 and the mixed-precision
// kernels: addressing of particle fields and cells, per-lane shape functions,
// the Jacobian inverse and the locate search.  Each kernel translation unit
// compiles them with its own floating-point contraction setting.
#pragma once

#include <type_traits>

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "mpm_math.cuh"
#include "mpm_state.cuh"

namespace mpm_b200 {
namespace {

template <int DIM>
struct PV {  // value offsets within a cell-slot partial
  static constexpr int MASS = 0, MOM = 1, FEXT = 1 + DIM, FINT = 1 + 2 * DIM, N = 1 + 3 * DIM;
};

__device__ __forceinline__ void raise_err(const DevState& s, unsigned bits) { atomicOr(s.err, bits); }

// A slot in the deferred MohrCoulomb return list (one atomic per group of
// lanes that defer together).  Each particle defers at most once per step, so
// slots stay below the particle count.
__device__ __forceinline__ unsigned defer_slot(const DevState& s) {
  namespace cg = cooperative_groups;
  cg::coalesced_group g = cg::coalesced_threads();
  unsigned base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(s.nplastic, g.size());
  base = g.shfl(base, 0);
  return base + g.thread_rank();
}

// A slot in the deferred list of the value steps for particle p: from the
// front when its last return took at most one correction, from the back
// otherwise (see DevState::nplastic_heavy).  One atomic per class per group of
// lanes that defer together.
__device__ __forceinline__ unsigned defer_slot_by_cost(const DevState& s, int64_t p) {
  const bool heavy = s.rpass[p] > 1;
  const unsigned act = __activemask();
  const unsigned hv = __ballot_sync(act, heavy), lt = act & ~hv;
  const int lane = threadIdx.x & 31;
  const int lead_h = __ffs(hv) - 1, lead_l = __ffs(lt) - 1;
  unsigned base = 0;
  if (lane == lead_l) base = atomicAdd(s.nplastic, (unsigned)__popc(lt));
  if (lane == lead_h) base = atomicAdd(s.nplastic_heavy, (unsigned)__popc(hv));
  base = __shfl_sync(act, base, heavy ? lead_h : lead_l);
  const unsigned below = (1u << lane) - 1u;
  const unsigned k = base + (unsigned)__popc((heavy ? hv : lt) & below);
  return heavy ? (unsigned)(s.np - 1) - k : k;
}

// Slot of the t-th entry of the list filled by defer_slot_by_cost
// (n_light = *nplastic entries from the front, then the heavy ones).
__device__ __forceinline__ unsigned list_slot(const DevState& s, unsigned t, unsigned n_light) {
  return t < n_light ? t : (unsigned)(s.np - 1) - (t - n_light);
}

// Values V0 .. V0 + NVS - 1 of one cell-slot partial row of NVAL values:
// FP32 quadruples as one 16-byte access when the row length, the first value
// and the count are multiples of four; pairs as one 8- or 16-byte access when
// they are even (rows then start on a multiple of two values).
template <typename T, int NVAL, int V0, int NVS>
__device__ __forceinline__ void load_partial_row(const T* row, T* out) {
  if constexpr (sizeof(T) == 4 && NVAL % 4 == 0 && V0 % 4 == 0 && NVS % 4 == 0) {
    const float4* r4 = reinterpret_cast<const float4*>(row + V0);
#pragma unroll
    for (int k = 0; k < NVS / 4; ++k) {
      const float4 v = r4[k];
      out[4 * k] = v.x;
      out[4 * k + 1] = v.y;
      out[4 * k + 2] = v.z;
      out[4 * k + 3] = v.w;
    }
  } else if constexpr (NVAL % 2 == 0 && V0 % 2 == 0 && NVS % 2 == 0) {
    using T2 = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
    const T2* r2 = reinterpret_cast<const T2*>(row + V0);
#pragma unroll
    for (int k = 0; k < NVS / 2; ++k) {
      const T2 v = r2[k];
      out[2 * k] = v.x;
      out[2 * k + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int v = 0; v < NVS; ++v) out[v] = row[V0 + v];
  }
}

// Values V0 .. V0 + NVS - 1 of an FP32 partial row of NVAL values stored with
// the widest accesses load_partial_row would read them with.
template <int NVAL, int V0, int NVS>
__device__ __forceinline__ void store_partial_row(float* row, const float* in) {
  if constexpr (NVAL % 4 == 0 && V0 % 4 == 0 && NVS % 4 == 0) {
    float4* r4 = reinterpret_cast<float4*>(row + V0);
#pragma unroll
    for (int k = 0; k < NVS / 4; ++k) r4[k] = make_float4(in[4 * k], in[4 * k + 1], in[4 * k + 2], in[4 * k + 3]);
  } else if constexpr (NVAL % 2 == 0 && V0 % 2 == 0 && NVS % 2 == 0) {
    float2* r2 = reinterpret_cast<float2*>(row + V0);
#pragma unroll
    for (int k = 0; k < NVS / 2; ++k) r2[k] = make_float2(in[2 * k], in[2 * k + 1]);
  } else {
#pragma unroll
    for (int v = 0; v < NVS; ++v) row[V0 + v] = in[v];
  }
}

template <int DIM>
__device__ __forceinline__ void load_x(const DevState& s, int64_t p, double* x) {
#pragma unroll
  for (int d = 0; d < DIM; ++d) x[d] = s.pf[(int64_t)(PF<DIM>::X + d) * s.np + p];
}

// cell (i, j, k) of a tensor-product grid
template <int DIM>
__device__ __forceinline__ void cell_ijk(const DevState& s, int c, int* ijk) {
  ijk[0] = c % s.gcells[0];
  if constexpr (DIM == 2) {
    ijk[1] = c / s.gcells[0];
  } else {
    ijk[1] = (c / s.gcells[0]) % s.gcells[1];
    ijk[2] = c / (s.gcells[0] * s.gcells[1]);
  }
}

// local node n of a cell -> offset (di, dj, dk) (quadrilateral_element.tcc:1-7,
// hexahedron_element.tcc:1-13)
__device__ __forceinline__ int off_i(int n) { return ((n & 3) == 1 || (n & 3) == 2) ? 1 : 0; }
__device__ __forceinline__ int off_j(int n) { return ((n & 3) >= 2) ? 1 : 0; }
__device__ __forceinline__ int off_k(int n) { return n >= 4 ? 1 : 0; }

// node ids of a cell of a tensor-product grid
template <int DIM>
__device__ __forceinline__ void grid_cell_nodes(const DevState& s, int c, int* nid) {
  constexpr int NV = Elem<DIM>::NV;
  int ijk[3] = {0, 0, 0};
  cell_ijk<DIM>(s, c, ijk);
  const int nx = s.gcells[0] + 1, ny = s.gcells[1] + 1;
#pragma unroll
  for (int n = 0; n < NV; ++n) {
    const int i = ijk[0] + off_i(n), j = ijk[1] + off_j(n);
    if constexpr (DIM == 2)
      nid[n] = i + nx * j;
    else
      nid[n] = i + nx * (j + ny * (ijk[2] + off_k(n)));
  }
}

// The cells around node `node` of a tensor-product grid, in ascending cell
// id: their ids, the node's slot (local node) in each, and each cell's
// particle count (0 for positions outside the grid).  All counts are loaded
// before any is used.
template <int DIM>
__device__ __forceinline__ void grid_node_cells(const DevState& s, int node, int* cid, int* slot,
                                                int* count) {
  constexpr int NC = DIM == 2 ? 4 : 8;
  const int gx = s.gcells[0], gy = s.gcells[1], gz = s.gcells[2];
  const int nx = gx + 1, ny = gy + 1;
  const int i = node % nx;
  const int j = DIM == 2 ? node / nx : (node / nx) % ny;
  const int k = DIM == 2 ? 0 : node / (nx * ny);
#pragma unroll
  for (int q = 0; q < NC; ++q) {
    const int a = q & 1, b = (q >> 1) & 1, e = q >> 2;  // cell (i - 1 + a, j - 1 + b, k - 1 + e)
    const int ci = i - 1 + a, cj = j - 1 + b, ck = k - 1 + e;
    bool in = ci >= 0 && ci < gx && cj >= 0 && cj < gy;
    if constexpr (DIM == 3) in = in && ck >= 0 && ck < gz;
    const int c = DIM == 2 ? ci + gx * cj : ci + gx * (cj + gy * ck);
    cid[q] = in ? c : 0;
    // the node sits at offset (1 - a, 1 - b, 1 - e) in the cell
    slot[q] = (b ? (a ? 0 : 1) : (a ? 3 : 2)) + (DIM == 3 && !e ? 4 : 0);
    count[q] = in ? s.cnt[c] : 0;
  }
}

// node ids and nodal coordinates of a cell
template <int DIM>
__device__ __forceinline__ void cell_nodes_coords(const DevState& s, int c, int* nid, double* X) {
  constexpr int NV = Elem<DIM>::NV;
  if (s.structured) {
    int ijk[3] = {0, 0, 0};
    cell_ijk<DIM>(s, c, ijk);
    const int nx = s.gcells[0] + 1, ny = s.gcells[1] + 1;
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      const int i = ijk[0] + off_i(n), j = ijk[1] + off_j(n);
      if constexpr (DIM == 2) {
        nid[n] = i + nx * j;
        X[n * 2 + 0] = __ldg(&s.axis[0][i]);
        X[n * 2 + 1] = __ldg(&s.axis[1][j]);
      } else {
        const int k = ijk[2] + off_k(n);
        nid[n] = i + nx * (j + ny * k);
        X[n * 3 + 0] = __ldg(&s.axis[0][i]);
        X[n * 3 + 1] = __ldg(&s.axis[1][j]);
        X[n * 3 + 2] = __ldg(&s.axis[2][k]);
      }
    }
  } else {
#pragma unroll
    for (int n = 0; n < NV; ++n) nid[n] = __ldg(&s.cell_nodes[(int64_t)c * NV + n]);
#pragma unroll
    for (int n = 0; n < NV; ++n)
#pragma unroll
      for (int d = 0; d < DIM; ++d) X[n * DIM + d] = __ldg(&s.ncoord[(int64_t)d * s.nn + nid[n]]);
  }
}

// J^-1 at xi (quadrilateral_element.tcc:295-309, hexahedron_element.tcc:307-321)
template <int DIM, typename R>
__device__ __forceinline__ void jacobian_inverse(const R* xi, const R* X, R* inv) {
  constexpr int NV = Elem<DIM>::NV;
  R G[NV * DIM];
  grad_shapefn<DIM>(xi, G);
  R J[DIM * DIM];
#pragma unroll
  for (int r = 0; r < DIM; ++r)
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      R a = G[0 * DIM + r] * X[0 * DIM + c];
#pragma unroll
      for (int n = 1; n < NV; ++n) a = a + G[n * DIM + r] * X[n * DIM + c];
      J[r * DIM + c] = a;
    }
  inverse<DIM>(J, inv);
}

// Map of local (xi) gradients to physical (x) gradients in one cell:
// dN/dx_c = sum_k dN/dxi_k J^-1[c][k] (quadrilateral_element.tcc:295-309,
// hexahedron_element.tcc:307-321, with J^-1 from the nodal coordinates).
//
// BOX: the cell is an axis-aligned box of a tensor-product grid, whose
// Jacobian is diag(len / 2) at every xi; dN/dx_c = dN/dxi_c * (2 / len_c)
// from the per-axis table, with no nodal coordinates and no per-point J.
// The products with the zero entries of J^-1 that the general map adds can
// change only the sign of a zero.
template <int DIM, bool BOX, typename R>
struct CellMap;

template <int DIM, typename R>
struct CellMap<DIM, true, R> {
  R ihl[DIM];
  __device__ __forceinline__ void grad(const R* g, R* d) const {
#pragma unroll
    for (int c = 0; c < DIM; ++c) d[c] = g[c] * ihl[c];
  }
};

template <int DIM, typename R>
struct CellMap<DIM, false, R> {
  R inv[DIM * DIM];
  __device__ __forceinline__ void grad(const R* g, R* d) const {
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      R a = g[0] * inv[c * DIM + 0];
#pragma unroll
      for (int k = 1; k < DIM; ++k) a = a + g[k] * inv[c * DIM + k];
      d[c] = a;
    }
  }
};

// the map of cell c at xi (X: the nodal coordinates, not read for a box)
template <int DIM, bool BOX, typename R>
__device__ __forceinline__ CellMap<DIM, BOX, R> cell_map(const DevState& s, int c, const R* xi,
                                                         const R* X) {
  CellMap<DIM, BOX, R> m;
  if constexpr (BOX) {
    int ijk[3] = {0, 0, 0};
    cell_ijk<DIM>(s, c, ijk);
#pragma unroll
    for (int d = 0; d < DIM; ++d) m.ihl[d] = R(__ldg(&s.axis_ihl[d][ijk[d]]));
  } else {
    jacobian_inverse<DIM>(xi, X, m.inv);
  }
  return m;
}

// node ids of cell c and, off a tensor-product grid, its nodal coordinates
template <int DIM, bool BOX>
__device__ __forceinline__ void cell_nodes_for(const DevState& s, int c, int* nid, double* X) {
  if constexpr (BOX)
    grid_cell_nodes<DIM>(s, c, nid);
  else
    cell_nodes_coords<DIM>(s, c, nid, X);
}

// dN_n/dx for one local node n
template <int DIM, class Map>
__device__ __forceinline__ void dn_dx_node(const double* xi, const Map& map, int n, double* Dn) {
  constexpr int NV = Elem<DIM>::NV;
  double G[NV * DIM];
  grad_shapefn<DIM>(xi, G);  // folded to the needed entries by the compiler
  map.grad(&G[n * DIM], Dn);
}

// The matrix M of the mapping velocity v + M r_i of particle p in cell c
// (position x, local coordinates xi): B D^-1 (AFF 1) with the shape tensor
// D = sum_i N_i r_i r_i^T, or B (AFF 2).
template <int DIM, int AFF>
__device__ __forceinline__ void mapping_velocity_matrix(const DevState& s, int64_t p, int c,
                                                        const double* x, const double* xi,
                                                        double* M) {
  constexpr int NV = Elem<DIM>::NV;
  double B[DIM * DIM];
#pragma unroll
  for (int q = 0; q < DIM * DIM; ++q) B[q] = s.mapb[(int64_t)q * s.np + p];
  if constexpr (AFF == 2) {
#pragma unroll
    for (int q = 0; q < DIM * DIM; ++q) M[q] = B[q];
  } else {
    int nid[NV];
    double X[NV * DIM], N[NV], T[DIM * DIM], Ti[DIM * DIM];
    cell_nodes_coords<DIM>(s, c, nid, X);
    shapefn<DIM>(xi, N);
#pragma unroll
    for (int q = 0; q < DIM * DIM; ++q) T[q] = 0.;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double r[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) r[d] = X[i * DIM + d] - x[d];
#pragma unroll
      for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int b = 0; b < DIM; ++b) T[a * DIM + b] += (N[i] * r[a]) * r[b];
    }
    inverse<DIM>(T, Ti);
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
      for (int b = 0; b < DIM; ++b) {
        double sum = B[a * DIM + 0] * Ti[0 * DIM + b];
#pragma unroll
        for (int k = 1; k < DIM; ++k) sum = sum + B[a * DIM + k] * Ti[k * DIM + b];
        M[a * DIM + b] = sum;
      }
  }
}

// ------------------------------------------------------------ P2G cell tiles
// Threads per tile: 256 on a tensor-product grid; 128 on a general mesh,
// whose staged rows add J^-1 and whose threads need more registers, and with
// an affine or Taylor mapping velocity (AFF), whose rows add the matrix.
template <bool BOX, int AFF = 0>
constexpr int p2g_tile_t() { return BOX && !AFF ? 256 : 128; }

// Particle ids of one cell in ascending order (the fill order is not
// deterministic), by the cell's NV threads of a block (k = 0 .. NV - 1):
// thread k ranks entries k, k + NV, ... (sort_per_thread<NV>() of them, 16
// per cell) against the whole segment; after a block barrier the caller
// writes them to their ranks (ids are distinct).  A longer segment is left to
// thread 0.
template <int NV>
constexpr int sort_per_thread() { return 16 / NV; }
template <int NV>
__device__ __forceinline__ bool rank_cell_segment(const int32_t* seg, int n, int k, int32_t* id,
                                                  int* rank) {
  if (n > 16) return false;
#pragma unroll
  for (int r = 0; r < sort_per_thread<NV>(); ++r) {
    const int i = k + NV * r;
    if (i < n) {
      const int32_t e = seg[i];
      int below = 0;
      for (int j = 0; j < n; ++j) below += seg[j] < e ? 1 : 0;
      id[r] = e;
      rank[r] = below;
    }
  }
  return true;
}

__device__ __forceinline__ void insertion_sort(int32_t* seg, int n) {
  for (int a = 1; a < n; ++a) {
    const int32_t key = seg[a];
    int b = a - 1;
    while (b >= 0 && seg[b] > key) {
      seg[b + 1] = seg[b];
      --b;
    }
    seg[b + 1] = key;
  }
}

// The ranking and the writes, with the block barriers between and after
// them: every thread of the block calls this (n = 0 for threads without a
// cell).
template <int NV>
__device__ __forceinline__ void sort_cell_ids(int32_t* seg, int n, int k) {
  constexpr int SPT = sort_per_thread<NV>();
  int32_t id[SPT];
  int rank[SPT];
  const bool ranked = rank_cell_segment<NV>(seg, n, k, id, rank);
  __syncthreads();
  if (ranked) {
#pragma unroll
    for (int r = 0; r < SPT; ++r)
      if (k + NV * r < n) seg[rank[r]] = id[r];
  } else if (k == 0) {
    insertion_sort(seg, n);
  }
  __syncthreads();
}

// Shape function and natural gradient of one local node n, with shapefn /
// grad_shapefn's operations and grouping (the constant first, then the x, y
// and z factors in that order, skipping the differentiated one).
template <int DIM, typename R>
__device__ __forceinline__ void node_shape(const R* xi, int n, R& N, R* G) {
  const bool px = off_i(n), py = off_j(n);
  const R a = px ? 1 + xi[0] : 1 - xi[0];
  const R b = py ? 1 + xi[1] : 1 - xi[1];
  if constexpr (DIM == 2) {
    const R e = R(0.25);
    N = e * a * b;
    G[0] = (px ? e : -e) * b;
    G[1] = (py ? e : -e) * a;
  } else {
    const bool pz = off_k(n);
    const R z = pz ? 1 + xi[2] : 1 - xi[2];
    const R e = R(0.125);
    N = e * a * b * z;
    G[0] = (px ? e : -e) * b * z;
    G[1] = (py ? e : -e) * a * z;
    G[2] = (pz ? e : -e) * a * b;
  }
}


// ------------------------------------------------------------------ locate
// cell.tcc:335-384 for cell c: the Cartesian local coordinates, or on a
// general mesh with s.iso the isoparametric ones
template <int DIM>
__device__ __forceinline__ bool cell_point_in(const DevState& s, int c, const double* x,
                                              double* xi) {
  const CellGeom& g = s.geom[c];
  if (s.iso) {
    constexpr int NV = Elem<DIM>::NV;
    int nid[NV];
    double X[NV * DIM];
    cell_nodes_coords<DIM>(s, c, nid, X);
    return point_in_cell_iso<DIM>(x, X, g.centroid, g.mean_length, xi);
  }
  return point_in_cell<DIM>(x, g.centroid, g.len, g.mean_length, xi);
}

// Local coordinates of a particle at x in the cell it was last located in,
// bit-identical to the value the locate step found (same function, same
// inputs): the Cartesian formula on box cells and without s.iso, else the
// isoparametric map, clamped to +-(1 - eps) as the locate step does.
template <int DIM, bool BOX>
__device__ __forceinline__ void particle_xi(const DevState& s, int c, const double* x,
                                            double* xi) {
  const CellGeom& g = s.geom[c];
  if constexpr (!BOX) {
    if (s.iso) {
      constexpr int NV = Elem<DIM>::NV;
      int nid[NV];
      double X[NV * DIM];
      cell_nodes_coords<DIM>(s, c, nid, X);
      iso_local_xi<DIM>(x, X, xi);
#pragma unroll
      for (int i = 0; i < DIM; ++i) {
        if (xi[i] < -1. + kDblEps) xi[i] = -1. + kDblEps;
        if (xi[i] > 1. - kDblEps) xi[i] = 1. - kDblEps;
      }
      return;
    }
  }
  local_xi<DIM>(x, g.centroid, g.len, xi);
}

// mesh.tcc:1116-1151: the current cell, then neighbours in ascending id
template <int DIM>
__device__ __forceinline__ int locate_near(const DevState& s, const double* x, int c) {
  double xi[DIM];
  if (cell_point_in<DIM>(s, c, x, xi)) return c;
  if (s.structured) {
    // neighbours of a tensor-product cell: the 3^dim - 1 cells around it,
    // ascending id (the node-sharing cells of mesh.tcc:287-306)
    int ijk[3] = {0, 0, 0};
    cell_ijk<DIM>(s, c, ijk);
    const int kmin = DIM == 3 ? ijk[2] - 1 : 0, kmax = DIM == 3 ? ijk[2] + 1 : 0;
    for (int k = kmin; k <= kmax; ++k) {
      if (DIM == 3 && (k < 0 || k >= s.gcells[2])) continue;
      for (int j = ijk[1] - 1; j <= ijk[1] + 1; ++j) {
        if (j < 0 || j >= s.gcells[1]) continue;
        for (int i = ijk[0] - 1; i <= ijk[0] + 1; ++i) {
          if (i < 0 || i >= s.gcells[0]) continue;
          const int nc = DIM == 2 ? i + s.gcells[0] * j : i + s.gcells[0] * (j + s.gcells[1] * k);
          if (nc == c) continue;
          if (cell_point_in<DIM>(s, nc, x, xi)) return nc;
        }
      }
    }
    return -1;
  }
  const int b = s.nb_off[c], e = s.nb_off[c + 1];
  for (int k = b; k < e; ++k) {
    const int nc = s.nb[k];
    if (cell_point_in<DIM>(s, nc, x, xi)) return nc;
  }
  return -1;
}


// ------------------------------------------------------------ counting sort
// The passes of the per-step counting sort of particles by cell, as bodies
// that a one-kernel-per-pass launch and the persistent step kernel share.
// Per-cell counts and each particle's slot within its cell.  Particles are
// stored mostly in cell order, so the lanes of a warp form runs of equal
// cells: each run's first lane adds the run's length with one atomic and the
// others take the following slots.  The slot order within a cell is not
// deterministic either way, and P2G sorts every cell's segment.  Every lane
// of the warp takes part (p at or beyond np is an empty lane).  Against one
// atomic per distinct cell of the warp (__match_any_sync): the 512-slope
// ensemble's sort 0.180 -> 0.165 ms, the 4M column's unchanged.
__device__ __forceinline__ void count_particle(const DevState& s, int64_t p) {
  const bool in = p < s.np;
  const int lane = threadIdx.x & 31;
  int c = in ? s.cell[p] : -1;
  if (c >= s.ncells) raise_err(s, ERR_BADCELL);
  const bool valid = c >= 0 && c < s.ncells;
  if (!valid) c = -1 - lane;  // a run of its own
  const int prev = __shfl_up_sync(0xffffffffu, c, 1);
  const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || c != prev);
  const unsigned upto = lane == 31 ? 0xffffffffu : (2u << lane) - 1u;  // lanes 0..lane
  const int head = 31 - __clz(heads & upto);
  const unsigned above = heads & ~upto;
  const int next = above ? __ffs(above) - 1 : 32;
  int base = 0;
  if (lane == head && valid) base = atomicAdd(&s.cnt[c], next - head);
  base = __shfl_sync(0xffffffffu, base, head);
  if (in) s.rank[p] = valid ? base + (lane - head) : -1;
}

// The particle's place in the cell-sorted order (start of its cell + rank).
__device__ __forceinline__ void fill_particle(const DevState& s, int64_t p) {
  if (p >= s.np) return;
  const int c = s.cell[p];
  if (c < 0 || c >= s.ncells) return;
  s.order[s.start[c] + s.rank[p]] = (int32_t)p;
}

// The exhaustive locate of the particles that left their cell's neighbourhood
// in G2P (mesh.tcc:1116-1151 over all cells); listed entries begin, begin +
// stride, ...
template <int DIM>
__device__ __forceinline__ void locate_lost(const DevState& s, int remove_lost, unsigned begin,
                                            unsigned stride) {
  const unsigned count = *s.nlost;
  for (unsigned k = begin; k < count; k += stride) {
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
        if (!(f >= 0.) || f >= (double)s.bn[d])
          inside = false;
        else
          b[d] = (int)f;
      }
      if (inside) {
        const int64_t bi = ((int64_t)b[2] * s.bn[1] + b[1]) * s.bn[0] + b[0];
        for (int j = s.bin_off[bi]; j < s.bin_off[bi + 1]; ++j) {
          const int cid = s.bin_cells[j];
          double xi[DIM];
          if (cell_point_in<DIM>(s, cid, x, xi)) {
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

}  // namespace
}  // namespace mpm_b200
