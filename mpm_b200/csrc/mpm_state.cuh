// mpm_state.cuh -- device-resident state of one solver and its field layout.
//
// Particles are structure-of-arrays: every scalar field is a contiguous array
// of np doubles, so a warp reads 32 consecutive particles' value of a field
// in one 256-byte transaction.  Fields that never change in 2D (stress yz/xz,
// strain zz/yz/xz, the third row and column of F) are not stored in 2D.
#pragma once

#include <cstdint>

#include "mpm_math.cuh"

namespace mpm_b200 {

// particle field offsets (units of np doubles)
template <int DIM>
struct PF;
template <>
struct PF<3> {
  static constexpr int X = 0, U = 3, V = 6, S = 9, E = 15, F = 21, VOL = 30, RHO = 31,
                       MASS = 32, NF = 33;
  static constexpr int NS = 6, NE = 6, NFG = 9;
};
template <>
struct PF<2> {
  // stress xx,yy,zz,xy; strain xx,yy,xy; F 00,01,10,11
  static constexpr int X = 0, U = 2, V = 4, S = 6, E = 10, F = 13, VOL = 17, RHO = 18,
                       MASS = 19, NF = 20;
  static constexpr int NS = 4, NE = 3, NFG = 4;
};

// Mixed precision: FP64 buffer [x (DIM), u (DIM), pdstrain] (DevState::pf
// points at it, so x and u keep the FP64 offsets) and an FP32 buffer with
// v, stress, strain, H = F - I, the initial volume and density, P = V/V0 - 1
// (volume and density follow as V0 (1 + P) and rho0 / (1 + P)) and the mass.
// Slowly varying quantities are stored as deviations so that FP32 keeps the
// small per-step increments.
template <int DIM>
struct PDX {
  static constexpr int X = 0, U = DIM, PDS = 2 * DIM, ND = 2 * DIM + 1;
};
template <int DIM>
struct PM;
template <>
struct PM<3> {
  static constexpr int V = 0, S = 3, E = 9, H = 15, V0 = 24, RHO0 = 25, JP = 26, MASS = 27, NF = 28;
};
template <>
struct PM<2> {
  static constexpr int V = 0, S = 2, E = 6, H = 9, V0 = 13, RHO0 = 14, JP = 15, MASS = 16, NF = 17;
};
constexpr int SVF_N = 8;  // MohrCoulomb state in FP32: SV_YIELD .. SV_THETA

// node field offsets (units of nn doubles)
template <int DIM>
struct NF {
  static constexpr int MASS = 0, MOM = 1, FEXT = 1 + DIM, FINT = 1 + 2 * DIM,
                       NACC_FIELDS = 1 + 3 * DIM,  // accumulated by P2G, zeroed every step
                       VEL = 1 + 3 * DIM, ACC = 1 + 4 * DIM, NNF = 1 + 5 * DIM;
};

// Mixed-precision nodal velocity and acceleration: one record per node of
// nfv_stride floats, 16-byte aligned, so that a particle kernel gathers a node
// with one (2D: v0 v1 a0 a1) or two (3D: v0 v1 v2 a0 | a1 a2 - -) 16-byte loads.
constexpr int nfv_stride(int dim) { return dim == 3 ? 8 : 4; }
// Values of a mixed-precision cell-slot partial row: mass, momentum (DIM) and
// internal force (DIM) -- the body force is gravity times the nodal mass,
// formed by the node update (the FP64 rows also carry it, 1 + 3 DIM) -- padded
// to 8 (3D) or 6 (2D) floats, so that a row moves in 16- or 8-byte accesses.
constexpr int mixed_nval(int dim) { return dim == 3 ? 8 : 6; }

// particle velocity constraint record: mask bit d => v[d] = value[d]
struct ParticleVC {
  uint32_t mask;
  uint32_t pad;
  double value[3];
};

enum ErrorBits : unsigned {
  ERR_OUTSIDE = 1u,     // a particle left the mesh (locate_particles on)
  ERR_NONFINITE = 2u,   // NaN or Inf in a particle position
  ERR_BADCELL = 4u,     // corrupt cell index found by a bounds check
  ERR_TIMEOUT = 8u      // a bounded wait (copy, scan chain, grid barrier) ran out
};

struct DevState {
  int64_t np = 0;          // particle rows
  double* pf = nullptr;    // [PF::NF][np]
  double* sv = nullptr;    // [SV_N][np] MohrCoulomb state (null when no MC)
  int32_t* cell = nullptr; // [np] current cell, -1 removed
  uint16_t* mat = nullptr; // [np] material slot
  int16_t* pvc = nullptr;  // [np] particle velocity constraint slot (-1 none)

  int64_t nn = 0;          // nodes
  double* nf = nullptr;    // [NF::NNF][nn]
  uint8_t* active = nullptr;     // [nn] node belongs to a cell holding particles
  int32_t* bc_index = nullptr;   // [nn] slot in bcs or -1

  int64_t ncells = 0;
  int32_t* cell_nodes = nullptr; // [ncells][NV]
  double* ncoord = nullptr;      // [DIM][nn]
  CellGeom* geom = nullptr;      // [ncells]
  int32_t* nb_off = nullptr;     // [ncells + 1] neighbour CSR (ascending ids)
  int32_t* nb = nullptr;

  // uniform bins over the cells' containment spheres, for the exhaustive
  // search (equivalent to scanning every cell in id order)
  int32_t* bin_off = nullptr;
  int32_t* bin_cells = nullptr;
  double bmin[3] = {0, 0, 0};
  double bsize[3] = {1, 1, 1};
  int32_t bn[3] = {1, 1, 1};

  // tensor-product grid (node (i,j,k) = i + nx*(j + ny*k) at (ax[i], ay[j],
  // az[k]); lexicographic cells): the exhaustive search needs only the
  // 3^dim cells around the axis interval that holds the point
  int structured = 0;
  int32_t gcells[3] = {1, 1, 1};     // cells per axis
  const double* axis[3] = {nullptr, nullptr, nullptr};  // node coordinates per axis
  const double* axis_ihl[3] = {nullptr, nullptr, nullptr};  // 2 / cell length per axis interval
  double* mapb = nullptr;  // [DIM * DIM][np] mapping matrix (ASFLIP, TPIC, APIC), row-major
  int iso = 0;             // general cells take isoparametric local coordinates

  // general meshes: cells around each node, ascending cell id, with the
  // node's local index (slot) in that cell
  int32_t* nc_off = nullptr;     // [nn + 1]
  int32_t* nc_cell = nullptr;
  int8_t* nc_slot = nullptr;
  double* dndx_c = nullptr;      // [ncells][NV][DIM] dN/dx at the cell centroid

  // per-step counting sort of particles by cell and the cell-slot partial
  // sums of P2G (mass, momentum, external force, internal force per slot)
  int32_t* cnt = nullptr;        // [ncells] particles per cell
  int32_t* start = nullptr;      // [ncells + 1] exclusive scan of cnt
  int32_t* rank = nullptr;       // [np] position of the particle within its cell
  int32_t* order = nullptr;      // [np] particle ids grouped by cell
  int32_t* bsum = nullptr;       // scan block totals
  double* partials = nullptr;    // [ncells][NV][1 + 3 DIM]

  double* xnext = nullptr;       // [DIM][np] MUSL: positions at the end of the step
  int32_t* lost = nullptr;       // [np] particles not found in cell or neighbours
  unsigned* nlost = nullptr;
  // particles whose MohrCoulomb trial stress is plastic this step, with the
  // inputs of their deferred return: strain increment (6) and density
  int32_t* plist = nullptr;      // [np]
  double* pbuf = nullptr;        // [7][np] (FP64 path)
  float* pbuf_f = nullptr;       // [7][np] (mixed path, same allocation)
  unsigned* nplastic = nullptr;
  // The value steps fill the list from both ends: points whose last return
  // took at most one correction from slot 0 up (nplastic of them), the others
  // from slot np - 1 down (nplastic_heavy), so that the lanes of a warp in the
  // return kernel carry returns of similar length.  rpass[p] is the number of
  // corrections of particle p's last return (0 for a point never returned).
  unsigned* nplastic_heavy = nullptr;
  uint8_t* rpass = nullptr;      // [np]
  unsigned* err = nullptr;       // ErrorBits

  // mixed precision (null on the FP64 path)
  float* pm = nullptr;            // [PM::NF][np]
  float* svf = nullptr;           // [SVF_N][np]
  float* nfv = nullptr;           // [nn][nfv_stride(DIM)] nodal velocity, acceleration
  float* partials_f = nullptr;    // [ncells][NV][1 + 3 DIM]
  float* dndx_cf = nullptr;       // [ncells][NV][DIM]
  const MaterialT<float>* mats_f = nullptr;

  int any_softening = 0;          // some MohrCoulomb material softens (phi..tc vary)
  // test hook: the staged G2P's first copy wait runs out on purpose (after its
  // copies have landed), exercising the ERR_TIMEOUT path without a fault
  int test_wait_timeout = 0;

  // tangents (derivatives with respect to NT material parameters), each in the
  // layout of its value array; null unless sensitivities are enabled
  double* pft[2] = {nullptr, nullptr};       // particle fields, layout of pf
  double* svt[2] = {nullptr, nullptr};       // MohrCoulomb state, layout of sv
  double* nft[2] = {nullptr, nullptr};       // nodal v, a, layout of nf
  double* partt[2] = {nullptr, nullptr};     // cell-slot partials
  const void* mats_t = nullptr;              // [materials] MaterialT<Dual>
  double* tpbuf = nullptr;                   // [7][1 + NT][np] deferred-return inputs
  double tangent_mass_floor = 0.0;           // nodes lighter than this carry no tangents
  const MaterialParams* mats = nullptr;
  const NodeBC* bcs = nullptr;
  const ParticleVC* pvcs = nullptr;
};

}  // namespace mpm_b200
