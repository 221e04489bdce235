// mpm_kernels.h -- launch entry points shared by the kernel translation units
// and the C-ABI host code.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "mpm_state.cuh"

namespace mpm_b200 {

struct StepArgs {
  int scheme;        // 0 USF, 1 USL
  int flip;          // 1 FLIP, 0 PIC
  int vupd;          // MPM_VELOCITY_*: 0 FLIP, 1 PIC, 2 ASFLIP, 3 TPIC, 4 APIC
  int remove_lost;   // locate_particles false: unlocatable particles removed
  double dt;
  double beta;       // FLIP/PIC blending ratio
  double damping;    // Cundall damping factor
  double g[3];       // gravity of this step (ramp applied)
  int phase;         // USL: 0 the whole step, 1 sort and P2G only, 2 the rest (node
                     // update onward) -- a slab run exchanges halo partials between them
  // Launch shape of the value steps (the results do not depend on it):
  // threads of a P2G cell tile on box cells (128 or 256), threads of a
  // node-kernel block (128 or 256), blocks per SM of the plastic-return kernel
  // (4, 8 or 16).  Zero selects the built-in default.
  int p2g_tile;
  int node_threads;
  int return_blocks_per_sm;
};

// The launch shape a step uses: the built-in defaults where a field is zero.
inline int tile_threads(const StepArgs& a, bool box) { return box && a.p2g_tile ? a.p2g_tile : (box ? 256 : 128); }
inline int node_block(const StepArgs& a) { return a.node_threads ? a.node_threads : 256; }
inline int return_blocks(const StepArgs& a) { return a.return_blocks_per_sm ? a.return_blocks_per_sm : 8; }

// Kernels of one step, for launch counting and per-kernel event timing.
enum KernelId {
  K_SORT = 0,       // counting sort of particles by cell (count, scan, fill)
  K_P2G,            // per-cell P2G of mass and momentum (and, in USL, forces)
  K_NODES_VEL,      // nodal velocity (USF) or full nodal update (USL)
  K_STRESS,         // USF: stress update
  K_P2G_FORCES,     // USF: per-cell P2G of the forces
  K_NODES_ACC,      // USF: nodal acceleration / velocity update
  K_G2P,            // G2P (+ USL stress update) + locate
  K_MC_RETURN,      // MohrCoulomb plastic returns deferred by the stress update
  K_LOCATE,         // exhaustive locate for particles that left their neighbourhood
  // the adjoint's reverse sweep
  K_ADJ_RECOMPUTE,  // sort, P2G and node update recomputed from the stored state
  K_ADJ_MATERIAL,   // elastic material reverse, plastic points listed
  K_ADJ_RETURN,     // plastic return-map reverse
  K_ADJ_KINEMATICS, // G2P reverse
  K_ADJ_SCATTER,    // node cotangents as cell-slot sums
  K_ADJ_NODES,      // node update reverse
  K_ADJ_P2G,        // P2G reverse (gather)
  K_NKERNELS
};
constexpr int SCAN_BLOCK = 4096;  // cells per block of the counting-sort scan
// particle arrays are padded to a multiple of this (the particle-kernel block
// size), so every block's slice of a field is a whole aligned segment
constexpr int PAD_PARTICLES = 128;
const char* kernel_name(int kid);

// Counts kernel launches; when enabled, brackets every phase (one kernel, or
// the SORT_KERNELS kernels of the counting sort) with a pair of CUDA events on
// the launching stream and accumulates their elapsed times.
constexpr int SORT_KERNELS = 5;  // count, two scan levels, scan add, fill
struct Profiler {
  bool enabled = false;
  int64_t launches = 0;
  double total_ms[K_NKERNELS] = {};
  int64_t count[K_NKERNELS] = {};
  void begin(int kid, cudaStream_t st, int kernels = 1);
  void end(int kid, cudaStream_t st);
  void collect();  // after the stream has been synchronised
  void reset();
  ~Profiler();
  struct Pending;
  void* impl = nullptr;
};

void launch_step_fp64(int dim, const DevState& s, const StepArgs& a, cudaStream_t st,
                      Profiler& prof);
void launch_step_mixed(int dim, const DevState& s, const StepArgs& a, cudaStream_t st,
                       Profiler& prof);
// The persistent form of the mixed USL step (FLIP or PIC, tensor-product
// grid): one cooperative launch runs `nsteps` whole steps, the passes of
// which are separated by grid barriers.  a.g is ignored: the gravity of step
// k is the ramp of *step + k applied to `gravity` (mpm_explicit.tcc:145-153),
// and the launch advances *step (device memory) by nsteps, so that a launch
// captured in a CUDA graph replays for any step.  `barrier` holds two words
// of device memory.  Returns the launch's error.
struct PersistentArgs {
  int64_t nsteps;
  long long* step;
  double gravity[3];
  double ramp;  // gravity ramping time (0: none)
  unsigned* barrier;
};
cudaError_t launch_steps_persistent_mixed(int dim, const DevState& s, const StepArgs& a,
                                          const PersistentArgs& q, cudaStream_t st);
// shared by both paths: the per-step counting sort and the exhaustive locate
void counting_sort(const DevState& s, cudaStream_t st);
void launch_locate_fallback(int dim, const DevState& s, int remove_lost, cudaStream_t st);
// PODParticle records (pod_particle.h:12-62): 74 fields, caller's layout
constexpr int POD_NFIELDS = 74;
struct PodLayout {
  int32_t offset[POD_NFIELDS];  // byte offset of each field in a record
  int64_t record_size;
};
struct PodAux {                 // per-particle data the step never changes
  const uint64_t* id;           // [np] particle id
  const double* nsize;          // [3][np] natural particle size
  const double* acc;            // [3][np] particle acceleration
  const int32_t* material_id;   // [material slot] material id
  const uint32_t* nstate;       // [material slot] number of state variables
};
// The C ABI's particle rows (mpm_gpu_particles: x, u, v n x 3; stress,
// strain n x 6; F n x 9; volume, mass, density n; svars n x 9) staged in one
// device buffer: the offset of each array in doubles, -1 when absent.  The
// device converts them to and from its own layout, so that loading and
// reading a state moves the caller's arrays with plain copies.
struct RowStage {
  int64_t n;
  double* base;
  int64_t x, u, v, stress, strain, F, volume, mass, density, svars;
};
// every array present; the device state's padding rows are zeroed
void launch_rows_to_state(int dim, bool mixed, bool any_mc, const DevState& s, const RowStage& r,
                          cudaStream_t st);
// the present arrays are written for the first r.n particles
void launch_state_to_rows(int dim, bool mixed, bool any_mc, const DevState& s, const RowStage& r,
                          cudaStream_t st);
void launch_pod_pack(int dim, bool mixed, const DevState& s, const PodAux& a, const PodLayout& L,
                     const int32_t* list, int64_t count, uint8_t* out, cudaStream_t st);
// Tangent (sensitivity) step: material parameters differentiated
enum { TP_YOUNGS_MODULUS = 0, TP_FRICTION = 1, TP_COHESION = 2, TP_DILATION = 3 };
struct TangentParam {
  int32_t material_slot;
  int32_t kind;
};
constexpr int MAX_TANGENTS = 2;
void launch_step_tangent(int dim, const DevState& s, const StepArgs& a, cudaStream_t st,
                         Profiler& prof);
size_t tangent_material_bytes();
// fills out (nmats MaterialT<Dual>) and sv_seed (nmats x SV_N x MAX_TANGENTS)
void make_tangent_materials(const MaterialParams* mats, int nmats, const TangentParam* params,
                            int nparams, void* out, double* sv_seed);
// The first half of a USL step (sort, P2G, node update) on the FP64 path.
void launch_p2g_nodes_fp64(int dim, const DevState& s, const StepArgs& a, cudaStream_t st);

// Reverse sweep of one FP64 USL step (kernels_adjoint.cu).  The particle
// cotangents adj ([x~ (DIM), v~ (DIM), sigma~ (NS), V~][np]) hold those of the
// state after the step on entry and of the state before it on return; theta
// ([nparams][np]) accumulates each particle's share of dL/dparameter.  The
// forward sort, P2G and node update of the step must have run on the
// step-start state (partials, nf, order).
struct AdjointArgs {
  double* adj = nullptr;
  double* deps = nullptr;    // [6][np] cotangent of the strain increment
  double* dsbar = nullptr;   // [NS][np] sigma~' of the listed plastic points (list order)
  double* coef = nullptr;    // [3 DIM + 6][np] coefficients of the node scatter
  double* theta = nullptr;   // [NT][np]
  double* apart = nullptr;   // [ncells][NV][2 DIM] cell-slot sums of v~, a~ of the nodes
  double* nbar = nullptr;    // [1 + 3 DIM][nn] cotangents of m, p, f_ext, f_int
  const void* mats_zero = nullptr;   // MaterialT<Dual> per slot, zero derivatives
  const void* mats_param = nullptr;  // MaterialT<Dual> per slot, derivatives = parameters
  const double* sv_seed = nullptr;   // [slot][SV_N][NT] d(initial state)/d(parameter)
  int nparams = 0;
  double mass_floor = 0.0;           // nodes lighter than this pass no cotangents
};
void launch_adjoint_step(int dim, const DevState& s, const AdjointArgs& A, const StepArgs& a,
                         cudaStream_t st, Profiler& prof);

void launch_material_batch_fp64(int dim, int64_t n, const MaterialParams& m, const double* stress,
                                const double* dstrain, const double* density, double* state,
                                double* out, cudaStream_t st);

}  // namespace mpm_b200
