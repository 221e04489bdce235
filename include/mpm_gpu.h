/*
 * mpm_gpu.h -- C ABI of the B200 explicit MPM step (libmpm_b200.so).
 *
 * Drop-in boundary for the explicit single-phase solver of geomechanics/mpm
 * (MPMExplicit<Tdim> with the USF/USL schemes).  Plain pointers and sizes
 * only; no C++ types, no exceptions cross this boundary.  Every call returns
 * an mpm_status (0 = success); mpm_gpu_last_error() describes the last
 * failure on a handle.  Host arrays passed in are copied before the call
 * returns; read-back calls write into caller-allocated arrays.
 *
 * Reference interfaces replaced (paths in the geomechanics/mpm tree):
 *   solver    include/solvers/mpm_explicit.tcc:24-199  MPMExplicit::solve
 *             include/solvers/mpm_scheme/mpm_scheme.tcc:19-261 (USF/USL)
 *   mesh      include/mesh/mesh.tcc:17-48, 211-256, 287-306 create nodes/cells
 *   material  include/materials/material.h:97-106 Material<Tdim>::compute_stress
 *             src/material.cc:30-53 factory keys LinearElastic2D/3D,
 *             MohrCoulomb2D/3D with the JSON property names of
 *             linear_elastic.tcc:20-24 and mohr_coulomb.tcc:9-71
 *   BCs       include/loads_bcs/constraints.tcc:83-217 nodal velocity /
 *             acceleration / friction constraints; mesh.tcc:1454-1467
 *             particle velocity constraints
 *   particles include/particles/particle.tcc:145-306 particle state (POD)
 *
 * Threading: one host thread per handle.  All device work of a handle runs
 * on its own CUDA stream; mpm_gpu_step() returns once the steps are queued
 * and their error word has been read (it synchronises the stream at the end
 * of the call).
 */
#ifndef MPM_GPU_H
#define MPM_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mpm_gpu_solver* mpm_gpu_t;

typedef enum {
  MPM_OK = 0,
  MPM_ERR_INVALID = -1,      /* bad argument or call order */
  MPM_ERR_CUDA = -2,         /* a CUDA call failed */
  MPM_ERR_OUTSIDE = -3,      /* particle(s) left the mesh, locate_particles on */
  MPM_ERR_NONFINITE = -4,    /* NaN/Inf detected in particle state */
  MPM_ERR_TIMEOUT = -5,      /* a bounded device wait gave up */
  MPM_ERR_ALLOC = -6,        /* device allocation failed */
  MPM_ERR_UNSUPPORTED = -7   /* feature outside the implemented path */
} mpm_status;

enum { MPM_SCHEME_USF = 0, MPM_SCHEME_USL = 1, MPM_SCHEME_MUSL = 2 };
/* particle velocity update, in the order of the reference's VelocityUpdate
 * (data_types.h:50) */
enum {
  MPM_VELOCITY_FLIP = 0,
  MPM_VELOCITY_PIC = 1,
  MPM_VELOCITY_ASFLIP = 2,
  MPM_VELOCITY_TPIC = 3,
  MPM_VELOCITY_APIC = 4
};
enum { MPM_PRECISION_FP64 = 0, MPM_PRECISION_MIXED = 1 };

/* Analysis settings (mpm_base.tcc:3-207; mpm_explicit.tcc:8-13, 145-153). */
typedef struct {
  int32_t dim;              /* 2 (quad4 / ED2Q4) or 3 (hex8 / ED3H8) */
  int32_t scheme;           /* MPM_SCHEME_USF / MPM_SCHEME_USL / MPM_SCHEME_MUSL (FP64 and
                               mixed; mpm_scheme_musl.tcc:20-35) */
  int32_t velocity_update;  /* MPM_VELOCITY_FLIP / PIC (particle.tcc:1018-1067), or the
                               affine ASFLIP / APIC and Taylor TPIC updates, which carry a
                               mapping matrix per particle (particle.tcc:630-721,
                               1071-1139, 1663-1730; USF and USL, FP64 and mixed) */
  int32_t precision;        /* MPM_PRECISION_FP64: every quantity in FP64, rounding as the
                               reference's CPU run (the parity mode);
                               MPM_PRECISION_MIXED: FP32 transfers and constitutive update
                               with FP64 positions, displacements, nodal mass division and
                               apex returns (no counterpart in the reference) */
  double blending_ratio;    /* velocity_update_settings.blending_ratio */
  double dt;
  double damping_factor;    /* damping {type: Cundall, damping_factor} */
  double gravity[3];
  double gravity_ramping_time;
  int32_t locate_particles; /* 1: a particle outside the mesh is an error,
                               0: it is removed (mpm_scheme.tcc:245-261) */
  int32_t device;           /* CUDA device ordinal */
} mpm_gpu_config;

/* Particle state, one row per particle, row-major.  x,u,v: n*3 (the third
 * column is ignored in 2D); stress, strain: n*6 Voigt (xx,yy,zz,xy,yz,xz,
 * engineering shear strain); F: n*9 row-major deformation gradient; volume,
 * mass, density: n; cell: n (cell id, -1 = removed); material: n (material
 * id); svars: n*9 MohrCoulomb state in the reference order (yield_state, phi,
 * psi, cohesion, tension_cutoff, epsilon, rho, theta, pdstrain; zero for
 * LinearElastic).  On load a NULL pointer means "default" (zeros; identity
 * F; initial material state); on read-back a NULL pointer is skipped. */
typedef struct {
  double* x;
  double* u;
  double* v;
  double* stress;
  double* strain;
  double* F;
  double* volume;
  double* mass;
  double* density;
  int64_t* cell;
  int32_t* material;
  double* svars;
} mpm_gpu_particles;

/* Local coordinates of the cells (mesh "isoparametric", mpm_base.tcc:767-784;
 * cell.tcc:335-384, 617-826): 1 the isoparametric map (the reference's
 * default), 0 the Cartesian formula of local_coordinates_point (the default
 * here).  On a tensor-product grid both give the same coordinates to rounding
 * and the Cartesian formula is used; on a general mesh 1 takes the inverse of
 * the bilinear / trilinear map.  Before mpm_gpu_initialise / particle loads;
 * FP64 and mixed precision, not with sensitivities. */
int mpm_gpu_set_isoparametric(mpm_gpu_t h, int32_t isoparametric);

/* The mapping matrix of the ASFLIP / APIC / TPIC velocity updates (the
 * particle's mapping_matrix_), n*9 row-major: its leading dim x dim block
 * (zeros elsewhere on read).  MPM_ERR_UNSUPPORTED for FLIP and PIC.  A new
 * particle starts from zero (particle.tcc:666-669). */
int mpm_gpu_read_mapping_matrix(mpm_gpu_t h, double* out);
int mpm_gpu_load_mapping_matrix(mpm_gpu_t h, const double* in);

/* Create a solver on cfg->device. */
int mpm_gpu_create(const mpm_gpu_config* cfg, mpm_gpu_t* out);
int mpm_gpu_destroy(mpm_gpu_t h);
const char* mpm_gpu_last_error(mpm_gpu_t h);

/* Mesh: node coordinates (nnodes*dim) and cell connectivity
 * (ncells*nodes_per_cell, node order of quadrilateral_element.tcc:1-7 /
 * hexahedron_element.tcc:1-13).  Replaces Mesh::create_nodes/create_cells
 * and find_cell_neighbours. */
int mpm_gpu_set_mesh(mpm_gpu_t h, int64_t nnodes, const double* coords, int64_t ncells,
                     int32_t nodes_per_cell, const int64_t* cell_nodes);

/* Material<Tdim> factory: type "LinearElastic2D/3D" or "MohrCoulomb2D/3D",
 * properties as the reference's JSON material object. */
int mpm_gpu_add_material(mpm_gpu_t h, int32_t id, const char* type, const char* json_props);

/* Nodal constraints (constraints.tcc:83-106, 192-217; node.tcc:349-505). */
int mpm_gpu_add_velocity_constraints(mpm_gpu_t h, int64_t n, const int64_t* node_ids,
                                     const int32_t* dirs, const double* values);
int mpm_gpu_add_acceleration_constraints(mpm_gpu_t h, int64_t n, const int64_t* node_ids,
                                         const int32_t* dirs, const double* values);
int mpm_gpu_add_friction_constraints(mpm_gpu_t h, int64_t n, const int64_t* node_ids,
                                     const int32_t* dirs, const int32_t* signs,
                                     const double* mu);

/* General (rotated) boundaries (mesh boundary_conditions "nodal_euler_angles",
 * mpm_base.tcc:1041-1063, mesh.tcc:1318-1345): node ids and dim Euler angles
 * per node (n*dim, radians).  The velocity, acceleration and friction
 * constraints of those nodes act on the components of the node's rotated
 * frame (node.tcc:370-483, 510-657). */
int mpm_gpu_set_nodal_euler_angles(mpm_gpu_t h, int64_t n, const int64_t* node_ids,
                                   const double* angles);

/* Create particles at coordinates (n*dim) with one material
 * (mesh.tcc:2114-2148 read_particles_file / create_particles). */
int mpm_gpu_add_particles(mpm_gpu_t h, int64_t n, const double* coords, int32_t material_id);

/* Material sets (mpm_base.tcc:448-472 "material_sets" -> Particle::assign_material
 * on every particle of a set, mesh.tcc:1175-1189): the particles with the given
 * ids (creation order, from 0) take material material_id; ids without a
 * particle are skipped, as the reference skips them.  Before
 * mpm_gpu_initialise, which derives mass and the material state from it. */
int mpm_gpu_assign_particle_materials(mpm_gpu_t h, int64_t n, const int64_t* pids,
                                      int32_t material_id);

/* Locate particles, volume = cell volume / particles in cell, mass =
 * volume * density, material state initialised (mpm_base.tcc:347-473,
 * particle.tcc:589-626, mpm_explicit.tcc:94-95).  Uploads the state. */
int mpm_gpu_initialise(mpm_gpu_t h);

/* Initial particle stresses, n*6 Voigt, in particle creation order
 * (mpm_base.tcc:1591-1625 particles_stresses, mesh.tcc:1502-1524).  After
 * mpm_gpu_initialise. */
int mpm_gpu_assign_particle_stresses(mpm_gpu_t h, int64_t n, const double* stress);

/* Particle velocity constraint on particle ids (n < 0: all particles)
 * (mesh.tcc:1454-1467, particle.tcc:1190-1194). */
int mpm_gpu_add_particle_velocity_constraint(mpm_gpu_t h, int64_t n, const int64_t* pids,
                                             int32_t dir, double velocity);

/* Replace the full particle state (e.g. restart from a checkpoint).  Arrays in
 * page-locked host memory (mpm_gpu_host_alloc, cudaHostAlloc or
 * cudaHostRegister; each array inside one such allocation) are copied by the
 * DMA engine directly; pageable arrays go through the library's own pinned
 * staging buffer, gathered on all host threads. */
int mpm_gpu_load_particles(mpm_gpu_t h, int64_t n, const mpm_gpu_particles* p);

/* Page-locked host memory for particle arrays that are loaded and read often
 * (no counterpart in the reference): *ptr receives `bytes` bytes, NULL with
 * MPM_ERR_ALLOC when the host cannot pin them; free with mpm_gpu_host_free. */
int mpm_gpu_host_alloc(size_t bytes, void** ptr);
int mpm_gpu_host_free(void* ptr);

/* Advance nsteps explicit steps (mpm_explicit.tcc:112-190). */
int mpm_gpu_step(mpm_gpu_t h, int64_t nsteps);

/* As mpm_gpu_step, and report the device time of the steps, measured with
 * CUDA events on the solver's stream (the reference logs the same span as
 * "solver duration", mpm_explicit.tcc:191-196). */
int mpm_gpu_step_timed(mpm_gpu_t h, int64_t nsteps, double* elapsed_ms);

/* Launch shape of the steps (no counterpart in the reference, whose steps
 * are host loops): threads of a P2G cell tile on a tensor-product grid (128
 * or 256), threads of a node-kernel block (128 or 256), blocks per SM of the
 * plastic-return kernel (4, 8 or 16); 0 keeps the built-in default (256, 256,
 * 8).  Results do not depend on it.  mpm_gpu_get_launch_shape writes the
 * three values in use.  mpm_gpu_autotune times each candidate over `steps`
 * steps (at least 3, after 2 untimed ones) of the solver's own state, one
 * field at a time, keeps
 * the fastest, and restores the particle state and step counter, so the run
 * then continues exactly as without it; report (report_len bytes, may be
 * NULL) receives the per-candidate milliseconds per step as JSON.  It holds a
 * copy of the particle state on the device meanwhile (MPM_ERR_ALLOC if that
 * does not fit).  Not with sensitivities on. */
int mpm_gpu_set_launch_shape(mpm_gpu_t h, int32_t p2g_tile, int32_t node_threads,
                             int32_t return_blocks_per_sm);
int mpm_gpu_get_launch_shape(mpm_gpu_t h, int32_t* shape);
int mpm_gpu_autotune(mpm_gpu_t h, int64_t steps, char* report, size_t report_len);

/* Persistent steps (the batched form's one-launch step; no counterpart in the
 * reference): with steps_per_launch > 0, mpm_gpu_step advances up to that
 * many whole steps per cooperative kernel launch (after the first launch of a
 * call, launches of that many steps replay a captured CUDA graph), every block resident, the
 * passes of a step (sort, P2G, node update, G2P and stress, plastic returns,
 * exhaustive locate) separated by grid barriers with bounded waits
 * (MPM_ERR_TIMEOUT when one runs out); 0 returns to one launch per pass,
 * replayed from a CUDA graph (the default).  Results are bit for bit those
 * of the per-pass launches.  Mixed precision, USL, FLIP or PIC, on a
 * tensor-product grid, without sensitivities (MPM_ERR_UNSUPPORTED
 * otherwise: here for the configuration, at mpm_gpu_step for the mesh and
 * sensitivities); per-kernel profiling steps run per pass. */
int mpm_gpu_set_persistent(mpm_gpu_t h, int32_t steps_per_launch);
/* The steps per persistent launch in use (0: off) and whether its launches of
 * that many steps replay a captured CUDA graph (1) or are launched directly (0:
 * none captured yet, or the capture was not possible). */
int mpm_gpu_get_persistent(mpm_gpu_t h, int32_t* steps_per_launch, int32_t* graph_replayed);

/* Per-kernel device timing (CUDA events around every launch on the solver's
 * stream).  Enabling or disabling resets the counters.  Kernel indices run
 * from 0 while the call succeeds; name receives a static string. */
int mpm_gpu_set_profiling(mpm_gpu_t h, int32_t enable);
int mpm_gpu_kernel_profile(mpm_gpu_t h, int32_t kernel, const char** name, double* total_ms,
                           int64_t* launches);
/* Kernels launched by this handle since profiling was last reset. */
int64_t mpm_gpu_launch_count(mpm_gpu_t h);

int64_t mpm_gpu_nparticles(mpm_gpu_t h);
int64_t mpm_gpu_current_step(mpm_gpu_t h);
/* The particle state into the caller's arrays (those given); page-locked ones
 * are written by the DMA engine directly, as in mpm_gpu_load_particles. */
int mpm_gpu_read_particles(mpm_gpu_t h, mpm_gpu_particles* out);

/* Particle output and checkpoint records.  Particle::pod (particle.tcc:180-306)
 * of every particle in the mesh, in particle order, packed on the device into
 * the caller's record layout: record i at records + i * record_size, field f
 * (the 74 PODParticle fields in declaration order, pod_particle.h:12-62) at
 * byte offset offsets[f] with size sizes[f] -- the reference's
 * pod::particle::dst_size / dst_offset / dst_sizes (pod_particle.cc), so a
 * std::vector<PODParticle> can receive them and go to H5TBmake_table as in
 * Mesh::write_particles_hdf5 (mesh.tcc:1573-1613).  Sizes must be 8 for the
 * doubles, id and cell_id, 4 for material_id and nstate_vars, 1 for the two
 * bools, each field aligned to its size, record_size a multiple of 8.
 * *nrecords receives the number of particles in the mesh; with capacity below
 * it nothing is written and MPM_ERR_INVALID is returned. */
int mpm_gpu_write_pod(mpm_gpu_t h, void* records, int64_t capacity, int64_t* nrecords,
                      size_t record_size, const size_t* offsets, const size_t* sizes,
                      int32_t nfields);

/* Checkpoint resume (MPMBase::checkpoint_resume, mpm_base.tcc:509-546;
 * Mesh::read_particles_hdf5, mesh.tcc:1663-1720; Particle::initialise_particle,
 * particle.tcc:21-175): replace the particles by n records in the layout of
 * mpm_gpu_write_pod.  Density is mass / volume; state variables are taken when
 * the record's nstate_vars matches the material's, else initialised; each
 * particle is located from its recorded cell (that cell, its neighbours, then
 * every cell in id order).  A particle outside the mesh is an error. */
int mpm_gpu_load_pod(mpm_gpu_t h, const void* records, int64_t n, size_t record_size,
                     const size_t* offsets, const size_t* sizes, int32_t nfields);

/* The particle output and checkpoint file (Mesh::write_particles_hdf5,
 * mesh.tcc:1573-1613; Mesh::read_particles_hdf5, mesh.tcc:1663-1720): the
 * PODParticle records of mpm_gpu_write_pod in the reference's own struct
 * layout (592-byte records, vtable slot first, pod_particle.h:12-62) written as
 * the HDF5 table H5TBmake_table makes -- dataset "table", compound type with
 * the field names and types of pod_particle.cc, chunks of 10000 records, no
 * compression, attributes CLASS, VERSION, TITLE, FIELD_<i>_NAME -- by the
 * library's own encoder (no HDF5 library involved).  mpm_gpu_load_hdf5 reads
 * such a table (by field name) and resumes from it as mpm_gpu_load_pod. */
int mpm_gpu_write_hdf5(mpm_gpu_t h, const char* path);
int mpm_gpu_load_hdf5(mpm_gpu_t h, const char* path);

/* The table codec itself.  Field types: */
enum { MPM_H5_F64 = 0, MPM_H5_I64 = 1, MPM_H5_U64 = 2, MPM_H5_I32 = 3, MPM_H5_U32 = 4,
       MPM_H5_U8 = 5 };
/* nrecords records of record_size bytes; field f at offsets[f] with type
 * types[f] and name names[f]; chunk_records records per chunk (10000 in the
 * reference). */
int mpm_h5_write_table(const char* path, const char* title, int64_t nrecords, size_t record_size,
                       int32_t nfields, const char* const* names, const size_t* offsets,
                       const int32_t* types, const void* records, int64_t chunk_records);
/* *nrecords receives the table's record count; with records non-NULL (room for
 * capacity records of record_size bytes) the named fields are copied to the
 * given offsets (types must match).  err receives a message (errlen bytes). */
int mpm_h5_read_table(const char* path, int64_t* nrecords, size_t record_size, int32_t nfields,
                      const char* const* names, const size_t* offsets, const int32_t* types,
                      void* records, int64_t capacity, char* err, int64_t errlen);

/* Sensitivities (no counterpart in the reference): derivatives of the whole
 * particle state with respect to up to two material parameters, carried by
 * every step after this call (forward-mode differentiation of the FP64 USL
 * step: P2G, node update with its boundary conditions, G2P, strain, volume,
 * MohrCoulomb return; discrete decisions follow the values).  kinds[k]:
 * 0 Young's modulus (Pa), 1 friction angle (degrees; peak and residual),
 * 2 cohesion (Pa; peak and residual), 3 dilation angle (degrees; peak and
 * residual), of material material_ids[k].  The derivatives start at zero for
 * the particle fields and at the parameter's own derivative for the state
 * variables it initialises.  n = 0 turns sensitivities off.  FP64 precision
 * and USL only (MPM_ERR_UNSUPPORTED otherwise); loading particles turns them
 * off.  A step carrying derivatives costs about three value-only steps. */
int mpm_gpu_set_sensitivities(mpm_gpu_t h, int32_t n, const int32_t* material_ids,
                              const int32_t* kinds);
/* d(field)/d(parameter k) for every particle: out[k][p][c], k < n, with c < 3
 * for field 0 x, 1 u, 2 v and c < 6 for field 3 stress (unused components 0). */
int mpm_gpu_read_sensitivities(mpm_gpu_t h, int32_t field, double* out);

/* Reverse-mode adjoint (no counterpart in the reference): gradients of a
 * loss on the particles' final positions and velocities with respect to up to
 * two material parameters (kinds as mpm_gpu_set_sensitivities) and to the
 * initial positions, velocities and stresses, by the discrete adjoint of the
 * FP64 USL step (FLIP or PIC, tensor-product grid, non-softening materials):
 * reverse G2P as a deterministic cell-slot scatter, reverse node update with
 * its velocity and friction constraints, reverse P2G as a per-particle gather,
 * and the reverse MohrCoulomb return map (its local Jacobian by forward-mode
 * passes over the return the forward step ran).  Paths of the forward run:
 * mpm_explicit.tcc:112-190, particle.tcc:630-657, 893-949, 994-1067,
 * node.tcc:236-345, 510-657, mohr_coulomb.tcc:348-513.
 *
 * mpm_gpu_adjoint_record advances nsteps from the current state like
 * mpm_gpu_step, keeping the particle state every checkpoint_every steps on the
 * device (0: every step when half the free device memory holds them -- the
 * reverse sweep then recomputes no step -- else ceil(sqrt(nsteps)) apart;
 * ceil(nsteps / checkpoint_every) checkpoints plus checkpoint_every
 * states of one segment, each holding the fields the reverse sweep reads --
 * x, v, stress, volume, density, mass, MohrCoulomb state, cell: about 200 B
 * per particle in 3D; MPM_ERR_ALLOC with the size when that does not fit).  mpm_gpu_adjoint_reverse then takes
 * dL/dx and dL/dv at the end (n*3 rows; either may be NULL for zero), recomputes
 * each segment from its checkpoint and sweeps back through it, and writes
 * dL/dparameter (nparams) and, when not NULL, dL/dx0, dL/dv0 (n*3) and
 * dL/dstress0 (n*6) of the state at the start of the record.  It leaves the
 * solver at the recorded run's end state and may be called again with other
 * cotangents.  Nodes lighter than 1e-3 of the mean particle mass pass no
 * cotangents (as the tangent step passes no derivatives there), so the
 * gradient equals mpm_gpu_set_sensitivities's. */
int mpm_gpu_adjoint_record(mpm_gpu_t h, int64_t nsteps, int64_t checkpoint_every, int32_t nparams,
                           const int32_t* material_ids, const int32_t* kinds);
int mpm_gpu_adjoint_reverse(mpm_gpu_t h, const double* dL_dx, const double* dL_dv,
                            double* dL_dparams, double* dL_dx0, double* dL_dv0,
                            double* dL_dstress0);
/* Both in one call for the calibration loss L = sum over particles in the
 * mesh of |x_final - x_target|^2 (x_target n*3 rows): *loss and dL/dparameter. */
int mpm_gpu_adjoint_run(mpm_gpu_t h, int64_t nsteps, int64_t checkpoint_every, int32_t nparams,
                        const int32_t* material_ids, const int32_t* kinds, const double* x_target,
                        double* loss, double* dL_dparams);

/* Slab decomposition (the reference's MPI halo sum and particle migration,
 * mesh.tcc:187-205, 737-1040): a run split along x into slabs of whole cell
 * columns, one solver per rank, each holding its columns plus one ghost column
 * per side.  mpm_gpu_step_begin runs a USL step's sort and P2G;
 * mpm_gpu_halo_pack writes the cell-slot partial sums and particle counts of
 * one x-column of cells (layer, the column's x index) to dst, and
 * mpm_gpu_halo_unpack writes such a buffer into a column (the caller moves
 * the buffers between ranks, e.g. with NCCL); mpm_gpu_step_end runs the rest
 * of the step (node update, G2P, plastic returns, locate) and counts it.
 * Buffers hold mpm_gpu_halo_bytes bytes and are device memory.
 * mpm_gpu_layer_count counts the particles whose cell's x index is below x_lo
 * and at or above x_hi (the ones to migrate).  USL, FLIP / PIC, tensor-product
 * grids. */
int mpm_gpu_step_begin(mpm_gpu_t h);
int mpm_gpu_step_end(mpm_gpu_t h);
int mpm_gpu_halo_bytes(mpm_gpu_t h, int64_t* bytes);
int mpm_gpu_halo_pack(mpm_gpu_t h, int32_t layer, void* dst);
int mpm_gpu_halo_unpack(mpm_gpu_t h, int32_t layer, const void* src);
int mpm_gpu_layer_count(mpm_gpu_t h, int32_t x_lo, int32_t x_hi, int64_t* below, int64_t* above);

/* Set the step counter (the resume step of analysis.resume.step; it drives the
 * gravity ramp, mpm_explicit.tcc:145-153). */
int mpm_gpu_set_current_step(mpm_gpu_t h, int64_t step);

/* Device addresses of the particle state (for zero-copy interop, e.g. torch).
 * field: 0 x, 1 u, 2 v, 3 stress, 4 strain, 5 F, 6 volume, 7 density, 8 mass.
 * Returns the base address; component c of particle p is at
 * base[c * stride + p] (doubles); *ncomp receives the component count.
 * MPM_PRECISION_MIXED keeps only x and u in FP64 and returns
 * MPM_ERR_UNSUPPORTED for the other fields. */
int mpm_gpu_device_field(mpm_gpu_t h, int32_t field, void** base, int64_t* stride,
                         int32_t* ncomp);

/* Material<Tdim>::compute_stress on a batch of independent points, on the
 * device (the constitutive kernel of the step, exposed for unit checks):
 * stress, dstrain, out: n*6; density: n; state: n*9 in/out. */
int mpm_gpu_material_stress_batch(int32_t device, int32_t dim, const char* type,
                                  const char* json_props, int64_t n, const double* stress,
                                  const double* dstrain, const double* density, double* state,
                                  double* out);

/* The same constitutive update for callers that cannot allocate device memory
 * (a plugin inside another program's memory arena, a real-time loop with a
 * fixed memory budget).  No counterpart in the reference.  It allocates
 * nothing: the points are staged in a fixed array of the library's device
 * image (32768 points, 7.3 MB, held by every GPU that loads the library until
 * the process exits).  n above 32768 is rejected with MPM_ERR_INVALID and a
 * message in err (errlen bytes, may be NULL).  All calls on a device share
 * its array; the entry point serialises its callers on that device with a
 * per-device lock and waits for its copies, so its calls never overlap.  Its
 * first call on a device looks up the array's address with that device
 * current and keeps it: make that call before any stream capture begins, and
 * do not reset the device afterwards.  A blocking call on the legacy default
 * stream (synchronous copies), not one to make during a stream capture. */
int mpm_gpu_material_stress_batch_noalloc(int32_t device, int32_t dim, const char* type,
                                          const char* json_props, int64_t n,
                                          const double* stress, const double* dstrain,
                                          const double* density, double* state, double* out,
                                          char* err, int64_t errlen);

/* Library version string. */
const char* mpm_gpu_version(void);

#ifdef __cplusplus
}
#endif
#endif /* MPM_GPU_H */
