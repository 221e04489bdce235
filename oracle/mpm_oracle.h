/*
 * mpm_oracle.h -- C interface of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a plain C++17 restatement of the
 * reference explicit MPM step (geomechanics/mpm, MPMExplicit with USF/USL,
 * FLIP/PIC, quad4/hex8, LinearElastic and MohrCoulomb, velocity, acceleration
 * and friction constraints, Cundall damping, particle location).  Only the test
 * suite, the smoke check and the CPU-baseline leg of the benchmark may load it;
 * the product library never links or calls it.
 *
 * Every function in mpm_oracle.cpp cites the reference file:line it restates.
 * Eigen (a system dependency of the reference, not vendored, version not
 * pinned) is replaced by fixed-size arrays: sums are evaluated left to right,
 * 2x2/3x3 inverses by adjugate over determinant as Eigen's fixed-size inverse
 * does.  Where Eigen's SIMD reduction order differs the results differ in the
 * last ulp; parity is asserted with a relative tolerance, never bitwise, for
 * floating point, and bitwise for cell indices.
 */
#ifndef MPM_ORACLE_H
#define MPM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int32_t dim;              /* 2 or 3 */
  int32_t scheme;           /* 0 = USF, 1 = USL, 2 = MUSL */
  int32_t velocity_update;  /* 0 = FLIP, 1 = PIC, 2 = ASFLIP, 3 = TPIC, 4 = APIC
                               (data_types.h:50 VelocityUpdate order) */
  int32_t locate_particles; /* 1: unlocatable particle is an error, 0: removed */
  double blending_ratio;
  double dt;
  double damping_factor; /* Cundall */
  double gravity[3];
  double gravity_ramping_time;
  int32_t nthreads; /* 1 = deterministic golden mode */
  int32_t isoparametric; /* 1: local coordinates by the isoparametric map
                            (cell.tcc:617-826), 0: the Cartesian formula */
} mpmo_config;

/* Particle state as flat arrays, one record per particle (AoS in this API).
 * x,u,v,a: n*3; stress,strain,dstrain,strain_rate: n*6; F: n*9 (row-major);
 * svars: n*9 (MohrCoulomb state in the reference order yield_state, phi,
 * psi, cohesion, tension_cutoff, epsilon, rho, theta, pdstrain; zeros for
 * LinearElastic).  Any pointer may be NULL when not wanted. */
typedef struct {
  double* x;
  double* u;
  double* v;
  double* a;
  double* stress;
  double* strain;
  double* dstrain;
  double* strain_rate;
  double* F;
  double* volume;
  double* mass;
  double* density;
  double* xi;
  int64_t* cell;
  int32_t* material;
  double* svars;
  int32_t* status;
  double* mapping; /* n*9 row-major mapping matrix (affine / Taylor updates;
                      the leading dim x dim block) */
} mpmo_particles;

void* mpmo_create(const mpmo_config* cfg);
void mpmo_destroy(void* h);
const char* mpmo_last_error(void* h);

int mpmo_set_mesh(void* h, int64_t nnodes, const double* coords, int64_t ncells,
                  int32_t nodes_per_cell, const int64_t* cell_nodes);
/* type 0 = LinearElastic, 1 = MohrCoulomb; parameter order in mpm_oracle.cpp */
int mpmo_add_material(void* h, int32_t id, int32_t type, const double* params,
                      int32_t nparams);
int mpmo_add_velocity_constraints(void* h, int64_t n, const int64_t* nid,
                                  const int32_t* dir, const double* val);
int mpmo_add_acceleration_constraints(void* h, int64_t n, const int64_t* nid,
                                      const int32_t* dir, const double* val);
int mpmo_add_friction_constraints(void* h, int64_t n, const int64_t* nid,
                                  const int32_t* dir, const int32_t* sign_n,
                                  const double* mu);
/* General boundaries: dim Euler angles (radians) per node; the node's
 * velocity, acceleration and friction constraints then act in its rotated
 * frame (mesh.tcc:1318-1345, node.tcc:370-483, 510-657). */
int mpmo_set_nodal_euler_angles(void* h, int64_t n, const int64_t* nid, const double* angles);
/* Particle velocity constraint on a list of particle ids (set id -1 = all). */
int mpmo_add_particle_velocity_constraint(void* h, int64_t n,
                                          const int64_t* pids, int32_t dir,
                                          double velocity);
/* create particles from coordinates (Mesh::create_particles) */
int mpmo_add_particles(void* h, int64_t n, const double* coords,
                       int32_t material_id);
/* locate, compute_volume, compute_mass, initial acceleration = gravity */
int mpmo_initialise(void* h);
/* overwrite full particle state (after mpmo_add_particles / initialise) */
int mpmo_set_particles(void* h, const mpmo_particles* p);
int64_t mpmo_nparticles(void* h);
int mpmo_get_particles(void* h, mpmo_particles* p);
int mpmo_step(void* h, int64_t nsteps);
/* nodal state, 17 doubles per node: mass, momentum[3], fext[3], fint[3],
 * vel[3], acc[3], status */
int mpmo_get_nodes(void* h, double* out);
int mpmo_set_nodes(void* h, const double* in);
/* one phase of the scheme (mpm_scheme.tcc): 0 initialise (zero nodes,
 * activate, shape functions), 1 P2G mass + momentum, 2 nodal velocity,
 * 3 stress and strain, 4 body force (gravity[3]), 5 internal force,
 * 6 nodal acceleration/velocity (Cundall), 7 G2P, 8 locate */
int mpmo_phase(void* h, int32_t phase, double dt, const double* gravity);

/* ---- unit-level entry points used by the known-answer tests ---- */
/* shape functions and gradients at xi for a cell with nodal coordinates X
 * (nv x dim), N: nv, dndx: nv x dim, grad: nv x dim (natural) */
int mpmo_element_dn_dx(int32_t dim, const double* xi, const double* X,
                       double* N, double* grad, double* dndx);
/* one material stress update; state: 9 doubles (MC order) */
int mpmo_material_stress(int32_t dim, int32_t type, const double* params,
                         int32_t nparams, const double* stress,
                         const double* dstrain, double density, double* state,
                         double* stress_out);
/* MC yield state and derivative helpers at a stress, for KATs:
 * out: [epsilon, rho, theta, f_tension, f_shear, yield_type,
 *       df_dsigma(6), dp_dsigma(6), dp_dq, softening] */
int mpmo_mc_diagnostics(int32_t dim, const double* params, int32_t nparams,
                        const double* stress, double* state, double* out);

#ifdef __cplusplus
}
#endif
#endif
