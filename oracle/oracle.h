/*
 * CPU oracle for the update-stress-last (USL) explicit MPM step of
 * PyroclastMPM.  TEST INFRASTRUCTURE ONLY: the oracle is the checker that the
 * CUDA path is compared against (tests, smoke(), bench cpu_baseline); it is
 * never linked into or called by the product library.
 *
 * The file is compiled twice: with REAL=float (the reference's FP32 build,
 * CMake DOUBLE_PRECISION=OFF) and with REAL=double (the FP64 drift oracle).
 *
 * Parity pinning: the reference cannot be compiled here (its Eigen, spdlog and
 * VTK dependencies are absent), so this restatement is pinned against the
 * reference's own known-answer unit tests (tests/unit/test_spatialpartition.h,
 * test_shapefunctions.h, test_usl.h, test_particles.h, test_nodes.h), whose
 * vectors live in tests/golden/reference_unit_vectors.json.
 *
 * Layouts follow the reference containers (AoS, row-major):
 *   positions/velocities/f_ext [n][dim], stresses [n][3][3], F/L [n][dim][dim],
 *   psi [n][nsn], dpsi [n][nsn][dim], node moments [nodes][dim].
 */
#ifndef PMPM_ORACLE_H
#define PMPM_ORACLE_H

#ifndef REAL
#define REAL float
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Shape function ids, same numbering as the reference SFType
 * (include/pyroclastmpm/common/types_common.h:151-156). */
enum { OR_LINEAR = 0, OR_QUADRATIC = 1, OR_CUBIC = 2 };

/* Material ids (position in the solver's material list is the colour). */
enum {
  OR_MAT_NONE = 0,          /* Material base class: stress untouched      */
  OR_MAT_LINEAR_ELASTIC = 1,
  OR_MAT_NEWTON_FLUID = 2,
  OR_MAT_DRUCKER_PRAGER = 3,
  OR_MAT_VON_MISES = 4,      /* p = {K, G, yield_stress, H}; 3D only */
  OR_MAT_MODIFIED_CAM_CLAY = 5, /* p = {K, G, M, lam, kap, Vs, Pt, R} */
  OR_MAT_DRUCKER_PRAGER_CAP = 6 /* p = {K, G, M, lam, kap, Vs, Pt, R, beta, eta_bar} */
};

/* Boundary-condition ids. */
enum {
  OR_BC_NONE = 0,
  OR_BC_GRAVITY = 1,
  OR_BC_NODEDOMAIN = 2,
  OR_BC_BODYFORCE = 3,
  OR_BC_PLANARDOMAIN = 4,
  OR_BC_RIGIDBODY_LEVELSET = 5, /* reference mode: nearest rigid particle */
  OR_BC_RIGID_SDF = 6           /* analytic body, Coulomb contact (no reference) */
};

/* Mirrors the reference Grid (include/pyroclastmpm/common/types_common.h:250-291). */
typedef struct {
  int dim;
  REAL origin[3];
  REAL end[3];
  REAL cell_size;
  REAL inv_cell_size;
  int num_cells[3];
  int num_cells_total;
} or_grid;

/* Material parameters.
 *   LINEAR_ELASTIC: p = {E, pois, lame, shear, bulk, corrected(0/1)}
 *   NEWTON_FLUID:   p = {viscosity, bulk_modulus, gamma}
 *   DRUCKER_PRAGER: p = {bulk K, shear G, eta, eta_bar, kc, p_apex, has_apex, pois}
 *     (pois < 0: dp_rheo form, no per-particle parameters)
 *     yield  Phi = sqrt(J2) + eta*p - kc   (p = tr(sigma)/3, tension positive)
 */
typedef struct {
  int type;
  REAL density;
  REAL p[12];
} or_material;

/* Boundary-condition parameters (state that the reference mutates, the
 * current gravity vector, is kept in r[0..2]).
 *   GRAVITY:      r[0..2] gravity, r[3..5] gravity_end, i[0] is_ramp, i[1] ramp_step
 *   NODEDOMAIN:   i[0..2] face0_mode, i[3..5] face1_mode
 *   BODYFORCE:    i[0] mode_id (0 forces, 1 moments, 2 fixed), i[1] is_active,
 *                 values [nodes][dim], mask [nodes]
 *   PLANARDOMAIN: r[0..2] face0 friction (radians), r[3..5] face1 friction
 *   RIGIDBODY_LEVELSET: i[0] mode (0 STATIC, 1 LOOP_ROTATE), i[1] corrected
 *                 rotation, r[0..2] euler angles per second, r[3..5] COM,
 *                 r[6..8] accumulated euler angles (state)
 *   RIGID_SDF:    i[0] shape (0 sphere, 1 half-cylinder shell), i[1] axis,
 *                 r[0..2] centre at step 0, r[3..5] velocity, r[6] angular
 *                 velocity, r[7] friction, r[8..10] dims, r[11] contact
 *                 distance, r[12] angle at step 0
 */
typedef struct {
  int type;
  int i[8];
  REAL r[16];
  const REAL *values;
  const unsigned char *mask;
} or_bc;

typedef struct {
  or_grid grid;
  int shape_function;
  int nsn;               /* stencil slots per particle (2^D or 4^D) */
  REAL dt;
  REAL alpha;
  REAL small_mass_cutoff;
  int global_step;
  int particles_per_cell;
  int num_particles;

  /* particles */
  REAL *positions, *velocities, *stresses, *F, *velocity_gradient;
  REAL *masses, *volumes, *volumes_original, *forces_external;
  unsigned char *colors, *is_rigid, *is_active;
  REAL *psi, *dpsi;

  /* spatial partition */
  int *bins;
  unsigned int *hash_unsorted, *hash_sorted;
  int *sorted_index, *cell_start, *cell_end;

  /* nodes */
  REAL *node_masses, *node_moments, *node_moments_nt;
  int *node_ids, *node_types;

  /* materials / boundary conditions, in the solver's list order */
  int num_materials;
  or_material *materials;
  int num_bcs;
  or_bc *bcs;

  /* Drucker-Prager history: elastic strain [n][dim][dim], reference stress [n][3][3] */
  REAL *eps_e, *stress_ref;

  /* optional per-particle Drucker-Prager Young's modulus and friction angle
   * (degrees) [n], or NULL: replace the material's K, G, eta, kc (friction
   * form of the material only, p[7] = Poisson ratio >= 0) */
  REAL *youngs, *friction;

  /* 1: MUSL step (second momentum mapping, velocity gradient from it) */
  int musl;

  /* VonMises accumulated plastic strain [n] (elastic strain in eps_e);
   * Modified Cam Clay volumetric plastic strain alpha [n] */
  REAL *acc_eps_p;

  /* Modified Cam Clay preconsolidation pressure [n] */
  REAL *pc;
} or_sim;

void or_grid_init(or_grid *g, int dim, const REAL *origin, const REAL *end, REAL cell_size);
int or_num_surround_nodes(int dim, int shape_function);
void or_node_ids(const or_grid *g, int *node_ids);
void or_node_types(const or_grid *g, int shape_function, const int *node_ids, int *node_types);
void or_calculate_hash(const or_grid *g, int n, const REAL *x, int *bins,
                       unsigned int *hash_unsorted, unsigned int *hash_sorted);
void or_sort_hashes(int n, unsigned int *hash_sorted, int *sorted_index);
void or_bin_particles(const or_grid *g, int n, const unsigned int *hash_sorted,
                      int *cell_start, int *cell_end);
void or_partition(or_sim *s);
void or_shape_functions(or_sim *s);
void or_initial_volumes(or_sim *s);
void or_initial_masses(or_sim *s, int mat_id, REAL density);
void or_reset(or_sim *s);
void or_apply_on_particles(or_sim *s);
void or_p2g(or_sim *s);
void or_apply_on_nodes_moments(or_sim *s);
void or_g2p(or_sim *s);
void or_stress_update(or_sim *s);
void or_solve(or_sim *s);
void or_solve_nsteps(or_sim *s, int nsteps);
void or_dp_point(int dim, const REAL *L, REAL *stress, REAL *eps_e, const REAL *stress_ref,
                 REAL dt, const REAL *p, int velgrad_is_strain_increment);
/* One Modified Cam Clay update of a single material point (stress [3][3],
 * elastic strain [dim][dim], reference stress [3][3], alpha, pc; V the
 * particle's current volume). */
void or_mcc_point(int dim, const REAL *L, REAL *stress, REAL *eps_e, const REAL *stress_ref, REAL *alpha, REAL *pc,
                  REAL V, REAL dt, const or_material *m);
/* One Drucker-Prager cap update of a single material point (V0: original volume). */
void or_dpc_point(int dim, const REAL *L, REAL *stress, REAL *eps_e, const REAL *stress_ref, REAL *alpha, REAL *pc,
                  REAL V0, REAL dt, const or_material *m);

#ifdef __cplusplus
}
#endif
#endif
