/*
 * pmpm.h - C ABI of the B200-native update-stress-last (USL) MPM step.
 *
 * Drop-in replacement for the hot path of PyroclastMPM's USL solver.  Every
 * entry point names the reference interface it stands in for (paths relative
 * to the PyroclastMPM project root).  All state lives in one opaque handle
 * (no process globals), so several simulations may coexist in one process;
 * one handle must not be used from two host threads at once.
 *
 * Conventions
 *  - Every call returns an int status (pmpm_status); nothing calls exit().
 *  - Host arrays use the reference container layouts, particles in the order
 *    they were given (the "id" order), row-major:
 *      vectors [n][dim], stresses [n][3][3], F / velocity_gradient [n][dim][dim],
 *      node vectors [num_nodes][dim], node ids [num_nodes][3].
 *  - Kernels run on the handle's stream; calls that return data synchronise.
 *    Device faults of the step (a particle outside the grid, non-finite
 *    state) are accumulated on the device and reported by pmpm_synchronize.
 *  - Arithmetic is FP32, as the reference's DOUBLE_PRECISION=OFF build.
 */
#ifndef PMPM_H
#define PMPM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PMPM_MAX_MATERIALS 16
#define PMPM_MAX_BCS 16

typedef enum {
  PMPM_OK = 0,
  PMPM_ERR_INVALID_ARGUMENT = 1,
  PMPM_ERR_CUDA = 2,
  PMPM_ERR_OUT_OF_MEMORY = 3,
  PMPM_ERR_NOT_SUPPORTED = 4,
  PMPM_ERR_STATE = 5,          /* call order: e.g. a step before particles exist */
  PMPM_ERR_OUT_OF_DOMAIN = 16, /* a particle's cell lies outside the grid        */
  PMPM_ERR_NONFINITE = 17,     /* NaN or Inf appeared in particle positions      */
  PMPM_ERR_CELL_OVERFLOW = 18, /* more particles in one cell than the sort holds */
  PMPM_ERR_TIMEOUT = 19        /* a bounded wait inside a kernel ran out: the step's results are invalid */
} pmpm_status;

/* Shape functions: numbering of the reference SFType
 * (include/pyroclastmpm/common/types_common.h:151-156).  Quadratic has no
 * reference implementation (src/shapefunction/quadratic.cuh is empty). */
enum { PMPM_SHAPE_LINEAR = 0, PMPM_SHAPE_QUADRATIC = 1, PMPM_SHAPE_CUBIC = 2 };

/* Materials: the reference MaterialType variant
 * (include/pyroclastmpm/solver/solver.h:76-78) members on this path, plus
 * Drucker-Prager (cone + apex return mapping). */
enum {
  PMPM_MAT_NONE = 0,            /* Material base: stress untouched            */
  PMPM_MAT_LINEAR_ELASTIC = 1,  /* src/materials/linearelastic_inline.h:40-107 */
  PMPM_MAT_NEWTON_FLUID = 2,    /* src/materials/newtonfluid_inline.h:49-96    */
  PMPM_MAT_DRUCKER_PRAGER = 3,  /* src/materials/dp_rheo_inline.h:123-246      */
  /* J2 plasticity with linear hardening, 3D (src/materials/vonmises_inline.h:
   * 36-120; like Drucker-Prager, not a member of the reference's MaterialType) */
  PMPM_MAT_VON_MISES = 4,
  /* Modified Cam Clay with the reference's nonlinear (pressure-dependent)
   * elasticity: update_modifiedcamclay_nonlinear
   * (src/materials/modifiedcamclay_inline.h:321-511), the update the reference's
   * ModifiedCamClay::stress_update runs (src/materials/modifiedcamclay.cpp:
   * 148-178); a member of the reference's MaterialType */
  PMPM_MAT_MODIFIED_CAM_CLAY = 5,
  /* Drucker-Prager cone with a Cam-Clay-type cap and exponential hardening:
   * update_druckerpragercap (src/materials/druckerprager_cap_inline.h:370-554;
   * like Drucker-Prager, not a member of the reference's MaterialType) */
  PMPM_MAT_DRUCKER_PRAGER_CAP = 6
};

/* Boundary conditions: the reference BoundaryConditionType members on this
 * path (include/pyroclastmpm/solver/solver.h:80-82). */
enum {
  PMPM_BC_GRAVITY = 1,      /* src/boundaryconditions/gravity.cpp:65-88            */
  PMPM_BC_NODEDOMAIN = 2,   /* src/boundaryconditions/nodedomain_inline.h:40-87    */
  PMPM_BC_BODYFORCE = 3,    /* src/boundaryconditions/bodyforce_inline.h:41-59     */
  PMPM_BC_PLANARDOMAIN = 4, /* src/boundaryconditions/planardomain_inline.h:56-138 */
  /* RigidBodyLevelSet as the reference computes it: stick contact of nodes
   * with the nearest rigid particle (rigidbodylevelset_inline.h:65-199, 240-343,
   * rigidbodylevelset.cpp:92-275); linear shape functions only */
  PMPM_BC_RIGIDBODY_LEVELSET = 5,
  /* RigidBodyLevelSet with an analytic signed-distance body (sphere or
   * half-cylinder shell) in translation and rotation and Coulomb friction;
   * no reference counterpart (the reference's level set is the mode above) */
  PMPM_BC_RIGID_SDF = 6
};

/* Rigid-body modes (RigidBodyMode, include/pyroclastmpm/boundaryconditions/
 * rigidbodylevelset.h:33) and analytic shapes. */
enum { PMPM_RIGID_STATIC = 0, PMPM_RIGID_LOOP_ROTATE = 1 };
enum { PMPM_SDF_SPHERE = 0, PMPM_SDF_HALF_CYLINDER_SHELL = 1 };

/* Step flags. */
enum {
  /* keep the velocity gradient L of the last step in device memory (needed
   * for the velocity_gradient getter; the step itself does not need it) */
  PMPM_FLAG_KEEP_VELOCITY_GRADIENT = 1u << 0,
  /* deterministic reduction: P2G gathers each node's contributions in the
   * reference's fixed order (slot, then cell-sorted particle), so repeated
   * runs are bitwise identical; the default P2G accumulates in shared memory
   * in whatever order the threads arrive */
  PMPM_FLAG_DETERMINISTIC = 1u << 1,
  /* MUSL (modified update stress last; the reference declares the solver,
   * include/pyroclastmpm/solver/musl/musl.cuh, but does not build it): after
   * the USL grid update and a first G2P of velocities and positions, the new
   * particle momenta are mapped to the grid again (velocity conditions only)
   * and the velocity gradient for F and the stress update is taken from
   * that remapped field; all mappings of a step use its start-of-step weights */
  PMPM_FLAG_MUSL = 1u << 2
};

/* Material parameters; fill with the pmpm_material_* helpers.
 *   LINEAR_ELASTIC: {E, pois, lame, shear, bulk, corrected}
 *   NEWTON_FLUID:   {viscosity, bulk_modulus, gamma}
 *   DRUCKER_PRAGER: {K, G, eta, eta_bar, kc, p_apex, has_apex, pois}
 *                   (pois = -1 for the dp_rheo form, which takes no
 *                   per-particle E / friction angle)
 *                   yield sqrt(J2) + eta p - kc (p = tr(sigma)/3)
 *   VON_MISES:      {K, G, yield_stress, H}
 *   MODIFIED_CAM_CLAY: {K, G, M, lam, kap, Vs, Pt, R}
 *                   (R: preconsolidation ratio, pc = R p0 at initialize)
 *   DRUCKER_PRAGER_CAP: {K, G, M, lam, kap, Vs, Pt, R, beta, eta_bar} */
typedef struct {
  int type;
  float density;
  float params[12];
} pmpm_material;

/* Boundary-condition parameters; fill with the pmpm_bc_* helpers.
 *   GRAVITY:      reals[0..2] gravity, reals[3..5] gravity_end,
 *                 ints[0] is_ramp, ints[1] ramp_step
 *   NODEDOMAIN:   ints[0..2] face0_mode, ints[3..5] face1_mode (0 stick, 1 slip)
 *   BODYFORCE:    ints[0] mode (0 forces, 1 moments, 2 fixed), ints[1] active,
 *                 values [num_nodes][dim] and mask [num_nodes] (host, copied)
 *   PLANARDOMAIN: reals[0..2] face0 friction, reals[3..5] face1 friction
 *                 (radians; the pmpm_bc_planardomain helper converts degrees)
 *   RIGIDBODY_LEVELSET: ints[0] mode (PMPM_RIGID_*), ints[1] corrected rotation
 *                 (0: the reference's matrices, 1: proper Rz Ry Rx),
 *                 reals[0..2] euler angles per second, reals[3..5] COM
 *   RIGID_SDF:    ints[0] shape (PMPM_SDF_*), ints[1] axis (3D: 0, 1, 2; the
 *                 cross-section plane is (axis+1, axis+2) cyclic; 2D: the
 *                 plane is (x, y)), reals[0..2] centre at step 0,
 *                 reals[3..5] translational velocity, reals[6] angular
 *                 velocity about the axis (rad/s), reals[7] Coulomb friction
 *                 coefficient, reals[8..10] dimensions (sphere: radius;
 *                 shell: mid-surface radius, thickness, length along the
 *                 axis), reals[11] contact distance (nodes with signed
 *                 distance below it are in contact), reals[12] angle at step 0 */
typedef struct {
  int type;
  int ints[8];
  float reals[16];
  const float *values;
  const unsigned char *mask;
} pmpm_bc;

/* Everything the reference keeps in NodesContainer/Grid, the process-global
 * settings (set_globals, src/common/global_settings.cpp:161-176) and the
 * Solver's material/BC lists (src/solver/solver.cpp:69-104). */
typedef struct {
  int dim;                 /* 2 or 3 */
  float origin[3];
  float end[3];
  float cell_size;
  int shape_function;      /* PMPM_SHAPE_* */
  float dt;
  int particles_per_cell;
  float alpha;             /* FLIP/PIC blend, reference default 0.99 */
  int num_materials;
  const pmpm_material *materials;
  int num_bcs;
  const pmpm_bc *bcs;      /* applied in list order, as the reference */
  unsigned flags;          /* PMPM_FLAG_* */
  int device;              /* CUDA device ordinal */
  void *stream;            /* cudaStream_t; NULL: the handle creates its own */
  int resort_interval;     /* steps between physical re-sorts of particle
                              storage by cell (0: never); default 32 */
} pmpm_desc;

typedef struct pmpm_sim pmpm_sim;

/* Field ids for pmpm_get_field / pmpm_set_field (reference member names). */
typedef enum {
  PMPM_FIELD_POSITIONS = 0,          /* float [n][dim]    ParticlesContainer::positions_gpu        */
  PMPM_FIELD_VELOCITIES = 1,         /* float [n][dim]    ::velocities_gpu                         */
  PMPM_FIELD_STRESSES = 2,           /* float [n][3][3]   ::stresses_gpu                           */
  PMPM_FIELD_F = 3,                  /* float [n][dim][dim] ::F_gpu                                */
  PMPM_FIELD_VELOCITY_GRADIENT = 4,  /* float [n][dim][dim] ::velocity_gradient_gpu                */
  PMPM_FIELD_MASSES = 5,             /* float [n]         ::masses_gpu                             */
  PMPM_FIELD_VOLUMES = 6,            /* float [n]         ::volumes_gpu                            */
  PMPM_FIELD_VOLUMES_ORIGINAL = 7,   /* float [n]         ::volumes_original_gpu                   */
  PMPM_FIELD_COLORS = 8,             /* uint8 [n]         ::colors_gpu                             */
  PMPM_FIELD_IS_RIGID = 9,           /* uint8 [n]         ::is_rigid_gpu                           */
  PMPM_FIELD_IS_ACTIVE = 10,         /* uint8 [n]         ::is_active_gpu                          */
  PMPM_FIELD_FORCES_EXTERNAL = 11,   /* float [n][dim]    ::forces_external_gpu                    */
  PMPM_FIELD_EPS_E = 12,             /* float [n][dim][dim] Drucker-Prager elastic strain          */
  PMPM_FIELD_STRESS_REF = 13,        /* float [n][3][3]   Drucker-Prager reference stress          */
  PMPM_FIELD_YOUNGS_MODULUS = 14,    /* float [n]  per-particle Drucker-Prager E (no reference
                                        counterpart); first use fills it from the materials    */
  PMPM_FIELD_FRICTION_ANGLE = 15,    /* float [n]  per-particle Drucker-Prager friction angle (deg) */
  PMPM_FIELD_ACC_EPS_P = 16,         /* float [n]  VonMises accumulated plastic strain (acc_eps_p_gpu);
                                        Modified Cam Clay volumetric plastic strain (alpha_gpu) */
  PMPM_FIELD_PRECONSOLIDATION = 17,  /* float [n]  Modified Cam Clay preconsolidation pressure (pc_gpu) */
  PMPM_FIELD_NODE_MASSES = 20,       /* float [nodes]     NodesContainer::masses_gpu               */
  PMPM_FIELD_NODE_MOMENTS = 21,      /* float [nodes][dim] ::moments_gpu                           */
  PMPM_FIELD_NODE_MOMENTS_NT = 22,   /* float [nodes][dim] ::moments_nt_gpu                        */
  PMPM_FIELD_NODE_IDS = 23,          /* int   [nodes][3]  ::node_ids_gpu (unused axes 0)           */
  PMPM_FIELD_NODE_TYPES = 24,        /* int   [nodes][3]  ::node_types_gpu                         */
  PMPM_FIELD_BINS = 30,              /* int   [n][dim]    SpatialPartition::bins_gpu               */
  PMPM_FIELD_HASH_UNSORTED = 31,     /* uint32 [n]        ::hash_unsorted_gpu                      */
  PMPM_FIELD_HASH_SORTED = 32,       /* uint32 [n]        ::hash_sorted_gpu                        */
  PMPM_FIELD_SORTED_INDEX = 33,      /* int   [n]         ::sorted_index_gpu                       */
  PMPM_FIELD_CELL_START = 34,        /* int   [nodes]     ::cell_start_gpu (0 for empty cells)     */
  PMPM_FIELD_CELL_END = 35           /* int   [nodes]     ::cell_end_gpu (0 for empty cells)       */
} pmpm_field;

/* Human-readable status text. */
const char *pmpm_status_string(int status);

/* Material helpers: derived constants computed exactly as the reference
 * constructors do, in FP32.
 * LinearElastic::LinearElastic (src/materials/linearelastic.cpp:47-58);
 * corrected != 0 selects lame*tr(deps)*I + 2G*deps instead of the
 * reference's (lame + 2G)*deps (src/materials/linearelastic_inline.h:74-75). */
int pmpm_material_linear_elastic(float density, float E, float pois, int corrected, pmpm_material *out);
/* NewtonFluid::NewtonFluid (src/materials/newtonfluid.cpp:44-52). */
int pmpm_material_newton_fluid(float density, float viscosity, float bulk_modulus, float gamma,
                               pmpm_material *out);
/* Drucker-Prager with friction angle, dilatancy angle (degrees) and cohesion,
 * fitted to Mohr-Coulomb's outer cone: eta = 6 sin(phi)/(sqrt3 (3 - sin(phi))),
 * kc = 6 c cos(phi)/(sqrt3 (3 - sin(phi))), eta_bar likewise from psi.  The
 * cone and apex return follow update_dp_rheo (src/materials/dp_rheo_inline.h:
 * 123-246); there is no reference class with these parameters (the reference's
 * DP classes are not reachable from its USL solver). */
int pmpm_material_drucker_prager(float density, float E, float pois, float friction_deg,
                                 float dilatancy_deg, float cohesion, pmpm_material *out);
/* The reference DP_rheo parameters M (CSL slope), Pt (tensile pressure) and
 * dilatancy angle (degrees): DP_rheo::DP_rheo (src/materials/dp_rheo.cpp:45-70). */
int pmpm_material_dp_rheo(float density, float E, float pois, float M, float Pt, float dilatancy_deg,
                          pmpm_material *out);
/* VonMises::VonMises (src/materials/vonmises.cpp:31-44): 3D only */
int pmpm_material_von_mises(float density, float E, float pois, float yield_stress, float H, pmpm_material *out);
/* ModifiedCamClay::ModifiedCamClay (src/materials/modifiedcamclay.cpp:47-63):
 * M slope of the critical state line, lam / kap slopes of the virgin
 * consolidation and swelling lines, Vs solid volume (specific volume =
 * particle volume / Vs), R preconsolidation ratio, Pt tensile yield pressure;
 * beta is accepted and unused, as in the reference's update.  pmpm_initialize
 * then does ModifiedCamClay::initialize (:68-108): reference stress = current
 * stress, elastic strain and alpha = 0, pc = R p0 with p0 = -tr(sigma)/3. */
int pmpm_material_modified_cam_clay(float density, float E, float pois, float M, float lam, float kap, float Vs,
                                    float R, float Pt, float beta, pmpm_material *out);
/* DruckerPragerCap::DruckerPragerCap (src/materials/druckerprager_cap.cpp:
 * 43-67): as ModifiedCamClay, plus beta (cap ellipse ratio on its compressive
 * side) and the dilatancy angle in degrees (eta_bar = 6 sin(psi) /
 * (sqrt(3) (3 + sin(psi)))); the cone slope is eta = M / sqrt(3).  Initialize
 * as ModifiedCamClay (DruckerPragerCap::initialize, :72-108). */
int pmpm_material_drucker_prager_cap(float density, float E, float pois, float M, float lam, float kap, float Vs,
                                     float R, float Pt, float beta, float dilatancy_deg, pmpm_material *out);

/* Boundary-condition helpers (reference constructors). */
/* Gravity::Gravity (src/boundaryconditions/gravity.cpp:52-60) */
int pmpm_bc_gravity(const float *gravity, int is_ramp, int ramp_step, const float *gravity_end,
                    int dim, pmpm_bc *out);
/* NodeDomain::NodeDomain (src/boundaryconditions/nodedomain.cpp:33-37) */
int pmpm_bc_nodedomain(const int *face0_mode, const int *face1_mode, int dim, pmpm_bc *out);
/* BodyForce::BodyForce (src/boundaryconditions/bodyforce.cpp:44-61): mode
 * "forces" 0, "moments" 1, "fixed" 2 */
int pmpm_bc_bodyforce(int mode, const float *values, const unsigned char *mask, pmpm_bc *out);
/* PlanarDomain::PlanarDomain (src/boundaryconditions/planardomain.cpp:33-40):
 * friction angles in degrees, stored in radians */
int pmpm_bc_planardomain(const float *face0_friction_deg, const float *face1_friction_deg, int dim,
                         pmpm_bc *out);
/* RigidBodyLevelSet::RigidBodyLevelSet and ::set_mode_loop_rotate
 * (src/boundaryconditions/rigidbodylevelset.cpp:32-60).  mode STATIC keeps
 * the rigid particles' velocity at zero (the reference leaves its rotation
 * matrix unset in that mode; the identity is used).  euler_angles_per_second
 * and com may be NULL (zero). */
int pmpm_bc_rigidbodylevelset(int mode, const float *euler_angles_per_second, const float *com,
                              int corrected_rotation, int dim, pmpm_bc *out);
/* Analytic rigid body (no reference counterpart): shape PMPM_SDF_*, centre,
 * velocity (may be NULL), angular velocity about the axis, angle at step 0,
 * dims[3], Coulomb friction, contact distance.  Applied to the forward
 * moments of every node with mass whose position has signed distance below
 * the contact distance: the relative velocity's inward normal part is
 * removed and its tangential part reduced by friction (stick if the
 * tangential speed is below friction x the normal speed). */
int pmpm_bc_rigid_sdf(int shape, int axis, const float *center, const float *velocity, float angular_velocity,
                      float angle0, const float *dims, float friction, float contact_distance, int dim,
                      pmpm_bc *out);

/* Critical time step from the p-wave speed (src/common/tools.cpp:373-380,
 * LinearElastic::calculate_timestep, src/materials/linearelastic.cpp:96-105):
 * dt = factor * cell_size / sqrt((K + 4G/3) / density). */
int pmpm_calculate_timestep(float cell_size, float factor, float bulk_modulus, float shear_modulus,
                            float density, float *dt);
/* The same for a filled pmpm_material: LINEAR_ELASTIC and DRUCKER_PRAGER use
 * their K and G; NEWTON_FLUID uses K and G = 0 (sound speed sqrt(K/rho)). */
int pmpm_material_timestep(const pmpm_material *mat, float cell_size, float factor, float *dt);

/* Create a simulation: the Grid and NodesContainer constructors
 * (include/pyroclastmpm/common/types_common.h:260-272, src/nodes/nodes.cpp:
 * 55-83) and set_globals (src/common/global_settings.cpp:161-176), held per
 * handle instead of in process globals. */
int pmpm_create(const pmpm_desc *desc, pmpm_sim **out);

/* Release all device memory of the handle. */
int pmpm_destroy(pmpm_sim *sim);

/* Grid sizes: Grid::num_cells / num_cells_total. */
int pmpm_get_grid(const pmpm_sim *sim, int num_cells[3], int *num_cells_total, float *inv_cell_size);

/* Upload particles: ParticlesContainer::ParticlesContainer
 * (src/particles/particles.cpp:51-149).  Rigid particles are appended after
 * the others, as in the reference.  velocities/colors/rigid arrays may be NULL.
 * Masses and volumes start at -1 (unset), F at identity, stresses at zero. */
int pmpm_set_particles(pmpm_sim *sim, int num_particles, const float *positions, const float *velocities,
                       const unsigned char *colors, int num_rigid, const float *rigid_positions,
                       const float *rigid_velocities, const unsigned char *rigid_colors);

/* Solver::Solver set-up (src/solver/solver.cpp:69-104): partition, initial
 * volumes (src/particles/particles.cpp:345-365), initial masses per material
 * (:372-393); Drucker-Prager history starts from the current stresses. */
int pmpm_initialize(pmpm_sim *sim);

/* Copy a field out (reference layout, id order).  dst is host memory unless
 * on_device != 0.  bytes must equal the field's size. */
int pmpm_get_field(pmpm_sim *sim, int field, void *dst, size_t bytes, int on_device);

/* Copy a field in (the pybind property setters,
 * python/pybind/particles/particles_bind.cpp:179-301).  Stresses are stored
 * as symmetric tensors (upper triangle); 2D keeps xx, yy, xy and zz. */
int pmpm_set_field(pmpm_sim *sim, int field, const void *src, size_t bytes, int on_device);

/* Number of particles / nodes, bytes of one field. */
int pmpm_num_particles(const pmpm_sim *sim);
int pmpm_num_nodes(const pmpm_sim *sim);
size_t pmpm_field_bytes(const pmpm_sim *sim, int field);

/* ParticlesContainer::partition (src/particles/particles.cpp:332-339):
 * cell hash, stable sort by hash, cell start/end; bit-exact with the
 * reference (SpatialPartition, src/spatialpartition/spatialpartition.cpp:90-136). */
int pmpm_partition(pmpm_sim *sim);

/* calculate_shape_function (src/shapefunction/shapefunction.cpp:167-190):
 * psi [n][nsn] and dpsi [n][nsn][dim] in the reference slot order.  The step
 * never stores these (weights live in registers); this call materialises them
 * for inspection.  Requires a prior pmpm_partition. */
int pmpm_shape_functions(pmpm_sim *sim, float *psi, float *dpsi, int on_device);
int pmpm_num_surround_nodes(const pmpm_sim *sim);

/* USL::P2G (src/solver/usl/usl.cpp:118-161).  apply_bcs != 0 also applies the
 * node boundary conditions in list order (USL::solve :97-103), fused into the
 * P2G epilogue.  Requires a prior pmpm_partition. */
int pmpm_p2g(pmpm_sim *sim, int apply_bcs);

/* USL::G2P (src/solver/usl/usl.cpp:164-199); stress_update != 0 also runs
 * Solver::stress_update (src/solver/solver.cpp:110-121) fused per particle. */
int pmpm_g2p(pmpm_sim *sim, int stress_update);

/* Solver::stress_update alone, from the stored velocity gradient. */
int pmpm_stress_update(pmpm_sim *sim);
/* The MUSL stages after USL's P2G (a handle created with PMPM_FLAG_MUSL):
 * 1 MUSL::G2P_double_mapping (velocities, positions set aside),
 * 2 MUSL::P2G_double_mapping (momentum remap, velocity conditions),
 * 3 MUSL::G2P (velocity gradient, F, V, positions, stress update)
 * (include/pyroclastmpm/solver/musl/musl.cuh). */
int pmpm_musl_stage(pmpm_sim *sim, int stage);

/* USL::solve (src/solver/usl/usl.cpp:69-115) followed by increment_global
 * (src/common/global_settings.cpp:220-227), nsteps times: Solver::solve_nsteps
 * (src/solver/solver.cpp:125-134).  Asynchronous. */
int pmpm_solve(pmpm_sim *sim, int nsteps);

/* Diagnostic: one USL step (as pmpm_solve(sim, 1)) with CUDA events between
 * its phases on the handle's stream; returns the phase durations in ms:
 * ms[0] partition (hash, scan, scatter, in-cell sort, re-sort when due),
 * ms[1] P2G with the node epilogue, ms[2] G2P with the stress update.
 * launches (may be NULL) receives the number of kernels the step launched.
 * No reference counterpart (the reference logs only wall time,
 * src/solver/solver.cpp:153-169). */
int pmpm_profile_step(pmpm_sim *sim, float ms[3], int *launches);

/* Number of kernels the handle has launched since it was created. */
int pmpm_launch_count(const pmpm_sim *sim, long long *count);

/* Bound on the key scan's look-back wait (no reference counterpart: the
 * reference sorts with thrust and calls exit() on a CUDA error,
 * include/pyroclastmpm/common/types_common.h:170-187).  A CTA of the
 * one-launch scan polls its predecessors' published sums at most `spins`
 * times (default 4194304); past that it records PMPM_ERR_TIMEOUT, and the
 * kernels that index particles through the scan's offsets skip the step's
 * P2G instead of reading through an invalid prefix.  After PMPM_ERR_TIMEOUT
 * the particle state is invalid: set it again.  0 gives up at the first
 * poll that finds a predecessor not yet published. */
int pmpm_set_wait_limit(pmpm_sim *sim, long long spins);

/* The tag (1 .. 2^30 - 2) that the key scan's launch number `launch` stamps
 * on its published sums; consecutive launches alternate its parity, which
 * picks their ticket counters, across the counter's wrap as well.
 * Diagnostic, no reference counterpart. */
int pmpm_scan_tag(unsigned launch, unsigned *tag);

/* The autotuner's re-sort interval rule (pmpm_autotune) on given timings:
 * t_sort the time of one physical re-sort, step_ms[0 .. m) the times of m
 * consecutive steps after it (ms); *interval gets the K in {8, 16, 32, 64,
 * 128} minimising t_sort / K + slope K / 2.  Host only, no GPU work; no
 * reference counterpart. */
int pmpm_pick_resort_interval(float t_sort, const float *step_ms, int m, int *interval);

/* Number of grid nodes with mass above the cutoff after the last P2G
 * (the nodes the step actually updates). */
int pmpm_active_nodes(pmpm_sim *sim, int *count);

/* The global step counter (set_global_step / global_step_cpu). */
int pmpm_get_step(const pmpm_sim *sim, int *step);
int pmpm_set_step(pmpm_sim *sim, int step);

/* Wait for the handle's stream; returns the first device fault seen since
 * the last call (PMPM_ERR_OUT_OF_DOMAIN, ...) or PMPM_OK, and clears it. */
int pmpm_synchronize(pmpm_sim *sim);

/* The handle's CUDA stream (cudaStream_t) and device. */
void *pmpm_stream(const pmpm_sim *sim);

/* Single-point material update on host arrays of n points: the standalone
 * stress_update binding of the reference DP material
 * (python/pybind/materials/dp_rheo.cpp:57) generalised to any material here.
 * L [n][dim][dim] (or the strain increment itself when
 * velgrad_is_strain_increment != 0), stress [n][3][3] in/out, eps_e
 * [n][dim][dim] in/out, stress_ref [n][3][3], masses/volumes/volumes_original
 * [n] (Newtonian fluid only; may be NULL otherwise). */
int pmpm_material_point_update(const pmpm_material *mat, int dim, int n, float dt, const float *L,
                               float *stress, float *eps_e, const float *stress_ref, const float *masses,
                               const float *volumes, const float *volumes_original,
                               int velgrad_is_strain_increment, int device);

/* Spatial partition that allocates no device memory.  No counterpart in the
 * reference; it gives the results of pmpm_partition (reference hashing,
 * stable sort, cell ranges) to callers that cannot allocate device memory at
 * the point they need them, for example code inside a memory pool's or a
 * framework's allocation callback, or plug-ins held to a fixed device-memory
 * budget by their host application.  The caller passes device pointers: positions
 * [n][dim] (the particles in index order) in, and hash_unsorted [n],
 * sorted_index [n] (binned particles), cell_start and cell_end [cells] out,
 * with cells = num_cells[0] * num_cells[1] (* num_cells[2]).  Temporaries
 * live in one fixed device array inside the library: at most 131072
 * particles and 131072 cells (larger inputs return
 * PMPM_ERR_INVALID_ARGUMENT).  The first call on a device looks up that
 * array's address and, with CUDA's lazy module loading, is when the driver
 * loads this code and places the array; make that first call (a warm-up
 * call will do) before any stream capture and outside any allocation
 * callback.  Calls share the array, so calls that overlap on the GPU race:
 * serialise them.  Waits for `stream` (cudaStream_t, may be NULL) before
 * returning.  Returns PMPM_ERR_OUT_OF_DOMAIN when a particle's cell lies
 * outside the grid on any axis or a coordinate is not finite; the outputs
 * still follow the reference's flat hash (a particle whose flat index stays
 * inside the grid is binned where it points, one past it is left out).
 * Returns PMPM_ERR_CELL_OVERFLOW when one cell holds more than 2048
 * particles: that cell's entries of sorted_index are then not in ascending
 * order (the other outputs are complete). */
int pmpm_partition_noalloc(int dim, const float *origin, float cell_size, const int *num_cells,
                           const float *positions, int num_particles, unsigned *hash_unsorted,
                           int *sorted_index, int *cell_start, int *cell_end, void *stream);

/* Autotuner (no reference counterpart; the reference launches every kernel
 * with a fixed block of 64 threads, include/pyroclastmpm/common/types_common.h:
 * 205-229).  Tunes, from the current state, for this handle:
 *  - the P2G kernel where a configuration has more than one (3D quadratic:
 *    dual-cell z-sweep per node tile, or a warp per row of dual cells
 *    scattering into brick boxes) and the staging of the 3D sweeps (bulk
 *    copies of sorted records, or a gather through the sorted order): each
 *    (kernel, staging) pair is timed on `steps` steps;
 *  - the re-sort interval (when it is not 0): one physical re-sort is timed,
 *    then the chosen kernels on max(48, 4 steps) steps without re-sorts; the
 *    interval in {8, 16, 32, 64, 128} minimising t_sort / K + slope K / 2
 *    is kept (slope: the growth of the step time per step, fitted by least
 *    squares, less two standard errors of the fit, at least 0).
 * The particle state and the step counter are put back afterwards.
 * *chosen: the P2G kernel (1 sweep, 0 cell scatter); pmpm_get_tuning reports
 * all choices. */
int pmpm_autotune(pmpm_sim *s, int steps, int *chosen);
/* Selects the P2G kernel directly (the autotuner's choices: 1 sweep, 0 cell
 * scatter); PMPM_ERR_NOT_SUPPORTED where the configuration has only one.
 * The 3D quadratic sweep runs one work item per thread of its CTA (up to 640);
 * on a grid with a node count divisible by 8 along x or y, the tiles ending at
 * that face hold 27 (source, offset) pairs along it and more items than that,
 * so such grids run the cell scatter and selecting the sweep is refused. */
int pmpm_set_p2g_kernel(pmpm_sim *s, int variant);
/* Staging of the 3D sweep P2G kernels: 1 (default) the particles of each
 * row of source cells arrive in shared memory by one bulk copy
 * (cp.async.bulk on an mbarrier) from records written in sorted order just
 * before the P2G; 0 each particle's fields are gathered through the sorted
 * order.  PMPM_ERR_NOT_SUPPORTED without a 3D sweep (2D, deterministic). */
int pmpm_set_p2g_staging(pmpm_sim *s, int mode);
/* Steps between physical re-sorts of particle storage (0: never). */
int pmpm_set_resort_interval(pmpm_sim *s, int steps);
/* The handle's current choices: P2G kernel (as pmpm_set_p2g_kernel), staging
 * (as pmpm_set_p2g_staging, -1 where it does not apply), re-sort interval.
 * Any pointer may be NULL. */
int pmpm_get_tuning(const pmpm_sim *s, int *p2g_kernel, int *staging, int *resort_interval);

/* ---------------------------------------------------------------------------
 * Differentiable rollouts (no counterpart in the reference).  A rollout of
 * nsteps USL steps from the current state keeps the particle state every
 * checkpoint_every steps; the backward pass recomputes each segment from its
 * checkpoint and runs the adjoint kernels step by step, giving the gradient
 * of a loss on the final positions with respect to the per-particle
 * Drucker-Prager Young's modulus and friction angle (PMPM_FIELD_YOUNGS_MODULUS
 * / _FRICTION_ANGLE, filled from the materials if not set) and the initial
 * positions and velocities.  Quadratic shape functions; Drucker-Prager and
 * inert materials; Gravity and NodeDomain conditions.  The physical re-sort
 * is off while a rollout is held.
 * ------------------------------------------------------------------------- */
int pmpm_rollout_forward(pmpm_sim *s, int nsteps, int checkpoint_every);
/* Device memory for segments kept whole from the forward pass (every step's
 * state and P2G node data), so the backward pass recomputes none of them:
 * the last segments are kept while they fit.  bytes < 0 (default): 60 % of
 * the free device memory at the start of each rollout; 0: checkpoints only.
 * Gradients do not depend on it. */
int pmpm_rollout_set_memory(pmpm_sim *s, long long bytes);
/* Back to the state the last rollout started from (step counter included). */
int pmpm_rollout_reset(pmpm_sim *s);
/* grad_positions: dLoss/dx of the final positions [n][dim] (id order).
 * Outputs (each may be NULL): [n] dLoss/dE, [n] dLoss/dphi (per degree),
 * [n][dim] dLoss/dx0, [n][dim] dLoss/dv0.  All host or all device memory
 * (on_device).  Leaves the simulation at the rollout's initial state. */
int pmpm_rollout_backward(pmpm_sim *s, const float *grad_positions, int on_device, float *grad_youngs,
                          float *grad_friction, float *grad_positions0, float *grad_velocities0);

/* Vector-Jacobian product of the single-point Drucker-Prager update
 * (pmpm_material_point_update's material law; no reference counterpart):
 * given adjoints of the new stress [n][3][3] and elastic strain [n][dim][dim],
 * the adjoints of the velocity gradient [n][dim][dim], of the old elastic
 * strain [n][dim][dim] (one value per independent component, on both of its
 * entries) and, with per-particle youngs / friction (else NULL, and the
 * gradients are 0), of E and the friction angle (per degree).  method 0:
 * reverse mode (what the rollout adjoint uses); 1: forward-mode dual
 * numbers, an independent evaluation for cross-checks.  Host arrays. */
int pmpm_material_point_vjp(const pmpm_material *mat, int dim, int n, float dt, const float *L, const float *eps_e,
                            const float *stress_ref, const float *youngs, const float *friction,
                            const float *grad_stress, const float *grad_eps_e, float *grad_L, float *grad_eps_e_in,
                            float *grad_youngs, float *grad_friction, int method, int device);

/* ---------------------------------------------------------------------------
 * Batched ensembles.  No counterpart in the reference (its settings are
 * process globals: one simulation per process).  Many independent
 * simulations are stepped together with one kernel launch per phase for
 * all of them; each instance gives the results of a pmpm_sim created from
 * the same descriptor and particles.  Instances share the dimension, shape
 * function and flags; the grid, dt, materials and boundary conditions are
 * per instance (RIGIDBODY_LEVELSET's nearest-rigid-particle mode is not
 * supported).  The descriptors' device, stream and resort_interval are
 * replaced by the batch's.
 * ------------------------------------------------------------------------- */
typedef struct pmpm_batch pmpm_batch;

typedef struct {
  const pmpm_desc *desc;
  int num_particles;
  const float *positions;      /* [n][dim], host */
  const float *velocities;     /* [n][dim] or NULL */
  const unsigned char *colors; /* [n] or NULL */
} pmpm_instance;

int pmpm_batch_create(int num_instances, const pmpm_instance *instances, int device, void *stream,
                      int resort_interval, pmpm_batch **out);
int pmpm_batch_destroy(pmpm_batch *b);
/* Solver::Solver set-up for every instance (volumes, masses, partition). */
int pmpm_batch_initialize(pmpm_batch *b);
/* nsteps USL steps of every instance (Solver::solve_nsteps per instance). */
int pmpm_batch_solve(pmpm_batch *b, int nsteps);
int pmpm_batch_num_instances(const pmpm_batch *b);
int pmpm_batch_num_particles(const pmpm_batch *b, int instance);
/* Particle fields, node masses/moments/ids/types and bins of one instance,
 * as pmpm_get_field / pmpm_set_field (setters: particle fields only). */
int pmpm_batch_get_field(pmpm_batch *b, int instance, int field, void *dst, size_t bytes, int on_device);
int pmpm_batch_set_field(pmpm_batch *b, int instance, int field, const void *src, size_t bytes, int on_device);
/* Waits for the batch's work; returns the first device fault of any instance. */
int pmpm_batch_synchronize(pmpm_batch *b);
/* One step with CUDA-event times: ms[0] partition, ms[1] P2G, ms[2] G2P. */
int pmpm_batch_profile_step(pmpm_batch *b, float *ms, int *launches);
int pmpm_batch_launch_count(const pmpm_batch *b, long long *count);
/* pmpm_set_wait_limit for the batch's key scan. */
int pmpm_batch_set_wait_limit(pmpm_batch *b, long long spins);

#ifdef __cplusplus
}
#endif
#endif /* PMPM_H */
