/*
 * CPU oracle for the PyroclastMPM update-stress-last step.
 * TEST INFRASTRUCTURE ONLY (see oracle.h): used by tests/, smoke() and the
 * bench's CPU baseline as the checker; never part of the product path.
 *
 * Every function names the reference code it restates.  Paths are relative to
 * the PyroclastMPM project root.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef REAL real;

/* ------------------------------------------------------------------------ */
/* Grid and stencil windows                                                 */
/* ------------------------------------------------------------------------ */

/* Grid ctor: include/pyroclastmpm/common/types_common.h:260-272.
 * inv = 1/h and N_axis = (int)((end - origin)/h) + 1, all in REAL. */
void or_grid_init(or_grid *g, int dim, const REAL *origin, const REAL *end, REAL cell_size) {
  memset(g, 0, sizeof(*g));
  g->dim = dim;
  g->cell_size = cell_size;
  g->inv_cell_size = (real)1.0 / cell_size;
  g->num_cells_total = 1;
  for (int a = 0; a < 3; a++) {
    g->num_cells[a] = 1;
    if (a < dim) {
      g->origin[a] = origin[a];
      g->end[a] = end[a];
      real span = (real)(end[a] - origin[a]);
      g->num_cells[a] = (int)(span / cell_size) + 1;
    }
    g->num_cells_total *= g->num_cells[a];
  }
}

/* set_global_shapefunction: nsn = window^DIM, window 2 (linear) or 4
 * (src/common/global_settings.cpp:232-268).  Quadratic (absent from the
 * reference) uses the same 4-wide window as cubic; its fourth slot per axis
 * always carries a zero weight. */
int or_num_surround_nodes(int dim, int sf) {
  int w = (sf == OR_LINEAR) ? 2 : 4;
  int n = 1;
  for (int a = 0; a < dim; a++) n *= w;
  return n;
}

/* Window offsets of slot `sid`, in the reference's slot order
 * (src/common/global_settings.cpp:108-150): 2D is x-fastest then y; 3D is
 * z-fastest, then x, then y.  Linear offsets are {0,1}, the 4-wide ones
 * {-1,0,1,2}.  The P2G window is the negation (p2g = -g2p). */
static void window_offset(int dim, int sf, int sid, int w[3]) {
  int width = (sf == OR_LINEAR) ? 2 : 4;
  int lo = (sf == OR_LINEAR) ? 0 : -1;
  w[0] = w[1] = w[2] = 0;
  if (dim == 1) {
    w[0] = lo + sid;
  } else if (dim == 2) {
    w[0] = lo + sid % width;
    w[1] = lo + sid / width;
  } else {
    w[2] = lo + sid % width;
    w[0] = lo + (sid / width) % width;
    w[1] = lo + sid / (width * width);
  }
}

static inline int flat3(const or_grid *g, const int b[3]) {
  /* NODE_MEM_INDEX: include/pyroclastmpm/common/types_common.h:98-99,110 */
  return b[0] + b[1] * g->num_cells[0] + b[2] * g->num_cells[0] * g->num_cells[1];
}

/* NodesContainer::calculate_bin_ids (src/nodes/nodes.cpp:89-129): x-fastest. */
void or_node_ids(const or_grid *g, int *node_ids) {
  for (int z = 0; z < g->num_cells[2]; z++)
    for (int y = 0; y < g->num_cells[1]; y++)
      for (int x = 0; x < g->num_cells[0]; x++) {
        int idx = x + y * g->num_cells[0] + z * g->num_cells[0] * g->num_cells[1];
        node_ids[3 * idx + 0] = x;
        node_ids[3 * idx + 1] = y;
        node_ids[3 * idx + 2] = z;
      }
}

/* NodesContainer::calculate_bin_types (src/nodes/nodes.cpp:135-173), cubic
 * only: 1 at either end, 2 at index 1, 3 otherwise.  The reference's "left of
 * boundary" test can never be true, so type 4 is never assigned; that is kept. */
void or_node_types(const or_grid *g, int sf, const int *node_ids, int *node_types) {
  for (int i = 0; i < g->num_cells_total; i++)
    for (int a = 0; a < 3; a++) node_types[3 * i + a] = 0;
  if (sf != OR_CUBIC) return;
  for (int i = 0; i < g->num_cells_total; i++)
    for (int a = 0; a < g->dim; a++) {
      int id = node_ids[3 * i + a];
      int t;
      if (id == 0 || id == g->num_cells[a] - 1) t = 1;
      else if (id == 1) t = 2;
      else t = 3;
      node_types[3 * i + a] = t;
    }
}

/* ------------------------------------------------------------------------ */
/* Spatial partition                                                        */
/* ------------------------------------------------------------------------ */

/* calculate_hashes (src/spatialpartition/spatialpartition_inline.h:49-62):
 * bin = (int)((x - origin) * inv_h) (truncation), hash = NODE_MEM_INDEX as
 * unsigned; then SpatialPartition::calculate_hash copies the hashes into the
 * to-be-sorted array (src/spatialpartition/spatialpartition.cpp:90-110). */
void or_calculate_hash(const or_grid *g, int n, const REAL *x, int *bins,
                       unsigned int *hash_unsorted, unsigned int *hash_sorted) {
  int d = g->dim;
  for (int i = 0; i < n; i++) {
    int b[3] = {0, 0, 0};
    for (int a = 0; a < d; a++) {
      real rel = (real)(x[i * d + a] - g->origin[a]);
      rel = (real)(rel * g->inv_cell_size);
      b[a] = (int)rel;
    }
    for (int a = 0; a < d; a++) bins[i * d + a] = b[a];
    unsigned int h = (unsigned int)flat3(g, b);
    hash_unsorted[i] = h;
    hash_sorted[i] = h;
  }
}

/* SpatialPartition::sort_hashes (src/spatialpartition/spatialpartition.cpp:113-117):
 * stable sort of (hash, index) with index = 0..n-1 (reset, :80).  Stable LSD
 * radix sort on the 32-bit key. */
void or_sort_hashes(int n, unsigned int *hash_sorted, int *sorted_index) {
  unsigned int *kbuf = (unsigned int *)malloc(sizeof(unsigned int) * (size_t)(n > 0 ? n : 1));
  int *vbuf = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++) sorted_index[i] = i;
  unsigned int *ks = hash_sorted, *kd = kbuf;
  int *vs = sorted_index, *vd = vbuf;
  for (int shift = 0; shift < 32; shift += 8) {
    size_t count[257];
    memset(count, 0, sizeof(count));
    for (int i = 0; i < n; i++) count[((ks[i] >> shift) & 255u) + 1]++;
    for (int k = 0; k < 256; k++) count[k + 1] += count[k];
    for (int i = 0; i < n; i++) {
      size_t pos = count[(ks[i] >> shift) & 255u]++;
      kd[pos] = ks[i];
      vd[pos] = vs[i];
    }
    unsigned int *tk = ks; ks = kd; kd = tk;
    int *tv = vs; vs = vd; vd = tv;
  }
  /* four passes: the result is back in the caller's arrays */
  free(kbuf);
  free(vbuf);
}

/* bin_particles_kernel (src/spatialpartition/spatialpartition_inline.h:85-115):
 * start/end from adjacent-hash changes; empty cells keep 0/0 (reset fills 0).
 * Hashes >= num_cells_total (particles outside the grid) would write out of
 * bounds in the reference; they are skipped here. */
void or_bin_particles(const or_grid *g, int n, const unsigned int *hs, int *cell_start, int *cell_end) {
  unsigned int nt = (unsigned int)g->num_cells_total;
  for (int i = 0; i < g->num_cells_total; i++) cell_start[i] = cell_end[i] = 0;
  for (int t = 0; t < n; t++) {
    unsigned int h = hs[t];
    if (t < n - 1) {
      unsigned int nh = hs[t + 1];
      if (t == 0 && h < nt) cell_start[h] = t;
      if (h != nh) {
        if (h < nt) cell_end[h] = t + 1;
        if (nh < nt) cell_start[nh] = t + 1;
      }
    }
    if (t == n - 1 && h < nt) cell_end[h] = t + 1;
  }
}

/* ParticlesContainer::partition (src/particles/particles.cpp:332-339). */
void or_partition(or_sim *s) {
  or_calculate_hash(&s->grid, s->num_particles, s->positions, s->bins, s->hash_unsorted, s->hash_sorted);
  or_sort_hashes(s->num_particles, s->hash_sorted, s->sorted_index);
  or_bin_particles(&s->grid, s->num_particles, s->hash_sorted, s->cell_start, s->cell_end);
}

/* ------------------------------------------------------------------------ */
/* Shape functions                                                          */
/* ------------------------------------------------------------------------ */

/* linear / derivative_linear (src/shapefunction/linear.cuh:28-52): the weight
 * is evaluated in double and rounded; the derivative is 0 at r == 0 exactly. */
static real sf_linear(real r) {
  double ar = fabs((double)r);
  if (ar >= 1.0) return (real)0.0;
  return (real)(1.0 - ar);
}
static real sf_dlinear(real r, real inv_h) {
  if (r > (real)1.0 || r < (real)-1.0 || r == (real)0.0) return (real)0.0;
  if (r > (real)0.0) return -inv_h;
  return inv_h;
}

/* Boundary-modified cubic B-spline (src/shapefunction/cubic.cuh:28-197),
 * restated as Horner coefficient tables per node type and unit interval
 * [-2,-1), [-1,0), [0,1), [1,2).  Weight: ((c3 r + c2) r + c1) r + c0;
 * derivative: inv_h * ((d2 r + d1) r + d0).  Type 3 is the uniform cubic
 * B-spline; types 1 (grid end) and 2 (next to the end) are the boundary
 * variants; type 4 exists in the reference but is never assigned.  Evaluated
 * in double, then rounded, as in the reference. */
static const double CUBIC_W[5][4][4] = {
    /* type 0: zero everywhere (node types are only set for cubic grids) */
    {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}},
    /* type 1 */
    {{1.0 / 6.0, 1.0, 2.0, 4.0 / 3.0}, {-1.0 / 6.0, 0.0, 1.0, 1.0},
     {1.0 / 6.0, 0.0, -1.0, 1.0}, {-1.0 / 6.0, 1.0, -2.0, 4.0 / 3.0}},
    /* type 2 */
    {{0, 0, 0, 0}, {-1.0 / 3.0, -1.0, 0.0, 2.0 / 3.0},
     {0.5, -1.0, 0.0, 2.0 / 3.0}, {-1.0 / 6.0, 1.0, -2.0, 4.0 / 3.0}},
    /* type 3 */
    {{1.0 / 6.0, 1.0, 2.0, 4.0 / 3.0}, {-0.5, -1.0, 0.0, 2.0 / 3.0},
     {0.5, -1.0, 0.0, 2.0 / 3.0}, {-1.0 / 6.0, 1.0, -2.0, 4.0 / 3.0}},
    /* type 4 */
    {{1.0 / 6.0, 1.0, 2.0, 4.0 / 3.0}, {-0.5, -1.0, 0.0, 2.0 / 3.0},
     {1.0 / 3.0, -1.0, 0.0, 2.0 / 3.0}, {0, 0, 0, 0}},
};
static const double CUBIC_D[5][4][3] = {
    {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}},
    {{0.5, 2.0, 2.0}, {-0.5, 0.0, 1.0}, {0.5, 0.0, -1.0}, {-0.5, 2.0, -2.0}},
    {{0, 0, 0}, {-1.0, -2.0, 0.0}, {1.5, -2.0, 0.0}, {-0.5, 2.0, -2.0}},
    {{0.5, 2.0, 2.0}, {-1.5, -2.0, 0.0}, {1.5, -2.0, 0.0}, {-0.5, 2.0, -2.0}},
    {{0.5, 2.0, 2.0}, {-1.5, -2.0, 0.0}, {1.0, -2.0, 0.0}, {0, 0, 0}},
};
static int cubic_interval(real r) {
  if (r >= (real)-2.0 && r < (real)-1.0) return 0;
  if (r >= (real)-1.0 && r < (real)0.0) return 1;
  if (r >= (real)0.0 && r < (real)1.0) return 2;
  if (r >= (real)1.0 && r < (real)2.0) return 3;
  return -1;
}
static real sf_cubic(real r, int type) {
  int k = cubic_interval(r);
  if (k < 0 || type < 0 || type > 4) return (real)0.0;
  const double *c = CUBIC_W[type][k];
  double rd = (double)r;
  return (real)(((c[0] * rd + c[1]) * rd + c[2]) * rd + c[3]);
}
static real sf_dcubic(real r, real inv_h, int type) {
  int k = cubic_interval(r);
  if (k < 0 || type < 0 || type > 4) return (real)0.0;
  const double *c = CUBIC_D[type][k];
  double rd = (double)r;
  return (real)((double)inv_h * ((c[0] * rd + c[1]) * rd + c[2]));
}

/* Quadratic B-spline (no reference implementation: quadratic.cuh is a TODO).
 * Uniform C1 quadratic B-spline of support 3h:
 *   |r| < 1/2:        3/4 - r^2            d = -2 r
 *   1/2 <= |r| < 3/2: (3/2 - |r|)^2 / 2    d = -sign(r) (3/2 - |r|)
 * Boundary handling: a stencil node that falls outside the grid on an axis is
 * folded onto the nearest grid node of that axis, so the weights of any
 * particle inside the grid sum to one. */
static real sf_quadratic(real r) {
  real ar = (real)fabs((double)r);
  if (ar < (real)0.5) return (real)((real)0.75 - r * r);
  if (ar < (real)1.5) {
    real t = (real)((real)1.5 - ar);
    return (real)((real)0.5 * t * t);
  }
  return (real)0.0;
}
static real sf_dquadratic(real r, real inv_h) {
  real ar = (real)fabs((double)r);
  if (ar < (real)0.5) return (real)(inv_h * ((real)-2.0 * r));
  if (ar < (real)1.5) {
    real t = (real)((real)1.5 - ar);
    return (real)(inv_h * (r > (real)0.0 ? -t : t));
  }
  return (real)0.0;
}

/* Target node of a particle slot.  Linear/cubic follow the reference exactly:
 * node = flat(bin + w) as an unsigned index, valid iff < num_cells_total (so a
 * slot that leaves the grid on one axis may alias into a neighbouring row, as
 * in src/shapefunction/shapefunction.cpp:84-91 and
 * src/solver/usl/usl_inline.h:114-126).  Quadratic clamps each axis (fold). */
static int slot_target(const or_sim *s, const int b[3], const int w[3], int sel[3]) {
  const or_grid *g = &s->grid;
  int t[3];
  for (int a = 0; a < 3; a++) {
    sel[a] = b[a] + w[a];
    t[a] = sel[a];
    if (s->shape_function == OR_QUADRATIC && a < g->dim) {
      if (t[a] < 0) t[a] = 0;
      if (t[a] > g->num_cells[a] - 1) t[a] = g->num_cells[a] - 1;
    }
  }
  unsigned int h = (unsigned int)flat3(g, t);
  if (h >= (unsigned int)g->num_cells_total) return -1;
  return (int)h;
}

/* shape_function_kernel (src/shapefunction/shapefunction.cpp:70-142):
 * psi/dpsi per (particle, slot); relative coordinate
 * (x - origin)*inv_h - selected_bin; products N0*N1[*N2]. */
void or_shape_functions(or_sim *s) {
  const or_grid *g = &s->grid;
  int d = g->dim, nsn = s->nsn;
  for (int i = 0; i < s->num_particles; i++) {
    int b[3] = {0, 0, 0};
    for (int a = 0; a < d; a++) b[a] = s->bins[i * d + a];
    for (int sid = 0; sid < nsn; sid++) {
      int w[3], sel[3];
      window_offset(d, s->shape_function, sid, w);
      int node = slot_target(s, b, w, sel);
      if (node < 0) continue;
      real N[3] = {1, 1, 1}, dN[3] = {0, 0, 0};
      for (int a = 0; a < d; a++) {
        real rel = (real)(s->positions[i * d + a] - g->origin[a]);
        rel = (real)(rel * g->inv_cell_size);
        rel = (real)(rel - (real)sel[a]);
        if (s->shape_function == OR_LINEAR) {
          N[a] = sf_linear(rel);
          dN[a] = sf_dlinear(rel, g->inv_cell_size);
        } else if (s->shape_function == OR_CUBIC) {
          int type = s->node_types[3 * node + a];
          N[a] = sf_cubic(rel, type);
          dN[a] = sf_dcubic(rel, g->inv_cell_size, type);
        } else {
          N[a] = sf_quadratic(rel);
          dN[a] = sf_dquadratic(rel, g->inv_cell_size);
        }
      }
      real psi;
      real dpsi[3] = {0, 0, 0};
      if (d == 1) {
        psi = N[0];
        dpsi[0] = dN[0];
      } else if (d == 2) {
        psi = (real)(N[0] * N[1]);
        dpsi[0] = (real)(dN[0] * N[1]);
        dpsi[1] = (real)(dN[1] * N[0]);
      } else {
        psi = (real)((real)(N[0] * N[1]) * N[2]);
        dpsi[0] = (real)((real)(dN[0] * N[1]) * N[2]);
        dpsi[1] = (real)((real)(dN[1] * N[0]) * N[2]);
        dpsi[2] = (real)((real)(dN[2] * N[0]) * N[1]);
      }
      s->psi[(size_t)i * nsn + sid] = psi;
      for (int a = 0; a < d; a++) s->dpsi[((size_t)i * nsn + sid) * d + a] = dpsi[a];
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Particle set-up                                                          */
/* ------------------------------------------------------------------------ */

/* calculate_initial_volumes (src/particles/particles.cpp:345-365):
 * V = (REAL)pow(h, DIM) / ppc for particles whose volume is not set (> 0). */
void or_initial_volumes(or_sim *s) {
  int d = s->grid.dim;
  for (int i = 0; i < s->num_particles; i++) {
    if (s->volumes[i] > (real)0.0) continue;
    real v = (real)pow((double)s->grid.cell_size, (double)d);
    v = (real)(v / (real)s->particles_per_cell);
    s->volumes[i] = v;
  }
  memcpy(s->volumes_original, s->volumes, sizeof(real) * (size_t)s->num_particles);
}

/* calculate_initial_masses (src/particles/particles.cpp:372-393). */
void or_initial_masses(or_sim *s, int mat_id, REAL density) {
  for (int i = 0; i < s->num_particles; i++) {
    if ((int)s->colors[i] != mat_id || s->masses[i] > (real)0.0) continue;
    s->masses[i] = (real)(density * s->volumes[i]);
  }
}

/* USL::reset (src/solver/usl/usl.cpp:61-66) with NodesContainer::reset
 * (src/nodes/nodes.cpp:183-188), ParticlesContainer::reset
 * (src/particles/particles.cpp:162-175) and SpatialPartition::reset
 * (src/spatialpartition/spatialpartition.cpp:77-86). */
void or_reset(or_sim *s) {
  int d = s->grid.dim;
  size_t nn = (size_t)s->grid.num_cells_total, np = (size_t)s->num_particles;
  memset(s->node_masses, 0, sizeof(real) * nn);
  memset(s->node_moments, 0, sizeof(real) * nn * d);
  memset(s->node_moments_nt, 0, sizeof(real) * nn * d);
  memset(s->psi, 0, sizeof(real) * np * s->nsn);
  memset(s->dpsi, 0, sizeof(real) * np * s->nsn * d);
  memset(s->velocity_gradient, 0, sizeof(real) * np * d * d);
  memset(s->forces_external, 0, sizeof(real) * np * d);
  for (size_t i = 0; i < np; i++) s->sorted_index[i] = (int)i;
  memset(s->cell_start, 0, sizeof(int) * nn);
  memset(s->cell_end, 0, sizeof(int) * nn);
  memset(s->bins, 0, sizeof(int) * np * d);
}

/* ------------------------------------------------------------------------ */
/* Boundary conditions                                                      */
/* ------------------------------------------------------------------------ */

/* apply_planardomain (src/boundaryconditions/planardomain_inline.h:56-138):
 * radius = 0.5 V^(1/D); overlap with each face -> f_ext += (m/dt^2) *
 * overlap * (n - mu (v - (n.v) n)).  Friction is stored in radians and used
 * as the coefficient directly, as in the reference. */
static void planardomain(or_sim *s, const or_bc *bc) {
  const or_grid *g = &s->grid;
  int d = g->dim;
  real inv_dim = (real)((real)1.0 / (real)d);
  for (int i = 0; i < s->num_particles; i++) {
    const real *x = s->positions + (size_t)i * d;
    const real *v = s->velocities + (size_t)i * d;
#ifdef OR_DOUBLE
    double pv = pow((double)s->volumes[i], (double)inv_dim);
#else
    double pv = (double)powf((float)s->volumes[i], (float)inv_dim);
#endif
    real radius = (real)((real)0.5 * (real)pv);
    real mass = s->masses[i];
    real scale = (real)((double)mass / pow((double)s->dt, 2.0));
    for (int face = 0; face < 2; face++) {
      for (int a = 0; a < d; a++) {
        real overlap = face == 0 ? (real)(radius - (real)(x[a] - g->origin[a]))
                                 : (real)(radius - (real)(g->end[a] - x[a]));
        if (!(overlap > (real)0.0)) continue;
        real nrm[3] = {0, 0, 0};
        nrm[a] = face == 0 ? (real)1.0 : (real)-1.0;
        real mu = bc->r[3 * face + a];
        real ndotv = 0;
        for (int b = 0; b < d; b++) ndotv = (real)(ndotv + nrm[b] * v[b]);
        for (int b = 0; b < d; b++) {
          real tang = (real)(v[b] - (real)(ndotv * nrm[b]));
          real fric = (real)(nrm[b] - (real)(mu * tang));
          s->forces_external[(size_t)i * d + b] =
              (real)(s->forces_external[(size_t)i * d + b] + (real)((real)(scale * overlap) * fric));
        }
      }
    }
  }
}

/* USL::solve step 5: BoundaryCondition::apply_on_particles over the list. */
void or_apply_on_particles(or_sim *s) {
  for (int k = 0; k < s->num_bcs; k++)
    if (s->bcs[k].type == OR_BC_PLANARDOMAIN) planardomain(s, &s->bcs[k]);
}

/* Gravity::apply_on_nodes_moments (src/boundaryconditions/gravity.cpp:65-88)
 * and apply_gravity (src/boundaryconditions/gravity_inline.h:46-63).  The ramp
 * overwrites the stored gravity while step < ramp_step, so after the ramp the
 * last ramp value stays in force (reproduced). */
static void gravity(or_sim *s, or_bc *bc) {
  int d = s->grid.dim;
  int is_ramp = bc->i[0], ramp_step = bc->i[1];
  real ramp_factor = (real)((real)s->global_step / (real)ramp_step);
  if (is_ramp && s->global_step < ramp_step)
    for (int a = 0; a < d; a++) bc->r[a] = (real)(bc->r[3 + a] * ramp_factor);
  for (int n = 0; n < s->grid.num_cells_total; n++) {
    real m = s->node_masses[n];
    if (m <= (real)0.000000001) continue;
    for (int a = 0; a < d; a++) {
      real inc = (real)((real)(bc->r[a] * m) * s->dt);
      s->node_moments_nt[(size_t)n * d + a] = (real)(s->node_moments_nt[(size_t)n * d + a] + inc);
    }
  }
}

/* apply_nodedomain (src/boundaryconditions/nodedomain_inline.h:40-87). */
static void nodedomain(or_sim *s, const or_bc *bc) {
  int d = s->grid.dim;
  for (int n = 0; n < s->grid.num_cells_total; n++) {
    if (s->node_masses[n] <= (real)0.00001) continue;
    real *p = s->node_moments + (size_t)n * d;
    real *q = s->node_moments_nt + (size_t)n * d;
    for (int a = 0; a < d; a++) {
      int id = s->node_ids[3 * n + a];
      if (id < 1) {
        if (bc->i[a] == 0) {
          for (int b = 0; b < d; b++) p[b] = q[b] = (real)0.0;
        } else if (bc->i[a] == 1) {
          p[a] = (real)fmax(0.0, (double)p[a]);
          q[a] = (real)fmax(0.0, (double)q[a]);
        }
      } else if (id >= s->grid.num_cells[a] - 1) {
        if (bc->i[3 + a] == 0) {
          for (int b = 0; b < d; b++) p[b] = q[b] = (real)0.0;
        } else if (bc->i[3 + a] == 1) {
          p[a] = (real)fmin(0.0, (double)p[a]);
          q[a] = (real)fmin(0.0, (double)q[a]);
        }
      }
    }
  }
}

/* BodyForce::apply_on_nodes_moments (src/boundaryconditions/bodyforce.cpp:72-100)
 * and apply_bodymoments (src/boundaryconditions/bodyforce_inline.h:41-59):
 * "fixed" sets moments_nt, the other modes add to moments. */
static void bodyforce(or_sim *s, const or_bc *bc) {
  int d = s->grid.dim;
  if (!bc->i[1]) return;
  int fixed = bc->i[0] == 2;
  for (int n = 0; n < s->grid.num_cells_total; n++) {
    if (!bc->mask[n]) continue;
    for (int a = 0; a < d; a++) {
      if (fixed) s->node_moments_nt[(size_t)n * d + a] = bc->values[(size_t)n * d + a];
      else s->node_moments[(size_t)n * d + a] = (real)(s->node_moments[(size_t)n * d + a] + bc->values[(size_t)n * d + a]);
    }
  }
}

#ifdef OR_DOUBLE
#define RCOS cos
#define RSIN sin
#define RSQRT sqrt
#else
#define RCOS cosf
#define RSIN sinf
#define RSQRT sqrtf
#endif

/* 3x3 product, coefficients summed ((a0 b0 + a1 b1) + a2 b2). */
static void mat3_mul(const real *A, const real *B, real *C) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      real acc = (real)(A[3 * i] * B[j]);
      acc = (real)(acc + (real)(A[3 * i + 1] * B[3 + j]));
      C[3 * i + j] = (real)(acc + (real)(A[3 * i + 2] * B[6 + j]));
    }
}

/* RigidBodyLevelSet::update_animation (src/boundaryconditions/rigidbodylevelset.cpp:
 * 127-206).  LOOP_ROTATE: euler += rate dt; delta = previous - new.  2D:
 * R = [[cos d0, -sin d0], [sin d0, cos d0]].  3D as the reference assigns it:
 * Rx keeps (0,1) = -sin d0 and (1,0) = sin d0 of the 2D assignment under its
 * 3D entries, Rz is never assigned (zero), so R = Rz Ry Rx = 0; i[1] = 1 gives
 * the proper Rz(d2) Ry(d1) Rx(d0).  STATIC leaves the reference's matrix
 * unset; the identity is taken. */
static void rigid_rotation(or_sim *s, or_bc *bc, real *R) {
  int d = s->grid.dim;
  real R3[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (bc->i[0] == 1) {
    real dl[3];
    for (int a = 0; a < 3; a++) {
      real prev = bc->r[6 + a];
      bc->r[6 + a] = (real)(bc->r[6 + a] + (real)(bc->r[a] * s->dt));
      dl[a] = (real)(prev - bc->r[6 + a]);
    }
    real c0 = (real)RCOS(dl[0]), s0 = (real)RSIN(dl[0]);
    real c1 = (real)RCOS(dl[1]), s1 = (real)RSIN(dl[1]);
    real c2 = (real)RCOS(dl[2]), s2 = (real)RSIN(dl[2]);
    if (d == 2) {
      real M[9] = {c0, -s0, 0, s0, c0, 0, 0, 0, 1};
      memcpy(R3, M, sizeof(R3));
    } else {
      real Rx[9], Ry[9] = {c1, 0, s1, 0, 1, 0, -s1, 0, c1}, Rz[9], T[9];
      if (!bc->i[1]) {
        real X[9] = {1, -s0, 0, s0, c2, -s2, 0, s2, c2};
        memcpy(Rx, X, sizeof(X));
        memset(Rz, 0, sizeof(Rz));
      } else {
        real X[9] = {1, 0, 0, 0, c0, -s0, 0, s0, c0};
        real Z[9] = {c2, -s2, 0, s2, c2, 0, 0, 0, 1};
        memcpy(Rx, X, sizeof(X));
        memcpy(Rz, Z, sizeof(Z));
      }
      mat3_mul(Rz, Ry, T);
      mat3_mul(T, Rx, R3);
    }
  }
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++) R[a * d + b] = R3[3 * a + b];
}

/* RigidBodyLevelSet::apply_on_nodes_moments (src/boundaryconditions/
 * rigidbodylevelset.cpp:92-105): update_animation; set_velocities (CPU
 * branch, :245-275, update_rigid_velocity rigidbodylevelset_inline.h:240-299);
 * calculate_grid_normals_nn_rigid (rigidbodylevelset_inline.h:65-199) per
 * node; set_position (update_rigid_position, :329-343). */
static void rigid_nn(or_sim *s, or_bc *bc) {
  const or_grid *g = &s->grid;
  int d = g->dim;
  real R[9];
  rigid_rotation(s, bc, R);
  for (int i = 0; i < s->num_particles; i++) {
    if (!s->is_rigid[i]) continue;
    real r[3], u[3];
    for (int a = 0; a < d; a++) r[a] = (real)(s->positions[i * d + a] - bc->r[3 + a]);
    for (int a = 0; a < d; a++) {
      real acc = (real)(R[a * d] * r[0]);
      for (int b = 1; b < d; b++) acc = (real)(acc + (real)(R[a * d + b] * r[b]));
      u[a] = acc;
    }
    for (int a = 0; a < d; a++) s->velocities[i * d + a] = (real)((real)(u[a] - r[a]) / s->dt);
  }
  static const int W3[8][3] = {{0, 0, 0}, {0, 0, -1}, {-1, 0, 0}, {-1, 0, -1},
                               {0, -1, 0}, {0, -1, -1}, {-1, -1, 0}, {-1, -1, -1}};
  static const int W2[4][3] = {{0, 0, 0}, {-1, 0, 0}, {0, -1, 0}, {-1, -1, 0}};
  int nw = d == 3 ? 8 : 4;
  for (int n = 0; n < g->num_cells_total; n++) {
    real m = s->node_masses[n];
    if (m <= (real)0.000000001) continue;
    real normal[3] = {0, 0, 0};
    real min_dist = (real)999999999999999.;
    int min_id = -1;
    for (int sid = 0; sid < nw; sid++) {
      const int *w = d == 3 ? W3[sid] : W2[sid];
      int sb[3] = {0, 0, 0};
      for (int a = 0; a < d; a++) sb[a] = s->node_ids[3 * n + a] + w[a];
      unsigned int h = (unsigned int)flat3(g, sb);
      if (h >= (unsigned int)g->num_cells_total) continue;
      int cs = s->cell_start[h], ce = s->cell_end[h];
      for (int j = cs; j < ce; j++) {
        int pid = s->sorted_index[j];
        if (s->is_rigid[pid]) {
          real dist = 0;
          for (int a = 0; a < d; a++) {
            real rel = (real)((real)(s->positions[pid * d + a] - g->origin[a]) * g->inv_cell_size);
            rel = (real)(rel - (real)sb[a]);
            dist = a == 0 ? (real)(rel * rel) : (real)(dist + (real)(rel * rel));
          }
          if (dist < min_dist) {
            min_dist = dist;
            min_id = pid;
          }
        } else {
          const real *dp = s->dpsi + ((size_t)pid * s->nsn + sid) * d;
          for (int a = 0; a < d; a++) normal[a] = (real)(normal[a] + (real)(dp[a] * s->masses[pid]));
        }
      }
    }
    if (min_id < 0) continue;
    real sq = (real)(normal[0] * normal[0]);
    for (int a = 1; a < d; a++) sq = (real)(sq + (real)(normal[a] * normal[a]));
    if (sq > (real)0.0) {
      real len = (real)RSQRT(sq);
      for (int a = 0; a < d; a++) normal[a] = (real)(normal[a] / len);
    }
    real *p = s->node_moments + (size_t)n * d;
    real *q = s->node_moments_nt + (size_t)n * d;
    real v[3], vt[3], cv[3], cvt[3], rel = 0, rel_nt = 0;
    for (int a = 0; a < d; a++) {
      real vb = s->velocities[min_id * d + a];
      v[a] = (real)(p[a] / m);
      vt[a] = (real)(q[a] / m);
      cv[a] = (real)(v[a] - vb);
      cvt[a] = (real)(vt[a] - vb);
      rel = a == 0 ? (real)(cv[a] * normal[a]) : (real)(rel + (real)(cv[a] * normal[a]));
      rel_nt = a == 0 ? (real)(cvt[a] * normal[a]) : (real)(rel_nt + (real)(cvt[a] * normal[a]));
    }
    if (rel >= (real)0.0)
      for (int a = 0; a < d; a++) p[a] = (real)((real)(v[a] - cv[a]) * m);
    if (rel_nt >= (real)0.0)
      for (int a = 0; a < d; a++) q[a] = (real)((real)(vt[a] - cvt[a]) * m);
  }
  for (int i = 0; i < s->num_particles; i++) {
    if (!s->is_rigid[i]) continue;
    for (int a = 0; a < d; a++)
      s->positions[i * d + a] = (real)(s->positions[i * d + a] + (real)(s->velocities[i * d + a] * s->dt));
  }
}

/* Analytic rigid body (no reference counterpart).  Pose at time step*dt:
 * centre c0 + v t, angle angle0 + omega t about the axis.  Cross-section
 * plane (P, Q) = (axis+1, axis+2) cyclic in 3D, (x, y) in 2D.  Shell: the
 * half q <= 0 (local) of the annulus |rho - R| <= t/2, ends rounded with
 * radius t/2, extruded to length L along the axis (3D).  Returns the signed
 * distance of x and the outward unit normal. */
static real sdf_eval(int d, const or_bc *bc, const real *c, real cs, real sn, const real *x, real *nrm) {
  int A = d == 3 ? bc->i[1] : 2;
  int P = d == 3 ? (A + 1) % 3 : 0, Q = d == 3 ? (A + 2) % 3 : 1;
  real dd[3] = {0, 0, 0};
  for (int a = 0; a < d; a++) dd[a] = (real)(x[a] - c[a]);
  nrm[0] = nrm[1] = nrm[2] = 0;
  if (bc->i[0] == 0) {
    real r2 = 0;
    for (int a = 0; a < d; a++) r2 = (real)(r2 + (real)(dd[a] * dd[a]));
    real r = (real)RSQRT(r2);
    if (r > 0) {
      for (int a = 0; a < d; a++) nrm[a] = (real)(dd[a] / r);
    } else {
      nrm[Q] = 1;
    }
    return (real)(r - bc->r[8]);
  }
  real lp = (real)((real)(cs * dd[P]) + (real)(sn * dd[Q]));
  real lq = (real)((real)(cs * dd[Q]) - (real)(sn * dd[P]));
  real R = bc->r[8], ht = (real)((real)0.5 * bc->r[9]);
  real phi2, gp = 0, gq = 1;
  if (lq <= 0) {
    real rho = (real)RSQRT((real)((real)(lp * lp) + (real)(lq * lq)));
    phi2 = (real)((real)fabs((double)(rho - R)) - ht);
    if (rho > 0) {
      real sg = rho >= R ? (real)1 : (real)-1;
      gp = (real)((real)(sg * lp) / rho);
      gq = (real)((real)(sg * lq) / rho);
    }
  } else {
    real wp = (real)(lp - (lp >= 0 ? R : -R)), wq = lq;
    real w = (real)RSQRT((real)((real)(wp * wp) + (real)(wq * wq)));
    phi2 = (real)(w - ht);
    if (w > 0) {
      gp = (real)(wp / w);
      gq = (real)(wq / w);
    }
  }
  real phi = phi2, ga = 0;
  if (d == 3) {
    real la = dd[A];
    real hA = (real)((real)fabs((double)la) - (real)((real)0.5 * bc->r[10]));
    real sa = la >= 0 ? (real)1 : (real)-1;
    if (phi2 > 0 && hA > 0) {
      phi = (real)RSQRT((real)((real)(phi2 * phi2) + (real)(hA * hA)));
      gp = (real)((real)(phi2 * gp) / phi);
      gq = (real)((real)(phi2 * gq) / phi);
      ga = (real)((real)(hA * sa) / phi);
    } else if (hA > phi2) {
      phi = hA;
      gp = gq = 0;
      ga = sa;
    }
  }
  nrm[P] = (real)((real)(cs * gp) - (real)(sn * gq));
  nrm[Q] = (real)((real)(sn * gp) + (real)(cs * gq));
  if (d == 3) nrm[A] = ga;
  return phi;
}

/* Coulomb contact of the forward moments of every node with m > 1e-9 whose
 * signed distance is below the contact distance: relative velocity
 * v_rel = p_nt/m - v_body(x); if its normal part vn < 0, the normal part is
 * removed and the tangential part vt scaled by max(0, 1 + mu vn / |vt|). */
static void rigid_sdf(or_sim *s, const or_bc *bc) {
  const or_grid *g = &s->grid;
  int d = g->dim;
  int A = d == 3 ? bc->i[1] : 2;
  int P = d == 3 ? (A + 1) % 3 : 0, Q = d == 3 ? (A + 2) % 3 : 1;
  double t = (double)s->global_step * (double)s->dt;
  real c[3] = {0, 0, 0};
  for (int a = 0; a < d; a++) c[a] = (real)((double)bc->r[a] + (double)bc->r[3 + a] * t);
  double ang = (double)bc->r[12] + (double)bc->r[6] * t;
  real cs = (real)cos(ang), sn = (real)sin(ang);
  real mu = bc->r[7], omega = bc->r[6];
  for (int n = 0; n < g->num_cells_total; n++) {
    real m = s->node_masses[n];
    if (m <= (real)0.000000001) continue;
    real x[3] = {0, 0, 0}, nrm[3];
    for (int a = 0; a < d; a++)
      x[a] = (real)(g->origin[a] + (real)((real)s->node_ids[3 * n + a] * g->cell_size));
    real phi = sdf_eval(d, bc, c, cs, sn, x, nrm);
    if (!(phi < bc->r[11])) continue;
    real vb[3] = {bc->r[3], bc->r[4], bc->r[5]};
    vb[P] = (real)(vb[P] - (real)(omega * (real)(x[Q] - c[Q])));
    vb[Q] = (real)(vb[Q] + (real)(omega * (real)(x[P] - c[P])));
    real *q = s->node_moments_nt + (size_t)n * d;
    real vr[3] = {0, 0, 0}, vn = 0;
    for (int a = 0; a < d; a++) {
      vr[a] = (real)((real)(q[a] / m) - vb[a]);
      vn = (real)(vn + (real)(vr[a] * nrm[a]));
    }
    if (!(vn < 0)) continue;
    real vt2 = 0;
    for (int a = 0; a < d; a++) {
      vr[a] = (real)(vr[a] - (real)(vn * nrm[a]));
      vt2 = (real)(vt2 + (real)(vr[a] * vr[a]));
    }
    real vt = (real)RSQRT(vt2);
    real scale = vt <= (real)(-mu * vn) ? (real)0 : (real)((real)1 + (real)((real)(mu * vn) / vt));
    for (int a = 0; a < d; a++) q[a] = (real)((real)(vb[a] + (real)(vr[a] * scale)) * m);
  }
}

/* USL::solve step 8 (src/solver/usl/usl.cpp:97-103): list order. */
void or_apply_on_nodes_moments(or_sim *s) {
  for (int k = 0; k < s->num_bcs; k++) {
    or_bc *bc = &s->bcs[k];
    if (bc->type == OR_BC_GRAVITY) gravity(s, bc);
    else if (bc->type == OR_BC_NODEDOMAIN) nodedomain(s, bc);
    else if (bc->type == OR_BC_BODYFORCE) bodyforce(s, bc);
    else if (bc->type == OR_BC_RIGIDBODY_LEVELSET) rigid_nn(s, bc);
    else if (bc->type == OR_BC_RIGID_SDF) rigid_sdf(s, bc);
  }
}

/* ------------------------------------------------------------------------ */
/* P2G / G2P                                                                */
/* ------------------------------------------------------------------------ */

/* usl_p2g_kernel (src/solver/usl/usl_inline.h:82-180).  The reference is a
 * node-centric gather: for each node, for slot sid in order, for the particles
 * of cell (node + p2g_window[sid]) in sorted order.  The same per-node
 * summation order is produced here by a scatter with sid outermost and the
 * sorted particle order inside; the target node is flat(bin) + flat(window)
 * with the reference's single unsigned range check.  Per pair:
 *   m += psi m_p;  p += (psi m_p) v_p;  f += psi f_ext - V_p (sigma_p [dpsi;0]) */
void or_p2g(or_sim *s) {
  const or_grid *g = &s->grid;
  int d = g->dim, nsn = s->nsn;
  size_t nn = (size_t)g->num_cells_total;
  real *mass = (real *)calloc(nn, sizeof(real));
  real *mom = (real *)calloc(nn * d, sizeof(real));
  real *force = (real *)calloc(nn * d, sizeof(real));
  for (int sid = 0; sid < nsn; sid++) {
    int w[3];
    window_offset(d, s->shape_function, sid, w);
    for (int k = 0; k < s->num_particles; k++) {
      int j = s->sorted_index[k];
      if (s->hash_sorted[k] >= (unsigned int)g->num_cells_total) continue;
      int b[3] = {0, 0, 0}, sel[3];
      for (int a = 0; a < d; a++) b[a] = s->bins[j * d + a];
      if (s->shape_function == OR_QUADRATIC) {
        /* quadratic only: a particle binned outside the grid on any axis
         * takes no part in P2G (no folding of whole particles) */
        int out = 0;
        for (int a = 0; a < d; a++)
          if (b[a] < 0 || b[a] >= g->num_cells[a]) out = 1;
        if (out) continue;
      }
      int node = slot_target(s, b, w, sel);
      if (node < 0) continue;
      real psi = s->psi[(size_t)j * nsn + sid];
      const real *dpsi = s->dpsi + ((size_t)j * nsn + sid) * d;
      real sm = (real)(psi * s->masses[j]);
      mass[node] = (real)(mass[node] + sm);
      for (int a = 0; a < d; a++)
        mom[node * d + a] = (real)(mom[node * d + a] + (real)(sm * s->velocities[(size_t)j * d + a]));
      for (int a = 0; a < d; a++)
        force[node * d + a] = (real)(force[node * d + a] + (real)(psi * s->forces_external[(size_t)j * d + a]));
      real mv = (real)(-1.0 * (double)s->volumes[j]);
      const real *sig = s->stresses + (size_t)j * 9;
      real dp3[3] = {0, 0, 0};
      for (int a = 0; a < d; a++) dp3[a] = dpsi[a];
      for (int a = 0; a < d; a++) {
        real acc = (real)((real)(mv * sig[3 * a + 0]) * dp3[0]);
        acc = (real)(acc + (real)((real)(mv * sig[3 * a + 1]) * dp3[1]));
        acc = (real)(acc + (real)((real)(mv * sig[3 * a + 2]) * dp3[2]));
        force[node * d + a] = (real)(force[node * d + a] + acc);
      }
    }
  }
  for (size_t n = 0; n < nn; n++) {
    if (mass[n] <= s->small_mass_cutoff) continue;
    s->node_masses[n] = mass[n];
    for (int a = 0; a < d; a++) {
      s->node_moments[n * d + a] = mom[n * d + a];
      s->node_moments_nt[n * d + a] = (real)(mom[n * d + a] + (real)(force[n * d + a] * s->dt));
    }
  }
  free(mass);
  free(mom);
  free(force);
}

/* Determinant: 2x2 as m00 m11 - m10 m01; 3x3 by cofactors of the first row. */
static real det(int d, const real *A) {
  if (d == 1) return A[0];
  if (d == 2) return (real)((real)(A[0] * A[3]) - (real)(A[2] * A[1]));
  real c0 = (real)((real)(A[4] * A[8]) - (real)(A[5] * A[7]));
  real c1 = (real)((real)(A[3] * A[8]) - (real)(A[5] * A[6]));
  real c2 = (real)((real)(A[3] * A[7]) - (real)(A[4] * A[6]));
  return (real)((real)((real)(A[0] * c0) - (real)(A[1] * c1)) + (real)(A[2] * c2));
}

/* usl_g2p_kernel (src/solver/usl/usl_inline.h:245-332): slots leaving the grid
 * on any axis, or hitting a node with m <= cutoff, are skipped.
 *   dv += psi (v_nt - v_n);  v_pic += psi v_nt;  L += dpsi v_nt^T
 *   v <- (1 - alpha) v_pic + alpha (v + dv);  x += dt v_pic;
 *   F <- (I + L dt) F;  V = det(F) V0 */
void or_g2p(or_sim *s) {
  const or_grid *g = &s->grid;
  int d = g->dim, nsn = s->nsn;
  real one_minus_alpha = (real)(1.0 - (double)s->alpha);
  for (int i = 0; i < s->num_particles; i++) {
    int b[3] = {0, 0, 0};
    for (int a = 0; a < d; a++) b[a] = s->bins[i * d + a];
    real vinc[3] = {0, 0, 0}, dvinc[3] = {0, 0, 0}, L[9] = {0};
    for (int sid = 0; sid < nsn; sid++) {
      int w[3], sel[3];
      window_offset(d, s->shape_function, sid, w);
      int node = slot_target(s, b, w, sel);
      if (s->shape_function != OR_QUADRATIC) {
        int invalid = 0;
        for (int a = 0; a < d; a++)
          if (sel[a] < 0 || sel[a] >= g->num_cells[a]) invalid = 1;
        if (invalid) continue;
      }
      if (node < 0) continue;
      real m = s->node_masses[node];
      if (m <= s->small_mass_cutoff) continue;
      real psi = s->psi[(size_t)i * nsn + sid];
      const real *dpsi = s->dpsi + ((size_t)i * nsn + sid) * d;
      real vn[3], vnt[3];
      for (int a = 0; a < d; a++) {
        vn[a] = (real)(s->node_moments[(size_t)node * d + a] / m);
        vnt[a] = (real)(s->node_moments_nt[(size_t)node * d + a] / m);
      }
      for (int a = 0; a < d; a++) {
        dvinc[a] = (real)(dvinc[a] + (real)(psi * (real)(vnt[a] - vn[a])));
        vinc[a] = (real)(vinc[a] + (real)(psi * vnt[a]));
      }
      for (int a = 0; a < d; a++)
        for (int c = 0; c < d; c++) L[a * d + c] = (real)(L[a * d + c] + (real)(dpsi[a] * vnt[c]));
    }
    real *v = s->velocities + (size_t)i * d;
    real *x = s->positions + (size_t)i * d;
    for (int a = 0; a < d; a++) {
      v[a] = (real)((real)(one_minus_alpha * vinc[a]) + (real)(s->alpha * (real)(v[a] + dvinc[a])));
    }
    memcpy(s->velocity_gradient + (size_t)i * d * d, L, sizeof(real) * d * d);
    for (int a = 0; a < d; a++) x[a] = (real)(x[a] + (real)(s->dt * vinc[a]));
    real A[9], Fn[9];
    real *F = s->F + (size_t)i * d * d;
    for (int a = 0; a < d; a++)
      for (int c = 0; c < d; c++) A[a * d + c] = (real)((a == c ? (real)1.0 : (real)0.0) + (real)(L[a * d + c] * s->dt));
    for (int a = 0; a < d; a++)
      for (int c = 0; c < d; c++) {
        real acc = (real)(A[a * d + 0] * F[0 * d + c]);
        for (int k = 1; k < d; k++) acc = (real)(acc + (real)(A[a * d + k] * F[k * d + c]));
        Fn[a * d + c] = acc;
      }
    memcpy(F, Fn, sizeof(real) * d * d);
    s->volumes[i] = (real)(det(d, F) * s->volumes_original[i]);
  }
}

/* ------------------------------------------------------------------------ */
/* Materials                                                                */
/* ------------------------------------------------------------------------ */

/* update_linearelastic (src/materials/linearelastic_inline.h:40-107):
 * deps = 0.5 (L + L^T) dt; sigma_DIM += lame*deps*I + 2G*deps.  "lame * deps *
 * I" is a matrix product, so the reference adds (lame + 2G) deps (kept by
 * default).  corrected=1 gives the textbook lame tr(deps) I + 2G deps, with
 * sigma_zz += lame tr(deps) in 2D (plane strain). */
static void le_point(int d, const real *L, real *sig, real dt, const or_material *m) {
  real lame = m->p[2], shear = m->p[3];
  int corrected = m->p[5] != (real)0.0;
  real two_g = (real)(2.0 * (double)shear);
  real deps[9];
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++)
      deps[a * d + b] = (real)((real)((real)0.5 * (real)(L[a * d + b] + L[b * d + a])) * dt);
  real tr = 0;
  for (int a = 0; a < d; a++) tr = (real)(tr + deps[a * d + a]);
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++) {
      real inc;
      if (corrected)
        inc = (real)((a == b ? (real)(lame * tr) : (real)0.0) + (real)(two_g * deps[a * d + b]));
      else
        inc = (real)((real)(lame * deps[a * d + b]) + (real)(two_g * deps[a * d + b]));
      sig[3 * a + b] = (real)(sig[3 * a + b] + inc);
    }
  if (corrected && d == 2) sig[8] = (real)(sig[8] + (real)(lame * tr));
}

/* stress_update_newtonfluid (src/materials/newtonfluid_inline.h:49-96):
 * rho = m/V, rho0 = m/V0, p = -K((rho/rho0)^gamma - 1); sigma = p I_DIM +
 * (2 mu / 3) dev(D) on the DIM x DIM block only (other entries 0). */
static void nf_point(int d, const real *L, real *sig, real mass, real vol, real vol0, const or_material *m) {
  real visc = m->p[0], bulk = m->p[1], gamma = m->p[2];
  real rho = (real)(mass / vol), rho0 = (real)(mass / vol0);
#ifdef OR_DOUBLE
  real pw = (real)pow(rho / rho0, gamma);
#else
  real pw = (real)powf((float)(rho / rho0), (float)gamma);
#endif
  real pressure = (real)(-bulk * (real)(pw - (real)1.0));
  real D[9];
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++) D[a * d + b] = (real)((real)0.5 * (real)(L[a * d + b] + L[b * d + a]));
  real tr = 0;
  for (int a = 0; a < d; a++) tr = (real)(tr + D[a * d + a]);
  real third = (real)(1.0 / 3.0);
  real coef = (real)(2.0 * (double)visc / 3.0);
  for (int k = 0; k < 9; k++) sig[k] = (real)0.0;
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++) {
      real dev = (real)(D[a * d + b] - (a == b ? (real)((real)(third * tr)) : (real)0.0));
      real iso = a == b ? pressure : (real)0.0;
      sig[3 * a + b] = (real)(iso + (real)(dev * coef));
    }
}

/* Drucker-Prager cone + apex return mapping, restating update_dp_rheo
 * (src/materials/dp_rheo_inline.h:123-246) with return_mapping_cone (:50-65),
 * return_mapping_apex (:67-78) and update_plasticity (:80-96):
 *   deps = sym(L) dt - W eps_e + eps_e W,  W = skew(L) dt
 *   eps_tr = eps_e + deps;  p_tr = p_ref + K tr(eps_tr)
 *   s_tr = s_ref + 2G dev(eps_tr)  (zz deviator zeroed in 2D)
 *   Phi = sqrt(J2) + eta p_tr - kc;  elastic if Phi <= 0
 *   cone: dgamma = Phi/(K eta eta_bar + G); p = p_tr - K eta_bar dgamma;
 *         s = (1 - G dgamma / sqrt(J2)) s_tr
 *   apex (sqrt(J2) - G dgamma < 0): s = 0, p = p_apex
 *   eps_e = (s - s_ref)/2G + (p - p_ref)/(3K) I  (DIM x DIM block)
 * The reference writes eta (p - Pt); with kc = eta*Pt and p_apex = Pt the two
 * agree.  For eta_bar > 0 the reference's apex formula yields p = Pt, which is
 * p_apex here; for eta_bar = 0 (no dilatancy) the reference divides by zero,
 * while this step keeps the limit p = p_apex.
 * p = {K, G, eta, eta_bar, kc, p_apex, has_apex}. */
void or_dp_point(int d, const REAL *L, REAL *sig, REAL *eps_e, const REAL *sref, REAL dt,
                 const REAL *p, int velgrad_is_strain_increment) {
  real K = p[0], G = p[1], eta = p[2], eta_bar = p[3], kc = p[4], p_apex = p[5];
  int has_apex = p[6] != (real)0.0;
  real deps[9];
  if (velgrad_is_strain_increment) {
    for (int k = 0; k < d * d; k++) deps[k] = L[k];
  } else {
    real W[9];
    for (int a = 0; a < d; a++)
      for (int b = 0; b < d; b++) {
        deps[a * d + b] = (real)((real)((real)0.5 * (real)(L[a * d + b] + L[b * d + a])) * dt);
        W[a * d + b] = (real)((real)((real)0.5 * (real)(L[a * d + b] - L[b * d + a])) * dt);
      }
    for (int a = 0; a < d; a++)
      for (int b = 0; b < d; b++) {
        real we = 0, ew = 0;
        for (int k = 0; k < d; k++) {
          we = (real)(we + (real)(W[a * d + k] * eps_e[k * d + b]));
          ew = (real)(ew + (real)(eps_e[a * d + k] * W[k * d + b]));
        }
        deps[a * d + b] = (real)(deps[a * d + b] + (real)(-we + ew));
      }
  }
  real p_ref = (real)((real)(1.0 / 3.0) * (real)((real)(sref[0] + sref[4]) + sref[8]));
  real s_ref[9];
  for (int k = 0; k < 9; k++) s_ref[k] = sref[k];
  s_ref[0] = (real)(s_ref[0] - p_ref);
  s_ref[4] = (real)(s_ref[4] - p_ref);
  s_ref[8] = (real)(s_ref[8] - p_ref);
  real eps_tr[9];
  for (int k = 0; k < d * d; k++) eps_tr[k] = (real)(eps_e[k] + deps[k]);
  real ev = 0;
  for (int a = 0; a < d; a++) ev = (real)(ev + eps_tr[a * d + a]);
  real p_tr = (real)(p_ref + (real)(K * ev));
  real edev[9] = {0};
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++) edev[3 * a + b] = eps_tr[a * d + b];
  real third_ev = (real)((real)(1.0 / 3.0) * ev);
  for (int a = 0; a < 3; a++) edev[3 * a + a] = (real)(edev[3 * a + a] - third_ev);
  if (d < 3) edev[8] = (real)0.0;
  real two_g = (real)(2.0 * (double)G);
  real s_tr[9];
  for (int k = 0; k < 9; k++) s_tr[k] = (real)(s_ref[k] + (real)(two_g * edev[k]));
  real ss = 0;
  for (int k = 0; k < 9; k++) ss = (real)(ss + (real)(s_tr[k] * s_tr[k]));
  real J2 = (real)((real)0.5 * ss);
  real sqrtJ2 = (real)sqrt((double)J2);
  real Phi = (real)((real)(sqrtJ2 + (real)(eta * p_tr)) - kc);
  if (Phi <= (real)0.0) {
    for (int k = 0; k < 9; k++) sig[k] = s_tr[k];
    sig[0] = (real)(sig[0] + p_tr);
    sig[4] = (real)(sig[4] + p_tr);
    sig[8] = (real)(sig[8] + p_tr);
    for (int k = 0; k < d * d; k++) eps_e[k] = eps_tr[k];
    return;
  }
  double dgamma = (double)Phi / ((double)K * (double)eta * (double)eta_bar + (double)G);
  double p_next = (double)p_tr - (double)K * (double)eta_bar * dgamma;
  real s_next[9];
  int apex = has_apex && ((double)sqrtJ2 - (double)G * dgamma < 0.0);
  if (apex) {
    p_next = (double)p_apex;
    for (int k = 0; k < 9; k++) s_next[k] = (real)0.0;
  } else {
    double scale = 1.0 - ((double)G * dgamma) / (double)sqrtJ2;
    for (int k = 0; k < 9; k++) s_next[k] = (real)(scale * (double)s_tr[k]);
  }
  real pn = (real)p_next;
  for (int k = 0; k < 9; k++) sig[k] = s_next[k];
  sig[0] = (real)(sig[0] + pn);
  sig[4] = (real)(sig[4] + pn);
  sig[8] = (real)(sig[8] + pn);
  double inv2g = 1.0 / (2.0 * (double)G);
  real dpk = (real)(((double)pn - (double)p_ref) / (3.0 * (double)K));
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++) {
      real e = (real)((double)(real)(s_next[3 * a + b] - s_ref[3 * a + b]) * inv2g);
      if (a == b) e = (real)(e + dpk);
      eps_e[a * d + b] = e;
    }
}

/* Solver::stress_update (src/solver/solver.cpp:110-121): materials in list
 * order, each over all particles of its colour (LE and NF skip inactive
 * particles; the reference DP kernel does not check the flag). */
/* Drucker-Prager parameters of one particle from its Young's modulus and
 * friction angle (degrees): K = E / (3 (1 - 2 nu)), G = E / (2 (1 + nu)),
 * eta = 6 sin(phi) / (sqrt(3) (3 - sin(phi))), xi = 6 cos(phi) / (same),
 * kc = xi c, with nu = p[7], eta_bar = p[3] and the cohesion c recovered
 * from the material's kc and eta. */
static void dp_particle_params(const REAL *mp, REAL E, REAL phi_deg, REAL *out) {
  double nu = mp[7], s3 = sqrt(3.0);
  double eta_m = mp[2];
  double sn_m = 3.0 * s3 * eta_m / (6.0 + s3 * eta_m);
  double xi_m = 6.0 * sqrt(fmax(0.0, 1.0 - sn_m * sn_m)) / (s3 * (3.0 - sn_m));
  double c = xi_m > 0 ? (double)mp[4] / xi_m : 0.0;
  double phi = (double)phi_deg * 3.14159265358979323846 / 180.0;
  double sn = sin(phi), cs = cos(phi);
  double eta = 6.0 * sn / (s3 * (3.0 - sn)), xi = 6.0 * cs / (s3 * (3.0 - sn));
  out[0] = (REAL)((double)E / (3.0 * (1.0 - 2.0 * nu)));
  out[1] = (REAL)((double)E / (2.0 * (1.0 + nu)));
  out[2] = (REAL)eta;
  out[3] = mp[3];
  out[4] = (REAL)(xi * c);
  out[5] = eta > 0 ? (REAL)(xi * c / eta) : (REAL)0;
  out[6] = eta > 0 ? (REAL)1 : (REAL)0;
  out[7] = (REAL)nu;
}

/* update_vonmises (src/materials/vonmises_inline.h:36-120), 3D: trial
 * elastic strain eps + sym(L) dt, p = K tr, s = 2G dev, q = sqrt(3/2 s:s);
 * Phi = q - (sigma_y + H acc); Newton on dgamma in double until |Phi| <= 1e-7
 * (acc from the iterate before the last update); s *= 1 - 3G dgamma / q;
 * eps = s / 2G + tr/3 I. */
static void vm_point(const real *L, real *sig, real *eps, real *acc, real dt, const or_material *m) {
  real K = m->p[0], G = m->p[1], sy0 = m->p[2], H = m->p[3];
  real et[9];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++)
      et[3 * a + b] = (real)(eps[3 * a + b] + (real)((real)((real)0.5 * (real)(L[3 * a + b] + L[3 * b + a])) * dt));
  real ev = (real)((real)(et[0] + et[4]) + et[8]);
  real p = (real)(K * ev);
  real sv[9], ss = 0;
  for (int k = 0; k < 9; k++) {
    real e = et[k];
    if (k == 0 || k == 4 || k == 8) e = (real)(e - (real)((real)(1.0 / 3.0) * ev));
    sv[k] = (real)((real)(2.0 * G) * e);
    ss = (real)(ss + (real)(sv[k] * sv[k]));
  }
  real sy = (real)(sy0 + (real)(H * *acc));
  real q = (real)sqrt((double)(real)(1.5 * ss));
  real Phi = (real)(q - sy);
  if (Phi <= 0) {
    for (int k = 0; k < 9; k++) {
      sig[k] = (real)(sv[k] + ((k == 0 || k == 4 || k == 8) ? p : (real)0));
      eps[k] = et[k];
    }
    return;
  }
  double dgamma = 0.0, acc_eps = *acc;
  for (int it = 0; it < 100; it++) {
    acc_eps = (double)*acc + dgamma;
    double syi = (double)sy0 + (double)H * acc_eps;
    double phi = (double)q - 3.0 * (double)G * dgamma - syi;
    dgamma = dgamma - phi / (-3.0 * (double)G - (double)H);
    if (!(fabs(phi) > 1e-7)) break;
  }
  double fac = 1.0 - (3.0 * (double)G * dgamma) / (double)q;
  for (int k = 0; k < 9; k++) {
    real sc = (real)(fac * (double)sv[k]);
    int diag = k == 0 || k == 4 || k == 8;
    sig[k] = (real)(sc + (diag ? p : (real)0));
    eps[k] = (real)((double)sc / (2.0 * (double)G) + (diag ? (1.0 / 3.0) * (double)ev : 0.0));
  }
  *acc = (real)acc_eps;
}

/* update_modifiedcamclay_nonlinear (src/materials/modifiedcamclay_inline.h:
 * 321-511) and compute_yield_function (:57-63), pressures positive in
 * compression, in the reference's types: real for the trial state, the
 * volumetric increments and the yield function of the residual; double for
 * the Newton unknowns (lambda, alpha), p, q, p_s, the hardening slope H and
 * the 2 x 2 iteration matrix, inverted as its adjugate over the determinant.
 * The iteration stops at |R| <= 1e-2, the bound growing tenfold per
 * iteration after 1000 (in FP32 the residual's noise lies above 1e-2, so the
 * bound is what stops it).  Stress, elastic strain and pc take the last
 * evaluated iterate; alpha the updated unknowns.  V: current particle volume
 * (specific volume V / Vs).  p = {K, G, M, lam, kap, Vs, Pt, R}. */
static real mcc_yield(real p, real Pt, real ps, real q, real M) {
  real a = (real)((real)(ps - p) - Pt), b = (real)(q / M);
  return (real)((real)((real)(a * a) + (real)(b * b)) - (real)(ps * ps));
}

void or_mcc_point(int d, const REAL *L, REAL *sig, REAL *eps_e, const REAL *sref, REAL *alpha, REAL *pc, REAL V,
                  REAL dt, const or_material *m) {
  real K = m->p[0], G = m->p[1], M = m->p[2], lam = m->p[3], kap = m->p[4], Vs = m->p[5], Pt = m->p[6];
  real deps[9], W[9];
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++) {
      deps[a * d + b] = (real)((real)((real)0.5 * (real)(L[a * d + b] + L[b * d + a])) * dt);
      W[a * d + b] = (real)((real)((real)0.5 * (real)(L[a * d + b] - L[b * d + a])) * dt);
    }
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++) {
      real we = 0, ew = 0;
      for (int k = 0; k < d; k++) {
        we = (real)(we + (real)(W[a * d + k] * eps_e[k * d + b]));
        ew = (real)(ew + (real)(eps_e[a * d + k] * W[k * d + b]));
      }
      deps[a * d + b] = (real)(deps[a * d + b] + (real)(-we + ew));
    }
  real p_ref = (real)(-(real)(1.0 / 3.0) * (real)((real)(sref[0] + sref[4]) + sref[8]));
  real s_ref[9];
  for (int k = 0; k < 9; k++) s_ref[k] = sref[k];
  s_ref[0] = (real)(s_ref[0] + p_ref);
  s_ref[4] = (real)(s_ref[4] + p_ref);
  s_ref[8] = (real)(s_ref[8] + p_ref);
  real eps_tr[9], tr_prev = 0, tr_inc = 0, tr_tr = 0;
  for (int k = 0; k < d * d; k++) eps_tr[k] = (real)(eps_e[k] + deps[k]);
  for (int a = 0; a < d; a++) {
    tr_prev = (real)(tr_prev + eps_e[a * d + a]);
    tr_inc = (real)(tr_inc + deps[a * d + a]);
    tr_tr = (real)(tr_tr + eps_tr[a * d + a]);
  }
  real ev_tr = -tr_tr;
  real edev[9] = {0};
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++) edev[3 * a + b] = eps_tr[a * d + b];
  real third = (real)((1.0 / 3.0) * (double)ev_tr);
  for (int a = 0; a < 3; a++) edev[3 * a + a] = (real)(edev[3 * a + a] + third);
  if (d < 3) edev[8] = 0;
  real v_spec = (real)(V / Vs);
  real p_prev = (real)(-(double)(real)((real)(sig[0] + sig[4]) + sig[8]) / 3.0);
  real v_kap = (real)(v_spec / kap);
  real dev_tr = -tr_inc;
  real p_tr = (real)((double)p_prev / (1.0 - (double)(real)(v_kap * dev_tr)));
  real two_g = (real)(2.0 * (double)G);
  real s_tr[9];
  for (int k = 0; k < 9; k++) s_tr[k] = (real)(s_ref[k] + (real)(two_g * edev[k]));
  real ss = 0;
  for (int a = 0; a < 3; a++) {
    real row = 0;
    for (int k = 0; k < 3; k++) row = (real)(row + (real)(s_tr[3 * a + k] * s_tr[3 * a + k]));
    ss = (real)(ss + row);
  }
  real q_tr = (real)sqrt(1.5 * (double)ss);
  real pc_prev = *pc;
  real ps_tr = (real)(0.5 * (double)(real)(pc_prev + Pt));
  if (mcc_yield(p_tr, Pt, ps_tr, q_tr, M) <= (real)0.0) {
    for (int k = 0; k < 9; k++) sig[k] = s_tr[k];
    sig[0] = (real)(sig[0] - p_tr);
    sig[4] = (real)(sig[4] - p_tr);
    sig[8] = (real)(sig[8] - p_tr);
    for (int k = 0; k < d * d; k++) eps_e[k] = eps_tr[k];
    return;
  }
  real a_prev = *alpha;
  double lamb = 0.0, a_next = (double)a_prev, tol = 1e-2, conv;
  double p_next = 0.0, q_next = 0.0, ps_next = 0.0;
  real s_next[9], dev_e = 0;
  double vlt = (double)(real)(v_spec / (real)(lam - kap));
  double MM = (double)(real)(M * M), six_g = (double)(real)(6 * G), m12g = (double)(real)(-12 * G);
  int counter = 0;
  do {
    double lm = lamb, an = a_next;
    real dpv = (real)(an - (double)a_prev);
    dev_e = (real)(dev_tr - dpv);
    p_next = (double)p_prev / (1.0 - (double)(real)(v_kap * dev_e));
    q_next = (MM / (MM + six_g * lm)) * (double)q_tr;
    ps_next = 0.5 * ((double)pc_prev * (1.0 + vlt * (double)dpv) + (double)Pt);
    real cs = (real)(MM / (MM + 6.0 * (double)G * lm));
    for (int k = 0; k < 9; k++) s_next[k] = (real)(cs * s_tr[k]);
    double R0 = (double)mcc_yield((real)p_next, Pt, (real)ps_next, (real)q_next, M);
    double R1 = an - (double)a_prev + 2.0 * lm * (ps_next - p_next - (double)Pt);
    double omv = 1.0 - vlt * (double)dpv;
    double H = 0.5 * vlt * ((double)pc_prev / (omv * omv));
    double pbar = ps_next - p_next - (double)Pt;
    double d00 = (m12g / (MM + six_g * lm)) * (q_next / (double)M) * (q_next / (double)M);
    double d01 = (2.0 * pbar) * ((double)K + H) - 2.0 * ps_next * H;
    double d10 = 2.0 * pbar;
    double d11 = 1.0 + (2.0 * lm) * ((double)K + H);
    double inv_det = 1.0 / (d00 * d11 - d01 * d10);
    double i00 = d11 * inv_det, i01 = -d01 * inv_det, i10 = -d10 * inv_det, i11 = d00 * inv_det;
    lamb = lm - (i00 * R0 + i01 * R1);
    a_next = an - (i10 * R0 + i11 * R1);
    conv = sqrt(R0 * R0 + R1 * R1);
    if (counter > 1000) tol *= 10.0;
    counter += 1;
  } while (fabs(conv) > tol && counter < 1400);
  real pn = (real)p_next;
  for (int k = 0; k < 9; k++) sig[k] = s_next[k];
  sig[0] = (real)(sig[0] - pn);
  sig[4] = (real)(sig[4] - pn);
  sig[8] = (real)(sig[8] - pn);
  real evol = (real)((1.0 / 3.0) * (double)(real)(tr_prev + dev_e));
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++) {
      real e = (real)((real)(s_next[3 * a + b] - s_ref[3 * a + b]) / two_g);
      if (a == b) e = (real)(e - evol);
      eps_e[a * d + b] = e;
    }
  *alpha = (real)a_next;
  *pc = (real)(2.0 * ps_next - (double)Pt);
}

/* update_druckerpragercap (src/materials/druckerprager_cap_inline.h:370-554)
 * with return_mapping_cone (:124-141), return_mapping_apex (:143-156),
 * return_mapping_cap (:159-235), compute_pc / compute_a / compute_b (:56-84),
 * the yield functions (:94-111) and update_plasticity (:328-346), p =
 * tr(sigma)/3 (tension positive), in the reference's types: real for the
 * trial state, the yield functions' arguments, pc and a; double for the
 * return mappings.  Past the apex the return takes eta_bar dgamma =
 * (p_tr - Pt) / K directly (the reference divides by eta_bar and multiplies
 * back, 0/0 for eta_bar = 0).  The cap's Newton iteration stops at
 * |R| <= 0.1, the bound growing tenfold per iteration after 1000; its
 * results are the last evaluated iterate's.  V0: the particle's original
 * volume.  p = {K, G, M, lam, kap, Vs, Pt, R, beta, eta_bar}. */
static real dpc_pc(real v0, real pc_prev, real lam, real kap, real a_next, real a_prev) {
  real C = (real)(v0 / (real)(lam - kap));
  return (real)((real)exp((double)(real)(C * (real)(a_next - a_prev))) * pc_prev);
}

static real dpc_cap_yield(real p, real Pt, real a, real q, real b, real M) {
  real pa = (real)((real)(p - Pt) + a), qm = (real)(q / M);
  return (real)((1.0 / (double)(real)(b * b)) * (double)pa * (double)pa + (double)(real)(qm * qm) -
                (double)(real)(a * a));
}

void or_dpc_point(int d, const REAL *L, REAL *sig, REAL *eps_e, const REAL *sref, REAL *alpha, REAL *pc, REAL V0,
                  REAL dt, const or_material *m) {
  real K = m->p[0], G = m->p[1], M = m->p[2], lam = m->p[3], kap = m->p[4], Vs = m->p[5], Pt = m->p[6];
  real beta = m->p[8], eta_bar = m->p[9];
  real deps[9], W[9];
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++) {
      deps[a * d + b] = (real)((real)((real)0.5 * (real)(L[a * d + b] + L[b * d + a])) * dt);
      W[a * d + b] = (real)((real)((real)0.5 * (real)(L[a * d + b] - L[b * d + a])) * dt);
    }
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++) {
      real we = 0, ew = 0;
      for (int k = 0; k < d; k++) {
        we = (real)(we + (real)(W[a * d + k] * eps_e[k * d + b]));
        ew = (real)(ew + (real)(eps_e[a * d + k] * W[k * d + b]));
      }
      deps[a * d + b] = (real)(deps[a * d + b] + (real)(-we + ew));
    }
  real p_ref = (real)((real)(1.0 / 3.0) * (real)((real)(sref[0] + sref[4]) + sref[8]));
  real s_ref[9];
  for (int k = 0; k < 9; k++) s_ref[k] = sref[k];
  s_ref[0] = (real)(s_ref[0] - p_ref);
  s_ref[4] = (real)(s_ref[4] - p_ref);
  s_ref[8] = (real)(s_ref[8] - p_ref);
  real eps_tr[9], ev = 0;
  for (int k = 0; k < d * d; k++) eps_tr[k] = (real)(eps_e[k] + deps[k]);
  for (int a = 0; a < d; a++) ev = (real)(ev + eps_tr[a * d + a]);
  real p_tr = (real)(p_ref + (real)(K * ev));
  real edev[9] = {0};
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++) edev[3 * a + b] = eps_tr[a * d + b];
  real third = (real)((1.0 / 3.0) * (double)ev);
  for (int a = 0; a < 3; a++) edev[3 * a + a] = (real)(edev[3 * a + a] - third);
  if (d < 3) edev[8] = 0;
  real two_g = (real)(2.0 * (double)G);
  real s_tr[9];
  for (int k = 0; k < 9; k++) s_tr[k] = (real)(s_ref[k] + (real)(two_g * edev[k]));
  real ss = 0;
  for (int a = 0; a < 3; a++) {
    real row = 0;
    for (int k = 0; k < 3; k++) row = (real)(row + (real)(s_tr[3 * a + k] * s_tr[3 * a + k]));
    ss = (real)(ss + row);
  }
  real J2 = (real)(0.5 * (double)ss);
  real q_tr = (real)sqrt(3.0 * (double)J2);
  real sqrtJ2 = (real)sqrt((double)J2);
  real eta = (real)(sqrt(1.0 / 3.0) * (double)M);
  real phi_cone = (real)(sqrtJ2 + (real)(eta * (real)(p_tr - Pt)));
  real v0 = (real)(V0 / Vs);
  real a_prev = *alpha, pc_prev = *pc;
  real a_tr = (real)((real)(pc_prev + Pt) / (real)(1 + beta));
  real b_tr = p_tr < (real)(Pt - a_tr) ? beta : (real)1;
  real phi_cap = dpc_cap_yield(p_tr, Pt, a_tr, q_tr, b_tr, M);
  if (phi_cone <= (real)0.0 && phi_cap <= (real)0.0) {
    for (int k = 0; k < 9; k++) sig[k] = s_tr[k];
    sig[0] = (real)(sig[0] + p_tr);
    sig[4] = (real)(sig[4] + p_tr);
    sig[8] = (real)(sig[8] + p_tr);
    for (int k = 0; k < d * d; k++) eps_e[k] = eps_tr[k];
    return;
  }
  double p_next = p_tr, pc_next = pc_prev, a_next = a_tr, al = a_prev;
  real s_next[9];
  for (int k = 0; k < 9; k++) s_next[k] = s_tr[k];
  int done = 0;
  if (phi_cone > (real)0.0) {
    double dg = (double)phi_cone / ((double)K * (double)eta * (double)eta_bar + (double)G);
    if ((double)sqrtJ2 - (double)G * dg < 0.0) {
      double edg = ((double)p_tr - (double)Pt) / (double)K;
      al = (double)a_prev - edg;
      p_next = (double)p_tr - (double)K * edg;
      for (int k = 0; k < 9; k++) s_next[k] = 0;
      pc_next = dpc_pc(v0, pc_prev, lam, kap, (real)al, a_prev);
      done = 1;
    } else {
      al = (double)a_prev - (double)eta_bar * dg;
      p_next = (double)p_tr - (double)K * (double)eta_bar * dg;
      real sc = (real)(1.0 - ((double)G * dg) / (double)sqrtJ2);
      for (int k = 0; k < 9; k++) s_next[k] = (real)(sc * s_tr[k]);
      pc_next = dpc_pc(v0, pc_prev, lam, kap, (real)al, a_prev);
      a_next = (real)((real)((real)pc_next + Pt) / (real)(1 + beta));
    }
  }
  if (!done && phi_cap > (real)0.0 && p_next < a_next) {
    double dgam = 0.0, alv = a_prev, tol = 1e-1, conv;
    double MM = (double)(real)(M * M), six_g = (double)(real)(6 * G), m12g = (double)(real)(-12 * G);
    int counter = 0;
    do {
      double dgn = dgam;
      al = alv;
      p_next = (double)p_tr + (double)K * (al - (double)a_prev);
      double q_next = (MM / (MM + six_g * dgn)) * (double)q_tr;
      pc_next = dpc_pc(v0, pc_prev, lam, kap, (real)al, a_prev);
      a_next = (real)((real)((real)pc_next + Pt) / (real)(1 + beta));
      double b_next = (real)p_next < (real)(Pt - (real)a_next) ? (double)beta : 1.0;
      real cs = (real)(MM / (MM + six_g * dgn));
      for (int k = 0; k < 9; k++) s_next[k] = (real)(cs * s_tr[k]);
      double R0 = (double)dpc_cap_yield((real)p_next, Pt, (real)a_next, (real)q_next, (real)b_next, M);
      double R1 = al - (double)a_prev + dgn * (2.0 / (b_next * b_next)) * (p_next - (double)Pt + a_next);
      double dPc = pc_next * ((double)v0 / ((double)lam - (double)kap));
      double H = dPc / (1.0 + (double)beta);
      double pbar = p_next - (double)Pt + a_next;
      double d00 = (m12g / (MM + six_g * dgn)) * (q_next / (double)M) * (q_next / (double)M);
      double d01 = ((2.0 * pbar) / (b_next * b_next)) * ((double)K + H) - 2.0 * a_next * H;
      double d10 = (2.0 * pbar) / (b_next * b_next);
      double d11 = 1.0 + ((2.0 * dgn) / (b_next * b_next)) * ((double)K + H);
      double inv_det = 1.0 / (d00 * d11 - d01 * d10);
      double i00 = d11 * inv_det, i01 = -d01 * inv_det, i10 = -d10 * inv_det, i11 = d00 * inv_det;
      dgam = dgn - (i00 * R0 + i01 * R1);
      alv = al - (i10 * R0 + i11 * R1);
      conv = sqrt(R0 * R0 + R1 * R1);
      counter++;
      if (counter > 1000) tol *= 10.0;
    } while (conv > tol && counter < 1400);
  }
  real pn = (real)p_next;
  for (int k = 0; k < 9; k++) sig[k] = s_next[k];
  sig[0] = (real)(sig[0] + pn);
  sig[4] = (real)(sig[4] + pn);
  sig[8] = (real)(sig[8] + pn);
  real dpk = (real)((p_next - (double)p_ref) / (3.0 * (double)K));
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++) {
      real e = (real)((real)(s_next[3 * a + b] - s_ref[3 * a + b]) / two_g);
      if (a == b) e = (real)(e + dpk);
      eps_e[a * d + b] = e;
    }
  *alpha = (real)al;
  *pc = (real)pc_next;
}

void or_stress_update(or_sim *s) {
  int d = s->grid.dim;
  for (int mid = 0; mid < s->num_materials; mid++) {
    const or_material *m = &s->materials[mid];
    for (int i = 0; i < s->num_particles; i++) {
      if ((int)s->colors[i] != mid) continue;
      const real *L = s->velocity_gradient + (size_t)i * d * d;
      real *sig = s->stresses + (size_t)i * 9;
      if (m->type == OR_MAT_LINEAR_ELASTIC) {
        if (!s->is_active[i]) continue;
        le_point(d, L, sig, s->dt, m);
      } else if (m->type == OR_MAT_NEWTON_FLUID) {
        if (!s->is_active[i]) continue;
        nf_point(d, L, sig, s->masses[i], s->volumes[i], s->volumes_original[i], m);
      } else if (m->type == OR_MAT_DRUCKER_PRAGER) {
        const REAL *prm = m->p;
        REAL pp[8];
        if (s->youngs && m->p[7] >= 0) {
          dp_particle_params(m->p, s->youngs[i], s->friction[i], pp);
          prm = pp;
        }
        or_dp_point(d, L, sig, s->eps_e + (size_t)i * d * d, s->stress_ref + (size_t)i * 9, s->dt, prm, 0);
      } else if (m->type == OR_MAT_VON_MISES && d == 3) {
        vm_point(L, sig, s->eps_e + (size_t)i * 9, s->acc_eps_p + i, s->dt, m);
      } else if (m->type == OR_MAT_MODIFIED_CAM_CLAY) {
        or_mcc_point(d, L, sig, s->eps_e + (size_t)i * d * d, s->stress_ref + (size_t)i * 9, s->acc_eps_p + i,
                     s->pc + i, s->volumes[i], s->dt, m);
      } else if (m->type == OR_MAT_DRUCKER_PRAGER_CAP) {
        or_dpc_point(d, L, sig, s->eps_e + (size_t)i * d * d, s->stress_ref + (size_t)i * 9, s->acc_eps_p + i,
                     s->pc + i, s->volumes_original[i], s->dt, m);
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* One USL step                                                             */
/* ------------------------------------------------------------------------ */

/* USL::solve (src/solver/usl/usl.cpp:69-115).  apply_on_nodes_f_ext has no
 * override in any boundary condition on this path, and the second
 * apply_on_particles call only writes f_ext, which the next reset clears. */
/* ------------------------------------------------------------------------ */
/* MUSL                                                                     */
/* ------------------------------------------------------------------------ */

/* MUSL (declared by the reference, include/pyroclastmpm/solver/musl/musl.cuh
 * and musl_kernels.cuh, not built there): G2P_double_mapping updates the
 * velocities (FLIP/PIC blend as USL G2P) and positions; P2G_double_mapping
 * maps the new momenta to the nodes (masses and moments; no forces), where
 * the velocity conditions apply again (NodeDomain, BodyForce "fixed", the
 * analytic rigid body); G2P then takes the velocity gradient from that field
 * for F, V and the stress update.  All three use the step's start-of-step
 * shape functions and bins. */
static void musl_g2p_velocities(or_sim *s, real *xnew) {
  const or_grid *g = &s->grid;
  int d = g->dim, nsn = s->nsn;
  real one_minus_alpha = (real)(1.0 - (double)s->alpha);
  for (int i = 0; i < s->num_particles; i++) {
    int b[3] = {0, 0, 0};
    for (int a = 0; a < d; a++) b[a] = s->bins[i * d + a];
    real vinc[3] = {0, 0, 0}, dvinc[3] = {0, 0, 0};
    for (int sid = 0; sid < nsn; sid++) {
      int w[3], sel[3];
      window_offset(d, s->shape_function, sid, w);
      int node = slot_target(s, b, w, sel);
      if (s->shape_function != OR_QUADRATIC) {
        int invalid = 0;
        for (int a = 0; a < d; a++)
          if (sel[a] < 0 || sel[a] >= g->num_cells[a]) invalid = 1;
        if (invalid) continue;
      }
      if (node < 0) continue;
      real m = s->node_masses[node];
      if (m <= s->small_mass_cutoff) continue;
      real psi = s->psi[(size_t)i * nsn + sid];
      for (int a = 0; a < d; a++) {
        real vn = (real)(s->node_moments[(size_t)node * d + a] / m);
        real vnt = (real)(s->node_moments_nt[(size_t)node * d + a] / m);
        dvinc[a] = (real)(dvinc[a] + (real)(psi * (real)(vnt - vn)));
        vinc[a] = (real)(vinc[a] + (real)(psi * vnt));
      }
    }
    real *v = s->velocities + (size_t)i * d;
    for (int a = 0; a < d; a++) {
      v[a] = (real)((real)(one_minus_alpha * vinc[a]) + (real)(s->alpha * (real)(v[a] + dvinc[a])));
      xnew[(size_t)i * d + a] = (real)(s->positions[(size_t)i * d + a] + (real)(s->dt * vinc[a]));
    }
  }
}

static void musl_remap(or_sim *s) {
  const or_grid *g = &s->grid;
  int d = g->dim, nsn = s->nsn;
  size_t nn = (size_t)g->num_cells_total;
  real *mass = (real *)calloc(nn, sizeof(real));
  real *mom = (real *)calloc(nn * d, sizeof(real));
  for (int sid = 0; sid < nsn; sid++) {
    int w[3];
    window_offset(d, s->shape_function, sid, w);
    for (int k = 0; k < s->num_particles; k++) {
      int j = s->sorted_index[k];
      if (s->hash_sorted[k] >= (unsigned int)g->num_cells_total) continue;
      int b[3] = {0, 0, 0}, sel[3];
      for (int a = 0; a < d; a++) b[a] = s->bins[j * d + a];
      if (s->shape_function == OR_QUADRATIC) {
        int out = 0;
        for (int a = 0; a < d; a++)
          if (b[a] < 0 || b[a] >= g->num_cells[a]) out = 1;
        if (out) continue;
      }
      int node = slot_target(s, b, w, sel);
      if (node < 0) continue;
      real sm = (real)(s->psi[(size_t)j * nsn + sid] * s->masses[j]);
      mass[node] = (real)(mass[node] + sm);
      for (int a = 0; a < d; a++)
        mom[node * d + a] = (real)(mom[node * d + a] + (real)(sm * s->velocities[(size_t)j * d + a]));
    }
  }
  memset(s->node_masses, 0, sizeof(real) * nn);
  memset(s->node_moments, 0, sizeof(real) * nn * d);
  memset(s->node_moments_nt, 0, sizeof(real) * nn * d);
  for (size_t n = 0; n < nn; n++) {
    if (mass[n] <= s->small_mass_cutoff) continue;
    s->node_masses[n] = mass[n];
    for (int a = 0; a < d; a++) {
      s->node_moments[n * d + a] = mom[n * d + a];
      s->node_moments_nt[n * d + a] = mom[n * d + a];
    }
  }
  free(mass);
  free(mom);
  for (int k = 0; k < s->num_bcs; k++) {
    or_bc *bc = &s->bcs[k];
    if (bc->type == OR_BC_NODEDOMAIN) nodedomain(s, bc);
    else if (bc->type == OR_BC_BODYFORCE && bc->i[0] == 2) bodyforce(s, bc);
    else if (bc->type == OR_BC_RIGID_SDF) rigid_sdf(s, bc);
  }
}

static void musl_g2p_gradient(or_sim *s, const real *xnew) {
  const or_grid *g = &s->grid;
  int d = g->dim, nsn = s->nsn;
  for (int i = 0; i < s->num_particles; i++) {
    int b[3] = {0, 0, 0};
    for (int a = 0; a < d; a++) b[a] = s->bins[i * d + a];
    real L[9] = {0};
    for (int sid = 0; sid < nsn; sid++) {
      int w[3], sel[3];
      window_offset(d, s->shape_function, sid, w);
      int node = slot_target(s, b, w, sel);
      if (s->shape_function != OR_QUADRATIC) {
        int invalid = 0;
        for (int a = 0; a < d; a++)
          if (sel[a] < 0 || sel[a] >= g->num_cells[a]) invalid = 1;
        if (invalid) continue;
      }
      if (node < 0) continue;
      real m = s->node_masses[node];
      if (m <= s->small_mass_cutoff) continue;
      const real *dpsi = s->dpsi + ((size_t)i * nsn + sid) * d;
      real vnt[3];
      for (int a = 0; a < d; a++) vnt[a] = (real)(s->node_moments_nt[(size_t)node * d + a] / m);
      for (int a = 0; a < d; a++)
        for (int c = 0; c < d; c++) L[a * d + c] = (real)(L[a * d + c] + (real)(dpsi[a] * vnt[c]));
    }
    memcpy(s->velocity_gradient + (size_t)i * d * d, L, sizeof(real) * d * d);
    for (int a = 0; a < d; a++) s->positions[(size_t)i * d + a] = xnew[(size_t)i * d + a];
    real A[9], Fn[9];
    real *F = s->F + (size_t)i * d * d;
    for (int a = 0; a < d; a++)
      for (int c = 0; c < d; c++) A[a * d + c] = (real)((a == c ? (real)1.0 : (real)0.0) + (real)(L[a * d + c] * s->dt));
    for (int a = 0; a < d; a++)
      for (int c = 0; c < d; c++) {
        real acc = (real)(A[a * d + 0] * F[0 * d + c]);
        for (int k = 1; k < d; k++) acc = (real)(acc + (real)(A[a * d + k] * F[k * d + c]));
        Fn[a * d + c] = acc;
      }
    memcpy(F, Fn, sizeof(real) * d * d);
    s->volumes[i] = (real)(det(d, F) * s->volumes_original[i]);
  }
}

void or_solve(or_sim *s) {
  or_reset(s);
  or_partition(s);
  or_shape_functions(s);
  or_apply_on_particles(s);
  or_p2g(s);
  or_apply_on_nodes_moments(s);
  if (s->musl) {
    real *xnew = (real *)malloc(sizeof(real) * (size_t)s->num_particles * s->grid.dim);
    musl_g2p_velocities(s, xnew);
    musl_remap(s);
    musl_g2p_gradient(s, xnew);
    free(xnew);
  } else {
    or_g2p(s);
  }
  or_stress_update(s);
}

/* Solver::solve_nsteps (src/solver/solver.cpp:125-134): solve, then
 * increment_global (src/common/global_settings.cpp:220-227). */
void or_solve_nsteps(or_sim *s, int nsteps) {
  for (int k = 0; k < nsteps; k++) {
    or_solve(s);
    s->global_step += 1;
  }
}
