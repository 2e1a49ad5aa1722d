// Device-side data layout and per-point math of the USL step (sm_100a).
//
// Layout in HBM (all FP32 unless noted), structure-of-arrays with one
// contiguous array per tensor component ("component-major"):
//   particle field f, component c, storage slot s  ->  f[c * stride + s]
// stride is the particle count rounded up to 64 so every component array
// starts 256-byte aligned.  Symmetric tensors keep only their independent
// components:
//   stress  2D: xx yy xy zz           3D: xx yy zz xy xz yz
//   eps_e   2D: xx yy xy              3D: xx yy zz xy xz yz
// F and the velocity gradient L are full dim x dim, row-major components.
// Grid nodes are dense, x-fastest (the reference NODE_MEM_INDEX order), one
// array per component: m, p (moments), pnt (moments_nt), v = p/m, vnt = pnt/m.
#pragma once

#include <cstdint>

#include "pmpm.h"

namespace pmpm {

constexpr int kMaxMat = PMPM_MAX_MATERIALS;
constexpr int kMaxBC = PMPM_MAX_BCS;

// fault word bits (first fault wins the status)
enum : int { kFaultOutOfDomain = 1, kFaultNonFinite = 2, kFaultCellOverflow = 4, kFaultWaitTimeout = 8 };

struct DevGrid {
  float origin[3];
  float end[3];
  float h, inv_h;
  int n[3];
  int ntotal;
  int tdim[3];  // tiles per axis
  int ntiles;
};

// Node tiles: the unit of P2G work and of grid activity tracking.
template <int D>
struct TileDims;
template <>
struct TileDims<2> {
  static constexpr int X = 16, Y = 16, Z = 1, N = 256;
};
template <>
struct TileDims<3> {
  static constexpr int X = 8, Y = 8, Z = 8, N = 512;
};

template <int D>
struct Sym {
  static constexpr int S = (D == 2) ? 4 : 6;  // stress components
  static constexpr int E = (D == 2) ? 3 : 6;  // elastic strain components
};

struct DevParticles {
  int n;
  int stride;
  float *x, *v, *F, *sig, *L, *m, *V, *V0, *fext, *eps, *sref;
  float *pE, *pphi;  // per-particle Young's modulus and friction angle (deg) of Drucker-Prager, or null
  float *acc;        // VonMises accumulated plastic strain / Modified Cam Clay alpha, or null
  float *pc;         // Modified Cam Clay preconsolidation pressure, or null
  uint8_t *color, *active, *rigid;
  int *id;             // original particle id of each storage slot
  unsigned int *hash;  // reference cell hash of the last partition
  int *slot;           // rank inside the key bin from the counting pass (-1: not binned)
  unsigned int *key;   // binning key of the last partition (scratch)
};

struct DevNodes {
  float *m, *p, *pnt;
  // v = p/m and v_nt = p_nt/m packed per node for the G2P gather:
  // 3D: vx vy vz - | vntx vnty vntz -  (two float4), 2D: vx vy vntx vnty
  float *vel;
  int *tile_epoch;  // tile active in the partition whose epoch it holds
  // active-tile queue of the 3D sweep P2G kernels (null where not used):
  // tile_list[0 .. tile_queue[epoch & 1]) are the tiles the binning pass of
  // that epoch marked; tile_queue[2 + parity] is a launch's fetch counter
  int *tile_list;
  int *tile_queue;
  // cell-scatter P2G: per node [m, p0 p1 p2, f0 f1 f2, -], zero outside P2G
  float *acc;
};

template <int D>
struct NodeVel {
  static constexpr int F = D == 3 ? 8 : 4;  // floats per node in DevNodes::vel
};

struct DevBins {
  // Binning key space.  Reference mode: the reference cell hash (key grid =
  // node grid).  Dual mode (quadratic, outside the deterministic mode): the
  // dual cell floor(x/h + 1/2), whose particles share one 3x3 (3x3x3) node
  // window; key grid = node grid + 1 per axis.
  int dual;
  int kd[3];
  int nkeys;
  int key_base;     // added to the stored particle keys (an instance's first key in a batch)
  int kb[3];        // dual-cell bricks per axis (8^3 dual cells each)
  int *brick_epoch; // brick holds particles in the partition whose epoch it holds (or null)
  int sentinel;     // particles outside the grid take key ntotal (batched ensembles)
  int *count;       // per key, zero between steps
  int *offset;      // exclusive prefix, nkeys + 1 entries
  int *order;       // sorted position -> storage slot
  int *block_sums;  // scan scratch
  int *scalars;     // [0] binned count, [1] unbinned counter, [2] big-cell count
  int *big_cells;   // cells too large for the in-register sort
  // P2G records of the 3D sweep kernels in sorted order (null where not
  // used): rec4 float4s per particle (4, or 5 with a PlanarDomain), written
  // by k_records just before each P2G launch, copied into shared memory by
  // the sweeps' bulk copies one row of source cells at a time
  float4 *rec;
  int rec4;
};

struct DevMaterial {
  int type;
  float density;
  // p[0..11]: the pmpm_material parameters; Drucker-Prager (friction-angle
  // form, which uses p[0..7]) also p[8] = cohesion, p[9] = friction angle,
  // for per-particle parameters
  float p[12];
};

struct DevBC {
  int type;
  int i[8];
  // gravity: r[0..2] is the gravity in force this step; rigid SDF body:
  // r[0..2] centre this step, r[12..13] cos and sin of its angle this step
  float r[16];
  const float *values;
  const uint8_t *mask;
};

struct StepArgs {
  DevGrid g;
  DevParticles P;
  DevNodes N;
  DevBins B;
  float dt, alpha, one_minus_alpha, cutoff;
  int epoch;
  unsigned flags;
  int *fault;
  int nmat;
  int nbc;
  int nbc_epi;      // node BCs [0, nbc_epi) run in the P2G epilogue, the rest after the rigid pass
  int rigid_shift;  // G2P also moves rigid particles by their set velocity (RigidBodyLevelSet)
  int remap;        // MUSL momentum remap: P2G without forces, velocity conditions only
  int musl_pass;    // G2P: 0 USL; MUSL 1 velocities (+ positions aside), 2 gradient, F, V, stress
  float *musl_x;    // MUSL: new positions between the two G2P passes
  int has_planar;
  int has_sref;
  int p2g_par;      // fetch counter of this P2G launch (tile queue)
  int bin_next;     // G2P: bin the new positions for the next partition
  unsigned *hash_next;  // their reference hashes (swapped in by that partition)
  DevMaterial mat[kMaxMat];
  DevBC bc[kMaxBC];
};

// --------------------------------------------------------------------------
// index helpers
// --------------------------------------------------------------------------

__device__ __forceinline__ int flat_index(const DevGrid &g, int x, int y, int z) {
  return x + y * g.n[0] + z * g.n[0] * g.n[1];
}

// Cell coordinate of a position: (int)((x - origin) * inv_h), truncation
// toward zero, FP32 subtract then multiply (no contraction possible), as
// calculate_hashes (src/spatialpartition/spatialpartition_inline.h:49-62).
__device__ __forceinline__ float scaled_coord(float x, float o, float inv_h) {
  return __fmul_rn(__fsub_rn(x, o), inv_h);
}

// Boundary-modified cubic B-spline node type of a node index (one axis):
// NodesContainer::calculate_bin_types (src/nodes/nodes.cpp:135-173).
__device__ __forceinline__ int cubic_node_type(int i, int n) {
  if (i == 0 || i == n - 1) return 1;
  if (i == 1) return 2;
  return 3;
}

// --------------------------------------------------------------------------
// shape functions, one axis
// --------------------------------------------------------------------------

// Horner coefficients of the boundary-modified cubic B-spline by node type
// (0..4) and unit interval [-2,-1), [-1,0), [0,1), [1,2): weight
// ((c3 r + c2) r + c1) r + c0, derivative (d2 r + d1) r + d0 (times 1/h).
// Same piecewise polynomials as src/shapefunction/cubic.cuh:28-197.
__constant__ float kCubicW[5][4][4] = {
    {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}},
    {{1.0f / 6.0f, 1.0f, 2.0f, 4.0f / 3.0f},
     {-1.0f / 6.0f, 0.0f, 1.0f, 1.0f},
     {1.0f / 6.0f, 0.0f, -1.0f, 1.0f},
     {-1.0f / 6.0f, 1.0f, -2.0f, 4.0f / 3.0f}},
    {{0, 0, 0, 0},
     {-1.0f / 3.0f, -1.0f, 0.0f, 2.0f / 3.0f},
     {0.5f, -1.0f, 0.0f, 2.0f / 3.0f},
     {-1.0f / 6.0f, 1.0f, -2.0f, 4.0f / 3.0f}},
    {{1.0f / 6.0f, 1.0f, 2.0f, 4.0f / 3.0f},
     {-0.5f, -1.0f, 0.0f, 2.0f / 3.0f},
     {0.5f, -1.0f, 0.0f, 2.0f / 3.0f},
     {-1.0f / 6.0f, 1.0f, -2.0f, 4.0f / 3.0f}},
    {{1.0f / 6.0f, 1.0f, 2.0f, 4.0f / 3.0f},
     {-0.5f, -1.0f, 0.0f, 2.0f / 3.0f},
     {1.0f / 3.0f, -1.0f, 0.0f, 2.0f / 3.0f},
     {0, 0, 0, 0}},
};
__constant__ float kCubicD[5][4][3] = {
    {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}},
    {{0.5f, 2.0f, 2.0f}, {-0.5f, 0.0f, 1.0f}, {0.5f, 0.0f, -1.0f}, {-0.5f, 2.0f, -2.0f}},
    {{0, 0, 0}, {-1.0f, -2.0f, 0.0f}, {1.5f, -2.0f, 0.0f}, {-0.5f, 2.0f, -2.0f}},
    {{0.5f, 2.0f, 2.0f}, {-1.5f, -2.0f, 0.0f}, {1.5f, -2.0f, 0.0f}, {-0.5f, 2.0f, -2.0f}},
    {{0.5f, 2.0f, 2.0f}, {-1.5f, -2.0f, 0.0f}, {1.0f, -2.0f, 0.0f}, {0, 0, 0}},
};

// The four cubic weights of one axis where all four nodes b - 1 .. b + 2 of a
// particle at u = b + t (t in [0, 1)) are of interior type 3, with their
// derivatives times inv_h, evaluated together from t and s = 1 - t.  They
// are the type-3 pieces of the table above (src/shapefunction/cubic.cuh:
// 28-197) at r = t + 1, t, t - 1, t - 2: (2 - r)^3 / 6 = s^3 / 6,
// r^3 / 2 - r^2 + 2/3, -r^3 / 2 - r^2 + 2/3 = s^3 / 2 - s^2 + 2/3 and
// (2 + r)^3 / 6 = t^3 / 6 (derivatives -s^2 / 2, 1.5 t^2 - 2t,
// 2s - 1.5 s^2, t^2 / 2); the same polynomials, FP32 rounding apart.
__device__ __forceinline__ void cubic_interior_weights(float t, float inv_h, float N[4], float dN[4]) {
  const float s = 1.0f - t;
  const float t2 = t * t, s2 = s * s;
  const float t3 = t2 * t, s3 = s2 * s;
  N[0] = s3 * (1.0f / 6.0f);
  N[1] = fmaf(0.5f, t3, (2.0f / 3.0f) - t2);
  N[2] = fmaf(0.5f, s3, (2.0f / 3.0f) - s2);
  N[3] = t3 * (1.0f / 6.0f);
  dN[0] = (-0.5f * s2) * inv_h;
  dN[1] = fmaf(1.5f, t2, -2.0f * t) * inv_h;
  dN[2] = fmaf(-1.5f, s2, 2.0f * s) * inv_h;
  dN[3] = (0.5f * t2) * inv_h;
}

// Weight and derivative of one axis for relative coordinate r (in cells).
// linear: src/shapefunction/linear.cuh:28-52 (derivative 0 at r == 0);
// quadratic: uniform C1 quadratic B-spline of support 3h;
// cubic: table above, node type `type`.
template <int SF>
__device__ __forceinline__ void axis_weight(float r, float inv_h, int type, float &N, float &dN) {
  if (SF == PMPM_SHAPE_LINEAR) {
    float ar = fabsf(r);
    N = ar >= 1.0f ? 0.0f : 1.0f - ar;
    if (r > 1.0f || r < -1.0f || r == 0.0f)
      dN = 0.0f;
    else
      dN = r > 0.0f ? -inv_h : inv_h;
  } else if (SF == PMPM_SHAPE_QUADRATIC) {
    // both pieces evaluated and selected: no divergence between lanes whose
    // nodes sit at different stencil offsets
    const float ar = fabsf(r);
    const float t = 1.5f - ar;
    const float n_in = 0.75f - r * r, dn_in = inv_h * (-2.0f * r);
    const float n_out = 0.5f * t * t, dn_out = inv_h * (r > 0.0f ? -t : t);
    const bool inner = ar < 0.5f, outer = ar < 1.5f;
    N = inner ? n_in : (outer ? n_out : 0.0f);
    dN = inner ? dn_in : (outer ? dn_out : 0.0f);
  } else {
    int k = -1;
    if (r >= -2.0f && r < -1.0f)
      k = 0;
    else if (r >= -1.0f && r < 0.0f)
      k = 1;
    else if (r >= 0.0f && r < 1.0f)
      k = 2;
    else if (r >= 1.0f && r < 2.0f)
      k = 3;
    if (k < 0) {
      N = 0.0f;
      dN = 0.0f;
    } else {
      const float *c = kCubicW[type][k];
      const float *d = kCubicD[type][k];
      N = ((c[0] * r + c[1]) * r + c[2]) * r + c[3];
      dN = inv_h * ((d[0] * r + d[1]) * r + d[2]);
    }
  }
}

// Stencil geometry per shape function: window width and first offset in the
// reference slot tables (src/common/global_settings.cpp:108-150); the
// quadratic B-spline has three non-zero nodes per axis inside that window.
template <int SF>
struct Stencil;
template <>
struct Stencil<PMPM_SHAPE_LINEAR> {
  static constexpr int WIN = 2, WLO = 0, K = 2;
};
template <>
struct Stencil<PMPM_SHAPE_QUADRATIC> {
  static constexpr int WIN = 4, WLO = -1, K = 3;
};
template <>
struct Stencil<PMPM_SHAPE_CUBIC> {
  static constexpr int WIN = 4, WLO = -1, K = 4;
};

// Window offset of reference slot `sid` (2D x-fastest; 3D z-fastest, then x,
// then y).
template <int D, int SF>
__device__ __forceinline__ void window_offset(int sid, int w[3]) {
  constexpr int W = Stencil<SF>::WIN, LO = Stencil<SF>::WLO;
  w[0] = w[1] = w[2] = 0;
  if (D == 2) {
    w[0] = LO + sid % W;
    w[1] = LO + sid / W;
  } else {
    w[2] = LO + sid % W;
    w[0] = LO + (sid / W) % W;
    w[1] = LO + sid / (W * W);
  }
}

// --------------------------------------------------------------------------
// symmetric tensor helpers
// --------------------------------------------------------------------------

// index of (a,b) in the symmetric stress storage
template <int D>
__device__ __forceinline__ int sig_index(int a, int b) {
  if (D == 2) {
    if (a == b) return a == 2 ? 3 : a;
    if (a + b == 1) return 2;  // xy
    return -1;                 // xz / yz are not stored in 2D
  } else {
    if (a == b) return a;
    int s = a + b;  // 1: xy, 2: xz, 3: yz
    return 2 + s;
  }
}
template <int D>
__device__ __forceinline__ int eps_index(int a, int b) {
  if (D == 2) {
    if (a == b) return a;
    return 2;
  } else {
    if (a == b) return a;
    return 2 + a + b;
  }
}

template <int D>
__device__ __forceinline__ void load_sig3(const DevParticles &P, int s, float S[9]) {
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      int k = sig_index<D>(a, b);
      S[3 * a + b] = k < 0 ? 0.0f : P.sig[k * P.stride + s];
    }
}
template <int D>
__device__ __forceinline__ void store_sig3(const DevParticles &P, int s, const float S[9]) {
  if (D == 2) {
    P.sig[0 * P.stride + s] = S[0];
    P.sig[1 * P.stride + s] = S[4];
    P.sig[2 * P.stride + s] = S[1];
    P.sig[3 * P.stride + s] = S[8];
  } else {
    P.sig[0 * P.stride + s] = S[0];
    P.sig[1 * P.stride + s] = S[4];
    P.sig[2 * P.stride + s] = S[8];
    P.sig[3 * P.stride + s] = S[1];
    P.sig[4 * P.stride + s] = S[2];
    P.sig[5 * P.stride + s] = S[5];
  }
}

// --------------------------------------------------------------------------
// materials (per point)
// --------------------------------------------------------------------------

// update_linearelastic (src/materials/linearelastic_inline.h:40-107):
// deps = sym(L) dt; sigma_DIM += lame*deps + 2G*deps (the reference's matrix
// product lame*deps*I); corrected: lame tr(deps) I + 2G deps (+ plane strain zz).
template <int D>
__device__ __forceinline__ void le_update(const DevMaterial &mt, const float *L, float dt, float S[9]) {
  float lame = mt.p[2], two_g = 2.0f * mt.p[3];
  bool corrected = mt.p[5] != 0.0f;
  float deps[9];
  float tr = 0.0f;
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) deps[a * D + b] = (0.5f * (L[a * D + b] + L[b * D + a])) * dt;
#pragma unroll
  for (int a = 0; a < D; a++) tr += deps[a * D + a];
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) {
      float e = deps[a * D + b];
      float inc = corrected ? ((a == b ? lame * tr : 0.0f) + two_g * e) : (lame * e + two_g * e);
      S[3 * a + b] += inc;
    }
  if (corrected && D == 2) S[8] += lame * tr;
}

// stress_update_newtonfluid (src/materials/newtonfluid_inline.h:49-96):
// pressure from the Tait law on rho/rho0 = V0/V; deviator (2 mu / 3) dev(D).
template <int D>
__device__ __forceinline__ void nf_update(const DevMaterial &mt, const float *L, float mass, float vol,
                                          float vol0, float S[9]) {
  float visc = mt.p[0], bulk = mt.p[1], gamma = mt.p[2];
  float rho = mass / vol, rho0 = mass / vol0;
  float pressure = -bulk * (powf(rho / rho0, gamma) - 1.0f);
  float Dm[9];
  float tr = 0.0f;
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) Dm[a * D + b] = 0.5f * (L[a * D + b] + L[b * D + a]);
#pragma unroll
  for (int a = 0; a < D; a++) tr += Dm[a * D + a];
  const float third = 1.0f / 3.0f;
  (void)visc;
  const float c2 = mt.p[3];  // 2 mu / 3, computed on the host in FP64 and rounded
#pragma unroll
  for (int k = 0; k < 9; k++) S[k] = 0.0f;
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) {
      float dev = Dm[a * D + b] - (a == b ? third * tr : 0.0f);
      S[3 * a + b] = (a == b ? pressure : 0.0f) + dev * c2;
    }
}

// Drucker-Prager cone/apex return mapping: update_dp_rheo
// (src/materials/dp_rheo_inline.h:123-246), return_mapping_cone (:50-65),
// return_mapping_apex (:67-78), update_plasticity (:80-96).  eps (D x D,
// full) and sref (3 x 3) are local copies; the yield function is
// sqrt(J2) + eta p - kc, the apex return sets s = 0 and p = p_apex.
// Scalars of the return are evaluated in FP64 as in the reference.
template <int D>
__device__ __forceinline__ void dp_update(const float *prm, const float *L, float dt, float eps[9],
                                          const float sref[9], float S[9], bool velgrad_is_increment) {
  const float K = prm[0], G = prm[1], eta = prm[2], eta_bar = prm[3], kc = prm[4], p_apex = prm[5];
  const bool has_apex = prm[6] != 0.0f;
  float deps[9];
  if (velgrad_is_increment) {
#pragma unroll
    for (int k = 0; k < D * D; k++) deps[k] = L[k];
  } else {
    float W[9];
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int b = 0; b < D; b++) {
        deps[a * D + b] = (0.5f * (L[a * D + b] + L[b * D + a])) * dt;
        W[a * D + b] = (0.5f * (L[a * D + b] - L[b * D + a])) * dt;
      }
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int b = 0; b < D; b++) {
        float we = 0.0f, ew = 0.0f;
#pragma unroll
        for (int k = 0; k < D; k++) {
          we += W[a * D + k] * eps[k * D + b];
          ew += eps[a * D + k] * W[k * D + b];
        }
        deps[a * D + b] += -we + ew;
      }
  }
  const float p_ref = (1.0f / 3.0f) * ((sref[0] + sref[4]) + sref[8]);
  float s_ref[9];
#pragma unroll
  for (int k = 0; k < 9; k++) s_ref[k] = sref[k];
  s_ref[0] -= p_ref;
  s_ref[4] -= p_ref;
  s_ref[8] -= p_ref;
  float eps_tr[9];
#pragma unroll
  for (int k = 0; k < D * D; k++) eps_tr[k] = eps[k] + deps[k];
  float ev = 0.0f;
#pragma unroll
  for (int a = 0; a < D; a++) ev += eps_tr[a * D + a];
  const float p_tr = p_ref + K * ev;
  float edev[9];
#pragma unroll
  for (int k = 0; k < 9; k++) edev[k] = 0.0f;
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) edev[3 * a + b] = eps_tr[a * D + b];
  const float third_ev = (1.0f / 3.0f) * ev;
#pragma unroll
  for (int a = 0; a < 3; a++) edev[3 * a + a] -= third_ev;
  if (D < 3) edev[8] = 0.0f;
  const float two_g = 2.0f * G;
  float s_tr[9];
  float ss = 0.0f;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    s_tr[k] = s_ref[k] + two_g * edev[k];
    ss += s_tr[k] * s_tr[k];
  }
  const float J2 = 0.5f * ss;
  const float sqrtJ2 = sqrtf(J2);
  const float Phi = (sqrtJ2 + eta * p_tr) - kc;
  if (Phi <= 0.0f) {
#pragma unroll
    for (int k = 0; k < 9; k++) S[k] = s_tr[k];
    S[0] += p_tr;
    S[4] += p_tr;
    S[8] += p_tr;
#pragma unroll
    for (int k = 0; k < D * D; k++) eps[k] = eps_tr[k];
    return;
  }
  const double dgamma = (double)Phi / ((double)K * (double)eta * (double)eta_bar + (double)G);
  double p_next = (double)p_tr - (double)K * (double)eta_bar * dgamma;
  float s_next[9];
  const bool apex = has_apex && ((double)sqrtJ2 - (double)G * dgamma < 0.0);
  if (apex) {
    p_next = (double)p_apex;
#pragma unroll
    for (int k = 0; k < 9; k++) s_next[k] = 0.0f;
  } else {
    const double scale = 1.0 - ((double)G * dgamma) / (double)sqrtJ2;
#pragma unroll
    for (int k = 0; k < 9; k++) s_next[k] = (float)(scale * (double)s_tr[k]);
  }
  const float pn = (float)p_next;
#pragma unroll
  for (int k = 0; k < 9; k++) S[k] = s_next[k];
  S[0] += pn;
  S[4] += pn;
  S[8] += pn;
  const double inv2g = 1.0 / (2.0 * (double)G);
  const float dpk = (float)(((double)pn - (double)p_ref) / (3.0 * (double)K));
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) {
      float e = (float)((double)(s_next[3 * a + b] - s_ref[3 * a + b]) * inv2g);
      if (a == b) e += dpk;
      eps[a * D + b] = e;
    }
}

// Drucker-Prager parameters {K, G, eta, eta_bar, kc, p_apex, has_apex} of one
// particle from its Young's modulus E and friction angle phi (degrees), with
// the material's Poisson ratio (p[7]), dilatancy (eta_bar, p[3]) and
// cohesion (p[8]): the outer-cone fit of pmpm_material_drucker_prager.
__device__ __forceinline__ void dp_particle_params(const DevMaterial &mt, float E, float phi_deg, float prm[8]) {
  const float nu = mt.p[7], c = mt.p[8];
  const float phi = phi_deg * 0.017453292519943295f;
  const float sn = sinf(phi), cs = cosf(phi);
  const float den = 1.7320508075688772f * (3.0f - sn);
  const float eta = 6.0f * sn / den, xi = 6.0f * cs / den;
  prm[0] = E / (3.0f * (1.0f - 2.0f * nu));
  prm[1] = E / (2.0f * (1.0f + nu));
  prm[2] = eta;
  prm[3] = mt.p[3];
  prm[4] = xi * c;
  prm[5] = eta > 0.0f ? prm[4] / eta : 0.0f;
  prm[6] = eta > 0.0f ? 1.0f : 0.0f;
  prm[7] = nu;
}

// update_vonmises (src/materials/vonmises_inline.h:36-120), 3D: elastic
// strain eps (3x3, updated), accumulated plastic strain acc (updated), stress
// S (written).  deps = sym(L) dt; trial p = K tr(eps_tr), s = 2G dev(eps_tr);
// Phi = sqrt(3/2 s:s) - (sigma_y + H acc); the reference's Newton iteration
// on dgamma (in double, |Phi| <= 1e-7) with acc taken before the last update.
__device__ __forceinline__ void vm_update(const float *prm, const float *L, float dt, float eps[9], float &acc,
                                          float S[9]) {
  const float K = prm[0], G = prm[1], sy0 = prm[2], H = prm[3];
  float eps_tr[9];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) eps_tr[3 * a + b] = eps[3 * a + b] + (0.5f * (L[3 * a + b] + L[3 * b + a])) * (float)dt;
  const float ev = (eps_tr[0] + eps_tr[4]) + eps_tr[8];
  const float p = K * ev;
  float s[9], ss = 0.0f;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    float e = eps_tr[k];
    if (k == 0 || k == 4 || k == 8) e -= (1.0f / 3.0f) * ev;
    s[k] = 2.0f * G * e;
    ss += s[k] * s[k];
  }
  const float sy = sy0 + H * acc;
  const float q = sqrtf(1.5f * ss);
  const float Phi = q - sy;
  if (Phi <= 0.0f) {
#pragma unroll
    for (int k = 0; k < 9; k++) {
      S[k] = s[k] + ((k == 0 || k == 4 || k == 8) ? p : 0.0f);
      eps[k] = eps_tr[k];
    }
    return;
  }
  double dgamma = 0.0, acc_eps = acc;
  for (int it = 0; it < 100; it++) {
    acc_eps = (double)acc + dgamma;
    const double syi = (double)sy0 + (double)H * acc_eps;
    const double phi = (double)q - 3.0 * (double)G * dgamma - syi;
    dgamma = dgamma - phi / (-3.0 * (double)G - (double)H);
    if (!(fabs(phi) > 1e-7)) break;
  }
  const double fac = 1.0 - (3.0 * (double)G * dgamma) / (double)q;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const float sc = (float)(fac * (double)s[k]);
    const bool diag = k == 0 || k == 4 || k == 8;
    S[k] = sc + (diag ? p : 0.0f);
    eps[k] = (float)((double)sc / (2.0 * (double)G) + (diag ? (1.0 / 3.0) * (double)ev : 0.0));
  }
  acc = (float)acc_eps;
}

// Small-strain increment of the co-rotational stress updates
// (src/materials/modifiedcamclay_inline.h:350-362, dp_rheo_inline.h:155-161):
// deps = sym(L) dt - W eps + eps W with W = skew(L) dt (D x D).
template <int D>
__device__ __forceinline__ void corotational_increment(const float *L, float dt, const float eps[9], float deps[9]) {
  float W[9];
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) {
      deps[a * D + b] = (0.5f * (L[a * D + b] + L[b * D + a])) * dt;
      W[a * D + b] = (0.5f * (L[a * D + b] - L[b * D + a])) * dt;
    }
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) {
      float we = 0.0f, ew = 0.0f;
#pragma unroll
      for (int k = 0; k < D; k++) {
        we += W[a * D + k] * eps[k * D + b];
        ew += eps[a * D + k] * W[k * D + b];
      }
      deps[a * D + b] += -we + ew;
    }
}

// Modified Cam Clay with pressure-dependent elasticity:
// update_modifiedcamclay_nonlinear (src/materials/modifiedcamclay_inline.h:
// 321-511), yield function compute_yield_function (:57-63).  Pressures are
// positive in compression.  V is the particle's current volume (specific
// volume V / Vs), S holds the previous stress on entry and the new one on
// exit, eps the D x D elastic strain, alpha the volumetric plastic strain,
// pc the preconsolidation pressure.
//   trial: p = p_prev / (1 - (v/kap) dev_e), s = dev(sref) + 2G dev(eps + deps)
//   (zz deviator zeroed in 2D), q = sqrt(3/2 s:s);
//   yield f = (p_s - p - Pt)^2 + (q/M)^2 - p_s^2 with p_s = (pc + Pt)/2;
//   plastic: Newton on (lambda, alpha) with the reference's residuals and
//   its 2 x 2 iteration matrix (which takes dp/dalpha as -K), until
//   |R| <= 1e-2, the bound growing tenfold per iteration after 1000.  The
//   iteration runs in FP64 (the reference mixes FP32 and FP64 there; with
//   FP32 residuals it needs the growing bound to stop); stress, strain and
//   pc come from the last evaluated iterate, alpha from the updated one.
__device__ __forceinline__ float mcc_yield(float p, float Pt, float ps, float q, float M) {
  return (ps - p - Pt) * (ps - p - Pt) + (q / M) * (q / M) - ps * ps;
}

template <int D>
__device__ __forceinline__ void mcc_update(const float *prm, const float *L, float dt, float V, float eps[9],
                                           const float sref[9], float S[9], float &alpha, float &pc) {
  const float K = prm[0], G = prm[1], M = prm[2], lam = prm[3], kap = prm[4], Vs = prm[5], Pt = prm[6];
  float deps[9];
  corotational_increment<D>(L, dt, eps, deps);
  const float p_ref = -(1.0f / 3.0f) * ((sref[0] + sref[4]) + sref[8]);
  float s_ref[9];
#pragma unroll
  for (int k = 0; k < 9; k++) s_ref[k] = sref[k];
  s_ref[0] += p_ref;
  s_ref[4] += p_ref;
  s_ref[8] += p_ref;
  float eps_tr[9], tr_prev = 0.0f, tr_inc = 0.0f, tr_tr = 0.0f;
#pragma unroll
  for (int k = 0; k < D * D; k++) eps_tr[k] = eps[k] + deps[k];
#pragma unroll
  for (int a = 0; a < D; a++) {
    tr_prev += eps[a * D + a];
    tr_inc += deps[a * D + a];
    tr_tr += eps_tr[a * D + a];
  }
  const float ev_tr = -tr_tr;
  float edev[9];
#pragma unroll
  for (int k = 0; k < 9; k++) edev[k] = 0.0f;
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) edev[3 * a + b] = eps_tr[a * D + b];
#pragma unroll
  for (int a = 0; a < 3; a++) edev[3 * a + a] += (1.0f / 3.0f) * ev_tr;
  if (D < 3) edev[8] = 0.0f;
  const float v_spec = V / Vs;
  const float p_prev = -((S[0] + S[4]) + S[8]) / 3.0f;
  const float v_kap = v_spec / kap;
  const float dev_tr = -tr_inc;
  const float p_tr = p_prev / (1.0f - v_kap * dev_tr);
  float s_tr[9], ss = 0.0f;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    s_tr[k] = s_ref[k] + 2.0f * G * edev[k];
    ss += s_tr[k] * s_tr[k];
  }
  const float q_tr = sqrtf(1.5f * ss);
  const float pc_prev = pc;
  const float f_tr = mcc_yield(p_tr, Pt, 0.5f * (pc_prev + Pt), q_tr, M);
  if (f_tr <= 0.0f) {
#pragma unroll
    for (int k = 0; k < 9; k++) S[k] = s_tr[k] - ((k == 0 || k == 4 || k == 8) ? p_tr : 0.0f);
#pragma unroll
    for (int k = 0; k < D * D; k++) eps[k] = eps_tr[k];
    return;
  }
  const double Kd = K, Gd = G, Md = M, MM = Md * Md, Ptd = Pt, pcd = pc_prev, a_prev = alpha;
  const double vlt = (double)v_spec / ((double)lam - (double)kap);
  double lamb = 0.0, a_next = a_prev, tol = 1e-2;
  double p = p_tr, c = 1.0, ps = 0.5 * (pcd + Ptd), dev_e = dev_tr;
  for (int it = 0; it < 1400; it++) {
    const double dpv = a_next - a_prev;
    dev_e = (double)dev_tr - dpv;
    p = (double)p_prev / (1.0 - (double)v_kap * dev_e);
    c = MM / (MM + 6.0 * Gd * lamb);
    const double q = c * (double)q_tr;
    ps = 0.5 * (pcd * (1.0 + vlt * dpv) + Ptd);
    const double pbar = ps - p - Ptd;
    const double R0 = pbar * pbar + (q / Md) * (q / Md) - ps * ps;
    const double R1 = dpv + 2.0 * lamb * pbar;
    const double omv = 1.0 - vlt * dpv;
    const double H = 0.5 * vlt * (pcd / (omv * omv));
    const double d00 = (-12.0 * Gd / (MM + 6.0 * Gd * lamb)) * (q / Md) * (q / Md);
    const double d01 = 2.0 * pbar * (Kd + H) - 2.0 * ps * H;
    const double d10 = 2.0 * pbar;
    const double d11 = 1.0 + 2.0 * lamb * (Kd + H);
    const double det = d00 * d11 - d01 * d10;
    lamb -= (d11 * R0 - d01 * R1) / det;
    a_next -= (d00 * R1 - d10 * R0) / det;
    const double conv = sqrt(R0 * R0 + R1 * R1);
    if (it > 1000) tol *= 10.0;
    if (!(conv > tol)) break;
  }
  const float cf = (float)c, pn = (float)p;
  const float two_g = (float)(2.0 * Gd);
  const float evol = (float)((1.0 / 3.0) * ((double)tr_prev + dev_e));
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const float sk = cf * s_tr[k];
    S[k] = sk - ((k == 0 || k == 4 || k == 8) ? pn : 0.0f);
    s_tr[k] = sk;
  }
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) eps[a * D + b] = (s_tr[3 * a + b] - s_ref[3 * a + b]) / two_g - (a == b ? evol : 0.0f);
  alpha = (float)a_next;
  pc = (float)(2.0 * ps - Ptd);
}

// Drucker-Prager cone with a cap: update_druckerpragercap
// (src/materials/druckerprager_cap_inline.h:370-554) with return_mapping_cone
// (:124-141), return_mapping_apex (:143-156), return_mapping_cap (:159-235),
// compute_pc / compute_a / compute_b (:56-84), the yield functions (:94-111)
// and update_plasticity (:328-346).  Pressure p = tr(sigma)/3 (tension
// positive).  Cone: sqrt(J2) + eta (p - Pt), eta = M / sqrt(3); cap:
// (p - Pt + a)^2 / b^2 + (q/M)^2 - a^2 with a = (pc + Pt) / (1 + beta) and
// b = beta beyond the cap's centre (p < Pt - a), else 1; hardening
// pc = pc_prev exp(v0 / (lam - kap) (alpha - alpha_prev)), v0 = V0 / Vs.
// The cone return is closed form; past the apex the stress goes to p = Pt,
// s = 0 (the apex's eta_bar dgamma is (p_tr - Pt) / K; the reference divides
// by eta_bar and multiplies back, which is 0/0 for eta_bar = 0, where this
// keeps the limit).  The cap return is the reference's Newton iteration on
// (dgamma, alpha) from the trial state, in FP64, until |R| <= 0.1 with the
// bound growing tenfold per iteration after 1000; its results are the last
// evaluated iterate's.  V0: the particle's original volume.
template <int D>
__device__ __forceinline__ void dpc_update(const float *prm, const float *L, float dt, float V0, float eps[9],
                                           const float sref[9], float S[9], float &alpha, float &pc) {
  const float K = prm[0], G = prm[1], M = prm[2], lam = prm[3], kap = prm[4], Vs = prm[5], Pt = prm[6];
  const float beta = prm[8], eta_bar = prm[9];
  float deps[9];
  corotational_increment<D>(L, dt, eps, deps);
  const float p_ref = (1.0f / 3.0f) * ((sref[0] + sref[4]) + sref[8]);
  float s_ref[9];
#pragma unroll
  for (int k = 0; k < 9; k++) s_ref[k] = sref[k];
  s_ref[0] -= p_ref;
  s_ref[4] -= p_ref;
  s_ref[8] -= p_ref;
  float eps_tr[9], ev = 0.0f;
#pragma unroll
  for (int k = 0; k < D * D; k++) eps_tr[k] = eps[k] + deps[k];
#pragma unroll
  for (int a = 0; a < D; a++) ev += eps_tr[a * D + a];
  const float p_tr = p_ref + K * ev;
  float edev[9];
#pragma unroll
  for (int k = 0; k < 9; k++) edev[k] = 0.0f;
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) edev[3 * a + b] = eps_tr[a * D + b];
#pragma unroll
  for (int a = 0; a < 3; a++) edev[3 * a + a] -= (1.0f / 3.0f) * ev;
  if (D < 3) edev[8] = 0.0f;
  float s_tr[9], ss = 0.0f;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    s_tr[k] = s_ref[k] + 2.0f * G * edev[k];
    ss += s_tr[k] * s_tr[k];
  }
  const float J2 = 0.5f * ss;
  const float q_tr = sqrtf(3.0f * J2);
  const float sqrtJ2 = sqrtf(J2);
  const float eta = 0.57735026918962576f * M;
  const float phi_cone = sqrtJ2 + eta * (p_tr - Pt);
  const double C = ((double)V0 / (double)Vs) / ((double)lam - (double)kap);
  const float a_tr = (pc + Pt) / (1.0f + beta);
  const float b_tr = p_tr < Pt - a_tr ? beta : 1.0f;
  const float phi_cap =
      (float)((1.0 / ((double)b_tr * b_tr)) * (double)(p_tr - Pt + a_tr) * (double)(p_tr - Pt + a_tr) +
              (double)((q_tr / M) * (q_tr / M)) - (double)(a_tr * a_tr));
  if (phi_cone <= 0.0f && phi_cap <= 0.0f) {
#pragma unroll
    for (int k = 0; k < 9; k++) S[k] = s_tr[k] + ((k == 0 || k == 4 || k == 8) ? p_tr : 0.0f);
#pragma unroll
    for (int k = 0; k < D * D; k++) eps[k] = eps_tr[k];
    return;
  }
  const double Kd = K, Gd = G, Md = M, MM = Md * Md, Ptd = Pt, a_prev = alpha, pc_prev = pc;
  double p = p_tr, pcn = pc_prev, an = a_tr, al = a_prev;
  float s[9];
#pragma unroll
  for (int k = 0; k < 9; k++) s[k] = s_tr[k];
  bool done = false;
  if (phi_cone > 0.0f) {
    const double dg = (double)phi_cone / (Kd * (double)eta * (double)eta_bar + Gd);
    if ((double)sqrtJ2 - Gd * dg < 0.0) {
      const double edg = ((double)p_tr - Ptd) / Kd;
      al = a_prev - edg;
      p = (double)p_tr - Kd * edg;
#pragma unroll
      for (int k = 0; k < 9; k++) s[k] = 0.0f;
      pcn = exp(C * (al - a_prev)) * pc_prev;
      done = true;
    } else {
      al = a_prev - (double)eta_bar * dg;
      p = (double)p_tr - Kd * (double)eta_bar * dg;
      const float sc = (float)(1.0 - (Gd * dg) / (double)sqrtJ2);
#pragma unroll
      for (int k = 0; k < 9; k++) s[k] = sc * s_tr[k];
      pcn = exp(C * (al - a_prev)) * pc_prev;
      an = (pcn + Ptd) / (1.0 + (double)beta);
    }
  }
  if (!done && phi_cap > 0.0f && p < an) {
    double dgam = 0.0, alv = a_prev, tol = 0.1;
    for (int it = 1; it <= 1400; it++) {
      al = alv;
      p = (double)p_tr + Kd * (al - a_prev);
      const double c = MM / (MM + 6.0 * Gd * dgam);
      const double q = c * (double)q_tr;
      pcn = exp(C * (al - a_prev)) * pc_prev;
      an = (pcn + Ptd) / (1.0 + (double)beta);
      const double b = p < Ptd - an ? (double)beta : 1.0;
      const float cf = (float)c;
#pragma unroll
      for (int k = 0; k < 9; k++) s[k] = cf * s_tr[k];
      const double pbar = p - Ptd + an;
      const double R0 = pbar * pbar / (b * b) + (q / Md) * (q / Md) - an * an;
      const double R1 = al - a_prev + dgam * (2.0 / (b * b)) * pbar;
      const double H = pcn * C / (1.0 + (double)beta);
      const double d00 = (-12.0 * Gd / (MM + 6.0 * Gd * dgam)) * (q / Md) * (q / Md);
      const double d01 = (2.0 * pbar / (b * b)) * (Kd + H) - 2.0 * an * H;
      const double d10 = 2.0 * pbar / (b * b);
      const double d11 = 1.0 + (2.0 * dgam / (b * b)) * (Kd + H);
      const double det = d00 * d11 - d01 * d10;
      dgam -= (d11 * R0 - d01 * R1) / det;
      alv -= (d00 * R1 - d10 * R0) / det;
      const double conv = sqrt(R0 * R0 + R1 * R1);
      if (it > 1000) tol *= 10.0;
      if (!(conv > tol)) break;
    }
  }
  const float pn = (float)p;
  const float dpk = (float)((p - (double)p_ref) / (3.0 * Kd));
  const float two_g = (float)(2.0 * Gd);
#pragma unroll
  for (int k = 0; k < 9; k++) S[k] = s[k] + ((k == 0 || k == 4 || k == 8) ? pn : 0.0f);
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) eps[a * D + b] = (s[3 * a + b] - s_ref[3 * a + b]) / two_g + (a == b ? dpk : 0.0f);
  alpha = (float)al;
  pc = (float)pcn;
}

// --------------------------------------------------------------------------
// node epilogue: P2G result -> boundary conditions -> velocities
// --------------------------------------------------------------------------

// Writes one node's final values: mass, moments, forward moments and the
// packed velocities (0 where the mass is at or below the cutoff, which G2P
// then adds as zero, as the reference skips those nodes).
template <int D>
__device__ __forceinline__ void write_node(const StepArgs &a, int node, float mass, const float p[3],
                                           const float pnt[3], bool live) {
  const int nt = a.g.ntotal;
  a.N.m[node] = mass;
  float v[3] = {0.0f, 0.0f, 0.0f}, vn[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int c = 0; c < D; c++) {
    a.N.p[c * nt + node] = p[c];
    a.N.pnt[c * nt + node] = pnt[c];
    v[c] = live ? p[c] / mass : 0.0f;
    vn[c] = live ? pnt[c] / mass : 0.0f;
  }
  float4 *vel = reinterpret_cast<float4 *>(a.N.vel);
  if (D == 3) {
    vel[2 * (size_t)node] = make_float4(v[0], v[1], v[2], 0.0f);
    vel[2 * (size_t)node + 1] = make_float4(vn[0], vn[1], vn[2], 0.0f);
  } else {
    vel[node] = make_float4(v[0], v[1], vn[0], vn[1]);
  }
}

// Analytic rigid body of a PMPM_BC_RIGID_SDF condition: signed distance of
// world point x and the outward unit normal there.  The cross-section plane
// is (P, Q) with P = axis+1, Q = axis+2 (cyclic) in 3D and (x, y) in 2D; the
// body's local frame is turned by its angle about the axis.  Shell: the half
// q <= 0 of the annulus |rho - R| <= t/2 in local coordinates, ends rounded
// with radius t/2, extruded to length L along the axis in 3D.
template <int D>
__device__ __forceinline__ float rigid_sdf(const DevBC &bc, const float x[3], float nrm[3]) {
  const int A = D == 3 ? bc.i[1] : 2;
  const int P = D == 3 ? (A + 1) % 3 : 0, Q = D == 3 ? (A + 2) % 3 : 1;
  float d[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int c = 0; c < D; c++) d[c] = x[c] - bc.r[c];
  nrm[0] = nrm[1] = nrm[2] = 0.0f;
  if (bc.i[0] == PMPM_SDF_SPHERE) {
    float r2 = 0.0f;
#pragma unroll
    for (int c = 0; c < D; c++) r2 += d[c] * d[c];
    const float r = sqrtf(r2);
    if (r > 0.0f) {
#pragma unroll
      for (int c = 0; c < D; c++) nrm[c] = d[c] / r;
    } else {
      nrm[Q] = 1.0f;
    }
    return r - bc.r[8];
  }
  const float cs = bc.r[12], sn = bc.r[13];
  const float lp = cs * d[P] + sn * d[Q], lq = cs * d[Q] - sn * d[P];
  const float R = bc.r[8], ht = 0.5f * bc.r[9];
  float phi2, gp = 0.0f, gq = 1.0f;
  if (lq <= 0.0f) {
    const float rho = sqrtf(lp * lp + lq * lq);
    phi2 = fabsf(rho - R) - ht;
    if (rho > 0.0f) {
      const float sg = rho >= R ? 1.0f : -1.0f;
      gp = sg * lp / rho;
      gq = sg * lq / rho;
    }
  } else {
    const float wp = lp - (lp >= 0.0f ? R : -R), wq = lq;
    const float w = sqrtf(wp * wp + wq * wq);
    phi2 = w - ht;
    if (w > 0.0f) {
      gp = wp / w;
      gq = wq / w;
    }
  }
  float phi = phi2, ga = 0.0f;
  if (D == 3) {
    const float la = d[A];
    const float hA = fabsf(la) - 0.5f * bc.r[10];
    const float sa = la >= 0.0f ? 1.0f : -1.0f;
    if (phi2 > 0.0f && hA > 0.0f) {
      phi = sqrtf(phi2 * phi2 + hA * hA);
      gp = phi2 * gp / phi;
      gq = phi2 * gq / phi;
      ga = hA * sa / phi;
    } else if (hA > phi2) {
      phi = hA;
      gp = gq = 0.0f;
      ga = sa;
    }
  }
  nrm[P] = cs * gp - sn * gq;
  nrm[Q] = sn * gp + cs * gq;
  if (D == 3) nrm[A] = ga;
  return phi;
}

// Coulomb contact of a node's forward moments with an analytic rigid body.
template <int D>
__device__ __forceinline__ void rigid_sdf_contact(const StepArgs &a, const DevBC &bc, const int nc[3], float m,
                                                  float pnt[3]) {
  float x[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int c = 0; c < D; c++) x[c] = __fadd_rn(a.g.origin[c], __fmul_rn((float)nc[c], a.g.h));
  float nrm[3];
  const float phi = rigid_sdf<D>(bc, x, nrm);
  if (!(phi < bc.r[11])) return;
  const int A = D == 3 ? bc.i[1] : 2;
  const int P = D == 3 ? (A + 1) % 3 : 0, Q = D == 3 ? (A + 2) % 3 : 1;
  float vb[3] = {bc.r[3], bc.r[4], bc.r[5]};
  const float w = bc.r[6];
  vb[P] -= w * (x[Q] - bc.r[Q]);
  vb[Q] += w * (x[P] - bc.r[P]);
  float vr[3] = {0.0f, 0.0f, 0.0f};
  float vn = 0.0f;
#pragma unroll
  for (int c = 0; c < D; c++) {
    vr[c] = pnt[c] / m - vb[c];
    vn += vr[c] * nrm[c];
  }
  if (!(vn < 0.0f)) return;
  float vt2 = 0.0f;
#pragma unroll
  for (int c = 0; c < D; c++) {
    vr[c] -= vn * nrm[c];
    vt2 += vr[c] * vr[c];
  }
  const float vt = sqrtf(vt2);
  const float mu = bc.r[7];
  const float scale = vt <= -mu * vn ? 0.0f : 1.0f + mu * vn / vt;
#pragma unroll
  for (int c = 0; c < D; c++) pnt[c] = (vb[c] + vr[c] * scale) * m;
}

// Applies the node boundary conditions in list order to (p, pnt) of node
// `node` with coordinates nc and mass m:
//   Gravity    (src/boundaryconditions/gravity_inline.h:46-63): pnt += g m dt, m > 1e-9
//   NodeDomain (src/boundaryconditions/nodedomain_inline.h:40-87): m > 1e-5;
//              face0 where id < 1, face1 where id >= n-1; mode 0 zeroes both
//              vectors, mode 1 clamps the normal component
//   BodyForce  (src/boundaryconditions/bodyforce_inline.h:41-59): masked nodes;
//              "fixed" sets pnt, other modes add to p
//   rigid SDF  m > 1e-9: Coulomb contact of pnt with the analytic body
template <int D>
__device__ __forceinline__ void node_bcs_range(const StepArgs &a, int node, const int nc[3], float m, float p[3],
                                               float pnt[3], int k0, int k1) {
  for (int k = k0; k < k1; k++) {
    const DevBC &bc = a.bc[k];
    // the MUSL remap carries no forces: only conditions on velocities apply
    if (a.remap && (bc.type == PMPM_BC_GRAVITY || (bc.type == PMPM_BC_BODYFORCE && bc.i[0] != 2))) continue;
    if (bc.type == PMPM_BC_GRAVITY) {
      if (m > 0.000000001f) {
#pragma unroll
        for (int c = 0; c < D; c++) pnt[c] += (bc.r[c] * m) * a.dt;
      }
    } else if (bc.type == PMPM_BC_NODEDOMAIN) {
      if (m > 0.00001f) {
#pragma unroll
        for (int c = 0; c < D; c++) {
          if (nc[c] < 1) {
            if (bc.i[c] == 0) {
#pragma unroll
              for (int e = 0; e < D; e++) p[e] = pnt[e] = 0.0f;
            } else if (bc.i[c] == 1) {
              p[c] = fmaxf(0.0f, p[c]);
              pnt[c] = fmaxf(0.0f, pnt[c]);
            }
          } else if (nc[c] >= a.g.n[c] - 1) {
            if (bc.i[3 + c] == 0) {
#pragma unroll
              for (int e = 0; e < D; e++) p[e] = pnt[e] = 0.0f;
            } else if (bc.i[3 + c] == 1) {
              p[c] = fminf(0.0f, p[c]);
              pnt[c] = fminf(0.0f, pnt[c]);
            }
          }
        }
      }
    } else if (bc.type == PMPM_BC_BODYFORCE) {
      if (bc.i[1] && bc.mask[node]) {
        if (bc.i[0] == 2) {
#pragma unroll
          for (int c = 0; c < D; c++) pnt[c] = bc.values[(size_t)node * D + c];
        } else {
#pragma unroll
          for (int c = 0; c < D; c++) p[c] += bc.values[(size_t)node * D + c];
        }
      }
    } else if (bc.type == PMPM_BC_RIGID_SDF) {
      if (m > 0.000000001f) rigid_sdf_contact<D>(a, bc, nc, m, pnt);
    }
  }
}

// The node boundary conditions of the P2G epilogue: the list up to the first
// nearest-rigid-particle RigidBodyLevelSet, which needs the finished grid.
template <int D>
__device__ __forceinline__ void node_bcs(const StepArgs &a, int node, const int nc[3], float m, float p[3],
                                         float pnt[3]) {
  node_bcs_range<D>(a, node, nc, m, p, pnt, 0, a.nbc_epi);
}

}  // namespace pmpm
