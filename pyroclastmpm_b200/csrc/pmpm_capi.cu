// Host side of the C ABI (include/pmpm.h): handle lifetime, device memory,
// field conversion between the reference layouts and the SoA device layout,
// and the launch sequence of one USL step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

#include "pmpm.h"
#include "pmpm_adjoint.cuh"
#include "pmpm_kernels.cuh"

using namespace pmpm;

namespace {

constexpr int kTPB = 256;

inline int blocks_for(long long n, int tpb = kTPB) { return (int)((n + tpb - 1) / tpb); }

#define PMPM_CUDA(call)                                                                   \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      fprintf(stderr, "pmpm: CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                                  \
      return PMPM_ERR_CUDA;                                                               \
    }                                                                                     \
  } while (0)

#define PMPM_LAUNCHED()                                                                   \
  do {                                                                                    \
    cudaError_t e_ = cudaGetLastError();                                                  \
    if (e_ != cudaSuccess) {                                                              \
      fprintf(stderr, "pmpm: launch error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                                  \
      return PMPM_ERR_CUDA;                                                               \
    }                                                                                     \
  } while (0)

#define PMPM_TRY(expr)        \
  do {                        \
    int st_ = (expr);         \
    if (st_ != PMPM_OK) return st_; \
  } while (0)

template <typename T>
int dalloc(T **p, size_t count) {
  *p = nullptr;
  if (count == 0) return PMPM_OK;
  cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
  if (e == cudaErrorMemoryAllocation) return PMPM_ERR_OUT_OF_MEMORY;
  PMPM_CUDA(e);
  return PMPM_OK;
}

template <typename T>
void dfree(T *&p) {
  if (p) cudaFree((void *)p);
  p = nullptr;
}

// Single-pass key scan state: per-chunk tagged status words and the ticket
// counters of alternate launches (both zeroed once at allocation).
struct ScanState {
  unsigned long long *status = nullptr;
  int *ticket = nullptr;
  unsigned launches = 0;
  long long spin_limit = 1ll << 22;  // look-back polls before a CTA gives up
};

unsigned scan_tag(unsigned launch) { return launch % 0x3ffffffeu + 1u; }

int alloc_scan(ScanState &sc, int nblocks) {
  PMPM_TRY(dalloc(&sc.status, (size_t)nblocks));
  PMPM_TRY(dalloc(&sc.ticket, 2));
  PMPM_CUDA(cudaMemset(sc.status, 0, sizeof(unsigned long long) * nblocks));
  PMPM_CUDA(cudaMemset(sc.ticket, 0, 2 * sizeof(int)));
  return PMPM_OK;
}

void free_scan(ScanState &sc) {
  dfree(sc.status);
  dfree(sc.ticket);
}

// count -> offset (exclusive), counts cleared, scalars reset; one launch
int launch_scan(ScanState &sc, int *count, int nkeys, int *offset, int *scalars, int *fault, int nblocks,
                cudaStream_t st) {
  // 30-bit tag, never 0 (zeroed status words carry no tag); the modulus is
  // even so that consecutive launches always alternate the tag's parity,
  // which selects the ticket counter (each launch resets the other one)
  const unsigned tag = scan_tag(sc.launches);
  sc.launches += 1;
  k_scan_onepass<<<nblocks, kScanThreads, 0, st>>>(count, nkeys, offset, sc.status, sc.ticket, scalars, fault, tag,
                                                   nblocks, sc.spin_limit);
  PMPM_LAUNCHED();
  return PMPM_OK;
}

struct GravityState {
  int bc_index;
  float current[3];
};

// RigidBodyLevelSet in the reference's mode: animation state of
// RigidBodyLevelSet::update_animation (src/boundaryconditions/rigidbodylevelset.cpp:127-206).
struct RigidState {
  int mode = PMPM_RIGID_STATIC, corrected = 0;
  float rate[3] = {0, 0, 0};   // euler_angles_per_second
  float com[3] = {0, 0, 0};
  float euler[3] = {0, 0, 0};  // accumulated euler angles
};

// Analytic rigid body: pose at step 0 and its motion.
struct SdfState {
  int bc_index;
  double c0[3], v[3], omega, angle0;
};

}  // namespace

struct pmpm_sim {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int dim = 2, shape = 0;
  DevGrid g{};
  float dt = 0, alpha = 0.99f;
  int ppc = 1;
  unsigned flags = 0;
  int resort_interval = 32;
  std::vector<DevMaterial> mats;
  std::vector<DevBC> bcs;
  std::vector<float *> bc_values;
  std::vector<uint8_t *> bc_masks;
  std::vector<GravityState> gravity;
  int rbls_index = -1;  // the nearest-rigid-particle RigidBodyLevelSet in the BC list
  RigidState rigid;
  std::vector<SdfState> sdf;
  bool rigid_shift_pending = false;  // the next G2P moves rigid particles by their set velocity
  float *musl_x = nullptr;           // MUSL: new positions between the two G2P passes
  int remap_now = 0, musl_pass_now = 0;
  // differentiable rollout: checkpoints of the particle state (storage-slot
  // order, so the physical re-sort is off while a rollout is held)
  struct Rollout {
    int every = 0, nsteps = 0, start_step = 0;
    std::vector<float *> ckpt;
    float *seg = nullptr;
    int seg_states = 0;
    char *seg_nodes = nullptr;  // node data of each segment step's P2G
    std::vector<int> seg_epoch;
    // segments kept whole from the forward pass (no recompute), as memory allows
    long long budget = -1;  // bytes for kept segments; < 0: 60 % of free device memory
    std::vector<float *> keep_state;
    std::vector<char *> keep_nodes;
    std::vector<std::vector<int>> keep_epoch;
    size_t keep_per = 0, keep_nodeb = 0;
    int keep_every = 0;
    AdjState A{};
    bool held = false;
  } ro;
  bool has_planar = false, has_dp = false, has_sref = false;
  bool has_vm = false;  // a VonMises material: elastic strain and accumulated plastic strain
  bool has_mcc = false; // a Modified Cam Clay or Drucker-Prager cap material: elastic strain, alpha, pc

  // particles (two storage sets, swapped by the physical re-sort)
  int n = 0, stride = 0;
  DevParticles P[2]{};
  int cur = 0;
  int *slot = nullptr;
  // nodes
  DevNodes N{};
  int *node_epoch = nullptr;  // epoch of the P2G that last wrote each tile
  // bins
  DevBins B{};
  int nscan_blocks = 0;
  ScanState scan;
  bool dual = false;  // quadratic 3D fast path bins by dual cell
  int kd[3] = {1, 1, 1};
  int nkeys = 0;
  int nbricks = 0;     // dual-cell bricks (cell-scatter P2G)
  int p2g_variant = 1; // 3D quadratic: 0 cell scatter, 1 dual sweep (pmpm_autotune picks)
  bool dual3_fits = true;  // every dual-sweep tile's work items fit the CTA's threads
  int p2g_staging = 1; // 3D sweeps: 1 bulk copies of sorted records, 0 gather through the order
  int num_sms = 1;       // persistent P2G grids: CTAs per SM x this
  // the last step's G2P binned the current positions for the next partition
  // (3D quadratic): counts, slots, keys and marks are in place
  bool keys_fresh = false;
  unsigned *hash_next = nullptr;  // reference hashes binned ahead [stride]
  unsigned p2g_seq = 0;  // queue-driven P2G launches so far (fetch counter parity)
  bool tuning = false; // no physical re-sort while the autotuner times variants
  int *key = nullptr;  // binning key scratch
  int *fault = nullptr;
  // staging for field conversion
  void *staging = nullptr;
  size_t staging_bytes = 0;

  long long launches = 0;
  int step = 0;
  int epoch = -1;
  int p2g_epoch = -2;
  int steps_since_sort = 0;
  bool partitioned = false;
};

namespace {

int ensure_staging(pmpm_sim *s, size_t bytes) {
  if (s->staging_bytes >= bytes) return PMPM_OK;
  if (s->staging) cudaFree(s->staging);
  s->staging = nullptr;
  s->staging_bytes = 0;
  cudaError_t e = cudaMalloc(&s->staging, bytes);
  if (e == cudaErrorMemoryAllocation) return PMPM_ERR_OUT_OF_MEMORY;
  PMPM_CUDA(e);
  s->staging_bytes = bytes;
  return PMPM_OK;
}

void free_rollout(pmpm_sim *s);

void free_particles(pmpm_sim *s) {
  free_rollout(s);
  for (int k = 0; k < 2; k++) {
    DevParticles &P = s->P[k];
    dfree(P.x);
    dfree(P.v);
    dfree(P.F);
    dfree(P.sig);
    dfree(P.L);
    dfree(P.m);
    dfree(P.V);
    dfree(P.V0);
    dfree(P.fext);
    dfree(P.eps);
    dfree(P.sref);
    dfree(P.color);
    dfree(P.active);
    dfree(P.rigid);
    dfree(P.id);
    dfree(P.hash);
    dfree(P.pE);
    dfree(P.pphi);
    dfree(P.acc);
    dfree(P.pc);
    P = DevParticles{};
  }
  dfree(s->slot);
  dfree(s->key);
  dfree(s->hash_next);
  dfree(s->B.order);
  dfree(s->B.rec);
  dfree(s->musl_x);
  s->n = 0;
  s->stride = 0;
}

int alloc_particle_set(pmpm_sim *s, DevParticles &P) {
  const int D = s->dim, st = s->stride;
  const int S = D == 2 ? 4 : 6, E = D == 2 ? 3 : 6;
  P.n = s->n;
  P.stride = st;
  PMPM_TRY(dalloc(&P.x, (size_t)D * st));
  PMPM_TRY(dalloc(&P.v, (size_t)D * st));
  PMPM_TRY(dalloc(&P.F, (size_t)D * D * st));
  PMPM_TRY(dalloc(&P.sig, (size_t)S * st));
  PMPM_TRY(dalloc(&P.L, (size_t)D * D * st));
  PMPM_TRY(dalloc(&P.m, (size_t)st));
  PMPM_TRY(dalloc(&P.V, (size_t)st));
  PMPM_TRY(dalloc(&P.V0, (size_t)st));
  if (s->has_planar) PMPM_TRY(dalloc(&P.fext, (size_t)D * st));
  if (s->has_dp) {
    PMPM_TRY(dalloc(&P.eps, (size_t)E * st));
    PMPM_TRY(dalloc(&P.sref, (size_t)S * st));
  }
  if (s->has_vm || s->has_mcc) PMPM_TRY(dalloc(&P.acc, (size_t)st));
  if (s->has_mcc) PMPM_TRY(dalloc(&P.pc, (size_t)st));
  PMPM_TRY(dalloc(&P.color, (size_t)st));
  PMPM_TRY(dalloc(&P.active, (size_t)st));
  PMPM_TRY(dalloc(&P.rigid, (size_t)st));
  PMPM_TRY(dalloc(&P.id, (size_t)st));
  PMPM_TRY(dalloc(&P.hash, (size_t)st));
  return PMPM_OK;
}

StepArgs make_args(pmpm_sim *s) {
  StepArgs a;
  memset(&a, 0, sizeof(a));
  a.g = s->g;
  a.P = s->P[s->cur];
  a.P.slot = s->slot;
  a.P.key = (unsigned *)s->key;
  a.N = s->N;
  a.B = s->B;
  a.B.dual = s->dual ? 1 : 0;
  for (int c = 0; c < 3; c++) a.B.kd[c] = s->kd[c];
  a.B.nkeys = s->nkeys;
  a.dt = s->dt;
  a.alpha = s->alpha;
  a.one_minus_alpha = (float)(1.0 - (double)s->alpha);
  a.cutoff = 0.000000001f;
  a.epoch = s->epoch;
  a.flags = s->flags;
  a.fault = s->fault;
  a.nmat = (int)s->mats.size();
  a.nbc = (int)s->bcs.size();
  a.nbc_epi = s->rbls_index >= 0 ? s->rbls_index : a.nbc;
  a.rigid_shift = s->rigid_shift_pending ? 1 : 0;
  a.remap = s->remap_now;
  a.musl_pass = s->musl_pass_now;
  a.musl_x = s->musl_x;
  a.has_planar = s->has_planar ? 1 : 0;
  a.has_sref = s->has_sref ? 1 : 0;
  for (int k = 0; k < a.nmat; k++) a.mat[k] = s->mats[k];
  for (int k = 0; k < a.nbc; k++) a.bc[k] = s->bcs[k];
  for (const GravityState &gs : s->gravity)
    for (int c = 0; c < 3; c++) a.bc[gs.bc_index].r[c] = gs.current[c];
  return a;
}

// Gravity::apply_on_nodes_moments (src/boundaryconditions/gravity.cpp:68-73):
// while step < ramp_step the stored gravity becomes gravity_end * step/ramp_step.
void update_gravity(pmpm_sim *s) {
  for (GravityState &gs : s->gravity) {
    const DevBC &bc = s->bcs[gs.bc_index];
    const int is_ramp = bc.i[0], ramp_step = bc.i[1];
    const float ramp_factor = (float)s->step / (float)ramp_step;
    if (is_ramp && s->step < ramp_step)
      for (int c = 0; c < 3; c++) gs.current[c] = bc.r[3 + c] * ramp_factor;
  }
}

// Pose of the analytic rigid bodies at the current step (time step * dt).
void update_bodies(pmpm_sim *s) {
  const double t = (double)s->step * (double)s->dt;
  for (const SdfState &b : s->sdf) {
    DevBC &bc = s->bcs[b.bc_index];
    for (int c = 0; c < 3; c++) bc.r[c] = (float)(b.c0[c] + b.v[c] * t);
    const double ang = b.angle0 + b.omega * t;
    bc.r[12] = (float)std::cos(ang);
    bc.r[13] = (float)std::sin(ang);
  }
}

// 3x3 product in Eigen's coefficient order: ((a0 b0 + a1 b1) + a2 b2).
void matmul3(const float *A, const float *B, float *C) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) C[3 * i + j] = (A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j]) + A[3 * i + 2] * B[6 + j];
}

// RigidBodyLevelSet::update_animation (src/boundaryconditions/rigidbodylevelset.cpp:
// 127-206): LOOP_ROTATE advances the euler angles by rate * dt and rotates by
// delta = previous - new.  The reference's 3D matrices are kept by default:
// Rx carries both the 2D and the 3D entries and Rz stays zero, so R = Rz Ry Rx
// is zero; `corrected` builds the proper Rz(d2) Ry(d1) Rx(d0).  STATIC: the
// reference leaves R unset; the identity is used (rigid velocity zero).
void rigid_rotation(pmpm_sim *s, float *R) {
  const int D = s->dim;
  RigidState &r = s->rigid;
  float R3[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (r.mode == PMPM_RIGID_LOOP_ROTATE) {
    float d[3];
    for (int c = 0; c < 3; c++) {
      const float prev = r.euler[c];
      r.euler[c] = r.euler[c] + r.rate[c] * s->dt;
      d[c] = prev - r.euler[c];
    }
    const float c0 = std::cos(d[0]), s0 = std::sin(d[0]);
    const float c1 = std::cos(d[1]), s1 = std::sin(d[1]);
    const float c2 = std::cos(d[2]), s2 = std::sin(d[2]);
    if (D == 2) {
      const float M[9] = {c0, -s0, 0, s0, c0, 0, 0, 0, 1};
      memcpy(R3, M, sizeof(R3));
    } else if (!r.corrected) {
      const float Rx[9] = {1, -s0, 0, s0, c2, -s2, 0, s2, c2};
      const float Ry[9] = {c1, 0, s1, 0, 1, 0, -s1, 0, c1};
      const float Rz[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      float T[9];
      matmul3(Rz, Ry, T);
      matmul3(T, Rx, R3);
    } else {
      const float Rx[9] = {1, 0, 0, 0, c0, -s0, 0, s0, c0};
      const float Ry[9] = {c1, 0, s1, 0, 1, 0, -s1, 0, c1};
      const float Rz[9] = {c2, -s2, 0, s2, c2, 0, 0, 0, 1};
      float T[9];
      matmul3(Rz, Ry, T);
      matmul3(T, Rx, R3);
    }
  }
  for (int i = 0; i < D; i++)
    for (int j = 0; j < D; j++) R[i * D + j] = R3[3 * i + j];
}

// The nearest-rigid-particle RigidBodyLevelSet after P2G: rigid velocities,
// then node contact and the node BCs listed after it; G2P then also moves
// the rigid particles by their set velocity.
template <int D>
int launch_rigid(pmpm_sim *s) {
  if (s->rbls_index < 0) return PMPM_OK;
  RigidMotion rm;
  memset(&rm, 0, sizeof(rm));
  rigid_rotation(s, rm.R);
  for (int c = 0; c < 3; c++) rm.com[c] = s->rigid.com[c];
  StepArgs a = make_args(s);
  k_rigid_velocity<D><<<blocks_for(s->n), kTPB, 0, s->stream>>>(a, rm);
  PMPM_LAUNCHED();
  k_rigid_nodes<D><<<s->g.ntiles, TileDims<D>::N, 0, s->stream>>>(a, s->rbls_index);
  PMPM_LAUNCHED();
  s->launches += 2;
  s->rigid_shift_pending = true;
  return PMPM_OK;
}

template <int D, int SF>
int launch_partition(pmpm_sim *s) {
  s->epoch += 1;
  StepArgs a = make_args(s);
  cudaStream_t st = s->stream;
  if (!s->keys_fresh) {
    k_hash_count<D, SF><<<blocks_for(s->n), kTPB, 0, st>>>(a);
    PMPM_LAUNCHED();
  } else {
    s->launches -= 1;  // binned by the last step's G2P
    std::swap(s->P[s->cur].hash, s->hash_next);
  }
  s->keys_fresh = false;
  s->launches += 7;
  if (D == 3 && !(s->flags & PMPM_FLAG_DETERMINISTIC)) {
    // active queue of the persistent 3D sweep P2G kernels: tiles (dual
    // sweep) or pairs of tiles stacked in z (linear and cubic sweeps)
    if (SF == PMPM_SHAPE_QUADRATIC) {
      k_tile_list<<<(s->g.ntiles + 255) / 256, 256, 0, st>>>(s->N.tile_epoch, s->g.ntiles, s->epoch,
                                                            s->N.tile_list, s->N.tile_queue);
    } else {
      const int plane = s->g.tdim[0] * s->g.tdim[1];
      const int nunits = plane * ((s->g.tdim[2] + 1) / 2);
      k_pair_list<<<(nunits + 255) / 256, 256, 0, st>>>(s->N.tile_epoch, plane, s->g.tdim[2], s->epoch,
                                                        s->N.tile_list, s->N.tile_queue);
    }
    PMPM_LAUNCHED();
    s->launches += 1;
  }
  PMPM_TRY(launch_scan(s->scan, s->B.count, s->nkeys, s->B.offset, s->B.scalars, s->fault, s->nscan_blocks, st));
  s->launches -= 2;  // one scan launch instead of three
  k_scatter<<<blocks_for((s->n + kScatterPer - 1) / kScatterPer), kTPB, 0, st>>>(a);
  PMPM_LAUNCHED();
  // ids in order inside each bin: needed by the deterministic gather and by
  // the nearest-rigid-particle search (the reference's first minimum); the
  // other P2G paths accumulate in any order, and the reference partition
  // views are built from the stored hashes
  if ((s->flags & PMPM_FLAG_DETERMINISTIC) || s->rbls_index >= 0) {
    k_sort_cells<<<blocks_for(s->nkeys), kTPB, 0, st>>>(a);
    PMPM_LAUNCHED();
    k_sort_big<<<148, 1024, 0, st>>>(a);
    PMPM_LAUNCHED();
  } else {
    s->launches -= 2;
  }
  s->partitioned = true;
  return PMPM_OK;
}

template <int D>
int launch_reorder(pmpm_sim *s) {
  StepArgs a = make_args(s);
  DevParticles dst = s->P[1 - s->cur];
  const bool move_L = (s->flags & PMPM_FLAG_KEEP_VELOCITY_GRADIENT) != 0;
  k_reorder<D><<<blocks_for(s->n), kTPB, 0, s->stream>>>(a, dst, move_L ? 1 : 0, s->has_planar ? 1 : 0);
  PMPM_LAUNCHED();
  s->launches += 1;
  s->cur = 1 - s->cur;
  s->steps_since_sort = 0;
  return PMPM_OK;
}

template <int D, int SF>
int launch_p2g(pmpm_sim *s, int apply_bcs) {
  if (apply_bcs && !s->remap_now) {
    update_gravity(s);
    update_bodies(s);
  }
  StepArgs a = make_args(s);
  if (s->flags & PMPM_FLAG_DETERMINISTIC) {
    k_p2g_gather<D, SF><<<s->g.ntiles, TileDims<D>::N, 0, s->stream>>>(a, apply_bcs, s->node_epoch);
  } else if (D == 3 && s->dual) {
    const int dev = s->device < 64 ? s->device : 63;
    static bool attr_set[64] = {false};  // per device
    if (!attr_set[dev]) {
      PMPM_CUDA(cudaFuncSetAttribute(k_p2g_dual3<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     dual3_smem_bytes<false, true>()));
      PMPM_CUDA(cudaFuncSetAttribute(k_p2g_dual3<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     dual3_smem_bytes<true, true>()));
      PMPM_CUDA(cudaFuncSetAttribute(k_p2g_dual3<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     dual3_smem_bytes<false, false>()));
      PMPM_CUDA(cudaFuncSetAttribute(k_p2g_dual3<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     dual3_smem_bytes<true, false>()));
      attr_set[dev] = true;
    }
    if (s->p2g_variant == 1 && s->dual3_fits) {
      // (bulk staging: sorted records of this partition's particles first)
      // persistent CTAs over the active-tile queue
      if (s->p2g_staging) {
        if (s->has_planar)
          k_records<PMPM_SHAPE_QUADRATIC, true, true><<<blocks_for(s->n), kTPB, 0, s->stream>>>(a);
        else
          k_records<PMPM_SHAPE_QUADRATIC, true, false><<<blocks_for(s->n), kTPB, 0, s->stream>>>(a);
        PMPM_LAUNCHED();
        s->launches += 1;
      }
      a.p2g_par = (int)(s->p2g_seq++ & 1u);
      const int grid = std::min(s->g.ntiles, s->num_sms);
      if (s->p2g_staging) {
        if (s->has_planar)
          k_p2g_dual3<true, true><<<grid, Dual3::NT, dual3_smem_bytes<true, true>(), s->stream>>>(a, apply_bcs,
                                                                                                  s->node_epoch);
        else
          k_p2g_dual3<false, true><<<grid, Dual3::NT, dual3_smem_bytes<false, true>(), s->stream>>>(a, apply_bcs,
                                                                                                    s->node_epoch);
      } else {
        if (s->has_planar)
          k_p2g_dual3<true, false><<<grid, Dual3::NT, dual3_smem_bytes<true, false>(), s->stream>>>(a, apply_bcs,
                                                                                                    s->node_epoch);
        else
          k_p2g_dual3<false, false><<<grid, Dual3::NT, dual3_smem_bytes<false, false>(), s->stream>>>(
              a, apply_bcs, s->node_epoch);
      }
    } else {
      constexpr int cbytes = cells3_smem_bytes();
      static bool cattr_set[64] = {false};  // per device
      if (!cattr_set[dev]) {
        PMPM_CUDA(cudaFuncSetAttribute(k_p2g_cells3, cudaFuncAttributeMaxDynamicSharedMemorySize, cbytes));
        cattr_set[dev] = true;
      }
      k_p2g_cells3<<<s->nbricks, Cells3::NT, cbytes, s->stream>>>(a);
      PMPM_LAUNCHED();
      k_node_epilogue<3><<<s->g.ntiles, TileDims<3>::N, 0, s->stream>>>(a, apply_bcs, s->node_epoch);
      s->launches += 1;
    }
  } else if (D == 3) {
    const int dev = s->device < 64 ? s->device : 63;
    static bool attr_set[64] = {false};  // per device
    if (!attr_set[dev]) {
      PMPM_CUDA(cudaFuncSetAttribute(k_p2g_sweep3<SF, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     sweep3_smem_bytes<SF, false, true>()));
      PMPM_CUDA(cudaFuncSetAttribute(k_p2g_sweep3<SF, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     sweep3_smem_bytes<SF, true, true>()));
      PMPM_CUDA(cudaFuncSetAttribute(k_p2g_sweep3<SF, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     sweep3_smem_bytes<SF, false, false>()));
      PMPM_CUDA(cudaFuncSetAttribute(k_p2g_sweep3<SF, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     sweep3_smem_bytes<SF, true, false>()));
      attr_set[dev] = true;
    }
    if (s->p2g_staging) {
      if (s->has_planar)
        k_records<SF, false, true><<<blocks_for(s->n), kTPB, 0, s->stream>>>(a);
      else
        k_records<SF, false, false><<<blocks_for(s->n), kTPB, 0, s->stream>>>(a);
      PMPM_LAUNCHED();
      s->launches += 1;
    }
    a.p2g_par = (int)(s->p2g_seq++ & 1u);
    const int grid = std::min(s->g.ntiles, s->num_sms);
    constexpr int NT3 = Sweep3<SF>::NT;
    if (s->p2g_staging) {
      if (s->has_planar)
        k_p2g_sweep3<SF, true, true><<<grid, NT3, sweep3_smem_bytes<SF, true, true>(), s->stream>>>(a, apply_bcs,
                                                                                                   s->node_epoch);
      else
        k_p2g_sweep3<SF, false, true><<<grid, NT3, sweep3_smem_bytes<SF, false, true>(), s->stream>>>(
            a, apply_bcs, s->node_epoch);
    } else {
      if (s->has_planar)
        k_p2g_sweep3<SF, true, false><<<grid, NT3, sweep3_smem_bytes<SF, true, false>(), s->stream>>>(
            a, apply_bcs, s->node_epoch);
      else
        k_p2g_sweep3<SF, false, false><<<grid, NT3, sweep3_smem_bytes<SF, false, false>(), s->stream>>>(
            a, apply_bcs, s->node_epoch);
    }
  } else {
    k_p2g_tile<D, SF><<<s->g.ntiles, TileDims<D>::N, 0, s->stream>>>(a, apply_bcs, s->node_epoch);
  }
  PMPM_LAUNCHED();
  s->launches += 1;
  s->p2g_epoch = s->epoch;
  if (apply_bcs && !s->remap_now) PMPM_TRY(launch_rigid<D>(s));
  return PMPM_OK;
}

// Invalidates binning done ahead by a step's G2P (particle state is about to
// change outside a step): its counts are cleared, its marks are harmless.
int drop_fresh_keys(pmpm_sim *s) {
  if (!s->keys_fresh) return PMPM_OK;
  s->keys_fresh = false;
  PMPM_CUDA(cudaMemsetAsync(s->B.count, 0, sizeof(int) * (size_t)s->nkeys, s->stream));
  return PMPM_OK;
}

// bin_next: the step loop's final G2P also bins the new positions (see
// k_g2p); any other G2P changes positions, so earlier binning is dropped.
template <int D, int SF>
int launch_g2p(pmpm_sim *s, int do_stress, int store_L, bool bin_next = false) {
  PMPM_TRY(drop_fresh_keys(s));
  StepArgs a = make_args(s);
  a.bin_next = bin_next ? 1 : 0;
  a.hash_next = s->hash_next;
  if (s->has_vm || s->has_mcc)
    k_g2p<D, SF, true><<<blocks_for(s->n, G2PLaunch<D, SF, true>::NT), G2PLaunch<D, SF, true>::NT, 0, s->stream>>>(
        a, do_stress, store_L);
  else
    k_g2p<D, SF, false><<<blocks_for(s->n, G2PLaunch<D, SF, false>::NT), G2PLaunch<D, SF, false>::NT, 0,
                          s->stream>>>(a, do_stress, store_L);
  PMPM_LAUNCHED();
  s->launches += 1;
  s->rigid_shift_pending = false;
  s->keys_fresh = bin_next;
  return PMPM_OK;
}

// MUSL after the first P2G: G2P of velocities and positions, momentum
// remap, G2P of the velocity gradient with F, V and the stress update.
template <int D, int SF>
int musl_tail(pmpm_sim *s, int store_L) {
  s->musl_pass_now = 1;
  int st = launch_g2p<D, SF>(s, 0, 0);
  if (st == PMPM_OK) {
    s->musl_pass_now = 0;
    s->remap_now = 1;  // node conditions on velocities only (node_bcs)
    st = launch_p2g<D, SF>(s, 1);
  }
  if (st == PMPM_OK) {
    s->remap_now = 0;
    s->musl_pass_now = 2;
    st = launch_g2p<D, SF>(s, 1, store_L);
  }
  s->remap_now = 0;
  s->musl_pass_now = 0;
  return st;
}

template <int D, int SF>
int step_once(pmpm_sim *s) {
  PMPM_TRY((launch_partition<D, SF>(s)));
  if (!s->ro.held && !s->tuning && s->resort_interval > 0 && s->steps_since_sort + 1 >= s->resort_interval) {
    PMPM_TRY(launch_reorder<D>(s));
  } else {
    s->steps_since_sort += 1;
  }
  PMPM_TRY((launch_p2g<D, SF>(s, 1)));
  const int store_L = (s->flags & PMPM_FLAG_KEEP_VELOCITY_GRADIENT) ? 1 : 0;
  if (s->flags & PMPM_FLAG_MUSL) {
    PMPM_TRY((musl_tail<D, SF>(s, store_L)));
  } else {
    // quadratic: the next partition's binning rides on this G2P (not while
    // the autotuner times kernels, nor with a PlanarDomain, whose particle
    // forces the binning pass computes; state restores drop the binning)
    const bool bin_next = s->dual && !s->tuning && s->rbls_index < 0 && !s->has_planar;
    PMPM_TRY((launch_g2p<D, SF>(s, 1, store_L, bin_next)));
  }
  s->step += 1;
  return PMPM_OK;
}

// Runtime (dim, shape function) -> template instantiation.
#define PMPM_DISPATCH(s, FN, ...)                                                   \
  ((s)->dim == 2                                                                    \
       ? ((s)->shape == PMPM_SHAPE_LINEAR      ? FN<2, PMPM_SHAPE_LINEAR>(__VA_ARGS__) \
          : (s)->shape == PMPM_SHAPE_QUADRATIC ? FN<2, PMPM_SHAPE_QUADRATIC>(__VA_ARGS__) \
                                               : FN<2, PMPM_SHAPE_CUBIC>(__VA_ARGS__))  \
       : ((s)->shape == PMPM_SHAPE_LINEAR      ? FN<3, PMPM_SHAPE_LINEAR>(__VA_ARGS__) \
          : (s)->shape == PMPM_SHAPE_QUADRATIC ? FN<3, PMPM_SHAPE_QUADRATIC>(__VA_ARGS__) \
                                               : FN<3, PMPM_SHAPE_CUBIC>(__VA_ARGS__)))

// ---------------------------------------------------------------------------
// field conversion kernels: reference AoS layout (id order) <-> SoA storage
// ---------------------------------------------------------------------------

// kind: 0 vector [dim], 1 full matrix [dim][dim], 2 stress/ref 3x3 from the
// symmetric storage, 3 eps [dim][dim] from symmetric, 4 scalar float,
// 5 uint8, 6 uint32 hash, 7 bins from positions
__global__ void k_get_particles(DevParticles P, int D, int kind, const void *src, void *dst, int extra) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.n) return;
  const int i = P.id[s], st = P.stride;
  if (kind == 0 || kind == 1) {
    const int nc = kind == 0 ? D : D * D;
    const float *f = (const float *)src;
    for (int c = 0; c < nc; c++) ((float *)dst)[(size_t)i * nc + c] = f[c * st + s];
  } else if (kind == 2) {
    const float *f = (const float *)src;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) {
        int k;
        if (D == 2) {
          k = (a == b) ? (a == 2 ? 3 : a) : (a + b == 1 ? 2 : -1);
        } else {
          k = (a == b) ? a : 2 + a + b;
        }
        ((float *)dst)[(size_t)i * 9 + 3 * a + b] = k < 0 ? 0.0f : f[k * st + s];
      }
  } else if (kind == 3) {
    const float *f = (const float *)src;
    for (int a = 0; a < D; a++)
      for (int b = 0; b < D; b++) {
        int k = (a == b) ? a : (D == 2 ? 2 : 2 + a + b);
        ((float *)dst)[(size_t)i * D * D + a * D + b] = f[k * st + s];
      }
  } else if (kind == 4) {
    ((float *)dst)[i] = ((const float *)src)[s];
  } else if (kind == 5) {
    ((uint8_t *)dst)[i] = ((const uint8_t *)src)[s];
  } else if (kind == 6) {
    ((unsigned *)dst)[i] = ((const unsigned *)src)[s];
  } else if (kind == 7) {
    const DevGrid *g = (const DevGrid *)src;
    for (int c = 0; c < D; c++)
      ((int *)dst)[(size_t)i * D + c] = (int)scaled_coord(P.x[c * st + s], g->origin[c], g->inv_h);
  }
  (void)extra;
}

__global__ void k_set_particles(DevParticles P, int D, int kind, const void *src, void *dst) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.n) return;
  const int i = P.id[s], st = P.stride;
  if (kind == 0 || kind == 1) {
    const int nc = kind == 0 ? D : D * D;
    for (int c = 0; c < nc; c++) ((float *)dst)[c * st + s] = ((const float *)src)[(size_t)i * nc + c];
  } else if (kind == 2) {
    const float *M = (const float *)src + (size_t)i * 9;
    float *f = (float *)dst;
    if (D == 2) {
      f[0 * st + s] = M[0];
      f[1 * st + s] = M[4];
      f[2 * st + s] = M[1];
      f[3 * st + s] = M[8];
    } else {
      f[0 * st + s] = M[0];
      f[1 * st + s] = M[4];
      f[2 * st + s] = M[8];
      f[3 * st + s] = M[1];
      f[4 * st + s] = M[2];
      f[5 * st + s] = M[5];
    }
  } else if (kind == 3) {
    const float *M = (const float *)src + (size_t)i * D * D;
    float *f = (float *)dst;
    if (D == 2) {
      f[0 * st + s] = M[0];
      f[1 * st + s] = M[3];
      f[2 * st + s] = M[1];
    } else {
      f[0 * st + s] = M[0];
      f[1 * st + s] = M[4];
      f[2 * st + s] = M[8];
      f[3 * st + s] = M[1];
      f[4 * st + s] = M[2];
      f[5 * st + s] = M[5];
    }
  } else if (kind == 4) {
    ((float *)dst)[s] = ((const float *)src)[i];
  } else if (kind == 5) {
    ((uint8_t *)dst)[s] = ((const uint8_t *)src)[i];
  }
}

// Node field out: nodes of tiles the last P2G did not write read as 0.
__global__ void k_get_nodes(DevGrid g, int D, int ncomp, const float *src, const int *node_epoch, int p2g_epoch,
                            float *dst) {
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= g.ntotal) return;
  const int c[3] = {node % g.n[0], (node / g.n[0]) % g.n[1], node / (g.n[0] * g.n[1])};
  int t = D == 2 ? tile_of<2>(g, c) : tile_of<3>(g, c);
  const bool valid = node_epoch[t] == p2g_epoch;
  for (int k = 0; k < ncomp; k++) dst[(size_t)node * ncomp + k] = valid ? src[(size_t)k * g.ntotal + node] : 0.0f;
}

// Solver::Solver set-up kernels.
__global__ void k_initial_volumes(DevParticles P, float vol) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.n) return;
  if (!(P.V[s] > 0.0f)) P.V[s] = vol;
  P.V0[s] = P.V[s];
}

__global__ void k_initial_masses(DevParticles P, int mat_id, float density) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.n) return;
  if ((int)P.color[s] != mat_id || P.m[s] > 0.0f) return;
  P.m[s] = density * P.V[s];
}

// Per-particle Drucker-Prager parameters from the particles' materials:
// E = 3 K (1 - 2 nu), friction angle of the material (0 elsewhere).
__global__ void k_fill_particle_params(DevParticles P, const DevMaterial *mats, int nmat) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.n) return;
  float E = 0.0f, phi = 0.0f;
  const int c = P.color[s];
  if (c < nmat && mats[c].type == PMPM_MAT_DRUCKER_PRAGER && mats[c].p[7] >= 0.0f) {
    E = 3.0f * mats[c].p[0] * (1.0f - 2.0f * mats[c].p[7]);
    phi = mats[c].p[9];
  }
  P.pE[s] = E;
  P.pphi[s] = phi;
}

__global__ void k_dp_init(DevParticles P, int D, int *nonzero_ref) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.n) return;
  const int S = D == 2 ? 4 : 6, E = D == 2 ? 3 : 6, st = P.stride;
  bool nz = false;
  for (int k = 0; k < S; k++) {
    float v = P.sig[k * st + s];
    P.sref[k * st + s] = v;
    nz = nz || v != 0.0f;
  }
  for (int k = 0; k < E; k++) P.eps[k * st + s] = 0.0f;
  if (nz) atomicOr(nonzero_ref, 1);
}

// ModifiedCamClay::initialize (src/materials/modifiedcamclay.cpp:68-108) and
// DruckerPragerCap::initialize (src/materials/druckerprager_cap.cpp:72-108),
// the part that is not the shared history reset of k_dp_init: per particle of
// a Modified Cam Clay or Drucker-Prager cap colour, alpha = 0 and pc = R p0 with p0 = -tr(sigma)/3
// (the reference applies one material's R to every particle; here each
// particle takes its own material's).
__global__ void k_mcc_init(StepArgs a, int D) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.P.n) return;
  const int st = a.P.stride;
  const int c = a.P.color[s];
  float pc = 0.0f;
  if (c < a.nmat && (a.mat[c].type == PMPM_MAT_MODIFIED_CAM_CLAY || a.mat[c].type == PMPM_MAT_DRUCKER_PRAGER_CAP)) {
    const float sxx = a.P.sig[0 * st + s], syy = a.P.sig[1 * st + s];
    const float szz = a.P.sig[(D == 2 ? 3 : 2) * st + s];
    const float p0 = (float)(-(double)((sxx + syy) + szz) / 3.0);
    pc = p0 * a.mat[c].p[7];
  }
  a.P.acc[s] = 0.0f;
  a.P.pc[s] = pc;
}

int field_info(const pmpm_sim *s, int field, size_t *bytes) {
  const size_t n = (size_t)s->n, D = (size_t)s->dim, nn = (size_t)s->g.ntotal;
  switch (field) {
    case PMPM_FIELD_POSITIONS:
    case PMPM_FIELD_VELOCITIES:
    case PMPM_FIELD_FORCES_EXTERNAL:
      *bytes = n * D * 4;
      return PMPM_OK;
    case PMPM_FIELD_STRESSES:
    case PMPM_FIELD_STRESS_REF:
      *bytes = n * 9 * 4;
      return PMPM_OK;
    case PMPM_FIELD_F:
    case PMPM_FIELD_VELOCITY_GRADIENT:
    case PMPM_FIELD_EPS_E:
      *bytes = n * D * D * 4;
      return PMPM_OK;
    case PMPM_FIELD_MASSES:
    case PMPM_FIELD_VOLUMES:
    case PMPM_FIELD_VOLUMES_ORIGINAL:
    case PMPM_FIELD_YOUNGS_MODULUS:
    case PMPM_FIELD_FRICTION_ANGLE:
    case PMPM_FIELD_ACC_EPS_P:
    case PMPM_FIELD_PRECONSOLIDATION:
    case PMPM_FIELD_HASH_UNSORTED:
    case PMPM_FIELD_HASH_SORTED:
    case PMPM_FIELD_SORTED_INDEX:
      *bytes = n * 4;
      return PMPM_OK;
    case PMPM_FIELD_COLORS:
    case PMPM_FIELD_IS_RIGID:
    case PMPM_FIELD_IS_ACTIVE:
      *bytes = n;
      return PMPM_OK;
    case PMPM_FIELD_NODE_MASSES:
    case PMPM_FIELD_CELL_START:
    case PMPM_FIELD_CELL_END:
      *bytes = nn * 4;
      return PMPM_OK;
    case PMPM_FIELD_NODE_MOMENTS:
    case PMPM_FIELD_NODE_MOMENTS_NT:
      *bytes = nn * D * 4;
      return PMPM_OK;
    case PMPM_FIELD_NODE_IDS:
    case PMPM_FIELD_NODE_TYPES:
      *bytes = nn * 3 * 4;
      return PMPM_OK;
    case PMPM_FIELD_BINS:
      *bytes = n * D * 4;
      return PMPM_OK;
    default:
      return PMPM_ERR_INVALID_ARGUMENT;
  }
}

// Allocates the per-particle Drucker-Prager parameters on first use (both
// storage sets) and fills them from the materials.
int ensure_particle_params(pmpm_sim *s) {
  if (s->P[0].pE) return PMPM_OK;
  if (s->n == 0) return PMPM_ERR_STATE;
  for (int k = 0; k < 2; k++) {
    PMPM_TRY(dalloc(&s->P[k].pE, (size_t)s->stride));
    PMPM_TRY(dalloc(&s->P[k].pphi, (size_t)s->stride));
  }
  DevMaterial *dm = nullptr;
  const int nmat = (int)s->mats.size();
  if (nmat > 0) {
    PMPM_CUDA(cudaMalloc(&dm, sizeof(DevMaterial) * nmat));
    PMPM_CUDA(cudaMemcpy(dm, s->mats.data(), sizeof(DevMaterial) * nmat, cudaMemcpyHostToDevice));
  }
  DevParticles P = s->P[s->cur];
  k_fill_particle_params<<<blocks_for(s->n), kTPB, 0, s->stream>>>(P, dm, nmat);
  const cudaError_t e = cudaGetLastError();
  PMPM_CUDA(cudaStreamSynchronize(s->stream));
  if (dm) cudaFree(dm);
  PMPM_CUDA(e);
  return PMPM_OK;
}

int copy_out(pmpm_sim *s, const void *dev_src, void *dst, size_t bytes, int on_device) {
  PMPM_CUDA(cudaMemcpyAsync(dst, dev_src, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                            s->stream));
  PMPM_CUDA(cudaStreamSynchronize(s->stream));
  return PMPM_OK;
}

// Sorted index and sorted hashes in the reference's layout: binned particles
// in cell order (ids ascending inside a cell), then the unbinned ones (hash
// >= num_cells_total) by (hash, id), as a stable sort of all hashes gives.
int sorted_views(pmpm_sim *s, std::vector<int> &sorted_index, std::vector<unsigned> &hash_sorted) {
  const int n = s->n;
  std::vector<int> id(n);
  std::vector<unsigned> hash(n);
  const DevParticles &P = s->P[s->cur];
  {
    // the reference permutation is the stable sort of the stored reference
    // hashes (the step's own bins may be dual cells, in any order inside)
    PMPM_CUDA(cudaMemcpyAsync(id.data(), P.id, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream));
    PMPM_CUDA(cudaMemcpyAsync(hash.data(), P.hash, sizeof(unsigned) * n, cudaMemcpyDeviceToHost, s->stream));
    PMPM_CUDA(cudaStreamSynchronize(s->stream));
    std::vector<unsigned> by_id(n);
    for (int k = 0; k < n; k++) by_id[id[k]] = hash[k];
    sorted_index.resize(n);
    hash_sorted.resize(n);
    std::iota(sorted_index.begin(), sorted_index.end(), 0);
    std::stable_sort(sorted_index.begin(), sorted_index.end(),
                     [&](int x, int y) { return by_id[x] < by_id[y]; });
    for (int k = 0; k < n; k++) hash_sorted[k] = by_id[sorted_index[k]];
    return PMPM_OK;
  }
  return PMPM_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" {

const char *pmpm_status_string(int status) {
  switch (status) {
    case PMPM_OK: return "ok";
    case PMPM_ERR_INVALID_ARGUMENT: return "invalid argument";
    case PMPM_ERR_CUDA: return "CUDA error";
    case PMPM_ERR_OUT_OF_MEMORY: return "out of device memory";
    case PMPM_ERR_NOT_SUPPORTED: return "not supported";
    case PMPM_ERR_STATE: return "call out of order (particles not set or not initialised)";
    case PMPM_ERR_OUT_OF_DOMAIN: return "a particle left the background grid";
    case PMPM_ERR_NONFINITE: return "non-finite particle position";
    case PMPM_ERR_CELL_OVERFLOW: return "too many particles in one cell";
    default: return "unknown status";
  }
}

int pmpm_material_linear_elastic(float density, float E, float pois, int corrected, pmpm_material *out) {
  if (!out) return PMPM_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  out->type = PMPM_MAT_LINEAR_ELASTIC;
  out->density = density;
  const float bulk = E / (3.0f * (1.0f - 2.0f * pois));
  const float shear = E / (2.0f * (1.0f + pois));
  const float lame = E * pois / ((1.0f + pois) * (1.0f - 2.0f * pois));
  float p[8] = {E, pois, lame, shear, bulk, corrected ? 1.0f : 0.0f, 0.0f, 0.0f};
  memcpy(out->params, p, sizeof(p));
  return PMPM_OK;
}

int pmpm_material_newton_fluid(float density, float viscosity, float bulk_modulus, float gamma,
                               pmpm_material *out) {
  if (!out) return PMPM_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  out->type = PMPM_MAT_NEWTON_FLUID;
  out->density = density;
  out->params[0] = viscosity;
  out->params[1] = bulk_modulus;
  out->params[2] = gamma;
  return PMPM_OK;
}

int pmpm_material_drucker_prager(float density, float E, float pois, float friction_deg, float dilatancy_deg,
                                 float cohesion, pmpm_material *out) {
  if (!out) return PMPM_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  out->type = PMPM_MAT_DRUCKER_PRAGER;
  out->density = density;
  const float bulk = E / (3.0f * (1.0f - 2.0f * pois));
  const float shear = E / (2.0f * (1.0f + pois));
  const double deg = 3.14159265358979323846 / 180.0;
  const double phi = (double)friction_deg * deg, psi = (double)dilatancy_deg * deg;
  const double s3 = std::sqrt(3.0);
  const double eta = 6.0 * std::sin(phi) / (s3 * (3.0 - std::sin(phi)));
  const double xi = 6.0 * std::cos(phi) / (s3 * (3.0 - std::sin(phi)));
  const double eta_bar = 6.0 * std::sin(psi) / (s3 * (3.0 - std::sin(psi)));
  const double kc = xi * (double)cohesion;
  out->params[0] = bulk;
  out->params[1] = shear;
  out->params[2] = (float)eta;
  out->params[3] = (float)eta_bar;
  out->params[4] = (float)kc;
  out->params[5] = eta > 0.0 ? (float)(kc / eta) : 0.0f;
  out->params[6] = eta > 0.0 ? 1.0f : 0.0f;
  out->params[7] = pois;
  return PMPM_OK;
}

int pmpm_material_von_mises(float density, float E, float pois, float yield_stress, float H, pmpm_material *out) {
  if (!out) return PMPM_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  out->type = PMPM_MAT_VON_MISES;
  out->density = density;
  out->params[0] = E / (3.0f * (1.0f - 2.0f * pois));
  out->params[1] = E / (2.0f * (1.0f + pois));
  out->params[2] = yield_stress;
  out->params[3] = H;
  return PMPM_OK;
}

int pmpm_material_modified_cam_clay(float density, float E, float pois, float M, float lam, float kap, float Vs,
                                    float R, float Pt, float beta, pmpm_material *out) {
  (void)beta;  // not used by the reference's update either
  if (!out) return PMPM_ERR_INVALID_ARGUMENT;
  if (!(lam != kap) || !(kap != 0.0f) || !(Vs != 0.0f) || !(M != 0.0f)) return PMPM_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  out->type = PMPM_MAT_MODIFIED_CAM_CLAY;
  out->density = density;
  out->params[0] = E / (3.0f * (1.0f - 2.0f * pois));
  out->params[1] = E / (2.0f * (1.0f + pois));
  out->params[2] = M;
  out->params[3] = lam;
  out->params[4] = kap;
  out->params[5] = Vs;
  out->params[6] = Pt;
  out->params[7] = R;
  return PMPM_OK;
}

int pmpm_material_drucker_prager_cap(float density, float E, float pois, float M, float lam, float kap, float Vs,
                                     float R, float Pt, float beta, float dilatancy_deg, pmpm_material *out) {
  PMPM_TRY(pmpm_material_modified_cam_clay(density, E, pois, M, lam, kap, Vs, R, Pt, beta, out));
  if (!(1.0f + beta != 0.0f)) return PMPM_ERR_INVALID_ARGUMENT;
  out->type = PMPM_MAT_DRUCKER_PRAGER_CAP;
  const double psi = (double)dilatancy_deg * 3.14159265358979323846 / 180.0;
  out->params[8] = beta;
  out->params[9] = (float)(6.0 * std::sin(psi) / (std::sqrt(3.0) * (3.0 + std::sin(psi))));
  return PMPM_OK;
}

int pmpm_material_dp_rheo(float density, float E, float pois, float M, float Pt, float dilatancy_deg,
                          pmpm_material *out) {
  if (!out) return PMPM_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  out->type = PMPM_MAT_DRUCKER_PRAGER;
  out->density = density;
  const float bulk = E / (3.0f * (1.0f - 2.0f * pois));
  const float shear = E / (2.0f * (1.0f + pois));
  const float psi = dilatancy_deg * (float)(3.14159265358979323846 / 180.0);
  const float eta_bar = (float)(6.0 * std::sin((double)psi) / (std::sqrt(3.0) * (3.0 + std::sin((double)psi))));
  const float eta = (float)(std::sqrt(1.0 / 3.0) * (double)M);
  out->params[0] = bulk;
  out->params[1] = shear;
  out->params[2] = eta;
  out->params[3] = eta_bar;
  out->params[4] = eta * Pt;
  out->params[5] = Pt;
  out->params[6] = 1.0f;
  out->params[7] = -1.0f;
  return PMPM_OK;
}

int pmpm_bc_gravity(const float *gravity, int is_ramp, int ramp_step, const float *gravity_end, int dim,
                    pmpm_bc *out) {
  if (!out || !gravity || dim < 2 || dim > 3) return PMPM_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  out->type = PMPM_BC_GRAVITY;
  for (int c = 0; c < dim; c++) {
    out->reals[c] = gravity[c];
    out->reals[3 + c] = gravity_end ? gravity_end[c] : 0.0f;
  }
  out->ints[0] = is_ramp ? 1 : 0;
  out->ints[1] = ramp_step;
  return PMPM_OK;
}

int pmpm_bc_nodedomain(const int *face0_mode, const int *face1_mode, int dim, pmpm_bc *out) {
  if (!out || dim < 2 || dim > 3) return PMPM_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  out->type = PMPM_BC_NODEDOMAIN;
  for (int c = 0; c < dim; c++) {
    out->ints[c] = face0_mode ? face0_mode[c] : 0;
    out->ints[3 + c] = face1_mode ? face1_mode[c] : 0;
  }
  return PMPM_OK;
}

int pmpm_bc_bodyforce(int mode, const float *values, const unsigned char *mask, pmpm_bc *out) {
  if (!out || !values || !mask || mode < 0 || mode > 2) return PMPM_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  out->type = PMPM_BC_BODYFORCE;
  out->ints[0] = mode;
  out->ints[1] = 1;
  out->values = values;
  out->mask = mask;
  return PMPM_OK;
}

int pmpm_bc_planardomain(const float *face0_friction_deg, const float *face1_friction_deg, int dim,
                         pmpm_bc *out) {
  if (!out || dim < 2 || dim > 3) return PMPM_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  out->type = PMPM_BC_PLANARDOMAIN;
  const float deg = (float)(3.14159265358979323846 / 180.0);
  for (int c = 0; c < dim; c++) {
    out->reals[c] = (face0_friction_deg ? face0_friction_deg[c] : 0.0f) * deg;
    out->reals[3 + c] = (face1_friction_deg ? face1_friction_deg[c] : 0.0f) * deg;
  }
  return PMPM_OK;
}

int pmpm_bc_rigidbodylevelset(int mode, const float *euler_angles_per_second, const float *com,
                              int corrected_rotation, int dim, pmpm_bc *out) {
  if (!out || dim < 2 || dim > 3 || (mode != PMPM_RIGID_STATIC && mode != PMPM_RIGID_LOOP_ROTATE))
    return PMPM_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  out->type = PMPM_BC_RIGIDBODY_LEVELSET;
  out->ints[0] = mode;
  out->ints[1] = corrected_rotation ? 1 : 0;
  for (int c = 0; c < dim; c++) {
    out->reals[c] = euler_angles_per_second ? euler_angles_per_second[c] : 0.0f;
    out->reals[3 + c] = com ? com[c] : 0.0f;
  }
  return PMPM_OK;
}

int pmpm_bc_rigid_sdf(int shape, int axis, const float *center, const float *velocity, float angular_velocity,
                      float angle0, const float *dims, float friction, float contact_distance, int dim,
                      pmpm_bc *out) {
  if (!out || !center || !dims || dim < 2 || dim > 3 || axis < 0 || axis > 2 ||
      (shape != PMPM_SDF_SPHERE && shape != PMPM_SDF_HALF_CYLINDER_SHELL) || !(friction >= 0.0f))
    return PMPM_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  out->type = PMPM_BC_RIGID_SDF;
  out->ints[0] = shape;
  out->ints[1] = dim == 2 ? 2 : axis;
  for (int c = 0; c < dim; c++) {
    out->reals[c] = center[c];
    out->reals[3 + c] = velocity ? velocity[c] : 0.0f;
  }
  out->reals[6] = angular_velocity;
  out->reals[7] = friction;
  for (int c = 0; c < 3; c++) out->reals[8 + c] = dims[c];
  if (shape == PMPM_SDF_SPHERE) out->reals[9] = out->reals[10] = 0.0f;
  out->reals[11] = contact_distance;
  out->reals[12] = angle0;
  return PMPM_OK;
}

int pmpm_calculate_timestep(float cell_size, float factor, float bulk_modulus, float shear_modulus,
                            float density, float *dt) {
  if (!dt || !(density > 0.0f) || !(cell_size > 0.0f)) return PMPM_ERR_INVALID_ARGUMENT;
  // c = (Real)sqrt((K + 4. G / 3.) / rho) in double, as the reference
  const float c = (float)std::sqrt(((double)bulk_modulus + 4.0 * (double)shear_modulus / 3.0) / (double)density);
  if (!(c > 0.0f)) return PMPM_ERR_INVALID_ARGUMENT;
  *dt = factor * (cell_size / c);
  return PMPM_OK;
}

int pmpm_material_timestep(const pmpm_material *mat, float cell_size, float factor, float *dt) {
  if (!mat) return PMPM_ERR_INVALID_ARGUMENT;
  switch (mat->type) {
    case PMPM_MAT_LINEAR_ELASTIC:
      return pmpm_calculate_timestep(cell_size, factor, mat->params[4], mat->params[3], mat->density, dt);
    case PMPM_MAT_NEWTON_FLUID:
      return pmpm_calculate_timestep(cell_size, factor, mat->params[1], 0.0f, mat->density, dt);
    case PMPM_MAT_DRUCKER_PRAGER:
    case PMPM_MAT_VON_MISES:
    case PMPM_MAT_MODIFIED_CAM_CLAY:
    case PMPM_MAT_DRUCKER_PRAGER_CAP:
      return pmpm_calculate_timestep(cell_size, factor, mat->params[0], mat->params[1], mat->density, dt);
    default:
      return PMPM_ERR_NOT_SUPPORTED;
  }
}

// Most (dual source, offset) pairs of any tile along an axis of n nodes, as
// the dual sweep builds them (build_dual_pairs): 24 inside the grid, 27 in a
// tile of eight node columns ending at the last node, where the clamped
// offsets of the face's dual cells fold onto that node (n a multiple of 8).
static int dual_pairs_max(int n) {
  int most = 0;
  for (int t0 = 0; t0 < n; t0 += TileDims<3>::X) {
    int cnt = 0;
    for (int si = 0; si < Dual3::NS; si++) {
      const int src = t0 - 1 + si;
      if (src < 0 || src > n) continue;
      for (int i = 0; i < 3; i++) {
        const int l = std::min(std::max(src - 1 + i, 0), n - 1) - t0;
        if (l >= 0 && l < TileDims<3>::X) cnt++;
      }
    }
    most = std::max(most, cnt);
  }
  return most;
}

// Binning key space: reference cells, or dual cells (floor(x/h + 1/2), one
// more per axis) for quadratic shape functions outside the deterministic mode.
// The dual sweep runs one work item per thread of its CTA: where a tile has
// more (27 pairs along x or y), the cell-row scatter P2G is used instead.
static void set_key_space(pmpm_sim *s) {
  s->dual = s->shape == PMPM_SHAPE_QUADRATIC && !(s->flags & PMPM_FLAG_DETERMINISTIC);
  s->nkeys = 1;
  for (int c = 0; c < 3; c++) {
    s->kd[c] = (s->dual && c < s->dim) ? s->g.n[c] + 1 : s->g.n[c];
    s->nkeys *= s->kd[c];
  }
  s->dual3_fits = !(s->dual && s->dim == 3) ||
                  dual_pairs_max(s->g.n[0]) * dual_pairs_max(s->g.n[1]) <= Dual3::NT * Dual3::IPT;
  if (!s->dual3_fits) s->p2g_variant = 0;
}

// Descriptor -> handle parameters: grid, materials and boundary conditions
// (BodyForce arrays are copied to the device; nothing else is allocated).
static int setup_handle(const pmpm_desc *desc, pmpm_sim *s) {
  if (desc->dim != 2 && desc->dim != 3) return PMPM_ERR_NOT_SUPPORTED;
  if (desc->shape_function < 0 || desc->shape_function > 2) return PMPM_ERR_INVALID_ARGUMENT;
  if (!(desc->cell_size > 0.0f) || desc->num_materials < 0 || desc->num_materials > PMPM_MAX_MATERIALS ||
      desc->num_bcs < 0 || desc->num_bcs > PMPM_MAX_BCS || desc->particles_per_cell <= 0)
    return PMPM_ERR_INVALID_ARGUMENT;
  if ((desc->num_materials > 0 && !desc->materials) || (desc->num_bcs > 0 && !desc->bcs))
    return PMPM_ERR_INVALID_ARGUMENT;
  s->device = desc->device;
  s->dim = desc->dim;
  s->shape = desc->shape_function;
  s->dt = desc->dt;
  s->alpha = desc->alpha;
  s->ppc = desc->particles_per_cell;
  s->flags = desc->flags;
  s->resort_interval = desc->resort_interval < 0 ? 0 : desc->resort_interval;
  // Grid (include/pyroclastmpm/common/types_common.h:260-272), FP32 as the reference
  DevGrid &g = s->g;
  g.h = desc->cell_size;
  g.inv_h = 1.0f / desc->cell_size;
  g.ntotal = 1;
  for (int c = 0; c < 3; c++) {
    g.n[c] = 1;
    g.origin[c] = 0.0f;
    g.end[c] = 0.0f;
    if (c < s->dim) {
      g.origin[c] = desc->origin[c];
      g.end[c] = desc->end[c];
      const float span = desc->end[c] - desc->origin[c];
      g.n[c] = (int)(span / desc->cell_size) + 1;
      if (g.n[c] < 1) return PMPM_ERR_INVALID_ARGUMENT;
    }
    g.ntotal *= g.n[c];
  }
  const int tsz[3] = {s->dim == 2 ? TileDims<2>::X : TileDims<3>::X, s->dim == 2 ? TileDims<2>::Y : TileDims<3>::Y,
                      s->dim == 2 ? 1 : TileDims<3>::Z};
  g.ntiles = 1;
  for (int c = 0; c < 3; c++) {
    g.tdim[c] = (g.n[c] + tsz[c] - 1) / tsz[c];
    g.ntiles *= g.tdim[c];
  }
  // materials
  for (int k = 0; k < desc->num_materials; k++) {
    const pmpm_material &m = desc->materials[k];
    if (m.type < PMPM_MAT_NONE || m.type > PMPM_MAT_DRUCKER_PRAGER_CAP) return PMPM_ERR_INVALID_ARGUMENT;
    if (m.type == PMPM_MAT_MODIFIED_CAM_CLAY || m.type == PMPM_MAT_DRUCKER_PRAGER_CAP) {
      s->has_mcc = true;
      s->has_dp = true;  // elastic strain and reference stress
    }
    if (m.type == PMPM_MAT_VON_MISES) {
      if (desc->dim != 3) return PMPM_ERR_NOT_SUPPORTED;  // the reference's VonMises is 3D only
      s->has_vm = true;
      s->has_dp = true;  // elastic-strain history arrays
    }
    DevMaterial dm;
    memset(&dm, 0, sizeof(dm));
    dm.type = m.type;
    dm.density = m.density;
    memcpy(dm.p, m.params, sizeof(m.params));
    if (m.type == PMPM_MAT_NEWTON_FLUID) dm.p[3] = (float)(2.0 * (double)m.params[0] / 3.0);
    if (m.type == PMPM_MAT_DRUCKER_PRAGER) {
      s->has_dp = true;
      // cohesion from kc = xi(phi) c, phi from eta = 6 sin(phi) / (sqrt(3) (3 - sin(phi)))
      const double eta = m.params[2], s3 = std::sqrt(3.0);
      const double sn = 3.0 * s3 * eta / (6.0 + s3 * eta);
      const double xi = 6.0 * std::sqrt(std::max(0.0, 1.0 - sn * sn)) / (s3 * (3.0 - sn));
      dm.p[8] = xi > 0.0 ? (float)((double)m.params[4] / xi) : 0.0f;
      dm.p[9] = (float)(std::asin(std::min(1.0, sn)) * 180.0 / 3.14159265358979323846);
    }
    s->mats.push_back(dm);
  }
  int st = PMPM_OK;
  // boundary conditions
  for (int k = 0; k < desc->num_bcs && st == PMPM_OK; k++) {
    const pmpm_bc &b = desc->bcs[k];
    DevBC db;
    memset(&db, 0, sizeof(db));
    db.type = b.type;
    memcpy(db.i, b.ints, sizeof(db.i));
    memcpy(db.r, b.reals, sizeof(db.r));
    if (b.type == PMPM_BC_GRAVITY) {
      GravityState gs;
      gs.bc_index = k;
      for (int c = 0; c < 3; c++) gs.current[c] = b.reals[c];
      s->gravity.push_back(gs);
    } else if (b.type == PMPM_BC_BODYFORCE) {
      if (!b.values || !b.mask) {
        st = PMPM_ERR_INVALID_ARGUMENT;
        break;
      }
      float *vals = nullptr;
      uint8_t *mask = nullptr;
      st = dalloc(&vals, (size_t)g.ntotal * s->dim);
      if (st == PMPM_OK) st = dalloc(&mask, (size_t)g.ntotal);
      if (st == PMPM_OK &&
          (cudaMemcpy(vals, b.values, sizeof(float) * g.ntotal * s->dim, cudaMemcpyHostToDevice) != cudaSuccess ||
           cudaMemcpy(mask, b.mask, g.ntotal, cudaMemcpyHostToDevice) != cudaSuccess))
        st = PMPM_ERR_CUDA;
      s->bc_values.push_back(vals);
      s->bc_masks.push_back(mask);
      db.values = vals;
      db.mask = mask;
    } else if (b.type == PMPM_BC_PLANARDOMAIN) {
      s->has_planar = true;
    } else if (b.type == PMPM_BC_RIGIDBODY_LEVELSET) {
      // the reference hard-codes the linear window (rigidbodylevelset_inline.h:88-101)
      if (s->rbls_index >= 0 || s->shape != PMPM_SHAPE_LINEAR || (s->flags & PMPM_FLAG_MUSL)) {
        st = PMPM_ERR_NOT_SUPPORTED;
        break;
      }
      if (b.ints[0] != PMPM_RIGID_STATIC && b.ints[0] != PMPM_RIGID_LOOP_ROTATE) {
        st = PMPM_ERR_INVALID_ARGUMENT;
        break;
      }
      s->rbls_index = k;
      s->rigid.mode = b.ints[0];
      s->rigid.corrected = b.ints[1] ? 1 : 0;
      for (int c = 0; c < 3; c++) {
        s->rigid.rate[c] = b.reals[c];
        s->rigid.com[c] = b.reals[3 + c];
      }
    } else if (b.type == PMPM_BC_RIGID_SDF) {
      const int shape = b.ints[0], axis = b.ints[1];
      const bool dims_ok = b.reals[8] > 0.0f && (shape == PMPM_SDF_SPHERE || (b.reals[9] > 0.0f && b.reals[10] > 0.0f));
      if ((shape != PMPM_SDF_SPHERE && shape != PMPM_SDF_HALF_CYLINDER_SHELL) || axis < 0 || axis > 2 || !dims_ok ||
          !(b.reals[7] >= 0.0f)) {
        st = PMPM_ERR_INVALID_ARGUMENT;
        break;
      }
      SdfState sd;
      sd.bc_index = k;
      for (int c = 0; c < 3; c++) {
        sd.c0[c] = c < s->dim ? b.reals[c] : 0.0;
        sd.v[c] = c < s->dim ? b.reals[3 + c] : 0.0;
        db.r[3 + c] = (float)sd.v[c];
      }
      sd.omega = b.reals[6];
      sd.angle0 = b.reals[12];
      s->sdf.push_back(sd);
    } else if (b.type != PMPM_BC_NODEDOMAIN) {
      st = PMPM_ERR_INVALID_ARGUMENT;
    }
    s->bcs.push_back(db);
  }
  return st;
}

int pmpm_create(const pmpm_desc *desc, pmpm_sim **out) {
  if (!desc || !out) return PMPM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (desc->dim != 2 && desc->dim != 3) return PMPM_ERR_NOT_SUPPORTED;
  if (desc->shape_function < 0 || desc->shape_function > 2) return PMPM_ERR_INVALID_ARGUMENT;
  if (!(desc->cell_size > 0.0f) || desc->num_materials < 0 || desc->num_materials > PMPM_MAX_MATERIALS ||
      desc->num_bcs < 0 || desc->num_bcs > PMPM_MAX_BCS || desc->particles_per_cell <= 0)
    return PMPM_ERR_INVALID_ARGUMENT;
  if ((desc->num_materials > 0 && !desc->materials) || (desc->num_bcs > 0 && !desc->bcs))
    return PMPM_ERR_INVALID_ARGUMENT;
  PMPM_CUDA(cudaSetDevice(desc->device));
  pmpm_sim *s = new pmpm_sim();
  int st = setup_handle(desc, s);
  if (st == PMPM_OK) {
    if (desc->stream) {
      s->stream = (cudaStream_t)desc->stream;
    } else if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) == cudaSuccess) {
      s->own_stream = true;
    } else {
      st = PMPM_ERR_CUDA;
    }
  }
  const DevGrid &g = s->g;
  // nodes and bins
  const size_t nn = (size_t)g.ntotal, D = (size_t)s->dim;
  if (st == PMPM_OK) st = dalloc(&s->N.m, nn);
  if (st == PMPM_OK) st = dalloc(&s->N.p, nn * D);
  if (st == PMPM_OK) st = dalloc(&s->N.pnt, nn * D);
  if (st == PMPM_OK) st = dalloc(&s->N.vel, nn * (s->dim == 3 ? NodeVel<3>::F : NodeVel<2>::F));
  if (st == PMPM_OK) st = dalloc(&s->N.tile_epoch, (size_t)g.ntiles);
  if (st == PMPM_OK) st = dalloc(&s->node_epoch, (size_t)g.ntiles);
  if (st == PMPM_OK) st = dalloc(&s->N.tile_list, (size_t)g.ntiles);
  if (st == PMPM_OK) st = dalloc(&s->N.tile_queue, 4);
  if (st == PMPM_OK && cudaMemset(s->N.tile_queue, 0, 4 * sizeof(int)) != cudaSuccess) st = PMPM_ERR_CUDA;
  if (st == PMPM_OK && cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device) != cudaSuccess)
    st = PMPM_ERR_CUDA;
  set_key_space(s);
  const size_t nk = (size_t)s->nkeys;
  s->nscan_blocks = (s->nkeys + kScanChunk - 1) / kScanChunk;
  if (st == PMPM_OK) st = dalloc(&s->B.count, nk);
  if (st == PMPM_OK) st = dalloc(&s->B.offset, nk + 1);
  if (st == PMPM_OK) st = dalloc(&s->B.block_sums, (size_t)s->nscan_blocks);
  if (st == PMPM_OK) st = alloc_scan(s->scan, s->nscan_blocks);
  if (st == PMPM_OK) st = dalloc(&s->B.scalars, 4);
  if (st == PMPM_OK) st = dalloc(&s->B.big_cells, nk);
  if (st == PMPM_OK && s->dual && s->dim == 3) {
    s->nbricks = 1;
    for (int c = 0; c < 3; c++) {
      s->B.kb[c] = (s->kd[c] + Cells3::B - 1) / Cells3::B;
      s->nbricks *= s->B.kb[c];
    }
    st = dalloc(&s->B.brick_epoch, (size_t)s->nbricks);
    if (st == PMPM_OK) st = dalloc(&s->N.acc, 8 * nn);
    if (st == PMPM_OK && (cudaMemset(s->B.brick_epoch, 0xff, sizeof(int) * s->nbricks) != cudaSuccess ||
                          cudaMemset(s->N.acc, 0, sizeof(float) * 8 * nn) != cudaSuccess))
      st = PMPM_ERR_CUDA;
  }
  if (st == PMPM_OK) st = dalloc(&s->fault, 1);
  if (st == PMPM_OK) {
    if (cudaMemset(s->B.count, 0, nk * sizeof(int)) != cudaSuccess ||
        cudaMemset(s->B.scalars, 0, 4 * sizeof(int)) != cudaSuccess ||
        cudaMemset(s->fault, 0, sizeof(int)) != cudaSuccess ||
        cudaMemset(s->N.tile_epoch, 0xff, g.ntiles * sizeof(int)) != cudaSuccess ||
        cudaMemset(s->node_epoch, 0xff, g.ntiles * sizeof(int)) != cudaSuccess ||
        cudaMemset(s->N.m, 0, nn * sizeof(float)) != cudaSuccess)
      st = PMPM_ERR_CUDA;
  }
  if (st != PMPM_OK) {
    pmpm_destroy(s);
    return st;
  }
  *out = s;
  return PMPM_OK;
}

int pmpm_destroy(pmpm_sim *s) {
  if (!s) return PMPM_ERR_INVALID_ARGUMENT;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  free_particles(s);
  dfree(s->N.m);
  dfree(s->N.p);
  dfree(s->N.pnt);
  dfree(s->N.vel);
  dfree(s->N.tile_epoch);
  dfree(s->N.tile_list);
  dfree(s->N.tile_queue);
  dfree(s->node_epoch);
  dfree(s->B.count);
  dfree(s->B.offset);
  dfree(s->B.block_sums);
  free_scan(s->scan);
  dfree(s->B.scalars);
  dfree(s->B.big_cells);
  dfree(s->B.brick_epoch);
  dfree(s->N.acc);
  dfree(s->fault);
  for (float *p : s->bc_values) dfree(p);
  for (uint8_t *p : s->bc_masks) dfree(p);
  if (s->staging) cudaFree(s->staging);
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return PMPM_OK;
}

int pmpm_get_grid(const pmpm_sim *s, int num_cells[3], int *num_cells_total, float *inv_cell_size) {
  if (!s) return PMPM_ERR_INVALID_ARGUMENT;
  if (num_cells)
    for (int c = 0; c < 3; c++) num_cells[c] = s->g.n[c];
  if (num_cells_total) *num_cells_total = s->g.ntotal;
  if (inv_cell_size) *inv_cell_size = s->g.inv_h;
  return PMPM_OK;
}

int pmpm_num_particles(const pmpm_sim *s) { return s ? s->n : -1; }
int pmpm_num_nodes(const pmpm_sim *s) { return s ? s->g.ntotal : -1; }
void *pmpm_stream(const pmpm_sim *s) { return s ? (void *)s->stream : nullptr; }

int pmpm_num_surround_nodes(const pmpm_sim *s) {
  if (!s) return -1;
  const int w = s->shape == PMPM_SHAPE_LINEAR ? 2 : 4;
  return s->dim == 2 ? w * w : w * w * w;
}

size_t pmpm_field_bytes(const pmpm_sim *s, int field) {
  size_t b = 0;
  if (!s || field_info(s, field, &b) != PMPM_OK) return 0;
  return b;
}

int pmpm_set_particles(pmpm_sim *s, int num_particles, const float *positions, const float *velocities,
                       const unsigned char *colors, int num_rigid, const float *rigid_positions,
                       const float *rigid_velocities, const unsigned char *rigid_colors) {
  if (!s || num_particles < 0 || num_rigid < 0 || (num_particles > 0 && !positions) ||
      (num_rigid > 0 && !rigid_positions) || num_particles + num_rigid < 1)
    return PMPM_ERR_INVALID_ARGUMENT;
  PMPM_CUDA(cudaSetDevice(s->device));
  PMPM_TRY(drop_fresh_keys(s));
  PMPM_CUDA(cudaStreamSynchronize(s->stream));
  free_particles(s);
  const int D = s->dim;
  const int n = num_particles + num_rigid;
  s->n = n;
  s->stride = (n + 63) / 64 * 64;
  s->cur = 0;
  PMPM_TRY(alloc_particle_set(s, s->P[0]));
  PMPM_TRY(alloc_particle_set(s, s->P[1]));
  PMPM_TRY(dalloc(&s->slot, (size_t)s->stride));
  PMPM_TRY(dalloc(&s->key, (size_t)s->stride));
  if (s->dual) PMPM_TRY(dalloc(&s->hash_next, (size_t)s->stride));
  PMPM_TRY(dalloc(&s->B.order, (size_t)s->stride));
  if (s->dim == 3 && !(s->flags & PMPM_FLAG_DETERMINISTIC)) {
    // sorted P2G records of the 3D sweep kernels (k_records)
    s->B.rec4 = s->has_planar ? 5 : 4;
    PMPM_TRY(dalloc(&s->B.rec, (size_t)s->stride * s->B.rec4));
  }
  if (s->flags & PMPM_FLAG_MUSL) PMPM_TRY(dalloc(&s->musl_x, (size_t)s->dim * s->stride));
  const int st = s->stride;
  const int S = D == 2 ? 4 : 6, E = D == 2 ? 3 : 6;
  // ParticlesContainer ctor (src/particles/particles.cpp:51-149): rigid particles appended
  std::vector<float> x((size_t)D * st, 0.0f), v((size_t)D * st, 0.0f), F((size_t)D * D * st, 0.0f);
  std::vector<float> m(st, -1.0f), V(st, -1.0f);
  std::vector<uint8_t> color(st, 0), rigid(st, 0), active(st, 1);
  std::vector<int> id(st, 0);
  for (int i = 0; i < n; i++) {
    const bool r = i >= num_particles;
    const int j = r ? i - num_particles : i;
    const float *px = r ? rigid_positions : positions;
    const float *pv = r ? rigid_velocities : velocities;
    const unsigned char *pc = r ? rigid_colors : colors;
    for (int c = 0; c < D; c++) {
      x[(size_t)c * st + i] = px[(size_t)j * D + c];
      v[(size_t)c * st + i] = pv ? pv[(size_t)j * D + c] : 0.0f;
    }
    for (int c = 0; c < D; c++) F[(size_t)(c * D + c) * st + i] = 1.0f;
    color[i] = pc ? pc[j] : 0;
    rigid[i] = r ? 1 : 0;
    id[i] = i;
  }
  DevParticles &P = s->P[0];
  PMPM_CUDA(cudaMemcpy(P.x, x.data(), sizeof(float) * x.size(), cudaMemcpyHostToDevice));
  PMPM_CUDA(cudaMemcpy(P.v, v.data(), sizeof(float) * v.size(), cudaMemcpyHostToDevice));
  PMPM_CUDA(cudaMemcpy(P.F, F.data(), sizeof(float) * F.size(), cudaMemcpyHostToDevice));
  PMPM_CUDA(cudaMemset(P.sig, 0, sizeof(float) * S * st));
  PMPM_CUDA(cudaMemset(P.L, 0, sizeof(float) * D * D * st));
  PMPM_CUDA(cudaMemset(s->P[1].L, 0, sizeof(float) * D * D * st));
  PMPM_CUDA(cudaMemcpy(P.m, m.data(), sizeof(float) * st, cudaMemcpyHostToDevice));
  PMPM_CUDA(cudaMemcpy(P.V, V.data(), sizeof(float) * st, cudaMemcpyHostToDevice));
  PMPM_CUDA(cudaMemcpy(P.V0, V.data(), sizeof(float) * st, cudaMemcpyHostToDevice));
  if (P.fext) PMPM_CUDA(cudaMemset(P.fext, 0, sizeof(float) * D * st));
  if (P.eps) PMPM_CUDA(cudaMemset(P.eps, 0, sizeof(float) * E * st));
  if (P.sref) PMPM_CUDA(cudaMemset(P.sref, 0, sizeof(float) * S * st));
  if (P.acc) PMPM_CUDA(cudaMemset(P.acc, 0, sizeof(float) * st));
  if (P.pc) PMPM_CUDA(cudaMemset(P.pc, 0, sizeof(float) * st));
  PMPM_CUDA(cudaMemcpy(P.color, color.data(), st, cudaMemcpyHostToDevice));
  PMPM_CUDA(cudaMemcpy(P.rigid, rigid.data(), st, cudaMemcpyHostToDevice));
  PMPM_CUDA(cudaMemcpy(P.active, active.data(), st, cudaMemcpyHostToDevice));
  PMPM_CUDA(cudaMemcpy(P.id, id.data(), sizeof(int) * st, cudaMemcpyHostToDevice));
  PMPM_CUDA(cudaMemset(P.hash, 0, sizeof(unsigned) * st));
  PMPM_CUDA(cudaMemset(s->B.order, 0, sizeof(int) * st));
  s->partitioned = false;
  s->steps_since_sort = 0;
  return PMPM_OK;
}

int pmpm_partition(pmpm_sim *s) {
  if (!s) return PMPM_ERR_INVALID_ARGUMENT;
  if (s->n == 0) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(s->device));
  return PMPM_DISPATCH(s, launch_partition, s);
}

int pmpm_initialize(pmpm_sim *s) {
  if (!s) return PMPM_ERR_INVALID_ARGUMENT;
  if (s->n == 0) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(s->device));
  PMPM_TRY(pmpm_partition(s));
  // particle storage starts in cell order (the re-sort interval counts from here)
  if (s->resort_interval > 0 && !s->ro.held) PMPM_TRY(s->dim == 2 ? launch_reorder<2>(s) : launch_reorder<3>(s));
  DevParticles &P = s->P[s->cur];
  // calculate_initial_volumes: (REAL)pow(h, DIM) / ppc
  float vol = (float)std::pow((double)s->g.h, (double)s->dim);
  vol = vol / (float)s->ppc;
  k_initial_volumes<<<blocks_for(s->n), kTPB, 0, s->stream>>>(P, vol);
  PMPM_LAUNCHED();
  for (int k = 0; k < (int)s->mats.size(); k++) {
    k_initial_masses<<<blocks_for(s->n), kTPB, 0, s->stream>>>(P, k, s->mats[k].density);
    PMPM_LAUNCHED();
  }
  if (s->has_dp) {
    int *flag = s->B.scalars + 3;
    PMPM_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s->stream));
    k_dp_init<<<blocks_for(s->n), kTPB, 0, s->stream>>>(P, s->dim, flag);
    PMPM_LAUNCHED();
    int h = 0;
    PMPM_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    PMPM_CUDA(cudaStreamSynchronize(s->stream));
    s->has_sref = h != 0;
  }
  if (s->has_mcc) {
    k_mcc_init<<<blocks_for(s->n), kTPB, 0, s->stream>>>(make_args(s), s->dim);
    PMPM_LAUNCHED();
  }
  PMPM_CUDA(cudaStreamSynchronize(s->stream));
  return PMPM_OK;
}

int pmpm_get_field(pmpm_sim *s, int field, void *dst, size_t bytes, int on_device) {
  if (!s || !dst) return PMPM_ERR_INVALID_ARGUMENT;
  size_t need = 0;
  PMPM_TRY(field_info(s, field, &need));
  if (bytes != need) return PMPM_ERR_INVALID_ARGUMENT;
  const bool particle_field = field < PMPM_FIELD_NODE_MASSES || field == PMPM_FIELD_BINS ||
                              (field >= PMPM_FIELD_HASH_UNSORTED && field <= PMPM_FIELD_SORTED_INDEX);
  if (particle_field && s->n == 0) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(s->device));
  const int D = s->dim;
  const DevParticles &P = s->P[s->cur];
  // host-computed fields
  if (field == PMPM_FIELD_NODE_IDS || field == PMPM_FIELD_NODE_TYPES || field == PMPM_FIELD_SORTED_INDEX ||
      field == PMPM_FIELD_HASH_SORTED || field == PMPM_FIELD_CELL_START || field == PMPM_FIELD_CELL_END) {
    std::vector<int> host(need / 4, 0);
    const DevGrid &g = s->g;
    if (field == PMPM_FIELD_NODE_IDS || field == PMPM_FIELD_NODE_TYPES) {
      for (int node = 0; node < g.ntotal; node++) {
        const int c[3] = {node % g.n[0], (node / g.n[0]) % g.n[1], node / (g.n[0] * g.n[1])};
        for (int a = 0; a < 3; a++) {
          int val = c[a];
          if (field == PMPM_FIELD_NODE_TYPES) {
            // calculate_bin_types (src/nodes/nodes.cpp:135-173): cubic grids only
            if (s->shape != PMPM_SHAPE_CUBIC || a >= D)
              val = 0;
            else
              val = (c[a] == 0 || c[a] == g.n[a] - 1) ? 1 : (c[a] == 1 ? 2 : 3);
          }
          host[(size_t)node * 3 + a] = val;
        }
      }
    } else if (field == PMPM_FIELD_SORTED_INDEX || field == PMPM_FIELD_HASH_SORTED) {
      std::vector<int> si;
      std::vector<unsigned> hs;
      PMPM_TRY(sorted_views(s, si, hs));
      if (field == PMPM_FIELD_SORTED_INDEX)
        memcpy(host.data(), si.data(), need);
      else
        memcpy(host.data(), hs.data(), need);
    } else {
      // cell_start / cell_end: 0 for empty cells (SpatialPartition::reset fills 0)
      std::vector<int> off(g.ntotal + 1, 0);
      if (s->dual) {
        std::vector<unsigned> hash(s->n);
        PMPM_CUDA(cudaMemcpyAsync(hash.data(), P.hash, sizeof(unsigned) * s->n, cudaMemcpyDeviceToHost, s->stream));
        PMPM_CUDA(cudaStreamSynchronize(s->stream));
        for (unsigned h : hash)
          if (h < (unsigned)g.ntotal) off[h + 1] += 1;
        for (int c = 0; c < g.ntotal; c++) off[c + 1] += off[c];
      } else {
        PMPM_CUDA(cudaMemcpyAsync(off.data(), s->B.offset, sizeof(int) * (g.ntotal + 1), cudaMemcpyDeviceToHost,
                                  s->stream));
        PMPM_CUDA(cudaStreamSynchronize(s->stream));
      }
      for (int c = 0; c < g.ntotal; c++) {
        const bool occupied = off[c + 1] > off[c];
        host[c] = occupied ? (field == PMPM_FIELD_CELL_START ? off[c] : off[c + 1]) : 0;
      }
    }
    if (on_device) {
      PMPM_CUDA(cudaMemcpy(dst, host.data(), need, cudaMemcpyHostToDevice));
    } else {
      memcpy(dst, host.data(), need);
    }
    return PMPM_OK;
  }
  PMPM_TRY(ensure_staging(s, need));
  if (field >= PMPM_FIELD_NODE_MASSES && field <= PMPM_FIELD_NODE_MOMENTS_NT) {
    const float *src = field == PMPM_FIELD_NODE_MASSES ? s->N.m : (field == PMPM_FIELD_NODE_MOMENTS ? s->N.p : s->N.pnt);
    const int ncomp = field == PMPM_FIELD_NODE_MASSES ? 1 : D;
    k_get_nodes<<<blocks_for(s->g.ntotal), kTPB, 0, s->stream>>>(s->g, D, ncomp, src, s->node_epoch, s->p2g_epoch,
                                                                  (float *)s->staging);
    PMPM_LAUNCHED();
    return copy_out(s, s->staging, dst, need, on_device);
  }
  int kind = -1;
  const void *src = nullptr;
  DevGrid *gdev = nullptr;
  switch (field) {
    case PMPM_FIELD_POSITIONS: kind = 0; src = P.x; break;
    case PMPM_FIELD_VELOCITIES: kind = 0; src = P.v; break;
    case PMPM_FIELD_FORCES_EXTERNAL:
      if (!P.fext) {
        PMPM_CUDA(cudaMemsetAsync(s->staging, 0, need, s->stream));
        return copy_out(s, s->staging, dst, need, on_device);
      }
      kind = 0;
      src = P.fext;
      break;
    case PMPM_FIELD_STRESSES: kind = 2; src = P.sig; break;
    case PMPM_FIELD_STRESS_REF:
      if (!P.sref) {
        PMPM_CUDA(cudaMemsetAsync(s->staging, 0, need, s->stream));
        return copy_out(s, s->staging, dst, need, on_device);
      }
      kind = 2;
      src = P.sref;
      break;
    case PMPM_FIELD_F: kind = 1; src = P.F; break;
    case PMPM_FIELD_VELOCITY_GRADIENT: kind = 1; src = P.L; break;
    case PMPM_FIELD_EPS_E:
      if (!P.eps) {
        PMPM_CUDA(cudaMemsetAsync(s->staging, 0, need, s->stream));
        return copy_out(s, s->staging, dst, need, on_device);
      }
      kind = 3;
      src = P.eps;
      break;
    case PMPM_FIELD_MASSES: kind = 4; src = P.m; break;
    case PMPM_FIELD_VOLUMES: kind = 4; src = P.V; break;
    case PMPM_FIELD_VOLUMES_ORIGINAL: kind = 4; src = P.V0; break;
    case PMPM_FIELD_ACC_EPS_P:
    case PMPM_FIELD_PRECONSOLIDATION:
      src = field == PMPM_FIELD_ACC_EPS_P ? P.acc : P.pc;
      if (!src) {
        PMPM_CUDA(cudaMemsetAsync(s->staging, 0, need, s->stream));
        return copy_out(s, s->staging, dst, need, on_device);
      }
      kind = 4;
      break;
    case PMPM_FIELD_YOUNGS_MODULUS:
    case PMPM_FIELD_FRICTION_ANGLE:
      PMPM_TRY(ensure_particle_params(s));
      kind = 4;
      src = field == PMPM_FIELD_YOUNGS_MODULUS ? s->P[s->cur].pE : s->P[s->cur].pphi;
      break;
    case PMPM_FIELD_COLORS: kind = 5; src = P.color; break;
    case PMPM_FIELD_IS_RIGID: kind = 5; src = P.rigid; break;
    case PMPM_FIELD_IS_ACTIVE: kind = 5; src = P.active; break;
    case PMPM_FIELD_HASH_UNSORTED: kind = 6; src = P.hash; break;
    case PMPM_FIELD_BINS: {
      kind = 7;
      PMPM_TRY(ensure_staging(s, need + sizeof(DevGrid) + 256));
      gdev = (DevGrid *)((char *)s->staging + ((need + 255) / 256) * 256);
      PMPM_CUDA(cudaMemcpyAsync(gdev, &s->g, sizeof(DevGrid), cudaMemcpyHostToDevice, s->stream));
      src = gdev;
      break;
    }
    default: return PMPM_ERR_INVALID_ARGUMENT;
  }
  k_get_particles<<<blocks_for(s->n), kTPB, 0, s->stream>>>(P, D, kind, src, s->staging, 0);
  PMPM_LAUNCHED();
  return copy_out(s, s->staging, dst, need, on_device);
}

int pmpm_set_field(pmpm_sim *s, int field, const void *src, size_t bytes, int on_device) {
  if (!s || !src) return PMPM_ERR_INVALID_ARGUMENT;
  size_t need = 0;
  PMPM_TRY(field_info(s, field, &need));
  if (bytes != need) return PMPM_ERR_INVALID_ARGUMENT;
  if (s->n == 0) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(s->device));
  PMPM_TRY(drop_fresh_keys(s));
  const DevParticles &P = s->P[s->cur];
  int kind = -1;
  void *dstp = nullptr;
  switch (field) {
    case PMPM_FIELD_POSITIONS: kind = 0; dstp = P.x; break;
    case PMPM_FIELD_VELOCITIES: kind = 0; dstp = P.v; break;
    case PMPM_FIELD_STRESSES: kind = 2; dstp = P.sig; break;
    case PMPM_FIELD_STRESS_REF: kind = 2; dstp = P.sref; break;
    case PMPM_FIELD_F: kind = 1; dstp = P.F; break;
    case PMPM_FIELD_VELOCITY_GRADIENT: kind = 1; dstp = P.L; break;
    case PMPM_FIELD_EPS_E: kind = 3; dstp = P.eps; break;
    case PMPM_FIELD_MASSES: kind = 4; dstp = P.m; break;
    case PMPM_FIELD_VOLUMES: kind = 4; dstp = P.V; break;
    case PMPM_FIELD_VOLUMES_ORIGINAL: kind = 4; dstp = P.V0; break;
    case PMPM_FIELD_ACC_EPS_P: kind = 4; dstp = P.acc; break;
    case PMPM_FIELD_PRECONSOLIDATION: kind = 4; dstp = P.pc; break;
    case PMPM_FIELD_YOUNGS_MODULUS:
    case PMPM_FIELD_FRICTION_ANGLE:
      PMPM_TRY(ensure_particle_params(s));
      kind = 4;
      dstp = field == PMPM_FIELD_YOUNGS_MODULUS ? s->P[s->cur].pE : s->P[s->cur].pphi;
      break;
    case PMPM_FIELD_COLORS: kind = 5; dstp = P.color; break;
    case PMPM_FIELD_IS_RIGID: kind = 5; dstp = P.rigid; break;
    case PMPM_FIELD_IS_ACTIVE: kind = 5; dstp = P.active; break;
    case PMPM_FIELD_FORCES_EXTERNAL: kind = 0; dstp = P.fext; break;
    default: return PMPM_ERR_NOT_SUPPORTED;
  }
  if (!dstp) return PMPM_ERR_NOT_SUPPORTED;  // field not held by this configuration
  const void *dsrc = src;
  if (!on_device) {
    PMPM_TRY(ensure_staging(s, need));
    PMPM_CUDA(cudaMemcpyAsync(s->staging, src, need, cudaMemcpyHostToDevice, s->stream));
    dsrc = s->staging;
  }
  k_set_particles<<<blocks_for(s->n), kTPB, 0, s->stream>>>(P, s->dim, kind, dsrc, dstp);
  PMPM_LAUNCHED();
  PMPM_CUDA(cudaStreamSynchronize(s->stream));
  return PMPM_OK;
}

int pmpm_shape_functions(pmpm_sim *s, float *psi, float *dpsi, int on_device) {
  if (!s || !psi || !dpsi) return PMPM_ERR_INVALID_ARGUMENT;
  if (s->n == 0) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(s->device));
  const size_t nsn = (size_t)pmpm_num_surround_nodes(s);
  const size_t bpsi = (size_t)s->n * nsn * 4, bdpsi = bpsi * s->dim;
  PMPM_TRY(ensure_staging(s, bpsi + bdpsi));
  float *dp = (float *)s->staging;
  float *dd = dp + (size_t)s->n * nsn;
  StepArgs a = make_args(s);
#define PMPM_SHAPE_LAUNCH(D, SF) k_shape_dump<D, SF><<<blocks_for(s->n), kTPB, 0, s->stream>>>(a, dp, dd)
  if (s->dim == 2) {
    if (s->shape == PMPM_SHAPE_LINEAR) PMPM_SHAPE_LAUNCH(2, PMPM_SHAPE_LINEAR);
    else if (s->shape == PMPM_SHAPE_QUADRATIC) PMPM_SHAPE_LAUNCH(2, PMPM_SHAPE_QUADRATIC);
    else PMPM_SHAPE_LAUNCH(2, PMPM_SHAPE_CUBIC);
  } else {
    if (s->shape == PMPM_SHAPE_LINEAR) PMPM_SHAPE_LAUNCH(3, PMPM_SHAPE_LINEAR);
    else if (s->shape == PMPM_SHAPE_QUADRATIC) PMPM_SHAPE_LAUNCH(3, PMPM_SHAPE_QUADRATIC);
    else PMPM_SHAPE_LAUNCH(3, PMPM_SHAPE_CUBIC);
  }
#undef PMPM_SHAPE_LAUNCH
  PMPM_LAUNCHED();
  const cudaMemcpyKind kd = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  PMPM_CUDA(cudaMemcpyAsync(psi, dp, bpsi, kd, s->stream));
  PMPM_CUDA(cudaMemcpyAsync(dpsi, dd, bdpsi, kd, s->stream));
  PMPM_CUDA(cudaStreamSynchronize(s->stream));
  return PMPM_OK;
}

int pmpm_p2g(pmpm_sim *s, int apply_bcs) {
  if (!s) return PMPM_ERR_INVALID_ARGUMENT;
  if (s->n == 0 || !s->partitioned) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(s->device));
  return PMPM_DISPATCH(s, launch_p2g, s, apply_bcs ? 1 : 0);
}

int pmpm_g2p(pmpm_sim *s, int stress_update) {
  if (!s) return PMPM_ERR_INVALID_ARGUMENT;
  if (s->n == 0 || !s->partitioned) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(s->device));
  return PMPM_DISPATCH(s, launch_g2p, s, stress_update ? 1 : 0, 1);
}

}  // extern "C"

namespace {
template <int D, int SF>
int musl_stage(pmpm_sim *s, int stage) {
  int st = PMPM_OK;
  if (stage == 1) {
    s->musl_pass_now = 1;
    st = launch_g2p<D, SF>(s, 0, 0);
  } else if (stage == 2) {
    s->remap_now = 1;
    st = launch_p2g<D, SF>(s, 1);
  } else {
    s->musl_pass_now = 2;
    st = launch_g2p<D, SF>(s, 1, 1);
  }
  s->musl_pass_now = 0;
  s->remap_now = 0;
  return st;
}
}  // namespace

extern "C" {

int pmpm_musl_stage(pmpm_sim *s, int stage) {
  if (!s || stage < 1 || stage > 3) return PMPM_ERR_INVALID_ARGUMENT;
  if (!(s->flags & PMPM_FLAG_MUSL)) return PMPM_ERR_STATE;
  if (s->n == 0 || !s->partitioned) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(s->device));
  return PMPM_DISPATCH(s, musl_stage, s, stage);
}

int pmpm_stress_update(pmpm_sim *s) {
  if (!s) return PMPM_ERR_INVALID_ARGUMENT;
  if (s->n == 0) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(s->device));
  StepArgs a = make_args(s);
  if (s->dim == 2)
    k_stress_update<2><<<blocks_for(s->n), kTPB, 0, s->stream>>>(a);
  else
    k_stress_update<3><<<blocks_for(s->n), kTPB, 0, s->stream>>>(a);
  PMPM_LAUNCHED();
  return PMPM_OK;
}

int pmpm_solve(pmpm_sim *s, int nsteps) {
  if (!s || nsteps < 0) return PMPM_ERR_INVALID_ARGUMENT;
  if (s->n == 0) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(s->device));
  for (int k = 0; k < nsteps; k++) PMPM_TRY(PMPM_DISPATCH(s, step_once, s));
  return PMPM_OK;
}

}  // extern "C"

namespace {
template <int D, int SF>
int profile_step(pmpm_sim *s, float *ms, int *launches) {
  cudaEvent_t ev[4];
  for (int k = 0; k < 4; k++) PMPM_CUDA(cudaEventCreate(&ev[k]));
  int n_launch = 0;
  PMPM_CUDA(cudaEventRecord(ev[0], s->stream));
  PMPM_TRY((launch_partition<D, SF>(s)));
  n_launch += ((s->flags & PMPM_FLAG_DETERMINISTIC) || s->rbls_index >= 0) ? 7 : 5;
  if (!s->ro.held && !s->tuning && s->resort_interval > 0 && s->steps_since_sort + 1 >= s->resort_interval) {
    PMPM_TRY(launch_reorder<D>(s));
    n_launch += 1;
  } else {
    s->steps_since_sort += 1;
  }
  PMPM_CUDA(cudaEventRecord(ev[1], s->stream));
  const long long lp0 = s->launches;
  PMPM_TRY((launch_p2g<D, SF>(s, 1)));
  n_launch += (int)(s->launches - lp0);
  PMPM_CUDA(cudaEventRecord(ev[2], s->stream));
  const int store_L = (s->flags & PMPM_FLAG_KEEP_VELOCITY_GRADIENT) ? 1 : 0;
  if (s->flags & PMPM_FLAG_MUSL) {
    PMPM_TRY((musl_tail<D, SF>(s, store_L)));
    n_launch += 3;
  } else {
    PMPM_TRY((launch_g2p<D, SF>(s, 1, store_L)));
    n_launch += 1;
  }
  PMPM_CUDA(cudaEventRecord(ev[3], s->stream));
  s->step += 1;
  PMPM_CUDA(cudaEventSynchronize(ev[3]));
  for (int k = 0; k < 3; k++) PMPM_CUDA(cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]));
  for (int k = 0; k < 4; k++) cudaEventDestroy(ev[k]);
  if (launches) *launches = n_launch;
  return PMPM_OK;
}

__global__ void k_count_active(const float *m, int n, float cutoff, int *count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool a = i < n && m[i] > cutoff;
  unsigned b = __ballot_sync(0xffffffffu, a);
  if ((threadIdx.x & 31) == 0 && b) atomicAdd(count, __popc(b));
}
}  // namespace

extern "C" {

int pmpm_profile_step(pmpm_sim *s, float ms[3], int *launches) {
  if (!s || !ms) return PMPM_ERR_INVALID_ARGUMENT;
  if (s->n == 0) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(s->device));
  return PMPM_DISPATCH(s, profile_step, s, ms, launches);
}

int pmpm_set_wait_limit(pmpm_sim *s, long long spins) {
  if (!s || spins < 0) return PMPM_ERR_INVALID_ARGUMENT;
  s->scan.spin_limit = spins;
  return PMPM_OK;
}

int pmpm_scan_tag(unsigned launch, unsigned *tag) {
  if (!tag) return PMPM_ERR_INVALID_ARGUMENT;
  *tag = scan_tag(launch);
  return PMPM_OK;
}

int pmpm_launch_count(const pmpm_sim *s, long long *count) {
  if (!s || !count) return PMPM_ERR_INVALID_ARGUMENT;
  *count = s->launches;
  return PMPM_OK;
}

int pmpm_active_nodes(pmpm_sim *s, int *count) {
  if (!s || !count) return PMPM_ERR_INVALID_ARGUMENT;
  PMPM_CUDA(cudaSetDevice(s->device));
  const int nn = s->g.ntotal;
  PMPM_TRY(ensure_staging(s, (size_t)nn * 4 + 256));
  float *m = (float *)s->staging;
  k_get_nodes<<<blocks_for(nn), kTPB, 0, s->stream>>>(s->g, s->dim, 1, s->N.m, s->node_epoch, s->p2g_epoch, m);
  PMPM_LAUNCHED();
  int *cnt = (int *)((char *)s->staging + (size_t)nn * 4 + 128 - ((size_t)nn * 4) % 128);
  PMPM_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int), s->stream));
  k_count_active<<<blocks_for(nn), kTPB, 0, s->stream>>>(m, nn, 0.000000001f, cnt);
  PMPM_LAUNCHED();
  PMPM_CUDA(cudaMemcpyAsync(count, cnt, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  PMPM_CUDA(cudaStreamSynchronize(s->stream));
  return PMPM_OK;
}

int pmpm_get_step(const pmpm_sim *s, int *step) {
  if (!s || !step) return PMPM_ERR_INVALID_ARGUMENT;
  *step = s->step;
  return PMPM_OK;
}

int pmpm_set_step(pmpm_sim *s, int step) {
  if (!s) return PMPM_ERR_INVALID_ARGUMENT;
  s->step = step;
  return PMPM_OK;
}

int pmpm_synchronize(pmpm_sim *s) {
  if (!s) return PMPM_ERR_INVALID_ARGUMENT;
  PMPM_CUDA(cudaSetDevice(s->device));
  int f = 0;
  PMPM_CUDA(cudaMemcpyAsync(&f, s->fault, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  PMPM_CUDA(cudaStreamSynchronize(s->stream));
  if (f) PMPM_CUDA(cudaMemset(s->fault, 0, sizeof(int)));
  if (f & kFaultWaitTimeout) return PMPM_ERR_TIMEOUT;  // the step's P2G did not run: reported first
  if (f & kFaultNonFinite) return PMPM_ERR_NONFINITE;
  if (f & kFaultOutOfDomain) return PMPM_ERR_OUT_OF_DOMAIN;
  if (f & kFaultCellOverflow) return PMPM_ERR_CELL_OVERFLOW;
  return PMPM_OK;
}

int pmpm_material_point_update(const pmpm_material *mat, int dim, int n, float dt, const float *L, float *stress,
                               float *eps_e, const float *stress_ref, const float *masses, const float *volumes,
                               const float *volumes_original, int velgrad_is_strain_increment, int device) {
  if (!mat || (dim != 2 && dim != 3) || n < 0 || !L || !stress) return PMPM_ERR_INVALID_ARGUMENT;
  if (mat->type == PMPM_MAT_DRUCKER_PRAGER && (!eps_e || !stress_ref)) return PMPM_ERR_INVALID_ARGUMENT;
  if (mat->type == PMPM_MAT_NEWTON_FLUID && (!masses || !volumes || !volumes_original))
    return PMPM_ERR_INVALID_ARGUMENT;
  if (n == 0) return PMPM_OK;
  PMPM_CUDA(cudaSetDevice(device));
  DevMaterial dm;
  dm.type = mat->type;
  dm.density = mat->density;
  memset(dm.p, 0, sizeof(dm.p));
  memcpy(dm.p, mat->params, sizeof(mat->params));
  if (mat->type == PMPM_MAT_NEWTON_FLUID) dm.p[3] = (float)(2.0 * (double)mat->params[0] / 3.0);
  const size_t dd = (size_t)dim * dim;
  std::vector<void *> bufs;
  auto up = [&](const float *h, size_t count, float **d) -> int {
    *d = nullptr;
    if (!h) return PMPM_OK;
    PMPM_TRY(dalloc(d, count));
    bufs.push_back(*d);
    PMPM_CUDA(cudaMemcpy(*d, h, count * 4, cudaMemcpyHostToDevice));
    return PMPM_OK;
  };
  float *dL, *dS, *dE, *dR, *dm_, *dV, *dV0;
  int st = up(L, n * dd, &dL);
  if (st == PMPM_OK) st = up(stress, (size_t)n * 9, &dS);
  if (st == PMPM_OK) st = up(eps_e, n * dd, &dE);
  if (st == PMPM_OK) st = up(stress_ref, (size_t)n * 9, &dR);
  if (st == PMPM_OK) st = up(masses, (size_t)n, &dm_);
  if (st == PMPM_OK) st = up(volumes, (size_t)n, &dV);
  if (st == PMPM_OK) st = up(volumes_original, (size_t)n, &dV0);
  if (st == PMPM_OK) {
    if (dim == 2)
      k_point_update<2><<<blocks_for(n), kTPB>>>(dm, n, dt, dL, dS, dE, dR, dm_, dV, dV0, velgrad_is_strain_increment);
    else
      k_point_update<3><<<blocks_for(n), kTPB>>>(dm, n, dt, dL, dS, dE, dR, dm_, dV, dV0, velgrad_is_strain_increment);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) st = PMPM_ERR_CUDA;
  }
  if (st == PMPM_OK && cudaMemcpy(stress, dS, (size_t)n * 9 * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    st = PMPM_ERR_CUDA;
  if (st == PMPM_OK && eps_e && cudaMemcpy(eps_e, dE, n * dd * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    st = PMPM_ERR_CUDA;
  for (void *p : bufs) cudaFree(p);
  return st;
}

}  // extern "C"

// ===========================================================================
// Batched ensembles
// ===========================================================================
//
// Many independent simulations stepped together: one launch per phase for
// all instances.  Instance i owns storage slots [first_i, first_i + n_i) of
// shared particle arrays, node sub-arrays at noff_i (component-major inside
// the instance), node tiles at toff_i and binning keys at koff_i (its cells
// plus one sentinel key for particles outside its grid).  The key space is
// instance-major, so the counting sort and the physical re-sort keep every
// instance inside its slot range, and one scan serves all instances.  Each
// instance's StepArgs view (grid, node and key sub-arrays, materials, BCs,
// dt) lives in device memory; the batched kernels copy it to shared memory
// and run the single-instance bodies.

struct pmpm_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int dim = 2, shape = 0;
  unsigned flags = 0;
  int resort_interval = 32;
  std::vector<pmpm_sim *> inst;  // per-instance parameters (grid, materials, BCs, dt)
  std::vector<int> np, first, noff, toff, koff;
  int n = 0, stride = 0, nn = 0, ntiles = 0, nkeys = 0;
  DevParticles P[2]{};
  int cur = 0;
  int *slot = nullptr, *key = nullptr;
  DevNodes N{};
  int *node_epoch = nullptr;
  DevBins B{};
  int nscan_blocks = 0;
  ScanState scan;
  int *fault = nullptr;
  std::vector<StepArgs> views;
  StepArgs *d_views = nullptr;
  std::vector<int> dynamic_bcs;  // instances whose BC state changes per step (gravity ramp, moving bodies)
  BatchBlock *d_blocks = nullptr;
  int nblocks = 0;
  int num_sms = 1;       // persistent P2G grid: 8 CTAs per SM x this
  unsigned p2g_seq = 0;  // P2G launches so far (fetch counter parity)
  bool keys_fresh = false;         // the last step's G2P binned the current positions
  unsigned *hash_next = nullptr;   // their reference hashes [stride]
  BatchTile *d_tiles = nullptr;
  bool has_dp = false, has_sref = false, has_planar = false;
  void *staging = nullptr;
  size_t staging_bytes = 0;
  long long launches = 0;
  int step = 0, epoch = -1, p2g_epoch = -2, steps_since_sort = 0;
  bool initialized = false;
};

namespace {

// The per-instance view a batched kernel runs on (P and epoch are set per launch).
StepArgs batch_view(pmpm_batch *b, int i) {
  pmpm_sim *h = b->inst[i];
  h->step = b->step;
  StepArgs a = make_args(h);
  const int D = b->dim;
  const int F = D == 3 ? NodeVel<3>::F : NodeVel<2>::F;
  a.N.m = b->N.m + b->noff[i];
  a.N.p = b->N.p + (size_t)D * b->noff[i];
  a.N.pnt = b->N.pnt + (size_t)D * b->noff[i];
  a.N.vel = b->N.vel + (size_t)F * b->noff[i];
  a.N.tile_epoch = b->N.tile_epoch + b->toff[i];
  a.B = b->B;
  a.B.dual = h->dual ? 1 : 0;
  for (int c = 0; c < 3; c++) a.B.kd[c] = h->kd[c];
  a.B.nkeys = h->nkeys + 1;  // the instance's keys and its sentinel
  a.B.key_base = b->koff[i];
  a.B.sentinel = 1;
  a.B.count = b->B.count + b->koff[i];
  a.B.offset = b->B.offset + b->koff[i];
  a.fault = b->fault;
  a.has_planar = h->has_planar ? 1 : 0;
  a.has_sref = b->has_sref ? 1 : 0;
  a.rigid_shift = 0;
  return a;
}

// The whole-batch arguments of the global phases (scatter, sorts, re-sort).
StepArgs batch_global_args(pmpm_batch *b) {
  StepArgs a;
  memset(&a, 0, sizeof(a));
  a.P = b->P[b->cur];
  a.P.slot = b->slot;
  a.P.key = (unsigned *)b->key;
  a.B = b->B;
  a.B.nkeys = b->nkeys;
  a.fault = b->fault;
  return a;
}

DevParticles batch_particles(pmpm_batch *b) {
  DevParticles P = b->P[b->cur];
  P.slot = b->slot;
  P.key = (unsigned *)b->key;
  return P;
}

// Non-owning single-instance handle over instance i's part of the batch
// (for the field getters and setters and the set-up kernels).
void batch_instance_handle(pmpm_batch *b, int i, pmpm_sim &v) {
  pmpm_sim *h = b->inst[i];
  v.device = b->device;
  v.stream = b->stream;
  v.dim = b->dim;
  v.shape = b->shape;
  v.g = h->g;
  v.dt = h->dt;
  v.alpha = h->alpha;
  v.ppc = h->ppc;
  v.flags = b->flags;
  v.mats = h->mats;
  v.has_dp = h->has_dp;
  v.has_planar = h->has_planar;
  v.has_sref = b->has_sref;
  v.n = b->np[i];
  v.stride = b->stride;
  v.cur = 0;
  DevParticles P = b->P[b->cur];
  const int o = b->first[i];
  auto off = [o](auto *p) { return p ? p + o : p; };
  P.n = v.n;
  P.x = off(P.x);
  P.v = off(P.v);
  P.F = off(P.F);
  P.sig = off(P.sig);
  P.L = off(P.L);
  P.m = off(P.m);
  P.V = off(P.V);
  P.V0 = off(P.V0);
  P.fext = off(P.fext);
  P.eps = off(P.eps);
  P.sref = off(P.sref);
  P.color = off(P.color);
  P.active = off(P.active);
  P.rigid = off(P.rigid);
  P.id = off(P.id);
  P.hash = off(P.hash);
  v.P[0] = P;
  const StepArgs a = batch_view(b, i);
  v.N = a.N;
  v.node_epoch = b->node_epoch + b->toff[i];
  v.B = a.B;
  v.fault = b->fault;
  v.staging = b->staging;
  v.staging_bytes = b->staging_bytes;
  v.epoch = b->epoch;
  v.p2g_epoch = b->p2g_epoch;
  v.partitioned = true;
}

void release_instance_handle(pmpm_batch *b, pmpm_sim &v) {
  b->staging = v.staging;
  b->staging_bytes = v.staging_bytes;
  v.staging = nullptr;
  v.stream = nullptr;
}

int upload_views(pmpm_batch *b, bool only_dynamic) {
  if (!only_dynamic) {
    for (int i = 0; i < (int)b->inst.size(); i++) b->views[i] = batch_view(b, i);
    PMPM_CUDA(cudaMemcpyAsync(b->d_views, b->views.data(), sizeof(StepArgs) * b->views.size(),
                              cudaMemcpyHostToDevice, b->stream));
    return PMPM_OK;
  }
  for (int i : b->dynamic_bcs) {
    pmpm_sim *h = b->inst[i];
    h->step = b->step;
    update_gravity(h);
    update_bodies(h);
    b->views[i] = batch_view(b, i);
    // pageable source: the call returns once the bytes are staged, so the
    // host copy may change for the next step
    PMPM_CUDA(cudaMemcpyAsync(b->d_views + i, &b->views[i], sizeof(StepArgs), cudaMemcpyHostToDevice, b->stream));
  }
  return PMPM_OK;
}

template <int D, int SF>
int batch_partition(pmpm_batch *b) {
  b->epoch += 1;
  cudaStream_t st = b->stream;
  if (b->keys_fresh) {
    std::swap(b->P[b->cur].hash, b->hash_next);  // binned by the last step's G2P
  } else {
    const DevParticles P = batch_particles(b);
    kb_hash_count<D, SF><<<b->nblocks, kTPB, 0, st>>>(b->d_views, b->d_blocks, P, b->epoch);
    PMPM_LAUNCHED();
    b->launches += 1;
  }
  b->keys_fresh = false;
  k_tile_list<<<(b->ntiles + 255) / 256, 256, 0, st>>>(b->N.tile_epoch, b->ntiles, b->epoch, b->N.tile_list,
                                                        b->N.tile_queue);
  PMPM_LAUNCHED();
  b->launches += 1;
  const StepArgs ga = batch_global_args(b);
  PMPM_TRY(launch_scan(b->scan, b->B.count, b->nkeys, b->B.offset, b->B.scalars, b->fault, b->nscan_blocks, st));
  k_scatter<<<blocks_for((b->n + kScatterPer - 1) / kScatterPer), kTPB, 0, st>>>(ga);
  PMPM_LAUNCHED();
  b->launches += 2;
  if (b->flags & PMPM_FLAG_DETERMINISTIC) {  // ids in order inside each bin for the gather
    k_sort_cells<<<blocks_for(b->nkeys), kTPB, 0, st>>>(ga);
    PMPM_LAUNCHED();
    k_sort_big<<<148, 1024, 0, st>>>(ga);
    PMPM_LAUNCHED();
    b->launches += 2;
  }
  return PMPM_OK;
}

template <int D>
int batch_reorder(pmpm_batch *b) {
  const StepArgs ga = batch_global_args(b);
  DevParticles dst = b->P[1 - b->cur];
  const bool move_L = (b->flags & PMPM_FLAG_KEEP_VELOCITY_GRADIENT) != 0;
  k_reorder<D><<<blocks_for(b->n), kTPB, 0, b->stream>>>(ga, dst, move_L ? 1 : 0, b->has_planar ? 1 : 0);
  PMPM_LAUNCHED();
  b->launches += 1;
  b->cur = 1 - b->cur;
  b->steps_since_sort = 0;
  return PMPM_OK;
}

template <int D, int SF>
int batch_step(pmpm_batch *b, float *ms) {
  cudaEvent_t ev[4];
  if (ms)
    for (int k = 0; k < 4; k++) PMPM_CUDA(cudaEventCreate(&ev[k]));
  if (ms) PMPM_CUDA(cudaEventRecord(ev[0], b->stream));
  PMPM_TRY((batch_partition<D, SF>(b)));
  if (b->resort_interval > 0 && b->steps_since_sort + 1 >= b->resort_interval) {
    PMPM_TRY(batch_reorder<D>(b));
  } else {
    b->steps_since_sort += 1;
  }
  if (ms) PMPM_CUDA(cudaEventRecord(ev[1], b->stream));
  if (!b->dynamic_bcs.empty()) PMPM_TRY(upload_views(b, true));
  const DevParticles P = batch_particles(b);
  const int gather = (b->flags & PMPM_FLAG_DETERMINISTIC) ? 1 : 0;
  {
    // persistent CTAs over the active-tile queue of this partition
    const int par = (int)(b->p2g_seq++ & 1u);
    const int grid = std::min(b->ntiles, 8 * b->num_sms);
    kb_p2g<D, SF><<<grid, TileDims<D>::N, 0, b->stream>>>(b->d_views, b->d_tiles, b->N.tile_list, b->N.tile_queue, par,
                                                           b->ntiles, P, b->epoch, 1, b->node_epoch, gather);
  }
  PMPM_LAUNCHED();
  b->p2g_epoch = b->epoch;
  if (ms) PMPM_CUDA(cudaEventRecord(ev[2], b->stream));
  const int store_L = (b->flags & PMPM_FLAG_KEEP_VELOCITY_GRADIENT) ? 1 : 0;
  // the next partition's binning rides on this G2P (not with a PlanarDomain,
  // whose particle forces the binning pass computes)
  const bool bin_next = !b->has_planar;
  const int view_words = (int)((b->has_planar ? sizeof(StepArgs) : offsetof(StepArgs, bc)) / sizeof(int));
  kb_g2p<D, SF><<<b->nblocks, kTPB, 0, b->stream>>>(b->d_views, b->d_blocks, P, b->epoch, 1, store_L,
                                                     bin_next ? 1 : 0, b->hash_next, view_words);
  PMPM_LAUNCHED();
  b->keys_fresh = bin_next;
  b->launches += 2;
  b->step += 1;
  if (ms) {
    PMPM_CUDA(cudaEventRecord(ev[3], b->stream));
    PMPM_CUDA(cudaEventSynchronize(ev[3]));
    for (int k = 0; k < 3; k++) PMPM_CUDA(cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]));
    for (int k = 0; k < 4; k++) cudaEventDestroy(ev[k]);
  }
  return PMPM_OK;
}

int batch_step_dispatch(pmpm_batch *b, float *ms) {
  if (b->dim == 2) {
    if (b->shape == PMPM_SHAPE_LINEAR) return batch_step<2, PMPM_SHAPE_LINEAR>(b, ms);
    if (b->shape == PMPM_SHAPE_QUADRATIC) return batch_step<2, PMPM_SHAPE_QUADRATIC>(b, ms);
    return batch_step<2, PMPM_SHAPE_CUBIC>(b, ms);
  }
  if (b->shape == PMPM_SHAPE_LINEAR) return batch_step<3, PMPM_SHAPE_LINEAR>(b, ms);
  if (b->shape == PMPM_SHAPE_QUADRATIC) return batch_step<3, PMPM_SHAPE_QUADRATIC>(b, ms);
  return batch_step<3, PMPM_SHAPE_CUBIC>(b, ms);
}

int batch_partition_dispatch(pmpm_batch *b) {
  if (b->dim == 2) {
    if (b->shape == PMPM_SHAPE_LINEAR) return batch_partition<2, PMPM_SHAPE_LINEAR>(b);
    if (b->shape == PMPM_SHAPE_QUADRATIC) return batch_partition<2, PMPM_SHAPE_QUADRATIC>(b);
    return batch_partition<2, PMPM_SHAPE_CUBIC>(b);
  }
  if (b->shape == PMPM_SHAPE_LINEAR) return batch_partition<3, PMPM_SHAPE_LINEAR>(b);
  if (b->shape == PMPM_SHAPE_QUADRATIC) return batch_partition<3, PMPM_SHAPE_QUADRATIC>(b);
  return batch_partition<3, PMPM_SHAPE_CUBIC>(b);
}

}  // namespace

extern "C" {

int pmpm_batch_destroy(pmpm_batch *b) {
  if (!b) return PMPM_ERR_INVALID_ARGUMENT;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (pmpm_sim *h : b->inst) pmpm_destroy(h);
  for (int k = 0; k < 2; k++) {
    DevParticles &P = b->P[k];
    for (void *p : {(void *)P.x, (void *)P.v, (void *)P.F, (void *)P.sig, (void *)P.L, (void *)P.m, (void *)P.V,
                    (void *)P.V0, (void *)P.fext, (void *)P.eps, (void *)P.sref, (void *)P.color, (void *)P.active,
                    (void *)P.rigid, (void *)P.id, (void *)P.hash})
      if (p) cudaFree(p);
  }
  for (void *p : {(void *)b->slot, (void *)b->key, (void *)b->hash_next, (void *)b->N.m, (void *)b->N.p, (void *)b->N.pnt, (void *)b->N.vel,
                  (void *)b->N.tile_epoch, (void *)b->N.tile_list, (void *)b->N.tile_queue, (void *)b->node_epoch,
                  (void *)b->B.count, (void *)b->B.offset,
                  (void *)b->B.order, (void *)b->B.block_sums, (void *)b->B.scalars, (void *)b->B.big_cells,
                  (void *)b->fault, (void *)b->d_views, (void *)b->d_blocks, (void *)b->d_tiles, b->staging})
    if (p) cudaFree(p);
  free_scan(b->scan);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return PMPM_OK;
}

int pmpm_batch_create(int num_instances, const pmpm_instance *instances, int device, void *stream,
                      int resort_interval, pmpm_batch **out) {
  if (!out || num_instances < 1 || !instances) return PMPM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  PMPM_CUDA(cudaSetDevice(device));
  pmpm_batch *b = new pmpm_batch();
  b->device = device;
  b->resort_interval = resort_interval < 0 ? 0 : resort_interval;
  int st = PMPM_OK;
  long long n = 0, nn = 0, nt = 0, nk = 0;
  for (int i = 0; i < num_instances && st == PMPM_OK; i++) {
    const pmpm_instance &in = instances[i];
    if (!in.desc || in.num_particles < 1 || !in.positions) {
      st = PMPM_ERR_INVALID_ARGUMENT;
      break;
    }
    pmpm_sim *h = new pmpm_sim();
    b->inst.push_back(h);
    st = setup_handle(in.desc, h);
    if (st != PMPM_OK) break;
    set_key_space(h);
    h->device = device;
    if (i == 0) {
      b->dim = h->dim;
      b->shape = h->shape;
      b->flags = h->flags;
    } else if (h->dim != b->dim || h->shape != b->shape || h->flags != b->flags) {
      st = PMPM_ERR_INVALID_ARGUMENT;  // one kernel instantiation serves the batch
      break;
    }
    if (h->rbls_index >= 0 || (h->flags & PMPM_FLAG_MUSL) || h->has_vm || h->has_mcc) {
      st = PMPM_ERR_NOT_SUPPORTED;
      break;
    }
    bool dyn = !h->sdf.empty();
    for (const GravityState &gs : h->gravity) dyn = dyn || h->bcs[gs.bc_index].i[0] != 0;
    if (dyn) b->dynamic_bcs.push_back(i);
    b->has_dp = b->has_dp || h->has_dp;
    b->has_planar = b->has_planar || h->has_planar;
    b->np.push_back(in.num_particles);
    b->first.push_back((int)n);
    b->noff.push_back((int)nn);
    b->toff.push_back((int)nt);
    b->koff.push_back((int)nk);
    n += in.num_particles;
    nn += h->g.ntotal;
    nt += h->g.ntiles;
    nk += (long long)h->nkeys + 1;
  }
  if (st == PMPM_OK && (n > INT32_MAX / 2 || nn > INT32_MAX / 8 || nk > INT32_MAX / 2)) st = PMPM_ERR_NOT_SUPPORTED;
  if (st != PMPM_OK) {
    pmpm_batch_destroy(b);
    return st;
  }
  b->n = (int)n;
  b->nn = (int)nn;
  b->ntiles = (int)nt;
  b->nkeys = (int)nk;
  b->stride = (b->n + 63) / 64 * 64;
  if (stream) {
    b->stream = (cudaStream_t)stream;
  } else if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess) {
    b->own_stream = true;
  } else {
    pmpm_batch_destroy(b);
    return PMPM_ERR_CUDA;
  }
  for (pmpm_sim *h : b->inst) h->stream = b->stream;
  const int D = b->dim;
  // particle storage: instance-major, local ids
  pmpm_sim shape_of;
  shape_of.dim = D;
  shape_of.n = b->n;
  shape_of.stride = b->stride;
  shape_of.has_dp = b->has_dp;
  shape_of.has_planar = b->has_planar;
  st = alloc_particle_set(&shape_of, b->P[0]);
  if (st == PMPM_OK) st = alloc_particle_set(&shape_of, b->P[1]);
  const size_t stv = (size_t)b->stride;
  if (st == PMPM_OK) st = dalloc(&b->slot, stv);
  if (st == PMPM_OK) st = dalloc(&b->key, stv);
  if (st == PMPM_OK) st = dalloc(&b->hash_next, stv);
  if (st == PMPM_OK) st = dalloc(&b->B.order, stv);
  const int F = D == 3 ? NodeVel<3>::F : NodeVel<2>::F;
  if (st == PMPM_OK) st = dalloc(&b->N.m, (size_t)b->nn);
  if (st == PMPM_OK) st = dalloc(&b->N.p, (size_t)b->nn * D);
  if (st == PMPM_OK) st = dalloc(&b->N.pnt, (size_t)b->nn * D);
  if (st == PMPM_OK) st = dalloc(&b->N.vel, (size_t)b->nn * F);
  if (st == PMPM_OK) st = dalloc(&b->N.tile_epoch, (size_t)b->ntiles);
  if (st == PMPM_OK) st = dalloc(&b->N.tile_list, (size_t)b->ntiles);
  if (st == PMPM_OK) st = dalloc(&b->N.tile_queue, 4);
  if (st == PMPM_OK && cudaMemset(b->N.tile_queue, 0, 4 * sizeof(int)) != cudaSuccess) st = PMPM_ERR_CUDA;
  if (st == PMPM_OK && cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    st = PMPM_ERR_CUDA;
  if (st == PMPM_OK) st = dalloc(&b->node_epoch, (size_t)b->ntiles);
  b->nscan_blocks = (b->nkeys + kScanChunk - 1) / kScanChunk;
  if (st == PMPM_OK) st = dalloc(&b->B.count, (size_t)b->nkeys);
  if (st == PMPM_OK) st = dalloc(&b->B.offset, (size_t)b->nkeys + 1);
  if (st == PMPM_OK) st = dalloc(&b->B.block_sums, (size_t)b->nscan_blocks);
  if (st == PMPM_OK) st = alloc_scan(b->scan, b->nscan_blocks);
  if (st == PMPM_OK) st = dalloc(&b->B.scalars, 4);
  if (st == PMPM_OK) st = dalloc(&b->B.big_cells, (size_t)b->nkeys);
  if (st == PMPM_OK) st = dalloc(&b->fault, 1);
  if (st == PMPM_OK && cudaMalloc(&b->d_views, sizeof(StepArgs) * num_instances) != cudaSuccess) st = PMPM_ERR_OUT_OF_MEMORY;
  // block and tile tables
  std::vector<BatchBlock> blocks;
  std::vector<BatchTile> tiles;
  for (int i = 0; i < num_instances && st == PMPM_OK; i++) {
    for (int s0 = 0; s0 < b->np[i]; s0 += kTPB)
      blocks.push_back({i, b->first[i] + s0, b->first[i] + std::min(s0 + kTPB, b->np[i])});
    for (int t = 0; t < b->inst[i]->g.ntiles; t++) tiles.push_back({i, t, b->toff[i] + t});
  }
  b->nblocks = (int)blocks.size();
  if (st == PMPM_OK && cudaMalloc(&b->d_blocks, sizeof(BatchBlock) * blocks.size()) != cudaSuccess)
    st = PMPM_ERR_OUT_OF_MEMORY;
  if (st == PMPM_OK && cudaMalloc(&b->d_tiles, sizeof(BatchTile) * tiles.size()) != cudaSuccess)
    st = PMPM_ERR_OUT_OF_MEMORY;
  if (st == PMPM_OK &&
      (cudaMemcpy(b->d_blocks, blocks.data(), sizeof(BatchBlock) * blocks.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(b->d_tiles, tiles.data(), sizeof(BatchTile) * tiles.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemset(b->B.count, 0, sizeof(int) * b->nkeys) != cudaSuccess ||
       cudaMemset(b->B.scalars, 0, 4 * sizeof(int)) != cudaSuccess || cudaMemset(b->fault, 0, sizeof(int)) != cudaSuccess ||
       cudaMemset(b->N.tile_epoch, 0xff, sizeof(int) * b->ntiles) != cudaSuccess ||
       cudaMemset(b->node_epoch, 0xff, sizeof(int) * b->ntiles) != cudaSuccess ||
       cudaMemset(b->N.m, 0, sizeof(float) * b->nn) != cudaSuccess))
    st = PMPM_ERR_CUDA;
  // particles (ParticlesContainer ctor per instance; ids local to the instance)
  if (st == PMPM_OK) {
    const size_t sv = (size_t)b->stride;
    const int S = D == 2 ? 4 : 6, E = D == 2 ? 3 : 6;
    std::vector<float> x((size_t)D * sv, 0.0f), v((size_t)D * sv, 0.0f), Fm((size_t)D * D * sv, 0.0f);
    std::vector<float> m(sv, -1.0f), V(sv, -1.0f);
    std::vector<uint8_t> color(sv, 0), zero(sv, 0), active(sv, 1);
    std::vector<int> id(sv, 0);
    for (int i = 0; i < num_instances; i++) {
      const pmpm_instance &in = instances[i];
      for (int j = 0; j < in.num_particles; j++) {
        const size_t s = (size_t)b->first[i] + j;
        for (int c = 0; c < D; c++) {
          x[c * sv + s] = in.positions[(size_t)j * D + c];
          v[c * sv + s] = in.velocities ? in.velocities[(size_t)j * D + c] : 0.0f;
          Fm[(c * D + c) * sv + s] = 1.0f;
        }
        color[s] = in.colors ? in.colors[j] : 0;
        id[s] = j;
      }
    }
    DevParticles &P = b->P[0];
    if (cudaMemcpy(P.x, x.data(), sizeof(float) * x.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(P.v, v.data(), sizeof(float) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(P.F, Fm.data(), sizeof(float) * Fm.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(P.sig, 0, sizeof(float) * S * sv) != cudaSuccess ||
        cudaMemset(P.L, 0, sizeof(float) * D * D * sv) != cudaSuccess ||
        cudaMemset(b->P[1].L, 0, sizeof(float) * D * D * sv) != cudaSuccess ||
        cudaMemcpy(P.m, m.data(), sizeof(float) * sv, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(P.V, V.data(), sizeof(float) * sv, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(P.V0, V.data(), sizeof(float) * sv, cudaMemcpyHostToDevice) != cudaSuccess ||
        (P.fext && cudaMemset(P.fext, 0, sizeof(float) * D * sv) != cudaSuccess) ||
        (P.eps && cudaMemset(P.eps, 0, sizeof(float) * E * sv) != cudaSuccess) ||
        (P.sref && cudaMemset(P.sref, 0, sizeof(float) * S * sv) != cudaSuccess) ||
        cudaMemcpy(P.color, color.data(), sv, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(P.rigid, zero.data(), sv, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(P.active, active.data(), sv, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(P.id, id.data(), sizeof(int) * sv, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(P.hash, 0, sizeof(unsigned) * sv) != cudaSuccess ||
        cudaMemset(b->B.order, 0, sizeof(int) * sv) != cudaSuccess)
      st = PMPM_ERR_CUDA;
  }
  if (st == PMPM_OK) {
    b->views.resize(num_instances);
    st = upload_views(b, false);
  }
  if (st == PMPM_OK && cudaStreamSynchronize(b->stream) != cudaSuccess) st = PMPM_ERR_CUDA;
  if (st != PMPM_OK) {
    pmpm_batch_destroy(b);
    return st;
  }
  *out = b;
  return PMPM_OK;
}

int pmpm_batch_num_instances(const pmpm_batch *b) { return b ? (int)b->inst.size() : -1; }

int pmpm_batch_num_particles(const pmpm_batch *b, int instance) {
  if (!b || instance < 0 || instance >= (int)b->inst.size()) return -1;
  return b->np[instance];
}

int pmpm_batch_initialize(pmpm_batch *b) {
  if (!b) return PMPM_ERR_INVALID_ARGUMENT;
  PMPM_CUDA(cudaSetDevice(b->device));
  PMPM_TRY(batch_partition_dispatch(b));
  // calculate_initial_volumes / calculate_initial_masses per instance
  for (int i = 0; i < (int)b->inst.size(); i++) {
    pmpm_sim v;
    batch_instance_handle(b, i, v);
    float vol = (float)std::pow((double)v.g.h, (double)v.dim);
    vol = vol / (float)v.ppc;
    int st = PMPM_OK;
    k_initial_volumes<<<blocks_for(v.n), kTPB, 0, b->stream>>>(v.P[0], vol);
    if (cudaGetLastError() != cudaSuccess) st = PMPM_ERR_CUDA;
    for (int k = 0; k < (int)v.mats.size() && st == PMPM_OK; k++) {
      k_initial_masses<<<blocks_for(v.n), kTPB, 0, b->stream>>>(v.P[0], k, v.mats[k].density);
      if (cudaGetLastError() != cudaSuccess) st = PMPM_ERR_CUDA;
    }
    release_instance_handle(b, v);
    PMPM_TRY(st);
  }
  if (b->has_dp) {
    DevParticles P = b->P[b->cur];
    P.n = b->n;
    int *flag = b->B.scalars + 3;
    PMPM_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), b->stream));
    k_dp_init<<<blocks_for(b->n), kTPB, 0, b->stream>>>(P, b->dim, flag);
    PMPM_LAUNCHED();
    int hflag = 0;
    PMPM_CUDA(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    PMPM_CUDA(cudaStreamSynchronize(b->stream));
    b->has_sref = hflag != 0;
  }
  PMPM_TRY(upload_views(b, false));
  PMPM_CUDA(cudaStreamSynchronize(b->stream));
  b->initialized = true;
  return PMPM_OK;
}

int pmpm_batch_solve(pmpm_batch *b, int nsteps) {
  if (!b || nsteps < 0) return PMPM_ERR_INVALID_ARGUMENT;
  if (!b->initialized) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(b->device));
  for (int k = 0; k < nsteps; k++) PMPM_TRY(batch_step_dispatch(b, nullptr));
  return PMPM_OK;
}

int pmpm_batch_profile_step(pmpm_batch *b, float *ms, int *launches) {
  if (!b || !ms) return PMPM_ERR_INVALID_ARGUMENT;
  if (!b->initialized) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(b->device));
  const long long l0 = b->launches;
  PMPM_TRY(batch_step_dispatch(b, ms));
  if (launches) *launches = (int)(b->launches - l0);
  return PMPM_OK;
}

static bool batch_field_ok(int field) {
  if (field == PMPM_FIELD_YOUNGS_MODULUS || field == PMPM_FIELD_FRICTION_ANGLE) return false;
  return field < PMPM_FIELD_NODE_MASSES || (field >= PMPM_FIELD_NODE_MASSES && field <= PMPM_FIELD_NODE_TYPES) ||
         field == PMPM_FIELD_BINS;
}

int pmpm_batch_get_field(pmpm_batch *b, int instance, int field, void *dst, size_t bytes, int on_device) {
  if (!b || instance < 0 || instance >= (int)b->inst.size()) return PMPM_ERR_INVALID_ARGUMENT;
  if (!batch_field_ok(field)) return PMPM_ERR_NOT_SUPPORTED;
  pmpm_sim v;
  batch_instance_handle(b, instance, v);
  const int st = pmpm_get_field(&v, field, dst, bytes, on_device);
  release_instance_handle(b, v);
  return st;
}

int pmpm_batch_set_field(pmpm_batch *b, int instance, int field, const void *src, size_t bytes, int on_device) {
  if (!b || instance < 0 || instance >= (int)b->inst.size()) return PMPM_ERR_INVALID_ARGUMENT;
  if (!batch_field_ok(field) || field >= PMPM_FIELD_NODE_MASSES) return PMPM_ERR_NOT_SUPPORTED;
  PMPM_CUDA(cudaSetDevice(b->device));
  if (b->keys_fresh) {  // particle state changes outside a step: redo the binning
    b->keys_fresh = false;
    PMPM_CUDA(cudaMemsetAsync(b->B.count, 0, sizeof(int) * (size_t)b->nkeys, b->stream));
  }
  pmpm_sim v;
  batch_instance_handle(b, instance, v);
  const int st = pmpm_set_field(&v, field, src, bytes, on_device);
  release_instance_handle(b, v);
  return st;
}

int pmpm_batch_synchronize(pmpm_batch *b) {
  if (!b) return PMPM_ERR_INVALID_ARGUMENT;
  PMPM_CUDA(cudaSetDevice(b->device));
  int f = 0;
  PMPM_CUDA(cudaMemcpyAsync(&f, b->fault, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  PMPM_CUDA(cudaStreamSynchronize(b->stream));
  if (f) PMPM_CUDA(cudaMemset(b->fault, 0, sizeof(int)));
  if (f & kFaultWaitTimeout) return PMPM_ERR_TIMEOUT;  // the step's P2G did not run: reported first
  if (f & kFaultNonFinite) return PMPM_ERR_NONFINITE;
  if (f & kFaultOutOfDomain) return PMPM_ERR_OUT_OF_DOMAIN;
  if (f & kFaultCellOverflow) return PMPM_ERR_CELL_OVERFLOW;
  return PMPM_OK;
}

int pmpm_batch_set_wait_limit(pmpm_batch *b, long long spins) {
  if (!b || spins < 0) return PMPM_ERR_INVALID_ARGUMENT;
  b->scan.spin_limit = spins;
  return PMPM_OK;
}

int pmpm_batch_launch_count(const pmpm_batch *b, long long *count) {
  if (!b || !count) return PMPM_ERR_INVALID_ARGUMENT;
  *count = b->launches;
  return PMPM_OK;
}

}  // extern "C"

// ===========================================================================
// Differentiable rollouts
// ===========================================================================

namespace {

// Floats per storage slot of one saved particle state: x, v, F, stress,
// elastic strain, volume.
int state_floats(const pmpm_sim *s) {
  const int D = s->dim;
  return D + D + D * D + (D == 2 ? 4 : 6) + (D == 2 ? 3 : 6) + 1;
}

// Up to eight device-to-device copies of 4-byte words in one launch (the
// rollout's state and node snapshots): blockIdx.y picks the copy.
struct CopyList {
  const void *src[8];
  void *dst[8];
  long long nbytes[8];
  int count = 0;
  void add(const void *from, void *to, size_t bytes) {
    src[count] = from;
    dst[count] = to;
    nbytes[count] = (long long)bytes;
    count++;
  }
};

__global__ void k_copy_list(CopyList c) {
  const int e = blockIdx.y;
  const char *src = (const char *)c.src[e];
  char *dst = (char *)c.dst[e];
  const long long nb = c.nbytes[e];
  const long long step = (long long)gridDim.x * blockDim.x;
  const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0) {
    const long long n4 = nb >> 4;
    for (long long i = t0; i < n4; i += step) reinterpret_cast<float4 *>(dst)[i] = reinterpret_cast<const float4 *>(src)[i];
    for (long long i = (n4 << 2) + t0; i < (nb >> 2); i += step)
      reinterpret_cast<float *>(dst)[i] = reinterpret_cast<const float *>(src)[i];
  } else {
    for (long long i = t0; i < (nb >> 2); i += step)
      reinterpret_cast<float *>(dst)[i] = reinterpret_cast<const float *>(src)[i];
  }
}

int launch_copy_list(pmpm_sim *s, const CopyList &c) {
  if (c.count == 0) return PMPM_OK;
  long long most = 0;
  for (int k = 0; k < c.count; k++) {
    if ((c.nbytes[k] & 3) || ((reinterpret_cast<uintptr_t>(c.src[k]) | reinterpret_cast<uintptr_t>(c.dst[k])) & 3))
      return PMPM_ERR_INVALID_ARGUMENT;
    most = std::max(most, c.nbytes[k]);
  }
  const long long blocks = std::min<long long>((most / 16 + 255) / 256 + 1, 8LL * s->num_sms);
  k_copy_list<<<dim3((unsigned)blocks, (unsigned)c.count), 256, 0, s->stream>>>(c);
  PMPM_LAUNCHED();
  s->launches += 1;
  return PMPM_OK;
}

int copy_state(pmpm_sim *s, float *buf, bool save) {
  if (!save) PMPM_TRY(drop_fresh_keys(s));
  const int D = s->dim, st = s->stride;
  const DevParticles &P = s->P[s->cur];
  float *arrays[6] = {P.x, P.v, P.F, P.sig, P.eps, P.V};
  const int ncomp[6] = {D, D, D * D, D == 2 ? 4 : 6, D == 2 ? 3 : 6, 1};
  size_t off = 0;
  CopyList c;
  for (int k = 0; k < 6; k++) {
    const size_t bytes = sizeof(float) * (size_t)ncomp[k] * st;
    if (arrays[k]) {
      if (save)
        c.add(arrays[k], buf + off, bytes);
      else
        c.add(buf + off, arrays[k], bytes);
    }
    off += (size_t)ncomp[k] * st;
  }
  return launch_copy_list(s, c);
}

void free_rollout(pmpm_sim *s) {
  for (float *p : s->ro.ckpt) cudaFree(p);
  s->ro.ckpt.clear();
  for (float *p : {s->ro.seg, s->ro.A.x, s->ro.A.v, s->ro.A.F, s->ro.A.sig, s->ro.A.eps, s->ro.A.gE, s->ro.A.gphi,
                   s->ro.A.node, s->ro.A.Lb})
    if (p) cudaFree(p);
  if (s->ro.seg_nodes) cudaFree(s->ro.seg_nodes);
  s->ro.seg_nodes = nullptr;
  s->ro.seg = nullptr;
  for (float *p : s->ro.keep_state)
    if (p) cudaFree(p);
  for (char *p : s->ro.keep_nodes)
    if (p) cudaFree(p);
  s->ro.keep_state.clear();
  s->ro.keep_nodes.clear();
  s->ro.keep_epoch.clear();
  s->ro.seg_states = 0;
  s->ro.A = AdjState{};
  s->ro.held = false;
}

int rollout_supported(const pmpm_sim *s) {
  if (s->shape != PMPM_SHAPE_QUADRATIC || s->has_planar || s->rbls_index >= 0 || (s->flags & PMPM_FLAG_MUSL))
    return PMPM_ERR_NOT_SUPPORTED;
  for (const DevMaterial &m : s->mats)
    if (m.type != PMPM_MAT_DRUCKER_PRAGER && m.type != PMPM_MAT_NONE) return PMPM_ERR_NOT_SUPPORTED;
  for (const DevBC &b : s->bcs)
    if (b.type != PMPM_BC_GRAVITY && b.type != PMPM_BC_NODEDOMAIN) return PMPM_ERR_NOT_SUPPORTED;
  return PMPM_OK;
}

// Bytes of one node snapshot: mass, moments, forward moments, packed
// velocities and the tile activity marks of one step's P2G.
size_t node_snapshot_bytes(const pmpm_sim *s) {
  const size_t nn = (size_t)s->g.ntotal, D = (size_t)s->dim;
  const size_t F = s->dim == 3 ? NodeVel<3>::F : NodeVel<2>::F;
  return sizeof(float) * nn * (1 + 2 * D + F) + sizeof(int) * (size_t)s->g.ntiles;
}

// The tile activity saved is the epoch of the P2G that wrote each tile (not
// the binning marks, which the step's G2P has already advanced to the next
// partition's tiles); restored into the marks the adjoint kernels read.
int copy_nodes(pmpm_sim *s, char *buf, bool save) {
  const size_t nn = (size_t)s->g.ntotal, D = (size_t)s->dim;
  const size_t F = s->dim == 3 ? NodeVel<3>::F : NodeVel<2>::F;
  void *arrays[5] = {s->N.m, s->N.p, s->N.pnt, s->N.vel, save ? s->node_epoch : s->N.tile_epoch};
  const size_t bytes[5] = {4 * nn, 4 * D * nn, 4 * D * nn, 4 * F * nn, 4 * (size_t)s->g.ntiles};
  size_t off = 0;
  CopyList c;
  for (int k = 0; k < 5; k++) {
    if (save)
      c.add(arrays[k], buf + off, bytes[k]);
    else
      c.add(buf + off, arrays[k], bytes[k]);
    off += bytes[k];
  }
  return launch_copy_list(s, c);
}

// The step's P2G alone (partition and P2G with the node conditions).
template <int D, int SF>
int p2g_only(pmpm_sim *s) {
  PMPM_TRY((launch_partition<D, SF>(s)));
  PMPM_TRY((launch_p2g<D, SF>(s, 1)));
  return PMPM_OK;
}

// Backward of one step whose state and P2G node data are in place.
template <int D, int SF>
int adjoint_step(pmpm_sim *s, int epoch) {
  AdjState &A = s->ro.A;
  PMPM_CUDA(cudaMemsetAsync(A.node, 0, sizeof(float) * 8 * (size_t)s->g.ntotal, s->stream));
  StepArgs a = make_args(s);
  a.epoch = epoch;  // the epoch the restored tile marks carry
  kadj_g2p_mat<D><<<blocks_for(s->n, 128), 128, 0, s->stream>>>(a, A);
  PMPM_LAUNCHED();
  kadj_g2p<D><<<blocks_for(s->n, 128), 128, 0, s->stream>>>(a, A);
  PMPM_LAUNCHED();
  kadj_grid<D><<<s->g.ntiles, TileDims<D>::N, 0, s->stream>>>(a, A);
  PMPM_LAUNCHED();
  kadj_p2g<D><<<blocks_for(s->n, 128), 128, 0, s->stream>>>(a, A);
  PMPM_LAUNCHED();
  s->launches += 4;
  return PMPM_OK;
}

int adjoint_step_dispatch(pmpm_sim *s, int epoch) {
  return s->dim == 2 ? adjoint_step<2, PMPM_SHAPE_QUADRATIC>(s, epoch)
                     : adjoint_step<3, PMPM_SHAPE_QUADRATIC>(s, epoch);
}

int to_id_order(pmpm_sim *s, int kind, const float *src, void *dst, size_t bytes, int on_device) {
  PMPM_TRY(ensure_staging(s, bytes));
  k_get_particles<<<blocks_for(s->n), kTPB, 0, s->stream>>>(s->P[s->cur], s->dim, kind, src, s->staging, 0);
  PMPM_LAUNCHED();
  return copy_out(s, s->staging, dst, bytes, on_device);
}

}  // namespace

extern "C" {

int pmpm_rollout_set_memory(pmpm_sim *s, long long bytes) {
  if (!s) return PMPM_ERR_INVALID_ARGUMENT;
  s->ro.budget = bytes;
  return PMPM_OK;
}

int pmpm_rollout_forward(pmpm_sim *s, int nsteps, int checkpoint_every) {
  if (!s || nsteps < 1 || checkpoint_every < 1) return PMPM_ERR_INVALID_ARGUMENT;
  if (s->n == 0) return PMPM_ERR_STATE;
  PMPM_TRY(rollout_supported(s));
  PMPM_CUDA(cudaSetDevice(s->device));
  PMPM_TRY(ensure_particle_params(s));
  const size_t per = (size_t)state_floats(s) * s->stride;
  const size_t nodeb = node_snapshot_bytes(s);
  const int every = checkpoint_every;
  const int ncp = (nsteps + every - 1) / every;
  if (s->ro.keep_per != per || s->ro.keep_nodeb != nodeb || s->ro.keep_every != every) {
    free_rollout(s);  // buffers sized for another layout
    s->ro.keep_per = per;
    s->ro.keep_nodeb = nodeb;
    s->ro.keep_every = every;
  }
  while ((int)s->ro.ckpt.size() < ncp) {
    float *buf = nullptr;
    if (cudaMalloc(&buf, per * sizeof(float)) != cudaSuccess) {
      free_rollout(s);
      return PMPM_ERR_OUT_OF_MEMORY;
    }
    s->ro.ckpt.push_back(buf);
  }
  // keep the last segments whole, as the memory budget allows
  const size_t segbytes = (size_t)every * (per * sizeof(float) + nodeb);
  size_t kept_now = 0;
  for (float *p : s->ro.keep_state)
    if (p) kept_now += segbytes;
  size_t budget;
  if (s->ro.budget < 0) {
    size_t free_b = 0, total_b = 0;
    PMPM_CUDA(cudaMemGetInfo(&free_b, &total_b));
    budget = (size_t)(0.6 * (double)(free_b + kept_now));
  } else {
    budget = (size_t)s->ro.budget;
  }
  const int nkeep = (int)std::min<size_t>((size_t)ncp, budget / segbytes);
  s->ro.keep_state.resize(std::max<size_t>(s->ro.keep_state.size(), (size_t)ncp), nullptr);
  s->ro.keep_nodes.resize(std::max<size_t>(s->ro.keep_nodes.size(), (size_t)ncp), nullptr);
  s->ro.keep_epoch.resize(std::max<size_t>(s->ro.keep_epoch.size(), (size_t)ncp));
  for (int c = 0; c < (int)s->ro.keep_state.size(); c++) {
    const bool want = c < ncp && c >= ncp - nkeep;
    if (want && !s->ro.keep_state[c]) {
      if (cudaMalloc(&s->ro.keep_state[c], per * every * sizeof(float)) != cudaSuccess ||
          cudaMalloc(&s->ro.keep_nodes[c], nodeb * every) != cudaSuccess) {
        free_rollout(s);
        return PMPM_ERR_OUT_OF_MEMORY;
      }
    } else if (!want && s->ro.keep_state[c]) {
      cudaFree(s->ro.keep_state[c]);
      cudaFree(s->ro.keep_nodes[c]);
      s->ro.keep_state[c] = nullptr;
      s->ro.keep_nodes[c] = nullptr;
    }
    if (want) s->ro.keep_epoch[c].assign(every, 0);
  }
  s->ro.every = every;
  s->ro.nsteps = nsteps;
  s->ro.start_step = s->step;
  s->ro.held = true;
  for (int k = 0; k < nsteps; k++) {
    const int c = k / every, j = k % every;
    if (j == 0) PMPM_TRY(copy_state(s, s->ro.ckpt[c], true));
    const bool keep = s->ro.keep_state[c] != nullptr;
    if (keep) PMPM_TRY(copy_state(s, s->ro.keep_state[c] + per * j, true));
    PMPM_TRY(PMPM_DISPATCH(s, step_once, s));
    if (keep) {
      PMPM_TRY(copy_nodes(s, s->ro.keep_nodes[c] + nodeb * j, true));
      s->ro.keep_epoch[c][j] = s->epoch;
    }
  }
  return PMPM_OK;
}

int pmpm_rollout_reset(pmpm_sim *s) {
  if (!s) return PMPM_ERR_INVALID_ARGUMENT;
  if (!s->ro.held || s->ro.ckpt.empty()) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(s->device));
  PMPM_TRY(copy_state(s, s->ro.ckpt[0], false));
  s->step = s->ro.start_step;
  PMPM_CUDA(cudaStreamSynchronize(s->stream));
  return PMPM_OK;
}

int pmpm_rollout_backward(pmpm_sim *s, const float *grad_positions, int on_device, float *grad_youngs,
                          float *grad_friction, float *grad_positions0, float *grad_velocities0) {
  if (!s || !grad_positions) return PMPM_ERR_INVALID_ARGUMENT;
  if (!s->ro.held) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(s->device));
  const int D = s->dim, st = s->stride;
  const int NS = D == 2 ? 4 : 6, NE = D == 2 ? 3 : 6;
  AdjState &A = s->ro.A;
  const int every = s->ro.every, nsteps = s->ro.nsteps;
  const size_t per = (size_t)state_floats(s) * st;
  if (!A.x) {
    PMPM_TRY(dalloc(&A.x, (size_t)D * st));
    PMPM_TRY(dalloc(&A.v, (size_t)D * st));
    PMPM_TRY(dalloc(&A.F, (size_t)D * D * st));
    PMPM_TRY(dalloc(&A.sig, (size_t)NS * st));
    PMPM_TRY(dalloc(&A.eps, (size_t)NE * st));
    PMPM_TRY(dalloc(&A.gE, (size_t)st));
    PMPM_TRY(dalloc(&A.gphi, (size_t)st));
    PMPM_TRY(dalloc(&A.node, (size_t)8 * s->g.ntotal));
    PMPM_TRY(dalloc(&A.Lb, (size_t)D * D * st));
  }
  const size_t nodeb = node_snapshot_bytes(s);
  bool need_seg = false;
  for (int c = 0; c * every < nsteps; c++) need_seg = need_seg || !s->ro.keep_state[c];
  if (need_seg && s->ro.seg_states < every) {
    if (s->ro.seg) cudaFree(s->ro.seg);
    if (s->ro.seg_nodes) cudaFree(s->ro.seg_nodes);
    s->ro.seg = nullptr;
    s->ro.seg_nodes = nullptr;
    s->ro.seg_states = 0;
    if (cudaMalloc(&s->ro.seg, per * every * sizeof(float)) != cudaSuccess) return PMPM_ERR_OUT_OF_MEMORY;
    if (cudaMalloc(&s->ro.seg_nodes, nodeb * every) != cudaSuccess) return PMPM_ERR_OUT_OF_MEMORY;
    s->ro.seg_states = every;
  }
  s->ro.seg_epoch.assign(every, 0);
  PMPM_CUDA(cudaMemsetAsync(A.v, 0, sizeof(float) * D * st, s->stream));
  PMPM_CUDA(cudaMemsetAsync(A.F, 0, sizeof(float) * D * D * st, s->stream));
  PMPM_CUDA(cudaMemsetAsync(A.sig, 0, sizeof(float) * NS * st, s->stream));
  PMPM_CUDA(cudaMemsetAsync(A.eps, 0, sizeof(float) * NE * st, s->stream));
  PMPM_CUDA(cudaMemsetAsync(A.gE, 0, sizeof(float) * st, s->stream));
  PMPM_CUDA(cudaMemsetAsync(A.gphi, 0, sizeof(float) * st, s->stream));
  PMPM_CUDA(cudaMemsetAsync(A.x, 0, sizeof(float) * D * st, s->stream));
  // loss gradient of the final positions (id order) into storage order
  {
    const size_t bytes = sizeof(float) * (size_t)s->n * D;
    const void *src = grad_positions;
    if (!on_device) {
      PMPM_TRY(ensure_staging(s, bytes));
      PMPM_CUDA(cudaMemcpyAsync(s->staging, grad_positions, bytes, cudaMemcpyHostToDevice, s->stream));
      src = s->staging;
    }
    DevParticles P = s->P[s->cur];
    k_set_particles<<<blocks_for(s->n), kTPB, 0, s->stream>>>(P, D, 0, src, A.x);
    PMPM_LAUNCHED();
  }
  const int ncp = (nsteps + every - 1) / every;
  for (int c = ncp - 1; c >= 0; c--) {
    const int k0 = c * every, k1 = std::min(k0 + every, nsteps);
    if (s->ro.keep_state[c]) {
      // kept from the forward pass: states and node data of every step
      for (int j = k1 - 1; j >= k0; j--) {
        PMPM_TRY(copy_state(s, s->ro.keep_state[c] + per * (j - k0), false));
        PMPM_TRY(copy_nodes(s, s->ro.keep_nodes[c] + nodeb * (j - k0), false));
        s->step = s->ro.start_step + j;
        PMPM_TRY(adjoint_step_dispatch(s, s->ro.keep_epoch[c][j - k0]));
      }
      continue;
    }
    PMPM_TRY(copy_state(s, s->ro.ckpt[c], false));
    s->step = s->ro.start_step + k0;
    // forward over the segment, keeping each step's state and P2G node data
    for (int j = k0; j < k1; j++) {
      PMPM_TRY(copy_state(s, s->ro.seg + per * (j - k0), true));
      if (j + 1 < k1)
        PMPM_TRY(PMPM_DISPATCH(s, step_once, s));
      else
        PMPM_TRY(s->dim == 2 ? (p2g_only<2, PMPM_SHAPE_QUADRATIC>(s)) : (p2g_only<3, PMPM_SHAPE_QUADRATIC>(s)));
      PMPM_TRY(copy_nodes(s, s->ro.seg_nodes + nodeb * (j - k0), true));
      s->ro.seg_epoch[j - k0] = s->epoch;
    }
    for (int j = k1 - 1; j >= k0; j--) {
      PMPM_TRY(copy_state(s, s->ro.seg + per * (j - k0), false));
      PMPM_TRY(copy_nodes(s, s->ro.seg_nodes + nodeb * (j - k0), false));
      s->step = s->ro.start_step + j;
      PMPM_TRY(adjoint_step_dispatch(s, s->ro.seg_epoch[j - k0]));
    }
  }
  s->step = s->ro.start_step;
  const size_t nb = sizeof(float) * (size_t)s->n;
  if (grad_youngs) PMPM_TRY(to_id_order(s, 4, A.gE, grad_youngs, nb, on_device));
  if (grad_friction) PMPM_TRY(to_id_order(s, 4, A.gphi, grad_friction, nb, on_device));
  if (grad_positions0) PMPM_TRY(to_id_order(s, 0, A.x, grad_positions0, nb * D, on_device));
  if (grad_velocities0) PMPM_TRY(to_id_order(s, 0, A.v, grad_velocities0, nb * D, on_device));
  PMPM_CUDA(cudaStreamSynchronize(s->stream));
  return PMPM_OK;
}

}  // extern "C"

extern "C" int pmpm_material_point_vjp(const pmpm_material *mat, int dim, int n, float dt, const float *L,
                                       const float *eps_e, const float *stress_ref, const float *youngs,
                                       const float *friction, const float *grad_stress, const float *grad_eps_e,
                                       float *grad_L, float *grad_eps_e_in, float *grad_youngs, float *grad_friction,
                                       int method, int device) {
  if (!mat || (dim != 2 && dim != 3) || n < 0 || !L || !eps_e || !stress_ref || !grad_stress || !grad_eps_e ||
      !grad_L || !grad_eps_e_in || !grad_youngs || !grad_friction || (method != 0 && method != 1) ||
      (!youngs != !friction))
    return PMPM_ERR_INVALID_ARGUMENT;
  if (mat->type != PMPM_MAT_DRUCKER_PRAGER) return PMPM_ERR_NOT_SUPPORTED;
  if (n == 0) return PMPM_OK;
  PMPM_CUDA(cudaSetDevice(device));
  pmpm_sim tmp;
  pmpm_desc d{};
  d.dim = dim;
  d.cell_size = 1.0f;
  d.particles_per_cell = 1;
  d.num_materials = 1;
  d.materials = mat;
  d.end[0] = d.end[1] = d.end[2] = 1.0f;
  PMPM_TRY(setup_handle(&d, &tmp));  // material constants as a simulation holds them
  const DevMaterial dm = tmp.mats[0];
  const size_t dd = (size_t)dim * dim;
  std::vector<void *> bufs;
  int st = PMPM_OK;
  auto up = [&](const float *h, size_t count) -> float * {
    float *p = nullptr;
    if (!h || st != PMPM_OK) return nullptr;
    if (cudaMalloc(&p, count * 4) != cudaSuccess) {
      st = PMPM_ERR_OUT_OF_MEMORY;
      return nullptr;
    }
    bufs.push_back(p);
    if (cudaMemcpy(p, h, count * 4, cudaMemcpyHostToDevice) != cudaSuccess) st = PMPM_ERR_CUDA;
    return p;
  };
  auto out = [&](size_t count) -> float * {
    float *p = nullptr;
    if (st != PMPM_OK) return nullptr;
    if (cudaMalloc(&p, count * 4) != cudaSuccess) {
      st = PMPM_ERR_OUT_OF_MEMORY;
      return nullptr;
    }
    bufs.push_back(p);
    return p;
  };
  float *dL = up(L, n * dd), *dE = up(eps_e, n * dd), *dR = up(stress_ref, (size_t)n * 9);
  float *dY = up(youngs, n), *dF = up(friction, n), *dgS = up(grad_stress, (size_t)n * 9);
  float *dgEo = up(grad_eps_e, n * dd);
  float *ogL = out(n * dd), *ogE = out(n * dd), *ogY = out(n), *ogF = out(n);
  if (st == PMPM_OK) {
    if (dim == 2)
      k_point_vjp<2><<<blocks_for(n, 128), 128>>>(dm, n, dt, dL, dE, dR, dY, dF, dgS, dgEo, ogL, ogE, ogY, ogF, method);
    else
      k_point_vjp<3><<<blocks_for(n, 128), 128>>>(dm, n, dt, dL, dE, dR, dY, dF, dgS, dgEo, ogL, ogE, ogY, ogF, method);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) st = PMPM_ERR_CUDA;
  }
  if (st == PMPM_OK && (cudaMemcpy(grad_L, ogL, n * dd * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
                        cudaMemcpy(grad_eps_e_in, ogE, n * dd * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
                        cudaMemcpy(grad_youngs, ogY, (size_t)n * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
                        cudaMemcpy(grad_friction, ogF, (size_t)n * 4, cudaMemcpyDeviceToHost) != cudaSuccess))
    st = PMPM_ERR_CUDA;
  for (void *p : bufs) cudaFree(p);
  for (float *p : tmp.bc_values) cudaFree(p);
  return st;
}

extern "C" int pmpm_set_p2g_kernel(pmpm_sim *s, int variant) {
  if (!s || (variant != 0 && variant != 1)) return PMPM_ERR_INVALID_ARGUMENT;
  if (!s->dual || s->dim != 3) return PMPM_ERR_NOT_SUPPORTED;
  if (variant == 1 && !s->dual3_fits) return PMPM_ERR_NOT_SUPPORTED;  // tiles with more items than threads
  s->p2g_variant = variant;
  return PMPM_OK;
}

extern "C" int pmpm_set_p2g_staging(pmpm_sim *s, int mode) {
  if (!s || (mode != 0 && mode != 1)) return PMPM_ERR_INVALID_ARGUMENT;
  if (!s->B.rec) return PMPM_ERR_NOT_SUPPORTED;
  s->p2g_staging = mode;
  return PMPM_OK;
}

extern "C" int pmpm_set_resort_interval(pmpm_sim *s, int steps) {
  if (!s || steps < 0) return PMPM_ERR_INVALID_ARGUMENT;
  s->resort_interval = steps;
  return PMPM_OK;
}

extern "C" int pmpm_get_tuning(const pmpm_sim *s, int *p2g_kernel, int *staging, int *resort_interval) {
  if (!s) return PMPM_ERR_INVALID_ARGUMENT;
  if (p2g_kernel) *p2g_kernel = s->p2g_variant;
  if (staging) *staging = s->B.rec ? s->p2g_staging : -1;
  if (resort_interval) *resort_interval = s->resort_interval;
  return PMPM_OK;
}

namespace {

// Re-sort interval from a cost model: a physical re-sort costs t_sort once;
// between re-sorts the step slows by about sigma per step as particles leave
// their sorted storage order (slope of the step times over the sampled
// steps, none re-sorted).  Steps per interval K cost t_sort / K + sigma K / 2
// on average; the candidate that minimises it is chosen.
int pick_resort_interval(float t_sort, const std::vector<float> &step_ms) {
  const int m = (int)step_ms.size();
  double sx = 0, sy = 0, sxx = 0, sxy = 0;
  for (int i = 0; i < m; i++) {
    sx += i;
    sy += step_ms[i];
    sxx += (double)i * i;
    sxy += (double)i * step_ms[i];
  }
  const double den = m * sxx - sx * sx;
  const double slope = den > 0 ? (m * sxy - sx * sy) / den : 0.0;
  // the growth counts only beyond two standard errors of the fitted slope:
  // step-to-step noise of a few microseconds otherwise reads as disorder
  // growth and picks short intervals whose re-sorts cost more than they save
  double se = 0.0;
  if (den > 0 && m > 2) {
    const double icpt = (sy - slope * sx) / m;
    double rss = 0.0;
    for (int i = 0; i < m; i++) {
      const double r = step_ms[i] - (icpt + slope * i);
      rss += r * r;
    }
    se = std::sqrt(rss / (m - 2) / (sxx - sx * sx / m));
  }
  const double sigma = std::max(0.0, slope - 2.0 * se);
  const int cands[] = {8, 16, 32, 64, 128};
  int best = 32;
  double best_cost = 1e300;
  for (int k : cands) {
    const double cost = t_sort / k + sigma * k / 2.0;
    if (cost < best_cost - 1e-12) {
      best_cost = cost;
      best = k;
    }
  }
  return best;
}

}  // namespace

extern "C" int pmpm_pick_resort_interval(float t_sort, const float *step_ms, int m, int *interval) {
  if (!step_ms || !interval || m < 1 || !(t_sort >= 0.0f)) return PMPM_ERR_INVALID_ARGUMENT;
  *interval = pick_resort_interval(t_sort, std::vector<float>(step_ms, step_ms + m));
  return PMPM_OK;
}

extern "C" int pmpm_autotune(pmpm_sim *s, int steps, int *chosen) {
  if (!s || steps < 1) return PMPM_ERR_INVALID_ARGUMENT;
  if (s->n == 0) return PMPM_ERR_STATE;
  PMPM_CUDA(cudaSetDevice(s->device));
  // candidates: (P2G kernel, staging) pairs this configuration has
  std::vector<std::pair<int, int>> cands;
  const bool dual3 = s->dual && s->dim == 3 && s->dual3_fits;
  const bool staged = s->B.rec != nullptr;
  for (int v : dual3 ? std::vector<int>{1, 0} : std::vector<int>{s->p2g_variant})
    for (int g : staged && v == 1 ? std::vector<int>{1, 0} : std::vector<int>{s->p2g_staging})
      cands.push_back({v, g});
  // time each candidate on the same state: save, step, restore (no re-sort meanwhile)
  const size_t per = (size_t)state_floats(s) * s->stride;
  const size_t extra = (size_t)(s->dim * s->dim + 2) * s->stride;  // L, alpha (or VonMises history) and pc
  float *saved = nullptr;
  if (cudaMalloc(&saved, (per + extra) * sizeof(float)) != cudaSuccess) return PMPM_ERR_OUT_OF_MEMORY;
  const int step0 = s->step;
  auto copy_extra = [&](bool save) -> int {
    const DevParticles &P = s->P[s->cur];
    const size_t nL = (size_t)s->dim * s->dim * s->stride;
    float *bL = saved + per, *bA = saved + per + nL;
    const cudaMemcpyKind kd = cudaMemcpyDeviceToDevice;
    if (P.L) PMPM_CUDA(cudaMemcpyAsync(save ? bL : P.L, save ? P.L : bL, nL * 4, kd, s->stream));
    if (P.acc) PMPM_CUDA(cudaMemcpyAsync(save ? bA : P.acc, save ? P.acc : bA, (size_t)s->stride * 4, kd, s->stream));
    float *bP = bA + s->stride;
    if (P.pc) PMPM_CUDA(cudaMemcpyAsync(save ? bP : P.pc, save ? P.pc : bP, (size_t)s->stride * 4, kd, s->stream));
    return PMPM_OK;
  };
  int st = copy_state(s, saved, true);
  if (st == PMPM_OK) st = copy_extra(true);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  std::pair<int, int> best_c = {s->p2g_variant, s->p2g_staging};
  std::vector<float> step_ms;
  s->tuning = true;
  for (size_t k = 0; k < cands.size() && st == PMPM_OK; k++) {
    s->p2g_variant = cands[k].first;
    s->p2g_staging = cands[k].second;
    st = PMPM_DISPATCH(s, step_once, s);  // warm-up (and first-launch set-up) of the candidate
    if (st != PMPM_OK) break;
    cudaEventRecord(e0, s->stream);
    for (int i = 0; i < steps && st == PMPM_OK; i++) st = PMPM_DISPATCH(s, step_once, s);
    cudaEventRecord(e1, s->stream);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) {
      best = ms;
      best_c = cands[k];
    }
    if (st == PMPM_OK) st = copy_state(s, saved, false);
    if (st == PMPM_OK) st = copy_extra(false);
    s->step = step0;
  }
  s->p2g_variant = best_c.first;
  s->p2g_staging = best_c.second;
  // re-sort interval: one physical re-sort timed (into the other storage
  // set), then the chosen kernels stepped on that sorted copy without
  // re-sorts, each step timed; the state returns to the original set after
  if (st == PMPM_OK && s->resort_interval > 0 && !s->ro.held) {
    const int since0 = s->steps_since_sort;
    float t_sort = 0.0f;
    st = PMPM_DISPATCH(s, step_once, s);  // fresh partition for the re-sort
    if (st == PMPM_OK) {
      cudaEventRecord(e0, s->stream);
      st = s->dim == 2 ? launch_reorder<2>(s) : launch_reorder<3>(s);
      cudaEventRecord(e1, s->stream);
      cudaEventSynchronize(e1);
      cudaEventElapsedTime(&t_sort, e0, e1);
    }
    if (st == PMPM_OK) {
      const int nsample = std::max(48, 4 * steps);
      std::vector<cudaEvent_t> ev(nsample + 1);
      for (auto &e : ev) cudaEventCreate(&e);
      cudaEventRecord(ev[0], s->stream);
      for (int i = 0; i < nsample && st == PMPM_OK; i++) {
        st = PMPM_DISPATCH(s, step_once, s);
        cudaEventRecord(ev[i + 1], s->stream);
      }
      cudaEventSynchronize(ev[nsample]);
      for (int i = 0; i < nsample && st == PMPM_OK; i++) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
        step_ms.push_back(ms);
      }
      for (auto &e : ev) cudaEventDestroy(e);
      s->cur = 1 - s->cur;  // back to the storage set the tuning started from
    }
    if (st == PMPM_OK) s->resort_interval = pick_resort_interval(t_sort, step_ms);
    if (st == PMPM_OK) st = copy_state(s, saved, false);
    if (st == PMPM_OK) st = copy_extra(false);
    s->steps_since_sort = since0;
    s->step = step0;
  }
  s->tuning = false;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamSynchronize(s->stream);
  cudaFree(saved);
  if (chosen) *chosen = best_c.first;
  return st;
}
