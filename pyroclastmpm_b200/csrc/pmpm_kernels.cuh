// sm_100a kernels of the USL step.
//
// One step (USL::solve, src/solver/usl/usl.cpp:69-115) runs as:
//   k_hash_count   cell hash per particle, per-cell counts (atomics), grid
//                  tile activity, PlanarDomain external force
//   k_scan_*       exclusive prefix over cells -> CSR offsets
//   k_scatter      particles into cell order
//   k_sort_cells / k_sort_big
//                  order inside each cell by particle id, which makes the
//                  permutation identical to the reference's stable sort and
//                  the P2G summation order deterministic
//   k_reorder      (every resort_interval steps) physical re-sort of particle
//                  storage into cell order
//   k_p2g_gather   one CTA per active node tile, one thread per node: P2G in
//                  the reference's per-node order with shape functions
//                  evaluated in registers, fused node epilogue (BCs, v = p/m)
//   k_g2p          one thread per particle: G2P, F, V and the material
//                  stress update fused
#pragma once

#include <cuda_runtime.h>

#include "pmpm_device.cuh"

namespace pmpm {

template <int B, int E>
struct IPow {
  static constexpr int value = B * IPow<B, E - 1>::value;
};
template <int B>
struct IPow<B, 0> {
  static constexpr int value = 1;
};

// --------------------------------------------------------------------------
// bulk copies into shared memory on an mbarrier (sm_90+ async proxy)
// --------------------------------------------------------------------------
//
// A CTA arms a barrier phase with the bytes it expects, any of its threads
// issue cp.async.bulk copies global -> shared that complete those bytes on
// the barrier, and every thread waits for the phase with a bounded poll.
// Plain per-CTA copies from this GPU's own memory: no cluster multicast.

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// the barrier's initialisation visible to the async proxy (the copy engine)
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// orders this thread's earlier shared-memory accesses before later
// async-proxy writes to the same memory
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// bytes (a multiple of 16) from 16-byte aligned global src to 16-byte aligned shared dst
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// one poll of the phase of the given parity; suspends the thread for at most
// about kBulkPollNs nanoseconds while the phase is incomplete
constexpr unsigned kBulkPollNs = 500;
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(kBulkPollNs)
      : "memory");
  return ok != 0;
}

// The copy state of one CTA: its barrier and a flag set once a wait gave up.
struct BulkState {
  unsigned long long bar;
  int failed;
};

// Waits for the barrier phase of the given parity.  After kBulkWaitPolls
// polls (about a second) the wait gives up, records kFaultWaitTimeout and
// marks the CTA's copies failed: later waits return at once and no further
// copies are issued, so the kernel finishes (its results are then invalid).
constexpr int kBulkWaitPolls = 1 << 21;
__device__ __forceinline__ bool mbar_wait(BulkState *bs, unsigned parity, int *fault) {
  if (*(volatile int *)&bs->failed) return false;
  for (int k = 0; k < kBulkWaitPolls; k++)
    if (mbar_try_wait(&bs->bar, parity)) return true;
  *(volatile int *)&bs->failed = 1;
  atomicOr(fault, kFaultWaitTimeout);
  return false;
}

// Sets up the CTA's copy state (one thread), before the block barrier that
// publishes it.
__device__ __forceinline__ void bulk_init(BulkState *bs) {
  bs->failed = 0;
  mbar_init(&bs->bar, 1);
  fence_mbar_init();
}

// binning_failed() read once per CTA and shared, for kernels whose threads
// must agree (block barriers follow).
__device__ __forceinline__ bool binning_failed_cta(const int *fault) {
  __shared__ int flag;
  if (threadIdx.x == 0) flag = (*(volatile const int *)fault & kFaultWaitTimeout) != 0;
  __syncthreads();
  return flag != 0;
}

template <int D>
__device__ __forceinline__ int tile_of(const DevGrid &g, const int c[3]) {
  using T = TileDims<D>;
  int tx = c[0] / T::X, ty = c[1] / T::Y, tz = (D == 3) ? c[2] / T::Z : 0;
  return tx + ty * g.tdim[0] + tz * g.tdim[0] * g.tdim[1];
}

// --------------------------------------------------------------------------
// binning
// --------------------------------------------------------------------------

// Marks tile t active in this partition.  Writers race harmlessly (all store
// the same value); the read first skips the store once the mark is set, as
// the cells of a tile mark it from many SMs (storing unconditionally made
// the bed's binning pass 0.23 -> 0.31 ms).
__device__ __forceinline__ void mark_tile(const StepArgs &a, int t, int epoch) {
  if (a.N.tile_epoch[t] != epoch) a.N.tile_epoch[t] = epoch;
}

// Active-tile queue of this partition: the tiles marked with its epoch, in
// tile order within each warp (one atomic per warp).  Runs after the binning
// pass; clears the next partition's count.
__global__ void __launch_bounds__(256) k_tile_list(const int *tile_epoch, int ntiles, int epoch, int *tile_list,
                                                   int *tile_queue) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int *count = &tile_queue[epoch & 1];
  if (t == 0) tile_queue[(epoch + 1) & 1] = 0;
  const bool on = t < ntiles && tile_epoch[t] == epoch;
  const unsigned m = __ballot_sync(0xffffffffu, on);
  if (!m) return;
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == __ffs(m) - 1) base = atomicAdd(count, __popc(m));
  base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
  if (on) {
    const int i = base + __popc(m & ((1u << lane) - 1u));
    if (i < ntiles) tile_list[i] = t;
  }
}

// Active queue of tile pairs stacked in z (tiles tz = 2k and 2k + 1 of one
// column; unit u = column + k * columns), for the linear and cubic sweeps:
// a pair is active when either tile is marked with this partition's epoch.
__global__ void __launch_bounds__(256) k_pair_list(const int *tile_epoch, int plane, int tdim2, int epoch,
                                                   int *list, int *queue) {
  const int nunits = plane * ((tdim2 + 1) / 2);
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  int *count = &queue[epoch & 1];
  if (u == 0) queue[(epoch + 1) & 1] = 0;
  bool on = false;
  if (u < nunits) {
    const int col = u % plane, tz = 2 * (u / plane);
    on = tile_epoch[col + tz * plane] == epoch || (tz + 1 < tdim2 && tile_epoch[col + (tz + 1) * plane] == epoch);
  }
  const unsigned m = __ballot_sync(0xffffffffu, on);
  if (!m) return;
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == __ffs(m) - 1) base = atomicAdd(count, __popc(m));
  base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
  if (on) {
    const int i = base + __popc(m & ((1u << lane) - 1u));
    if (i < nunits) list[i] = u;
  }
}

// Next tile of the active-tile queue for the whole CTA, or -1.
__device__ __forceinline__ int next_tile(const StepArgs &a, int *cur) {
  if (threadIdx.x == 0) *cur = atomicAdd(&a.N.tile_queue[2 + a.p2g_par], 1);
  __syncthreads();
  const int idx = *cur;
  __syncthreads();
  return idx < min(a.N.tile_queue[a.epoch & 1], a.g.ntiles) ? a.N.tile_list[idx] : -1;
}

// Marks every node tile the particle's P2G contributions or G2P reads touch.
template <int D, int SF>
__device__ __forceinline__ void mark_tiles(const StepArgs &a, const int b[3], unsigned hu, bool binned,
                                           bool in_axes, int epoch) {
  using T = TileDims<D>;
  constexpr int LO = Stencil<SF>::WLO, HI = Stencil<SF>::WLO + Stencil<SF>::WIN - 1;
  const DevGrid &g = a.g;
  if (SF == PMPM_SHAPE_QUADRATIC && !in_axes) return;  // takes no part in the step
  int tlo[3] = {0, 0, 0}, thi[3] = {0, 0, 0};
  bool empty = false, clipped = false;
  const int tsz[3] = {T::X, T::Y, T::Z};
#pragma unroll
  for (int c = 0; c < D; c++) {
    int lo = b[c] + LO, hi = b[c] + HI;
    if (lo < 0) {
      lo = 0;
      clipped = true;
    }
    if (hi > g.n[c] - 1) {
      hi = g.n[c] - 1;
      clipped = true;
    }
    if (lo > hi) empty = true;
    tlo[c] = lo / tsz[c];
    thi[c] = hi / tsz[c];
  }
  if (!empty) {
    for (int tz = tlo[2]; tz <= thi[2]; tz++)
      for (int ty = tlo[1]; ty <= thi[1]; ty++)
        for (int tx = tlo[0]; tx <= thi[0]; tx++) {
          int t = tx + ty * g.tdim[0] + tz * g.tdim[0] * g.tdim[1];
          mark_tile(a, t, epoch);
        }
  }
  if (SF != PMPM_SHAPE_QUADRATIC && clipped && binned) {
    // slots leaving the grid on an axis: the reference's flat index check lets
    // them land on a node of a neighbouring row (src/solver/usl/usl_inline.h:114-126)
    // A slot inside the grid on every axis is its own node, whose tile the
    // loop above marked (skipping them took the bed's binning pass from 0.23
    // to 0.19 ms: a warp holding a cell on a grid face walked all 64).  The
    // node of an aliased slot's flat index: one carry per axis where that
    // reproduces the index (the particle's own cell in the grid), else
    // divisions.
    constexpr int W = Stencil<SF>::WIN;
    const int nxy = g.n[0] * g.n[1];
    for (int wz = (D == 3 ? LO : 0); wz <= (D == 3 ? HI : 0); wz++) {
      const bool zin = D == 2 || (b[2] + wz >= 0 && b[2] + wz < g.n[2]);
      for (int wy = LO; wy < LO + W; wy++) {
        const bool yin = b[1] + wy >= 0 && b[1] + wy < g.n[1];
#pragma unroll
        for (int wx = LO; wx < LO + W; wx++) {
          if (zin && yin && b[0] + wx >= 0 && b[0] + wx < g.n[0]) continue;
          const int f = (int)hu + wx + wy * g.n[0] + wz * nxy;
          if ((unsigned)f >= (unsigned)g.ntotal) continue;
          int c[3] = {b[0] + wx, b[1] + wy, D == 3 ? b[2] + wz : 0};
#pragma unroll
          for (int k = 0; k < D - 1; k++) {
            if (c[k] < 0) {
              c[k] += g.n[k];
              c[k + 1] -= 1;
            } else if (c[k] >= g.n[k]) {
              c[k] -= g.n[k];
              c[k + 1] += 1;
            }
          }
          if (c[0] < 0 || c[0] >= g.n[0] || c[1] < 0 || c[1] >= g.n[1] || c[2] < 0 ||
              c[0] + c[1] * g.n[0] + c[2] * nxy != f) {
            c[0] = f % g.n[0];
            c[1] = (f / g.n[0]) % g.n[1];
            c[2] = f / nxy;
          }
          mark_tile(a, tile_of<D>(g, c), epoch);
        }
      }
    }
  }
}

// Dual binning: the particle's nodes are d - 1 .. d + 1 (clamped) per axis.
template <int D>
__device__ __forceinline__ void mark_tiles_dual(const StepArgs &a, const int d[3], int epoch) {
  using T = TileDims<D>;
  const DevGrid &g = a.g;
  const int tsz[3] = {T::X, T::Y, T::Z};
  int tlo[3] = {0, 0, 0}, thi[3] = {0, 0, 0};
#pragma unroll
  for (int c = 0; c < D; c++) {
    tlo[c] = max(d[c] - 1, 0) / tsz[c];
    thi[c] = min(d[c] + 1, g.n[c] - 1) / tsz[c];
  }
  for (int tz = tlo[2]; tz <= thi[2]; tz++)
    for (int ty = tlo[1]; ty <= thi[1]; ty++)
      for (int tx = tlo[0]; tx <= thi[0]; tx++) {
        const int t = tx + ty * g.tdim[0] + tz * g.tdim[0] * g.tdim[1];
        mark_tile(a, t, epoch);
      }
}

// apply_planardomain (src/boundaryconditions/planardomain_inline.h:56-138).
template <int D>
__device__ __forceinline__ void planar_force(const StepArgs &a, int s, const float x[3]) {
  const DevParticles &P = a.P;
  float f[3] = {0.0f, 0.0f, 0.0f};
  float v[3];
#pragma unroll
  for (int c = 0; c < D; c++) v[c] = P.v[c * P.stride + s];
  const float vol = P.V[s], mass = P.m[s];
  const float radius = 0.5f * powf(vol, 1.0f / (float)D);
  const float scale = (float)((double)mass / ((double)a.dt * (double)a.dt));
  for (int k = 0; k < a.nbc; k++) {
    const DevBC &bc = a.bc[k];
    if (bc.type != PMPM_BC_PLANARDOMAIN) continue;
    for (int face = 0; face < 2; face++) {
#pragma unroll
      for (int c = 0; c < D; c++) {
        float overlap = face == 0 ? radius - (x[c] - a.g.origin[c]) : radius - (a.g.end[c] - x[c]);
        if (!(overlap > 0.0f)) continue;
        float nrm = face == 0 ? 1.0f : -1.0f;
        float mu = bc.r[3 * face + c];
        float ndotv = nrm * v[c];
#pragma unroll
        for (int e = 0; e < D; e++) {
          float ne = (e == c) ? nrm : 0.0f;
          float tang = v[e] - ndotv * ne;
          f[e] += (scale * overlap) * (ne - mu * tang);
        }
      }
    }
  }
#pragma unroll
  for (int c = 0; c < D; c++) P.fext[c * P.stride + s] = f[c];
}

// Dual cell of a quadratic particle: the first of its three nodes plus one,
// chosen with the same comparison as the G2P window (frac < 1/2 -> b - 1).
__device__ __forceinline__ int dual_coord(float u, int b) { return (u - (float)(b - 1)) < 1.5f ? b : b + 1; }

// Called by every lane of a warp (valid = the lane has a particle): lanes
// of the warp that share a key add to its count with one atomic (particles
// stored in cell order after a re-sort mostly share keys with neighbours).
__device__ __forceinline__ int warp_bin_slot(int *count, unsigned key, bool add) {
  const unsigned kk = add ? key : 0xffffffffu;
  const unsigned peers = __match_any_sync(0xffffffffu, kk);
  int slot = -1;
  if (add) {
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&count[key], __popc(peers));
    base = __shfl_sync(peers, base, leader);
    slot = base + __popc(peers & ((1u << lane) - 1u));
  }
  return slot;
}

template <int D, int SF>
// epoch: the partition the marks are for (the G2P of a step bins for the
// next); hash_out: where the reference cell hashes go
__device__ __forceinline__ void hash_count_body(const StepArgs &a, int s, bool valid, int epoch, unsigned *hash_out) {
  const DevGrid &g = a.g;
  float x[3] = {0.0f, 0.0f, 0.0f}, u[3] = {0.0f, 0.0f, 0.0f};
  int b[3] = {0, 0, 0};
  bool in_axes = true;
  bool binned = false, sorted = false;
  unsigned key = 0, hu = 0;
  int dcell[3] = {0, 0, 0};
  bool ref_cells = false;
  if (valid) {
#pragma unroll
    for (int c = 0; c < D; c++) {
      x[c] = a.P.x[c * a.P.stride + s];
      u[c] = scaled_coord(x[c], g.origin[c], g.inv_h);
      b[c] = (int)u[c];
      in_axes = in_axes && b[c] >= 0 && b[c] < g.n[c];
    }
    hu = (unsigned)(b[0] + b[1] * g.n[0] + b[2] * g.n[0] * g.n[1]);
    hash_out[s] = hu;
    if (SF == PMPM_SHAPE_QUADRATIC && a.B.dual) {
      int d[3] = {0, 0, 0};
#pragma unroll
      for (int c = 0; c < D; c++) d[c] = dual_coord(u[c], b[c]);
      key = (unsigned)(d[0] + d[1] * a.B.kd[0] + d[2] * a.B.kd[0] * a.B.kd[1]);
      binned = in_axes;
#pragma unroll
      for (int c = 0; c < 3; c++) dcell[c] = d[c];
    } else {
      key = hu;
      binned = hu < (unsigned)g.ntotal;
      ref_cells = true;
    }
    // with a sentinel key (batched ensembles) a particle outside the grid is
    // sorted into its instance's extra last key, so instances keep their
    // storage ranges; it is reported as a fault either way
    sorted = binned;
    if (!binned && a.B.sentinel) {
      key = (unsigned)(a.B.nkeys - 1);  // the instance's last key
      sorted = true;
    }
  }
  const int slot = warp_bin_slot(a.B.count, key, sorted);
  if (!valid) return;
  // reference cells: all particles of a cell mark the same tiles, so the
  // cell's first arrival marks them (a particle outside the grid marks its own)
  if (ref_cells && (slot == 0 || !binned)) mark_tiles<D, SF>(a, b, hu, binned, in_axes, epoch);
  if (SF == PMPM_SHAPE_QUADRATIC && a.B.dual && binned && slot == 0) {
    // all particles of a dual cell share its tiles and brick: the cell's
    // first arrival marks them
    mark_tiles_dual<D>(a, dcell, epoch);
    if (a.B.brick_epoch) {
      const int bi = dcell[0] / 8 + (dcell[1] / 8) * a.B.kb[0] + (dcell[2] / 8) * a.B.kb[0] * a.B.kb[1];
      if (a.B.brick_epoch[bi] != epoch) a.B.brick_epoch[bi] = epoch;
    }
  }
  a.P.key[s] = (unsigned)a.B.key_base + key;
  a.P.slot[s] = slot;
  if (!binned || (SF == PMPM_SHAPE_QUADRATIC && !in_axes)) atomicOr(a.fault, kFaultOutOfDomain);
  if (a.has_planar) planar_force<D>(a, s, x);
}

template <int D, int SF>
__global__ void __launch_bounds__(256) k_hash_count(StepArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  hash_count_body<D, SF>(a, s, s < a.P.n, a.epoch, a.P.hash);
}

constexpr int kScanThreads = 1024;
constexpr int kScanPer = 16;
constexpr int kScanChunk = kScanThreads * kScanPer;

__device__ __forceinline__ int block_exclusive_scan(int v, int *smem_warp, int &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) smem_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int wv = lane < (blockDim.x >> 5) ? smem_warp[lane] : 0;
    int wi = wv;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    smem_warp[lane] = wi - wv;
    if (lane == 31) smem_warp[32] = wi;
  }
  __syncthreads();
  total = smem_warp[32];
  int r = smem_warp[warp] + incl - v;
  __syncthreads();
  return r;
}

// kScanPer consecutive keys per thread: 16-byte accesses when all are in range
__device__ __forceinline__ void load_keys(const int *p, int base, int n, int v[kScanPer]) {
  static_assert(kScanPer % 4 == 0, "vector width");
  if (base + kScanPer <= n) {
#pragma unroll
    for (int q = 0; q < kScanPer / 4; q++) {
      const int4 w = *reinterpret_cast<const int4 *>(p + base + 4 * q);
      v[4 * q] = w.x;
      v[4 * q + 1] = w.y;
      v[4 * q + 2] = w.z;
      v[4 * q + 3] = w.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < kScanPer; k++) v[k] = base + k < n ? p[base + k] : 0;
  }
}

// Single-pass exclusive scan of the per-key counts into offsets (decoupled
// look-back): each CTA takes a ticket in launch order, scans its chunk,
// publishes the chunk total and then the inclusive prefix in status[ticket]
// (tagged with the launch, so nothing is cleared between launches), and
// sums its predecessors' published values back to the first inclusive one.
// A CTA only waits on CTAs with smaller tickets, which are already running;
// the wait is bounded (kFaultWaitTimeout).  Clears the counts it consumed;
// the last CTA writes offset[n], the binned total and resets the per-step
// counters and the next launch's ticket counter.
constexpr unsigned long long kScanAggregate = 1ull << 32, kScanInclusive = 2ull << 32;

__global__ void __launch_bounds__(kScanThreads) k_scan_onepass(int *count, int n, int *offset,
                                                                unsigned long long *status, int *ticket,
                                                                int *scalars, int *fault, unsigned tag,
                                                                int nblocks, long long spin_limit) {
  __shared__ int sw[33];
  __shared__ int sh_block, sh_prefix;
  if (threadIdx.x == 0) sh_block = atomicAdd(&ticket[tag & 1u], 1);
  __syncthreads();
  const int blk = sh_block;
  const int base = blk * kScanChunk + threadIdx.x * kScanPer;
  int v[kScanPer];
  load_keys(count, base, n, v);
  int sum = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; k++) sum += v[k];
  int total;
  const int ex_local = block_exclusive_scan(sum, sw, total);
  if (threadIdx.x < 32) {
    // warp 0 looks back over 32 predecessors at a time: the nearest one with
    // an inclusive prefix ends the walk, the aggregates before it add up
    const int lane = threadIdx.x;
    const unsigned long long t = (unsigned long long)tag << 34;
    int prefix = 0;
    if (blk > 0) {
      if (lane == 0) atomicExch(&status[blk], t | kScanAggregate | (unsigned)total);
      int top = blk - 1;
      long long spins = 0;
      for (;;) {
        const int idx = top - lane;
        unsigned long long w = idx >= 0 ? atomicAdd(&status[idx], 0ull) : (t | kScanInclusive);
        const bool ready = (w >> 34) == (unsigned long long)tag;
        const unsigned incl = __ballot_sync(0xffffffffu, ready && (w & kScanInclusive));
        const unsigned rdy = __ballot_sync(0xffffffffu, ready);
        const int first = incl ? __ffs(incl) - 1 : 31;  // lanes 0..first are needed
        const unsigned need = first == 31 ? 0xffffffffu : ((1u << (first + 1)) - 1u);
        if ((rdy & need) != need) {
          if (++spins > spin_limit) {
            if (lane == 0) atomicOr(fault, kFaultWaitTimeout);
            break;
          }
          continue;
        }
        int val = lane <= first ? (int)(unsigned)(w & 0xffffffffull) : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
        prefix += val;
        if (incl) break;
        top -= 32;
      }
    }
    if (lane == 0) {
      atomicExch(&status[blk], t | kScanInclusive | (unsigned)(prefix + total));
      sh_prefix = prefix;
      if (blk == nblocks - 1) {
        offset[n] = prefix + total;
        scalars[0] = prefix + total;  // binned particles
        scalars[1] = 0;               // unbinned counter
        scalars[2] = 0;               // big-cell counter
        ticket[(tag + 1u) & 1u] = 0;
      }
    }
  }
  __syncthreads();
  int ex = ex_local + sh_prefix;
  if (base + kScanPer <= n) {
#pragma unroll
    for (int q = 0; q < kScanPer / 4; q++) {
      int4 o;
      o.x = ex;
      o.y = o.x + v[4 * q];
      o.z = o.y + v[4 * q + 1];
      o.w = o.z + v[4 * q + 2];
      ex = o.w + v[4 * q + 3];
      *reinterpret_cast<int4 *>(offset + base + 4 * q) = o;
      *reinterpret_cast<int4 *>(count + base + 4 * q) = make_int4(0, 0, 0, 0);
    }
  } else {
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
      if (base + k < n) {
        offset[base + k] = ex;
        count[base + k] = 0;
      }
      ex += v[k];
    }
  }
}

// True when this step's key scan gave up a bounded wait: its offsets are
// then not a valid prefix, so every kernel that indexes particles through
// them returns without work (the step reports PMPM_ERR_TIMEOUT).
__device__ __forceinline__ bool binning_failed(const int *fault) {
  return (*(volatile const int *)fault & kFaultWaitTimeout) != 0;
}

// Four consecutive particles per thread (kScatterPer): their slots and keys
// in one 16-byte load each where aligned, so four offset gathers are in
// flight per thread instead of one.
constexpr int kScatterPer = 4;
__global__ void __launch_bounds__(256) k_scatter(StepArgs a) {
  if (binning_failed(a.fault)) return;
  const int s0 = (blockIdx.x * blockDim.x + threadIdx.x) * kScatterPer;
  if (s0 >= a.P.n) return;
  int slot[kScatterPer], key[kScatterPer];
  const bool vec = s0 + kScatterPer <= a.P.n && ((reinterpret_cast<uintptr_t>(a.P.slot + s0) |
                                                  reinterpret_cast<uintptr_t>(a.P.key + s0)) & 15) == 0;
  if (vec) {
    const int4 sv = *reinterpret_cast<const int4 *>(a.P.slot + s0);
    const int4 kv = *reinterpret_cast<const int4 *>(a.P.key + s0);
    slot[0] = sv.x; slot[1] = sv.y; slot[2] = sv.z; slot[3] = sv.w;
    key[0] = kv.x; key[1] = kv.y; key[2] = kv.z; key[3] = kv.w;
  } else {
#pragma unroll
    for (int q = 0; q < kScatterPer; q++) {
      const bool in = s0 + q < a.P.n;
      slot[q] = in ? a.P.slot[s0 + q] : -2;
      key[q] = in && slot[q] >= 0 ? (int)a.P.key[s0 + q] : 0;
    }
  }
  int base[kScatterPer];
#pragma unroll
  for (int q = 0; q < kScatterPer; q++) base[q] = slot[q] >= 0 ? a.B.offset[key[q]] : 0;
#pragma unroll
  for (int q = 0; q < kScatterPer; q++) {
    if (slot[q] >= 0) {
      a.B.order[base[q] + slot[q]] = s0 + q;
    } else if (s0 + q < a.P.n) {  // not binned
      int k = atomicAdd(&a.B.scalars[1], 1);
      a.B.order[a.B.scalars[0] + k] = s0 + q;
    }
  }
}

constexpr int kSmallCell = 32;
constexpr int kBigCell = 2048;

// Orders each cell's particles by id; cells above kSmallCell go to k_sort_big.
__global__ void __launch_bounds__(256) k_sort_cells(StepArgs a) {
  if (binning_failed(a.fault)) return;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.B.nkeys) return;
  const int lo = a.B.offset[c], hi = a.B.offset[c + 1];
  const int cnt = hi - lo;
  if (cnt < 2) return;
  if (cnt > kSmallCell) {
    int k = atomicAdd(&a.B.scalars[2], 1);
    a.B.big_cells[k] = c;
    return;
  }
  int key[kSmallCell], val[kSmallCell];
  for (int i = 0; i < cnt; i++) {
    val[i] = a.B.order[lo + i];
    key[i] = a.P.id[val[i]];
  }
  for (int i = 1; i < cnt; i++) {
    int kk = key[i], vv = val[i];
    int j = i - 1;
    while (j >= 0 && key[j] > kk) {
      key[j + 1] = key[j];
      val[j + 1] = val[j];
      j--;
    }
    key[j + 1] = kk;
    val[j + 1] = vv;
  }
  for (int i = 0; i < cnt; i++) a.B.order[lo + i] = val[i];
}

// Bitonic sort in shared memory of each large cell (up to kBigCell entries).
__global__ void __launch_bounds__(1024) k_sort_big(StepArgs a) {
  __shared__ int key[kBigCell], val[kBigCell];
  if (binning_failed(a.fault)) return;
  const int nbig = a.B.scalars[2];
  for (int bi = blockIdx.x; bi < nbig; bi += gridDim.x) {
    const int c = a.B.big_cells[bi];
    const int lo = a.B.offset[c], cnt = a.B.offset[c + 1] - lo;
    if (cnt > kBigCell) {
      if (threadIdx.x == 0) atomicOr(a.fault, kFaultCellOverflow);
      continue;
    }
    int p2 = 1;
    while (p2 < cnt) p2 <<= 1;
    for (int i = threadIdx.x; i < p2; i += blockDim.x) {
      if (i < cnt) {
        val[i] = a.B.order[lo + i];
        key[i] = a.P.id[val[i]];
      } else {
        key[i] = 0x7fffffff;
        val[i] = -1;
      }
    }
    __syncthreads();
    for (int k = 2; k <= p2; k <<= 1) {
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int i = threadIdx.x; i < p2; i += blockDim.x) {
          int ixj = i ^ j;
          if (ixj > i) {
            bool up = (i & k) == 0;
            if ((key[i] > key[ixj]) == up) {
              int tk = key[i];
              key[i] = key[ixj];
              key[ixj] = tk;
              int tv = val[i];
              val[i] = val[ixj];
              val[ixj] = tv;
            }
          }
        }
        __syncthreads();
      }
    }
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) a.B.order[lo + i] = val[i];
    __syncthreads();
  }
}

// --------------------------------------------------------------------------
// P2G records of the 3D sweeps
// --------------------------------------------------------------------------
//
// Sorted position k of the binned particles -> rec[k * R4 ..]:
//   [0] (m, m vx, m vy, m vz)   [1] (Sxx, Sxy, Sxy, Syy)   [2] (Sxz, Syz, Szz, 0)
//   [3] (x, y, z, 0)            [4] PlanarDomain only: (f_ext, 0)
// with S = -V sigma; the MUSL momentum remap maps neither stress nor
// external force.  The sweeps copy a row of source cells (consecutive keys:
// one run of records) into shared memory with one bulk copy instead of
// gathering each particle's fields through the sorted order.  Written just
// before each P2G from the current particle state, so a P2G after any
// change of state (stage calls, field setters, MUSL) reads current values.
// DUAL: the dual-cell sweep (its cells hold only particles inside the grid;
// f_ext mapped for all); otherwise the linear/cubic sweep conventions (a
// quadratic particle outside the grid on an axis takes no part; f_ext only
// with mass).
template <int SF, bool DUAL, bool PLANAR>
__device__ __forceinline__ void make_record(const StepArgs &a, int s, float4 r[5]) {
  const DevParticles &P = a.P;
  const DevGrid &g = a.g;
  const int st = P.stride;
  const float x[3] = {P.x[s], P.x[st + s], P.x[2 * st + s]};
  bool drop = false;
  if (!DUAL && SF == PMPM_SHAPE_QUADRATIC) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const int b = (int)scaled_coord(x[c], g.origin[c], g.inv_h);
      drop = drop || b < 0 || b >= g.n[c];
    }
  }
  const float m = drop ? 0.0f : P.m[s];
  const float nv = (drop || a.remap) ? 0.0f : -P.V[s];
  const float Sxx = nv * P.sig[s], Syy = nv * P.sig[st + s], Szz = nv * P.sig[2 * st + s];
  const float Sxy = nv * P.sig[3 * st + s], Sxz = nv * P.sig[4 * st + s], Syz = nv * P.sig[5 * st + s];
  r[0] = make_float4(m, m * P.v[s], m * P.v[st + s], m * P.v[2 * st + s]);
  r[1] = make_float4(Sxx, Sxy, Sxy, Syy);
  r[2] = make_float4(Sxz, Syz, Szz, 0.0f);
  r[3] = make_float4(x[0], x[1], x[2], 0.0f);
  if (PLANAR) {
    const bool use = DUAL ? !a.remap : (m != 0.0f && !a.remap);
    r[4] = make_float4(use ? P.fext[s] : 0.0f, use ? P.fext[st + s] : 0.0f, use ? P.fext[2 * st + s] : 0.0f, 0.0f);
  }
}

template <int SF, bool DUAL, bool PLANAR>
__global__ void __launch_bounds__(256) k_records(StepArgs a) {
  if (binning_failed(a.fault)) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.B.scalars[0]) return;  // binned particles occupy sorted positions [0, binned)
  float4 r[5];
  make_record<SF, DUAL, PLANAR>(a, a.B.order[k], r);
  float4 *dst = a.B.rec + (size_t)k * (PLANAR ? 5 : 4);
#pragma unroll
  for (int q = 0; q < (PLANAR ? 5 : 4); q++) dst[q] = r[q];
}

// --------------------------------------------------------------------------
// physical re-sort of particle storage into cell order
// --------------------------------------------------------------------------

template <typename T>
__device__ __forceinline__ void move_comps(const T *src, T *dst, int ncomp, int stride, int from, int to) {
  if (!src) return;
  for (int c = 0; c < ncomp; c++) dst[c * stride + to] = src[c * stride + from];
}

template <int D>
__global__ void __launch_bounds__(256) k_reorder(StepArgs a, DevParticles dst, int move_L, int move_fext) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.P.n) return;
  const DevParticles &S = a.P;
  const int s = a.B.order[k];
  const int st = S.stride;
  move_comps(S.x, dst.x, D, st, s, k);
  move_comps(S.v, dst.v, D, st, s, k);
  move_comps(S.F, dst.F, D * D, st, s, k);
  move_comps(S.sig, dst.sig, Sym<D>::S, st, s, k);
  if (move_L) move_comps(S.L, dst.L, D * D, st, s, k);
  move_comps(S.m, dst.m, 1, st, s, k);
  move_comps(S.V, dst.V, 1, st, s, k);
  move_comps(S.V0, dst.V0, 1, st, s, k);
  if (move_fext) move_comps(S.fext, dst.fext, D, st, s, k);
  move_comps(S.eps, dst.eps, Sym<D>::E, st, s, k);
  move_comps(S.sref, dst.sref, Sym<D>::S, st, s, k);
  move_comps(S.color, dst.color, 1, st, s, k);
  move_comps(S.active, dst.active, 1, st, s, k);
  move_comps(S.rigid, dst.rigid, 1, st, s, k);
  move_comps(S.id, dst.id, 1, st, s, k);
  if (S.pE) {
    move_comps(S.pE, dst.pE, 1, st, s, k);
    move_comps(S.pphi, dst.pphi, 1, st, s, k);
  }
  if (S.acc) move_comps(S.acc, dst.acc, 1, st, s, k);
  if (S.pc) move_comps(S.pc, dst.pc, 1, st, s, k);
  move_comps(S.hash, dst.hash, 1, st, s, k);
  a.B.order[k] = k;  // storage is now in cell order
}

__global__ void __launch_bounds__(256) k_identity_order(int *order, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) order[k] = k;
}

// --------------------------------------------------------------------------
// P2G: node-tile gather with fused node epilogue
// --------------------------------------------------------------------------

// Adds the contributions of the particles at sorted positions [k0, k1) for
// window slot w to node nc (usl_p2g_kernel, src/solver/usl/usl_inline.h:
// 136-161): m += psi m_p; p += (psi m_p) v_p; f += psi f_ext - V_p sigma_p dpsi.
template <int D, int SF>
__device__ __forceinline__ void p2g_range(const StepArgs &a, int k0, int k1, const int w[3], const int nc[3],
                                          float &mass, float mom[3], float force[3]) {
  const DevParticles &P = a.P;
  const DevGrid &g = a.g;
  const int st = P.stride;
  for (int k = k0; k < k1; k++) {
    const int s = a.B.order[k];
    float u[3];
    int b[3];
    bool inside = true;
#pragma unroll
    for (int c = 0; c < D; c++) {
      u[c] = scaled_coord(P.x[c * st + s], g.origin[c], g.inv_h);
      b[c] = (int)u[c];
      inside = inside && b[c] >= 0 && b[c] < g.n[c];
    }
    if (SF == PMPM_SHAPE_QUADRATIC && !inside) continue;
    float N[3], dN[3];
#pragma unroll
    for (int c = 0; c < D; c++) {
      const float rel = u[c] - (float)(b[c] + w[c]);
      const int type = SF == PMPM_SHAPE_CUBIC ? cubic_node_type(nc[c], g.n[c]) : 0;
      axis_weight<SF>(rel, g.inv_h, type, N[c], dN[c]);
    }
    float psi, dpsi[3];
    if (D == 2) {
      psi = N[0] * N[1];
      dpsi[0] = dN[0] * N[1];
      dpsi[1] = dN[1] * N[0];
      dpsi[2] = 0.0f;
    } else {
      psi = N[0] * N[1] * N[2];
      dpsi[0] = dN[0] * N[1] * N[2];
      dpsi[1] = dN[1] * N[0] * N[2];
      dpsi[2] = dN[2] * N[0] * N[1];
    }
    const float sm = psi * P.m[s];
    mass += sm;
#pragma unroll
    for (int c = 0; c < D; c++) mom[c] += sm * P.v[c * st + s];
    if (a.has_planar && !a.remap) {
#pragma unroll
      for (int c = 0; c < D; c++) force[c] += psi * P.fext[c * st + s];
    }
    const float mv = a.remap ? 0.0f : -P.V[s];
    float S[9];
    load_sig3<D>(P, s, S);
#pragma unroll
    for (int c = 0; c < D; c++) {
      float acc = (mv * S[3 * c + 0]) * dpsi[0];
      acc += (mv * S[3 * c + 1]) * dpsi[1];
      if (D == 3) acc += (mv * S[3 * c + 2]) * dpsi[2];
      force[c] += acc;
    }
  }
}

template <int D, int SF>
__device__ __forceinline__ void p2g_gather_body(const StepArgs &a, int tile, int apply_bcs, int *node_epoch) {
  using T = TileDims<D>;
  const DevGrid &g = a.g;
  if (a.N.tile_epoch[tile] != a.epoch) return;
  if (threadIdx.x == 0) node_epoch[tile] = a.epoch;
  const int tx = tile % g.tdim[0], ty = (tile / g.tdim[0]) % g.tdim[1], tz = tile / (g.tdim[0] * g.tdim[1]);
  const int lx = threadIdx.x % T::X, ly = (threadIdx.x / T::X) % T::Y, lz = threadIdx.x / (T::X * T::Y);
  const int nc[3] = {tx * T::X + lx, ty * T::Y + ly, D == 3 ? tz * T::Z + lz : 0};
  if (nc[0] >= g.n[0] || nc[1] >= g.n[1] || nc[2] >= g.n[2]) return;
  const int node = flat_index(g, nc[0], nc[1], nc[2]);
  float mass = 0.0f, mom[3] = {0.0f, 0.0f, 0.0f}, force[3] = {0.0f, 0.0f, 0.0f};
  constexpr int NS = IPow<Stencil<SF>::WIN, D>::value;
  const int *off = a.B.offset;
  for (int sid = 0; sid < NS; sid++) {
    int w[3];
    window_offset<D, SF>(sid, w);
    if (SF == PMPM_SHAPE_QUADRATIC) {
      // cells whose slot w folds onto this node (axis-wise clamp preimage)
      int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
      bool empty = false;
#pragma unroll
      for (int c = 0; c < D; c++) {
        int l = nc[c] == 0 ? 0 : nc[c] - w[c];
        int h = nc[c] == g.n[c] - 1 ? g.n[c] - 1 : nc[c] - w[c];
        l = max(l, 0);
        h = min(h, g.n[c] - 1);
        if (l > h) empty = true;
        lo[c] = l;
        hi[c] = h;
      }
      if (empty) continue;
      for (int cz = lo[2]; cz <= hi[2]; cz++)
        for (int cy = lo[1]; cy <= hi[1]; cy++) {
          const int c0 = flat_index(g, lo[0], cy, cz), c1 = flat_index(g, hi[0], cy, cz);
          p2g_range<D, SF>(a, off[c0], off[c1 + 1], w, nc, mass, mom, force);
        }
    } else {
      const int cell = node - (w[0] + w[1] * g.n[0] + w[2] * g.n[0] * g.n[1]);
      if ((unsigned)cell >= (unsigned)g.ntotal) continue;
      p2g_range<D, SF>(a, off[cell], off[cell + 1], w, nc, mass, mom, force);
    }
  }
  // epilogue: the reference leaves nodes with m <= cutoff at their reset value (0)
  float p[3] = {0.0f, 0.0f, 0.0f}, pnt[3] = {0.0f, 0.0f, 0.0f};
  const bool live = mass > a.cutoff;
  if (live) {
#pragma unroll
    for (int c = 0; c < D; c++) {
      p[c] = mom[c];
      pnt[c] = mom[c] + force[c] * a.dt;
    }
  } else {
    mass = 0.0f;
  }
  if (apply_bcs) node_bcs<D>(a, node, nc, mass, p, pnt);
  write_node<D>(a, node, mass, p, pnt, live);
}

template <int D, int SF>
__global__ void __launch_bounds__(TileDims<D>::N) k_p2g_gather(StepArgs a, int apply_bcs, int *node_epoch) {
  if (binning_failed(a.fault)) return;
  p2g_gather_body<D, SF>(a, blockIdx.x, apply_bcs, node_epoch);
}

// --------------------------------------------------------------------------
// RigidBodyLevelSet, reference mode: nearest rigid particle stick contact
// --------------------------------------------------------------------------

struct RigidMotion {
  float R[9];  // row-major D x D rotation of this step
  float com[3];
};

// RigidBodyLevelSet::set_velocities, CPU branch, and update_rigid_velocity
// (src/boundaryconditions/rigidbodylevelset.cpp:245-275, rigidbodylevelset_inline.h:
// 240-299): v = (R (x - COM) - (x - COM)) / dt for rigid particles.
template <int D>
__global__ void __launch_bounds__(256) k_rigid_velocity(StepArgs a, RigidMotion rm) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const DevParticles &P = a.P;
  if (s >= P.n || !P.rigid[s]) return;
  const int st = P.stride;
  float r[3];
#pragma unroll
  for (int c = 0; c < D; c++) r[c] = __fsub_rn(P.x[c * st + s], rm.com[c]);
#pragma unroll
  for (int i = 0; i < D; i++) {
    float u = __fmul_rn(rm.R[i * D], r[0]);
#pragma unroll
    for (int j = 1; j < D; j++) u = __fadd_rn(u, __fmul_rn(rm.R[i * D + j], r[j]));
    P.v[i * st + s] = __fdiv_rn(__fsub_rn(u, r[i]), a.dt);
  }
}

// calculate_grid_normals_nn_rigid (src/boundaryconditions/rigidbodylevelset_inline.h:
// 65-199) for the nodes of the active tiles, then the node BCs listed after
// it.  Per node with m > 1e-9: over the linear P2G window cells (slot order,
// flattened index with the reference's single unsigned range check), the
// rigid particle nearest to its cell's corner (first strict minimum) gives
// the body velocity; the mass-weighted sum of the non-rigid particles' shape
// function gradients, normalised, the normal; p and p_nt each stick to the
// body velocity when (v - v_body) . n >= 0.  Linear shape functions only.
template <int D>
__global__ void __launch_bounds__(TileDims<D>::N) k_rigid_nodes(StepArgs a, int rb) {
  using T = TileDims<D>;
  const DevGrid &g = a.g;
  const DevParticles &P = a.P;
  const int tile = blockIdx.x;
  if (a.N.tile_epoch[tile] != a.epoch || binning_failed(a.fault)) return;
  const int tx = tile % g.tdim[0], ty = (tile / g.tdim[0]) % g.tdim[1], tz = tile / (g.tdim[0] * g.tdim[1]);
  const int lx = threadIdx.x % T::X, ly = (threadIdx.x / T::X) % T::Y, lz = threadIdx.x / (T::X * T::Y);
  const int nc[3] = {tx * T::X + lx, ty * T::Y + ly, D == 3 ? tz * T::Z + lz : 0};
  if (nc[0] >= g.n[0] || nc[1] >= g.n[1] || nc[2] >= g.n[2]) return;
  const int node = flat_index(g, nc[0], nc[1], nc[2]);
  const int nt = g.ntotal, st = P.stride;
  float m = a.N.m[node];
  float p[3] = {0.0f, 0.0f, 0.0f}, pnt[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int c = 0; c < D; c++) {
    p[c] = a.N.p[c * nt + node];
    pnt[c] = a.N.pnt[c * nt + node];
  }
  if (m > 0.000000001f) {
    float min_dist = 999999999999999.0f;
    int min_s = -1;
    float nrm[3] = {0.0f, 0.0f, 0.0f};
    constexpr int NS = D == 3 ? 8 : 4;
    for (int sid = 0; sid < NS; sid++) {
      int w[3];
      window_offset<D, PMPM_SHAPE_LINEAR>(sid, w);  // g2p offset; the cell is node - w
      const int cell = node - (w[0] + w[1] * g.n[0] + w[2] * g.n[0] * g.n[1]);
      if ((unsigned)cell >= (unsigned)nt) continue;
      for (int k = a.B.offset[cell]; k < a.B.offset[cell + 1]; k++) {
        const int s = a.B.order[k];
        float u[3];
#pragma unroll
        for (int c = 0; c < D; c++) u[c] = scaled_coord(P.x[c * st + s], g.origin[c], g.inv_h);
        if (P.rigid[s]) {
          float dist = 0.0f;
#pragma unroll
          for (int c = 0; c < D; c++) {
            const float rel = __fsub_rn(u[c], (float)(nc[c] - w[c]));
            dist = c == 0 ? __fmul_rn(rel, rel) : __fadd_rn(dist, __fmul_rn(rel, rel));
          }
          if (dist < min_dist) {
            min_dist = dist;
            min_s = s;
          }
        } else {
          // the particle's gradient for slot sid: node (own bin + w), zero
          // where that node is outside the flattened range
          int b[3];
#pragma unroll
          for (int c = 0; c < D; c++) b[c] = (int)u[c];
          const int tgt = flat_index(g, b[0] + w[0], b[1] + w[1], D == 3 ? b[2] + w[2] : 0);
          if ((unsigned)tgt >= (unsigned)nt) continue;
          float N[3], dN[3];
#pragma unroll
          for (int c = 0; c < D; c++)
            axis_weight<PMPM_SHAPE_LINEAR>(__fsub_rn(u[c], (float)(b[c] + w[c])), g.inv_h, 0, N[c], dN[c]);
          float dpsi[3];
          if (D == 2) {
            dpsi[0] = __fmul_rn(dN[0], N[1]);
            dpsi[1] = __fmul_rn(dN[1], N[0]);
          } else {
            dpsi[0] = __fmul_rn(__fmul_rn(dN[0], N[1]), N[2]);
            dpsi[1] = __fmul_rn(__fmul_rn(dN[1], N[0]), N[2]);
            dpsi[2] = __fmul_rn(__fmul_rn(dN[2], N[0]), N[1]);
          }
          const float mp = P.m[s];
#pragma unroll
          for (int c = 0; c < D; c++) nrm[c] = __fadd_rn(nrm[c], __fmul_rn(dpsi[c], mp));
        }
      }
    }
    if (min_s >= 0) {
      float sq = __fmul_rn(nrm[0], nrm[0]);
#pragma unroll
      for (int c = 1; c < D; c++) sq = __fadd_rn(sq, __fmul_rn(nrm[c], nrm[c]));
      if (sq > 0.0f) {
        const float len = __fsqrt_rn(sq);
#pragma unroll
        for (int c = 0; c < D; c++) nrm[c] = __fdiv_rn(nrm[c], len);
      }
      float vn[3], vnt[3], cv[3], cvt[3];
      float rel = 0.0f, rel_nt = 0.0f;
#pragma unroll
      for (int c = 0; c < D; c++) {
        const float vb = P.v[c * st + min_s];
        vn[c] = __fdiv_rn(p[c], m);
        vnt[c] = __fdiv_rn(pnt[c], m);
        cv[c] = __fsub_rn(vn[c], vb);
        cvt[c] = __fsub_rn(vnt[c], vb);
        rel = c == 0 ? __fmul_rn(cv[c], nrm[c]) : __fadd_rn(rel, __fmul_rn(cv[c], nrm[c]));
        rel_nt = c == 0 ? __fmul_rn(cvt[c], nrm[c]) : __fadd_rn(rel_nt, __fmul_rn(cvt[c], nrm[c]));
      }
      if (rel >= 0.0f) {
#pragma unroll
        for (int c = 0; c < D; c++) p[c] = __fmul_rn(__fsub_rn(vn[c], cv[c]), m);
      }
      if (rel_nt >= 0.0f) {
#pragma unroll
        for (int c = 0; c < D; c++) pnt[c] = __fmul_rn(__fsub_rn(vnt[c], cvt[c]), m);
      }
    }
  }
  node_bcs_range<D>(a, node, nc, m, p, pnt, rb + 1, a.nbc);
  write_node<D>(a, node, m, p, pnt, m > a.cutoff);
}

// --------------------------------------------------------------------------
// P2G, fast path: tile scatter into shared memory
// --------------------------------------------------------------------------
//
// One CTA per active node tile owns the tile's nodes.  It streams every
// particle of the cells that can reach those nodes (the tile plus a halo of
// the stencil width), evaluates the particle's per-axis weights once, and
// adds the contributions that land inside the tile to shared-memory
// accumulators (float atomics).  After a barrier each thread finishes one
// node: the same epilogue as the gather path.  Each (particle, node) pair is
// added by exactly one CTA, so no global atomics are needed; the summation
// order inside a node is not fixed (use the gather path for bitwise
// reproducibility).
//
// The halo is walked as rows of cells along x; a row is one contiguous range
// of the cell-sorted order.  Rows use the reference's flat cell arithmetic,
// so a row that runs past the grid's x extent continues into the next row of
// cells, exactly where the reference's gather (usl_inline.h:114-126) finds
// its aliased neighbours; overlapping row ranges are merged so each
// particle is visited once per tile.

template <int D, int SF>
struct P2GTileShape {
  using T = TileDims<D>;
  static constexpr int LO = Stencil<SF>::WLO;
  static constexpr int HI = Stencil<SF>::WLO + Stencil<SF>::WIN - 1;
  static constexpr int HX = T::X + HI - LO;
  static constexpr int HY = T::Y + HI - LO;
  static constexpr int HZ = D == 3 ? T::Z + HI - LO : 1;
  static constexpr int ROWS = HY * HZ;
  static constexpr int NACC = 1 + 2 * D;
};

// Particle phase of the tile P2G under dual-cell binning (quadratic): the
// source cells are the dual cells d in [t0 - 1, t0 + T] per axis, whose
// particles all reach the same nodes d - 1 .. d + 1 (clamped onto the grid).
// Each thread takes a contiguous chunk of the cell-sorted list; with RUN,
// consecutive particles of one dual cell are summed in registers and the
// cell's window is added to the shared accumulators once per run.
template <int D, bool RUN>
__device__ __forceinline__ void p2g_dual_particles(const StepArgs &a, const int t0[3], float *acc, int *row_k0,
                                                   int *row_pref, int *warp_tmp) {
  using T = TileDims<D>;
  constexpr int NT = T::N;
  constexpr int RY = T::Y + 2, RZ = D == 3 ? T::Z + 2 : 1;
  constexpr int ROWS = RY * RZ;
  constexpr int NW = D == 3 ? 27 : 9;  // window nodes
  constexpr int NV = 1 + 2 * D;        // mass, momentum, force
  const DevGrid &g = a.g;
  const DevParticles &P = a.P;
  const int st = P.stride;
  const int tid = threadIdx.x;
  const long long kd0 = a.B.kd[0], kd01 = (long long)a.B.kd[0] * a.B.kd[1];
  // ---- source rows (along x) -> sorted-order ranges ----
  int carry = 0;
  for (int it = 0; it < (ROWS + NT - 1) / NT; it++) {
    const int r = it * NT + tid;
    int cnt = 0, k0 = 0;
    if (r < ROWS) {
      const int dy = t0[1] - 1 + r % RY, dz = D == 3 ? t0[2] - 1 + r / RY : 0;
      const int dx0 = max(t0[0] - 1, 0), dx1 = min(t0[0] + T::X, g.n[0]);  // dual coordinates run 0 .. n
      const bool row_in = dy >= 0 && dy <= g.n[1] && (D == 2 || (dz >= 0 && dz <= g.n[2]));
      if (row_in && dx0 <= dx1) {
        const long long base = (long long)dy * kd0 + (long long)dz * kd01;
        k0 = a.B.offset[base + dx0];
        cnt = a.B.offset[base + dx1 + 1] - k0;
      }
    }
    int total;
    const int ex = block_exclusive_scan(cnt, warp_tmp, total);
    if (r < ROWS) {
      row_k0[r] = k0;
      row_pref[r] = carry + ex;
    }
    carry += total;
  }
  if (tid == 0) row_pref[ROWS] = carry;
  __syncthreads();
  const int ntot = row_pref[ROWS];
  // contiguous chunks; the lanes of a warp take chunks NT/32 apart
  const int chunk = (ntot + NT - 1) / NT;
  const int slot = (tid & 31) * (NT / 32) + (tid >> 5);
  const int j0 = slot * chunk, j1 = min(j0 + chunk, ntot);
  int row = 0;
  if (j0 < j1) {
    int lo = 0, hi = ROWS;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (row_pref[mid] <= j0) lo = mid; else hi = mid;
    }
    row = lo;
  }
  float run[RUN ? NW : 1][NV];
#pragma unroll
  for (int w = 0; w < (RUN ? NW : 1); w++)
#pragma unroll
    for (int v = 0; v < NV; v++) run[w][v] = 0.0f;
  int run_d[3] = {0, 0, 0};
  bool have_run = false;
  // adds a window's values (node k of each axis at d - 1 + k, clamped) to
  // the shared accumulators of the tile nodes it reaches
  auto add_window = [&](const int d[3], int w, const float *val) {
    const int kx = w % 3, ky = (w / 3) % 3, kz = D == 3 ? w / 9 : 0;
    const int nx = min(max(d[0] - 1 + kx, 0), g.n[0] - 1) - t0[0];
    const int ny = min(max(d[1] - 1 + ky, 0), g.n[1] - 1) - t0[1];
    const int nz = D == 3 ? min(max(d[2] - 1 + kz, 0), g.n[2] - 1) - t0[2] : 0;
    if (nx < 0 || nx >= T::X || ny < 0 || ny >= T::Y || nz < 0 || nz >= T::Z) return;
    const int ln = nx + T::X * (ny + T::Y * nz);
#pragma unroll
    for (int v = 0; v < NV; v++) atomicAdd(&acc[v * NT + ln], val[v]);
  };
  for (int j = j0; j < j1; j++) {
    while (row_pref[row + 1] <= j) row++;
    const int s = a.B.order[row_k0[row] + (j - row_pref[row])];
    float u[3] = {0, 0, 0};
    int d[3] = {0, 0, 0};
#pragma unroll
    for (int c = 0; c < D; c++) {
      u[c] = scaled_coord(P.x[c * st + s], g.origin[c], g.inv_h);
      d[c] = dual_coord(u[c], (int)u[c]);
    }
    if (RUN) {
      const bool same = have_run && d[0] == run_d[0] && d[1] == run_d[1] && (D == 2 || d[2] == run_d[2]);
      if (have_run && !same) {
#pragma unroll
        for (int w = 0; w < NW; w++) {
          add_window(run_d, w, run[w]);
#pragma unroll
          for (int v = 0; v < NV; v++) run[w][v] = 0.0f;
        }
      }
      have_run = true;
#pragma unroll
      for (int c = 0; c < 3; c++) run_d[c] = d[c];
    }
    float N[3][3], dN[3][3];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int k = 0; k < 3; k++) {
        N[c][k] = 1.0f;
        dN[c][k] = 0.0f;
        if (c < D) axis_weight<PMPM_SHAPE_QUADRATIC>(u[c] - (float)(d[c] - 1 + k), g.inv_h, 0, N[c][k], dN[c][k]);
      }
    const float m = P.m[s];
    float mv[3] = {0, 0, 0}, fx[3] = {0, 0, 0}, S[9];
#pragma unroll
    for (int c = 0; c < D; c++) mv[c] = m * P.v[c * st + s];
    if (a.has_planar && !a.remap) {
#pragma unroll
      for (int c = 0; c < D; c++) fx[c] = P.fext[c * st + s];
    }
    load_sig3<D>(P, s, S);
    const float nvol = a.remap ? 0.0f : -P.V[s];
#pragma unroll
    for (int k = 0; k < 9; k++) S[k] *= nvol;
#pragma unroll
    for (int w = 0; w < NW; w++) {
      const int kx = w % 3, ky = (w / 3) % 3, kz = D == 3 ? w / 9 : 0;
      float psi, dpsi[3];
      if (D == 2) {
        psi = N[0][kx] * N[1][ky];
        dpsi[0] = dN[0][kx] * N[1][ky];
        dpsi[1] = dN[1][ky] * N[0][kx];
        dpsi[2] = 0.0f;
      } else {
        psi = N[0][kx] * N[1][ky] * N[2][kz];
        dpsi[0] = dN[0][kx] * N[1][ky] * N[2][kz];
        dpsi[1] = dN[1][ky] * N[0][kx] * N[2][kz];
        dpsi[2] = dN[2][kz] * N[0][kx] * N[1][ky];
      }
      float val[NV];
      val[0] = psi * m;
#pragma unroll
      for (int c = 0; c < D; c++) {
        float f = psi * fx[c] + S[3 * c + 0] * dpsi[0] + S[3 * c + 1] * dpsi[1];
        if (D == 3) f += S[3 * c + 2] * dpsi[2];
        val[1 + c] = psi * mv[c];
        val[1 + D + c] = f;
      }
      if (RUN) {
#pragma unroll
        for (int v = 0; v < NV; v++) run[w][v] += val[v];
      } else {
        add_window(d, w, val);
      }
    }
  }
  if (RUN && have_run) {
#pragma unroll
    for (int w = 0; w < NW; w++) add_window(run_d, w, run[w]);
  }
}

template <int D, int SF>
__device__ __forceinline__ void p2g_tile_body(const StepArgs &a, int tile, int apply_bcs, int *node_epoch) {
  using T = TileDims<D>;
  using Sh = P2GTileShape<D, SF>;
  constexpr int NT = T::N;
  constexpr int K = Stencil<SF>::K;
  const DevGrid &g = a.g;
  if (a.N.tile_epoch[tile] != a.epoch) return;

  __shared__ float acc[Sh::NACC * NT];
  __shared__ int row_k0[Sh::ROWS];
  __shared__ int row_lo[Sh::ROWS], row_hi[Sh::ROWS];
  __shared__ int row_pref[Sh::ROWS + 1];
  __shared__ int warp_tmp[33];

  const int tid = threadIdx.x;
  const int t0[3] = {(tile % g.tdim[0]) * T::X, ((tile / g.tdim[0]) % g.tdim[1]) * T::Y,
                     D == 3 ? (tile / (g.tdim[0] * g.tdim[1])) * T::Z : 0};
#pragma unroll
  for (int k = 0; k < Sh::NACC; k++) acc[k * NT + tid] = 0.0f;
  if (tid == 0) node_epoch[tile] = a.epoch;

  bool dual_done = false;
  if constexpr (SF == PMPM_SHAPE_QUADRATIC) {
    static_assert(Sh::ROWS >= (TileDims<D>::Y + 2) * (D == 3 ? TileDims<D>::Z + 2 : 1), "dual source rows");
    if (a.B.dual) {
      // dual-cell binning: the source cells are the dual cells whose
      // windows reach the tile
      p2g_dual_particles<D, D == 2>(a, t0, acc, row_k0, row_pref, warp_tmp);
      dual_done = true;
    }
  }
  if (!dual_done) {
    // ---- halo rows -> flat cell intervals -> sorted-order ranges ----
    // Interior tiles (halo inside the grid) have disjoint, increasing row
    // intervals.  Near the grid boundary the reference's flat arithmetic can
    // make virtual rows overlap, so there the intervals are sorted and merged
    // (each particle must be visited once).
    bool interior = true;
    {
      const int tsz[3] = {T::X, T::Y, T::Z};
#pragma unroll
      for (int c = 0; c < D; c++)
        interior = interior && t0[c] - Sh::HI >= 0 && t0[c] + tsz[c] - 1 - Sh::LO <= g.n[c] - 1;
    }
    const bool merge = SF != PMPM_SHAPE_QUADRATIC && !interior;
    for (int r = tid; r < Sh::ROWS; r += NT) {
      const int cy = t0[1] - Sh::HI + r % Sh::HY;
      const int cz = D == 3 ? t0[2] - Sh::HI + r / Sh::HY : 0;
      int x0 = t0[0] - Sh::HI, x1 = t0[0] + T::X - 1 - Sh::LO;
      long long lo, hi;
      if (SF == PMPM_SHAPE_QUADRATIC) {
        const bool row_in = cy >= 0 && cy < g.n[1] && cz >= 0 && cz < g.n[2];
        x0 = max(x0, 0);
        x1 = min(x1, g.n[0] - 1);
        lo = flat_index(g, x0, cy, cz);
        hi = row_in ? (long long)flat_index(g, x1, cy, cz) : lo - 1;
      } else {
        const long long base = (long long)cy * g.n[0] + (long long)cz * g.n[0] * g.n[1];
        lo = max(base + x0, 0ll);
        hi = min(base + x1, (long long)g.ntotal - 1);
      }
      // keep 0 <= lo and hi <= ntotal - 1; lo > hi marks an empty row
      row_lo[r] = (int)min(max(lo, 0ll), (long long)g.ntotal);
      row_hi[r] = (int)max(min(hi, (long long)g.ntotal - 1), -1ll);
    }
    __syncthreads();
    if (merge && tid == 0) {
      // insertion sort by interval start, then clip each start past the
      // furthest end seen so far
      for (int i = 1; i < Sh::ROWS; i++) {
        const int l = row_lo[i], h = row_hi[i];
        int j = i - 1;
        while (j >= 0 && row_lo[j] > l) {
          row_lo[j + 1] = row_lo[j];
          row_hi[j + 1] = row_hi[j];
          j--;
        }
        row_lo[j + 1] = l;
        row_hi[j + 1] = h;
      }
      int maxend = -1;
      for (int i = 0; i < Sh::ROWS; i++) {
        if (row_lo[i] > row_hi[i]) continue;
        if (row_lo[i] <= maxend) row_lo[i] = maxend + 1;
        if (row_hi[i] > maxend) maxend = row_hi[i];
      }
    }
    __syncthreads();
    const int nrow_iter = (Sh::ROWS + NT - 1) / NT;
    int carry = 0;
    for (int it = 0; it < nrow_iter; it++) {
      const int r = it * NT + tid;
      int cnt = 0, k0 = 0;
      if (r < Sh::ROWS) {
        const int lo = row_lo[r], hi = row_hi[r];
        if (lo <= hi) {
          k0 = a.B.offset[lo];
          cnt = a.B.offset[hi + 1] - k0;
        }
      }
      int total;
      const int ex = block_exclusive_scan(cnt, warp_tmp, total);
      if (r < Sh::ROWS) {
        row_k0[r] = k0;
        row_pref[r] = carry + ex;
      }
      carry += total;
    }
    if (tid == 0) row_pref[Sh::ROWS] = carry;
    __syncthreads();
    const int ntot = row_pref[Sh::ROWS];

    // ---- particles: each thread takes one contiguous chunk of the list; the
    // lanes of a warp take chunks NT/32 apart, so their stencils rarely share
    // nodes (neighbouring chunks lie in neighbouring cells, whose stencils
    // overlap and would serialise the shared-memory atomics) ----
    const int chunk = (ntot + NT - 1) / NT;
    const int slot = (tid & 31) * (NT / 32) + (tid >> 5);
    const int j0 = slot * chunk, j1 = min(j0 + chunk, ntot);
    int row = 0;
    if (j0 < j1) {
      int lo = 0, hi = Sh::ROWS;  // last row with row_pref <= j0
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (row_pref[mid] <= j0) lo = mid; else hi = mid;
      }
      row = lo;
    }
    const DevParticles &P = a.P;
    const int st = P.stride;
    for (int j = j0; j < j1; j++) {
      while (row_pref[row + 1] <= j) row++;
      const int s = a.B.order[row_k0[row] + (j - row_pref[row])];
      float u[3] = {0, 0, 0};
      int b[3] = {0, 0, 0};
      bool inside = true;
#pragma unroll
      for (int c = 0; c < D; c++) {
        u[c] = scaled_coord(P.x[c * st + s], g.origin[c], g.inv_h);
        b[c] = (int)u[c];
        inside = inside && b[c] >= 0 && b[c] < g.n[c];
      }
      if (SF == PMPM_SHAPE_QUADRATIC && !inside) continue;
      // per-axis weights, target node coordinates and tile-local coordinates
      float N[3][K], dN[3][K];
      int loc[3][K];   // tile-local coordinate, or -1 outside the tile
      bool inrange[3][K];
      int woff[3] = {Stencil<SF>::WLO, Stencil<SF>::WLO, Stencil<SF>::WLO};
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int k = 0; k < K; k++) {
          N[c][k] = 1.0f;
          dN[c][k] = 0.0f;
          loc[c][k] = 0;
          inrange[c][k] = true;
        }
      const int tsz[3] = {T::X, T::Y, T::Z};
#pragma unroll
      for (int c = 0; c < D; c++) {
        if (SF == PMPM_SHAPE_QUADRATIC) woff[c] = (u[c] - (float)(b[c] - 1)) < 1.5f ? -1 : 0;
#pragma unroll
        for (int k = 0; k < K; k++) {
          const int sel = b[c] + woff[c] + k;
          const bool in = sel >= 0 && sel < g.n[c];
          const int node_c = SF == PMPM_SHAPE_QUADRATIC ? min(max(sel, 0), g.n[c] - 1) : sel;
          const int type = SF == PMPM_SHAPE_CUBIC ? cubic_node_type(in ? sel : 0, g.n[c]) : 0;
          axis_weight<SF>(u[c] - (float)sel, g.inv_h, type, N[c][k], dN[c][k]);
          inrange[c][k] = SF == PMPM_SHAPE_QUADRATIC ? true : in;
          const int l = node_c - t0[c];
          loc[c][k] = (l >= 0 && l < tsz[c]) ? l : -1;
        }
      }
      const float m = P.m[s];
      float mv[3], fx[3] = {0, 0, 0}, S[9];
#pragma unroll
      for (int c = 0; c < D; c++) mv[c] = m * P.v[c * st + s];
      if (a.has_planar && !a.remap) {
#pragma unroll
        for (int c = 0; c < D; c++) fx[c] = P.fext[c * st + s];
      }
      load_sig3<D>(P, s, S);
      const float nvol = a.remap ? 0.0f : -P.V[s];
#pragma unroll
      for (int k = 0; k < 9; k++) S[k] *= nvol;
      const unsigned hu = P.hash[s];
      constexpr int KZ = D == 3 ? K : 1;
#pragma unroll
      for (int ky = 0; ky < K; ky++) {
#pragma unroll
        for (int kx = 0; kx < K; kx++) {
#pragma unroll
          for (int kz = 0; kz < KZ; kz++) {
            int lx = loc[0][kx], ly = loc[1][ky], lz = D == 3 ? loc[2][kz] : 0;
            const bool all_in = inrange[0][kx] && inrange[1][ky] && (D == 2 || inrange[2][kz]);
            float tN[3] = {N[0][kx], N[1][ky], D == 3 ? N[2][kz] : 1.0f};
            float tdN[3] = {dN[0][kx], dN[1][ky], D == 3 ? dN[2][kz] : 0.0f};
            if (!all_in) {
              // reference aliasing: the slot leaves the grid on an axis; its
              // node is the flat index hash + flat(window offset)
              const int w[3] = {woff[0] + kx, woff[1] + ky, D == 3 ? woff[2] + kz : 0};
              const long long f = (long long)hu + w[0] + (long long)w[1] * g.n[0] +
                                  (long long)w[2] * g.n[0] * g.n[1];
              if (f < 0 || f >= g.ntotal) continue;
              const int fc[3] = {(int)(f % g.n[0]), (int)((f / g.n[0]) % g.n[1]),
                                 (int)(f / ((long long)g.n[0] * g.n[1]))};
              lx = fc[0] - t0[0];
              ly = fc[1] - t0[1];
              lz = D == 3 ? fc[2] - t0[2] : 0;
              if (lx < 0 || lx >= T::X || ly < 0 || ly >= T::Y || lz < 0 || lz >= T::Z) continue;
              if (SF == PMPM_SHAPE_CUBIC) {
                // node types of the aliased node (src/shapefunction/shapefunction.cpp:104-110)
#pragma unroll
                for (int c = 0; c < D; c++)
                  axis_weight<SF>(u[c] - (float)(b[c] + w[c]), g.inv_h, cubic_node_type(fc[c], g.n[c]), tN[c], tdN[c]);
              }
            } else if (lx < 0 || ly < 0 || lz < 0) {
              continue;
            }
            float psi, dpsi[3];
            if (D == 2) {
              psi = tN[0] * tN[1];
              dpsi[0] = tdN[0] * tN[1];
              dpsi[1] = tdN[1] * tN[0];
              dpsi[2] = 0.0f;
            } else {
              psi = tN[0] * tN[1] * tN[2];
              dpsi[0] = tdN[0] * tN[1] * tN[2];
              dpsi[1] = tdN[1] * tN[0] * tN[2];
              dpsi[2] = tdN[2] * tN[0] * tN[1];
            }
            const int ln = lx + T::X * (ly + T::Y * lz);
            atomicAdd(&acc[ln], psi * m);
#pragma unroll
            for (int c = 0; c < D; c++) {
              float f = psi * fx[c] + S[3 * c + 0] * dpsi[0] + S[3 * c + 1] * dpsi[1];
              if (D == 3) f += S[3 * c + 2] * dpsi[2];
              atomicAdd(&acc[(1 + c) * NT + ln], psi * mv[c]);
              atomicAdd(&acc[(1 + D + c) * NT + ln], f);
            }
          }
        }
      }
    }
  }
  __syncthreads();

  // ---- node epilogue (one node per thread) ----
  const int lx = tid % T::X, ly = (tid / T::X) % T::Y, lz = tid / (T::X * T::Y);
  const int nc[3] = {t0[0] + lx, t0[1] + ly, D == 3 ? t0[2] + lz : 0};
  if (nc[0] >= g.n[0] || nc[1] >= g.n[1] || nc[2] >= g.n[2]) return;
  const int node = flat_index(g, nc[0], nc[1], nc[2]);
  float mass = acc[tid];
  float p[3] = {0.0f, 0.0f, 0.0f}, pnt[3] = {0.0f, 0.0f, 0.0f};
  const bool live = mass > a.cutoff;
  if (live) {
#pragma unroll
    for (int c = 0; c < D; c++) {
      p[c] = acc[(1 + c) * NT + tid];
      pnt[c] = p[c] + acc[(1 + D + c) * NT + tid] * a.dt;
    }
  } else {
    mass = 0.0f;
  }
  if (apply_bcs) node_bcs<D>(a, node, nc, mass, p, pnt);
  write_node<D>(a, node, mass, p, pnt, live);
}

template <int D, int SF>
__global__ void __launch_bounds__(TileDims<D>::N, D == 2 ? 3 : 1) k_p2g_tile(StepArgs a, int apply_bcs, int *node_epoch) {
  if (binning_failed(a.fault)) return;
  p2g_tile_body<D, SF>(a, blockIdx.x, apply_bcs, node_epoch);
}

// --------------------------------------------------------------------------
// P2G, 3D fast path: z-sweep with register windows
// --------------------------------------------------------------------------
//
// One CTA per active work unit of two 8x8x8 node tiles stacked in z (8x8x16
// nodes, so a cubic unit reads 19 source layers for 16 node layers instead
// of 11 for 8).  Work item = (x pair, y pair), a pair being (source cell
// column, stencil offset) whose target node column lies in the unit.  Each item sweeps the source cell layers along z.  For every
// layer the CTA stages the particles of the layer's halo cells in shared
// memory (with their z weights, which every item needs), then each item adds
// its source cell's particles into a register window of the WIN z nodes
// that layer can reach.  The lowest window node is complete after the layer
// (later layers only reach higher nodes), so it is added to the shared tile
// accumulator and the window shifts: 7 shared-memory atomics per item and
// tile node instead of 7 per particle and node.
//
// Sources are virtual cells: node n takes slot w from cell flat(n) - flat(w),
// the reference gather's flat arithmetic (usl_inline.h:114-126), so cells
// past a grid face alias onto neighbouring rows exactly as there; the weight
// uses the particle's own bin (the reference psi), the cubic node type the
// target node's.  Quadratic sources are real cells and targets are clamped.

template <int SF>
struct Sweep3 {
  using T = TileDims<3>;
  static constexpr int WIN = Stencil<SF>::WIN;
  static constexpr int LO = Stencil<SF>::WLO;
  static constexpr int HI = Stencil<SF>::WLO + Stencil<SF>::WIN - 1;
  static constexpr int NS = T::X + WIN - 1;          // source cells per axis
  static constexpr int MAXPAIR = NS * WIN;           // (source, offset) pairs per axis
  static constexpr int NCELL = NS * NS;              // source cells per layer
  static constexpr int TZ = 2 * T::Z;                // nodes along z of a work unit (two tiles)
  static constexpr int NN = T::X * T::Y * TZ;        // nodes of a work unit
  static constexpr int NL = TZ + WIN - 1;            // source layers a unit reads
  static constexpr int NT = 1024;
  static constexpr int IPT = 1;                      // items per thread per round
  static constexpr int NZ4 = (2 * WIN + 3) / 4;     // float4s of z weights
  // staged floats per particle: the x and y weights of the WIN offsets
  // (float2 N, dN each), float4 (m, m vx, m vy, m vz), float4 (Sxx, Sxy, Sxy,
  // Syy), float4 (Sxz, Syz, Szz, 0), the z weights then derivatives of the
  // layer's WIN nodes (NZ4 float4s); a PlanarDomain adds float4 (f, 0);
  // S = -V sigma
  __host__ __device__ static constexpr int floats(bool planar) {
    return 4 * WIN + 12 + 4 * NZ4 + (planar ? 4 : 0);
  }
  // float4s of one P2G record (k_records), bulk-copied per row of source cells
  __host__ __device__ static constexpr int rec4(bool planar) { return planar ? 5 : 4; }
  static constexpr int NROWS = NL * NS;              // rows of source cells along x
  // static shared memory: pair lists, the all-layer cell table, scan scratch,
  // the copy barrier
  static constexpr int STATIC_BYTES =
      (4 * (2 * MAXPAIR + 2 + 2 * NL * NCELL + 1 + 33 + 1 + 2) + 255) / 256 * 256 + 256;
  // staged particles (and with bulk staging their records): 227 KB per CTA
  // less the static part and the node accumulators
  __host__ __device__ static constexpr int cap(bool planar, bool bulk) {
    return ((232448 - STATIC_BYTES - 7 * NN * 4) / (4 * floats(planar) + (bulk ? 16 * rec4(planar) : 0))) & ~7;
  }
};

template <int SF, bool PLANAR, bool BULK>
constexpr int sweep3_smem_bytes() {
  using W = Sweep3<SF>;
  return (7 * W::NN + W::cap(PLANAR, BULK) * W::floats(PLANAR)) * 4 +
         (BULK ? W::cap(PLANAR, BULK) * W::rec4(PLANAR) * 16 : 0);
}

// Issues the bulk copies of positions [p0, p1) of a work unit's particle
// list into raw[0 .. p1 - p0) (R4 float4s each) and arms the barrier with
// their bytes.  The list runs through the unit's table of source cells in
// order; a row of NS cells along x has consecutive binning keys, so its
// particles are one run of the sorted records: one copy per row that
// overlaps the piece, issued by the row's thread.  Every copy lies inside
// the binned records (sorted positions of the row's cells) and inside raw.
template <int NS, int R4>
__device__ __forceinline__ void issue_piece(const float4 *rec, const int *cell_k0, const int *cell_pref, int nrows,
                                            int p0, int p1, float4 *raw, BulkState *bs) {
  const int tid = threadIdx.x;
  if (*(volatile int *)&bs->failed) return;  // the CTA's copies stopped after a wait gave up
  unsigned long long *bar = &bs->bar;
  if (tid == 0) mbar_arrive_expect_tx(bar, (unsigned)(p1 - p0) * R4 * 16u);
  if (tid < nrows) {
    const int c0 = tid * NS;
    const int a0 = cell_pref[c0], b0 = cell_pref[c0 + NS];
    const int lo = max(a0, p0), hi = min(b0, p1);
    if (lo < hi) {
      // the row's first particle is the first particle of its first non-empty cell
      int k0 = 0;
      for (int i = 0; i < NS; i++) {
        if (cell_pref[c0 + i + 1] > cell_pref[c0 + i]) {
          k0 = cell_k0[c0 + i];
          break;
        }
      }
      fence_async_smem();
      bulk_copy_g2s(raw + (size_t)(lo - p0) * R4, rec + (size_t)(k0 + (lo - a0)) * R4, (unsigned)(hi - lo) * R4 * 16u,
                    bar);
    }
  }
}

// pair encoding: source (virtual, relative to tile origin - HI) in bits 0..7,
// stencil offset in bits 8..9, target local coordinate in bits 12..15, bit
// 16 set where the target lies inside the grid (every listed pair, except the
// padded target-major lists of the linear and cubic sweeps)
__device__ __forceinline__ int pair_src(int p) { return p & 0xff; }
__device__ __forceinline__ int pair_off(int p) { return (p >> 8) & 0x3; }
__device__ __forceinline__ int pair_tgt(int p) { return (p >> 12) & 0xf; }

template <int SF>
__device__ __forceinline__ int build_pairs(int t0, int n, int *pairs) {
  using W = Sweep3<SF>;
  constexpr int TS = W::T::X;
  int cnt = 0;
  for (int si = 0; si < W::NS; si++) {
    const int src = t0 - W::HI + si;
    if (SF == PMPM_SHAPE_QUADRATIC && (src < 0 || src >= n)) continue;
    for (int i = 0; i < W::WIN; i++) {
      int t = src + i + W::LO;
      if (SF == PMPM_SHAPE_QUADRATIC) t = min(max(t, 0), n - 1);
      const int l = t - t0;
      if (l < 0 || l >= TS || t >= n || t < 0) continue;
      pairs[cnt++] = si | (i << 8) | (l << 12) | (1 << 16);
    }
  }
  return cnt;
}

// Linear and cubic: every (target column l, stencil offset i) of the unit in
// target-major order, 8 WIN entries, so that the WIN pairs adding into one
// target are neighbouring work items (neighbouring lanes of a warp); the
// source column is l - i - LO + HI; bit 16 marks a target inside the grid.
template <int SF>
__device__ __forceinline__ int build_pairs_by_target(int t0, int n, int *pairs) {
  using W = Sweep3<SF>;
  int cnt = 0;
  for (int l = 0; l < W::T::X; l++)
    for (int i = 0; i < W::WIN; i++)
      pairs[cnt++] = (l - i - W::LO + W::HI) | (i << 8) | (l << 12) | (t0 + l < n ? 1 << 16 : 0);
  return cnt;
}
__device__ __forceinline__ bool pair_valid(int p) { return (p >> 16) & 1; }

// Staged slot of piece position j: an XOR swizzle inside aligned groups of
// eight, so lanes reading the same position of neighbouring cells (runs of
// about eight) hit different shared-memory banks.
__device__ __forceinline__ int sweep_slot(int j) { return j ^ ((j >> 3) & 7); }

// BULK: a piece's particles arrive as sorted records by bulk copy (k_records
// wrote them); otherwise each is gathered through the sorted order.
// bs / phase: the CTA's copy state and the parity of its barrier's next phase
template <int SF, bool PLANAR, bool BULK>
__device__ __forceinline__ void sweep3_tile(const StepArgs &a, int apply_bcs, int *node_epoch, int unit,
                                            BulkState *bs, unsigned &phase) {
  using W = Sweep3<SF>;
  using T = TileDims<3>;
  constexpr int NT = W::NT;
  constexpr int WIN = W::WIN;
  constexpr int SL = W::cap(PLANAR, BULK);
  constexpr int R4 = W::rec4(PLANAR);
  constexpr int TZ = W::TZ, NN = W::NN;
  const DevGrid &g = a.g;

  __shared__ int pairs_x[W::MAXPAIR], pairs_y[W::MAXPAIR];
  __shared__ int npair[2];
  // every layer's source cells: first sorted position and running prefix
  __shared__ int cell_k0[W::NL * W::NCELL], cell_pref[W::NL * W::NCELL + 1];
  __shared__ int warp_tmp[33];
  // dynamic shared memory: tile accumulators, then the staged particles
  // (arrays of SL slots, see Sweep3::floats); size sweep3_smem_bytes<SF, PLANAR>()
  extern __shared__ __align__(16) float dyn_smem[];
  float *acc = dyn_smem;                                    // [7][NN]
  float2(*st_wx)[SL] = (float2(*)[SL])(acc + 7 * NN);       // [WIN] x weights (N, dN) per offset
  float2(*st_wy)[SL] = st_wx + WIN;                         // [WIN]
  float4 *st_p = (float4 *)(st_wy + WIN);                   // (m, m v)
  float4 *st_s0 = st_p + SL;                                // (Sxx, Sxy, Sxy, Syy)
  float4 *st_s1 = st_s0 + SL;                               // (Sxz, Syz, Szz, 0)
  float4(*st_z)[SL] = (float4(*)[SL])(st_s1 + SL);          // [NZ4] z N[0..WIN), dN[0..WIN)
  float4 *st_f = (float4 *)(st_z + W::NZ4);                 // PLANAR: (f, 0)
  float4 *raw = (float4 *)(acc + 7 * NN + SL * W::floats(PLANAR));  // BULK: [SL][R4] records of the piece

  // work unit `unit`: the two tiles 2k, 2k + 1 along z of one tile column
  const int tid = threadIdx.x;
  const int plane = g.tdim[0] * g.tdim[1];
  const int col = unit % plane, tz0 = 2 * (unit / plane);
  const int t0[3] = {(col % g.tdim[0]) * T::X, (col / g.tdim[0]) * T::Y, tz0 * T::Z};
  for (int k = tid; k < 7 * NN; k += NT) acc[k] = 0.0f;
  if (tid == 0) {
    node_epoch[col + tz0 * plane] = a.epoch;
    if (tz0 + 1 < g.tdim[2]) node_epoch[col + (tz0 + 1) * plane] = a.epoch;
    npair[0] = SF == PMPM_SHAPE_QUADRATIC ? build_pairs<SF>(t0[0], g.n[0], pairs_x)
                                          : build_pairs_by_target<SF>(t0[0], g.n[0], pairs_x);
  } else if (tid == 32) {
    npair[1] = SF == PMPM_SHAPE_QUADRATIC ? build_pairs<SF>(t0[1], g.n[1], pairs_y)
                                          : build_pairs_by_target<SF>(t0[1], g.n[1], pairs_y);
  }
  __syncthreads();
  const int nx = npair[0], ny = npair[1];
  const int nitems = nx * ny;
  const int nrounds = (nitems + NT * W::IPT - 1) / (NT * W::IPT);

  // z range of source layers
  int cz_lo = t0[2] - W::HI, cz_hi = t0[2] + TZ - 1 - W::LO;
  if (SF == PMPM_SHAPE_QUADRATIC) {
    cz_lo = max(cz_lo, 0);
    cz_hi = min(cz_hi, g.n[2] - 1);
  }
  const int nlayers = cz_hi - cz_lo + 1;
  const long long nxny = (long long)g.n[0] * g.n[1];

  // ---- all layers' source cells -> sorted ranges, one prefix ----
  const int ntab = nlayers * W::NCELL;
  {
    constexpr int PER = (W::NL * W::NCELL + NT - 1) / NT;
    int cnt[PER];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < PER; k++) {
      const int idx = tid * PER + k;
      cnt[k] = 0;
      if (idx < ntab) {
        const int layer = idx / W::NCELL, vc = idx % W::NCELL;
        const int sx = t0[0] - W::HI + vc % W::NS, sy = t0[1] - W::HI + vc / W::NS;
        const long long f = sx + (long long)sy * g.n[0] + (long long)(cz_lo + layer) * nxny;
        const bool valid = SF == PMPM_SHAPE_QUADRATIC ? (sx >= 0 && sx < g.n[0] && sy >= 0 && sy < g.n[1])
                                                      : (f >= 0 && f < g.ntotal);
        int k0 = 0;
        if (valid) {
          k0 = a.B.offset[f];
          cnt[k] = a.B.offset[f + 1] - k0;
        }
        cell_k0[idx] = k0;
        sum += cnt[k];
      }
    }
    int total;
    int ex = block_exclusive_scan(sum, warp_tmp, total);
#pragma unroll
    for (int k = 0; k < PER; k++) {
      const int idx = tid * PER + k;
      if (idx < ntab) cell_pref[idx] = ex;
      ex += cnt[k];
    }
    if (tid == 0) cell_pref[ntab] = total;
  }
  __syncthreads();
  const int total = cell_pref[ntab];

  // table cell of position j of the unit's particle list
  auto locate = [&](int j) {
    int lo = 0, hi = ntab;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (cell_pref[mid] <= j) lo = mid; else hi = mid;
    }
    return lo;
  };
  // ---- stage particle list position j (record r, table cell lo) into slot jj ----
  auto stage_one = [&](int lo, const float4 *r, int jj) {
    const int layer = lo / W::NCELL, vc = lo - layer * W::NCELL;
    const int cz = cz_lo + layer;
    const float4 xp = r[3];
    const float xs[3] = {xp.x, xp.y, xp.z};
    float u[3];
    int b[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      u[c] = scaled_coord(xs[c], g.origin[c], g.inv_h);
      b[c] = (int)u[c];
    }
    // (m, m v), -V sigma as (xx, xy, xy, yy) (xz, yz, zz, 0), f_ext: k_records
    st_p[jj] = r[0];
    st_s0[jj] = r[1];
    st_s1[jj] = r[2];
    if (PLANAR) st_f[jj] = r[4];
    // weights of the WIN offsets per axis: r from the particle's own bin
    // (the reference psi), the cubic node type of the target the offset
    // reaches from the (possibly aliased) source cell the particle is
    // staged for.  Cubic at u >= 0: offset w sits on spline piece 2 - w
    // (r in [-w, 1 - w)), so its coefficients are the same for neighbouring
    // lanes; u < 0 takes the general form
    const int src[3] = {t0[0] - W::HI + vc % W::NS, t0[1] - W::HI + vc / W::NS, cz};
    float zf[4 * W::NZ4];
#pragma unroll
    for (int k = 0; k < 4 * W::NZ4; k++) zf[k] = 0.0f;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (SF == PMPM_SHAPE_CUBIC && u[c] >= 0.0f && src[c] + W::LO >= 2 && src[c] + W::LO + 3 <= g.n[c] - 2) {
        // all four targets are interior nodes (type 3) and the source cell
        // is the particle's own: the four weights together
        float N4[4], dN4[4];
        cubic_interior_weights(u[c] - (float)b[c], g.inv_h, N4, dN4);
#pragma unroll
        for (int k = 0; k < WIN; k++) {
          if (c == 0) st_wx[k][jj] = make_float2(N4[k], dN4[k]);
          else if (c == 1) st_wy[k][jj] = make_float2(N4[k], dN4[k]);
          else {
            zf[k] = N4[k];
            zf[WIN + k] = dN4[k];
          }
        }
        continue;
      }
#pragma unroll
      for (int k = 0; k < WIN; k++) {
        const int tgt = src[c] + k + W::LO;
        const int type = SF == PMPM_SHAPE_CUBIC ? cubic_node_type(min(max(tgt, 0), g.n[c] - 1), g.n[c]) : 0;
        const float r = u[c] - (float)(b[c] + k + W::LO);
        float N, dN;
        if (SF == PMPM_SHAPE_CUBIC && u[c] >= 0.0f) {
          const float *cw = kCubicW[type][WIN - 1 - k], *cd = kCubicD[type][WIN - 1 - k];
          N = ((cw[0] * r + cw[1]) * r + cw[2]) * r + cw[3];
          dN = g.inv_h * ((cd[0] * r + cd[1]) * r + cd[2]);
        } else {
          axis_weight<SF>(r, g.inv_h, type, N, dN);
        }
        if (c == 0) st_wx[k][jj] = make_float2(N, dN);
        else if (c == 1) st_wy[k][jj] = make_float2(N, dN);
        else {
          zf[k] = N;
          zf[WIN + k] = dN;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < W::NZ4; k++) st_z[k][jj] = make_float4(zf[4 * k], zf[4 * k + 1], zf[4 * k + 2], zf[4 * k + 3]);
  };

  constexpr int R = (SL + NT - 1) / NT;
  const int nrows = nlayers * W::NS;
  // storage slot of list position j (table cell lo), for the gathered staging
  auto slot_of = [&](int j, int lo) { return a.B.order[cell_k0[lo] + (j - cell_pref[lo])]; };
  for (int round = 0; round < nrounds; round++) {
    // the first piece's records are on their way while the items are set up
    if (BULK && total > 0)
      issue_piece<W::NS, R4>(a.B.rec, cell_k0, cell_pref, nrows, 0, min(SL, total), raw, bs);
    // this thread's items
    int item_cell[W::IPT], item_ix[W::IPT], item_iy[W::IPT], item_tl[W::IPT];
    int item_tx[W::IPT], item_ty[W::IPT];
    bool item_ok[W::IPT];
    // window of WIN z nodes per item: (m, m vx), (m vy, m vz), (fx, fy), fz
    float2 wa[W::IPT][WIN], wb[W::IPT][WIN], wc[W::IPT][WIN];
    float wz[W::IPT][WIN];
#pragma unroll
    for (int q = 0; q < W::IPT; q++) {
      const int it = (round * W::IPT + q) * NT + tid;
      const bool in = it < nitems;
      const int px = in ? pairs_x[it % nx] : 0;
      const int py = in ? pairs_y[it / nx] : 0;
      item_ok[q] = in && pair_valid(px) && pair_valid(py);
      item_cell[q] = pair_src(py) * W::NS + pair_src(px);
      item_ix[q] = pair_off(px);
      item_iy[q] = pair_off(py);
      item_tx[q] = pair_tgt(px);
      item_ty[q] = pair_tgt(py);
      item_tl[q] = item_tx[q] + T::X * item_ty[q];
#pragma unroll
      for (int k = 0; k < WIN; k++) {
        wa[q][k] = wb[q][k] = wc[q][k] = make_float2(0.0f, 0.0f);
        wz[q][k] = 0.0f;
      }
    }
    // Window node k of item q into the node accumulators at layer lz.  Called
    // by every thread of the CTA at the same point.  Linear and cubic: the
    // WIN lanes of one target column (neighbours, target-major pairs) sum
    // their values with shuffles and one of them adds them: WIN times fewer
    // shared-memory atomics, none colliding inside a warp.  Quadratic (its
    // folded pairs are not target-major): one atomic per item.
    constexpr bool REDUCE = SF != PMPM_SHAPE_QUADRATIC && W::IPT == 1;
    auto add_node = [&](int q, int k, int lz) {
      float v[7] = {wa[q][k].x, wa[q][k].y, wb[q][k].x, wb[q][k].y, wc[q][k].x, wc[q][k].y, wz[q][k]};
      if (REDUCE) {
#pragma unroll
        for (int c = 0; c < 7; c++) {
#pragma unroll
          for (int o = 1; o < WIN; o <<= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
        }
        if ((threadIdx.x & (WIN - 1)) != 0) return;
      }
      if (!item_ok[q]) return;
      const int ln = item_tl[q] + T::X * T::Y * lz;
#pragma unroll
      for (int c = 0; c < 7; c++) atomicAdd(&acc[c * NN + ln], v[c]);
    };
    // ---- the lowest window node of layer L is complete: flush, shift ----
    auto flush_shift = [&](int L) {
#pragma unroll
      for (int q = 0; q < W::IPT; q++) {
        {
          int tz = cz_lo + L + W::LO;
          if (SF == PMPM_SHAPE_QUADRATIC) tz = min(max(tz, 0), g.n[2] - 1);
          const int lz = tz - t0[2];
          if (lz >= 0 && lz < TZ && tz < g.n[2]) add_node(q, 0, lz);
        }
#pragma unroll
        for (int k = 0; k < WIN - 1; k++) {
          wa[q][k] = wa[q][k + 1];
          wb[q][k] = wb[q][k + 1];
          wc[q][k] = wc[q][k + 1];
          wz[q][k] = wz[q][k + 1];
        }
        wa[q][WIN - 1] = wb[q][WIN - 1] = wc[q][WIN - 1] = make_float2(0.0f, 0.0f);
        wz[q][WIN - 1] = 0.0f;
      }
    };
    // The unit's particles, all layers in z order, are positions
    // 0 .. total of the table; they are staged in pieces of SL positions
    // regardless of layer boundaries.  A piece's records arrive by bulk copy
    // (issued while the previous piece's items ran), are turned into
    // weights here, and the next piece's copies and table cells are started
    // before this piece's items run.
    int pf_lo[R], pf_s[R];
    int L = 0;  // layer whose particles the items add next
    for (int p0 = 0; p0 < total; p0 += SL) {
      const int p1 = min(p0 + SL, total);
      if (BULK) {
        mbar_wait(bs, phase, a.fault);
        phase ^= 1u;
      }
#pragma unroll
      for (int r = 0; r < R; r++) {
        const int j = p0 + tid + r * NT;
        if (j < p1) {
          const int lo = p0 > 0 ? pf_lo[r] : locate(j);
          if (BULK) {
            stage_one(lo, raw + (size_t)(j - p0) * R4, sweep_slot(j - p0));
          } else {
            float4 rc[5];
            make_record<SF, false, PLANAR>(a, p0 > 0 ? pf_s[r] : slot_of(j, lo), rc);
            stage_one(lo, rc, sweep_slot(j - p0));
          }
        }
      }
      __syncthreads();
      if (p1 < total) {
        const int n1 = min(p1 + SL, total);
        if (BULK) issue_piece<W::NS, R4>(a.B.rec, cell_k0, cell_pref, nrows, p1, n1, raw, bs);
#pragma unroll
        for (int r = 0; r < R; r++) {
          const int j = p1 + tid + r * NT;
          if (j < n1) {
            pf_lo[r] = locate(j);
            if (!BULK) pf_s[r] = slot_of(j, pf_lo[r]);
          }
        }
      }
      // ---- items: layers with particles before p1 add their part of the
      // piece; layers that end in it (empty ones included) are complete ----
      while (L < nlayers) {
        const int ls = cell_pref[L * W::NCELL], le = cell_pref[(L + 1) * W::NCELL];
        if (ls < p1) {
          const int *pref = cell_pref + L * W::NCELL;
#pragma unroll
          for (int q = 0; q < W::IPT; q++) {
            if (!item_ok[q]) continue;
            const int vc = item_cell[q];
            const int j0 = max(pref[vc], p0) - p0, j1 = min(pref[vc + 1], p1) - p0;
            const float2 *wxp = st_wx[item_ix[q]], *wyp = st_wy[item_iy[q]];
            auto add = [&](int jp) {
              const int j = sweep_slot(jp);
              const float2 wx = wxp[j], wy = wyp[j];
              const float4 pm = st_p[j], s0 = st_s0[j], s1 = st_s1[j];
              float zf[4 * W::NZ4];
#pragma unroll
              for (int k = 0; k < W::NZ4; k++) {
                const float4 z4 = st_z[k][j];
                zf[4 * k] = z4.x;
                zf[4 * k + 1] = z4.y;
                zf[4 * k + 2] = z4.z;
                zf[4 * k + 3] = z4.w;
              }
              const float nn = wx.x * wy.x;
              const float gx = wx.y * wy.x, gy = wx.x * wy.y;
              const float2 nn2 = make_float2(nn, nn);
              // f_c = Nz (f_ext,c nn + S_c0 gx + S_c1 gy) + dNz (S_c2 nn); x and
              // y components in packed FP32 pairs
              float2 A = __ffma2_rn(make_float2(s0.z, s0.w), make_float2(gy, gy),
                                    __fmul2_rn(make_float2(s0.x, s0.y), make_float2(gx, gx)));
              float Az = fmaf(s1.y, gy, s1.x * gx);
              if (PLANAR) {
                const float4 fe = st_f[j];
                A = __ffma2_rn(make_float2(fe.x, fe.y), nn2, A);
                Az = fmaf(fe.z, nn, Az);
              }
              const float2 B = __fmul2_rn(make_float2(s1.x, s1.y), nn2);
              const float Bz = s1.z * nn;
              const float2 mm = __fmul2_rn(make_float2(pm.x, pm.y), nn2), mv = __fmul2_rn(make_float2(pm.z, pm.w), nn2);
#pragma unroll
              for (int k = 0; k < WIN; k++) {
                const float Nz = zf[k], dNz = zf[WIN + k];
                const float2 n2 = make_float2(Nz, Nz), d2 = make_float2(dNz, dNz);
                wa[q][k] = __ffma2_rn(mm, n2, wa[q][k]);
                wb[q][k] = __ffma2_rn(mv, n2, wb[q][k]);
                wc[q][k] = __ffma2_rn(B, d2, __ffma2_rn(A, n2, wc[q][k]));
                wz[q][k] = fmaf(Bz, dNz, fmaf(Az, Nz, wz[q][k]));
              }
            };
            int j = j0;
            for (; j + 1 < j1; j += 2) {
              add(j);
              add(j + 1);
            }
            if (j < j1) add(j);
          }
        }
        if (le > p1) break;  // the layer goes on in the next piece
        flush_shift(L);
        L++;
      }
      __syncthreads();
    }
    for (; L < nlayers; L++) flush_shift(L);  // layers after the last particle
    // ---- remaining window nodes after the last layer ----
#pragma unroll
    for (int q = 0; q < W::IPT; q++) {
#pragma unroll
      for (int k = 0; k < WIN - 1; k++) {
        int tz = cz_hi + 1 + k + W::LO;
        if (SF == PMPM_SHAPE_QUADRATIC) tz = min(max(tz, 0), g.n[2] - 1);
        const int lz = tz - t0[2];
        if (lz >= 0 && lz < TZ && tz < g.n[2]) add_node(q, k, lz);
      }
    }
  }
  __syncthreads();

  // ---- node epilogue (two nodes per thread) ----
  for (int ln = tid; ln < NN; ln += NT) {
    const int lx = ln % T::X, ly = (ln / T::X) % T::Y, lz = ln / (T::X * T::Y);
    const int nc[3] = {t0[0] + lx, t0[1] + ly, t0[2] + lz};
    if (nc[0] >= g.n[0] || nc[1] >= g.n[1] || nc[2] >= g.n[2]) continue;
    const int node = flat_index(g, nc[0], nc[1], nc[2]);
    float mass = acc[ln];
    float p[3] = {0.0f, 0.0f, 0.0f}, pnt[3] = {0.0f, 0.0f, 0.0f};
    const bool live = mass > a.cutoff;
    if (live) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        p[c] = acc[(1 + c) * NN + ln];
        pnt[c] = p[c] + acc[(4 + c) * NN + ln] * a.dt;
      }
    } else {
      mass = 0.0f;
    }
    if (apply_bcs) node_bcs<3>(a, node, nc, mass, p, pnt);
    write_node<3>(a, node, mass, p, pnt, live);
  }
}

// One persistent CTA pass over the active-tile queue (grid: 1 CTA per SM).
template <int SF, bool PLANAR, bool BULK>
__global__ void __launch_bounds__(Sweep3<SF>::NT, 1) k_p2g_sweep3(StepArgs a, int apply_bcs, int *node_epoch) {
  __shared__ int cur;
  __shared__ BulkState bs;
  if (blockIdx.x == 0 && threadIdx.x == 0) a.N.tile_queue[2 + (a.p2g_par ^ 1)] = 0;  // the next launch's counter
  if (binning_failed_cta(a.fault)) return;
  if (threadIdx.x == 0) bulk_init(&bs);
  __syncthreads();
  unsigned phase = 0;
  for (int unit = next_tile(a, &cur); unit >= 0; unit = next_tile(a, &cur))
    sweep3_tile<SF, PLANAR, BULK>(a, apply_bcs, node_epoch, unit, &bs, phase);
}

// --------------------------------------------------------------------------
// P2G, 3D quadratic fast path: dual-cell z-sweep
// --------------------------------------------------------------------------
//
// Particles are binned by dual cell d = floor(x/h + 1/2), so every particle
// of a dual cell has the same three nodes d - 1 .. d + 1 per axis (clamped
// onto the grid: the boundary fold of the quadratic spline) and every
// (particle, node) pair the sweep visits carries weight.  Work item = (x
// pair, y pair), a pair being (dual source column, node offset 0..2) whose
// target lies in the tile; items sweep the dual layers along z with a
// three-node register window, as k_p2g_sweep3.  One CTA of 20 warps per SM
// (one item per thread) stages the tile's particles, all layers in z order,
// in pieces of up to 1,872 regardless of layer boundaries (two barriers per
// piece), and finds the next piece's storage slots while the items run.

struct Dual3 {
  using T = TileDims<3>;
  static constexpr int NS = T::X + 2;   // dual sources per axis
  static constexpr int MAXPAIR = NS * 3;
  static constexpr int NCELL = NS * NS;
  static constexpr int NL = T::Z + 2;   // dual layers a tile reads
  static constexpr int NT = 640;        // threads (20 warps), one CTA per SM
  static constexpr int IPT = 1;         // items per thread
  // staged bytes per particle: the x and y weights of the three offsets
  // (float2 N, dN each), float4 (m, m vx, m vy, m vz), float4 (Sxx, Sxy,
  // Sxy, Syy), float4 (Sxz, Syz, Szz, Nz2), float4 (Nz0, Nz1, dNz0, dNz1),
  // with a PlanarDomain float4 (f, 0); S = -V sigma
  __host__ __device__ static constexpr int slot_bytes(bool planar) { return 6 * 8 + 4 * 16 + (planar ? 16 : 0); }
  // float4s of one P2G record (k_records), bulk-copied per row of dual cells
  __host__ __device__ static constexpr int rec4(bool planar) { return planar ? 5 : 4; }
  static constexpr int NROWS = NL * NS;  // rows of dual cells along x
  // staged particles and their records: 227 KB of shared memory per CTA,
  // less the static tables (with the copy barrier) and the node accumulators
  static constexpr int STATIC_BYTES = 8704;
  __host__ __device__ static constexpr int cap(bool planar, bool bulk) {
    return ((232448 - STATIC_BYTES - 7 * T::N * 4) / (slot_bytes(planar) + (bulk ? 16 * rec4(planar) : 0))) & ~7;
  }
};

template <bool PLANAR, bool BULK>
constexpr int dual3_smem_bytes() {
  return 7 * TileDims<3>::N * 4 +
         Dual3::cap(PLANAR, BULK) * (Dual3::slot_bytes(PLANAR) + (BULK ? 16 * Dual3::rec4(PLANAR) : 0));
}

// Staged slot of chunk position j: an XOR swizzle inside aligned groups of
// eight, so lanes reading the same position of neighbouring cells (runs of
// about eight) hit different shared-memory banks with 8- and 16-byte loads.
__device__ __forceinline__ int dual_slot(int j) { return j ^ ((j >> 3) & 7); }

__device__ __forceinline__ int build_dual_pairs(int t0, int n, int *pairs) {
  int cnt = 0;
  for (int si = 0; si < Dual3::NS; si++) {
    const int src = t0 - 1 + si;
    if (src < 0 || src > n) continue;  // dual coordinates run 0 .. n
    for (int i = 0; i < 3; i++) {
      const int t = min(max(src - 1 + i, 0), n - 1);
      const int l = t - t0;
      if (l < 0 || l >= TileDims<3>::X) continue;
      pairs[cnt++] = si | (i << 8) | (l << 12);
    }
  }
  return cnt;
}

// Node epilogue for the nodes of a tile from shared accumulators acc[7][512]:
// the reference leaves nodes with m <= cutoff at their reset value (0).
__device__ __forceinline__ void tile_epilogue3(const StepArgs &a, int apply_bcs, const int t0[3], const float *acc,
                                               int tid, int nthreads) {
  using T = TileDims<3>;
  const DevGrid &g = a.g;
  for (int ln = tid; ln < T::N; ln += nthreads) {
    const int lx = ln % T::X, ly = (ln / T::X) % T::Y, lz = ln / (T::X * T::Y);
    const int nc[3] = {t0[0] + lx, t0[1] + ly, t0[2] + lz};
    if (nc[0] >= g.n[0] || nc[1] >= g.n[1] || nc[2] >= g.n[2]) continue;
    const int node = flat_index(g, nc[0], nc[1], nc[2]);
    float mass = acc[ln];
    float p[3] = {0.0f, 0.0f, 0.0f}, pnt[3] = {0.0f, 0.0f, 0.0f};
    const bool live = mass > a.cutoff;
    if (live) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        p[c] = acc[(1 + c) * T::N + ln];
        pnt[c] = p[c] + acc[(4 + c) * T::N + ln] * a.dt;
      }
    } else {
      mass = 0.0f;
    }
    if (apply_bcs) node_bcs<3>(a, node, nc, mass, p, pnt);
    write_node<3>(a, node, mass, p, pnt, live);
  }
}

// PLANAR: the handle has a PlanarDomain (per-particle external forces to map)
// BULK: a piece's particles arrive as sorted records by bulk copy (k_records
// wrote them); otherwise each is gathered through the sorted order.
// bs / phase: the CTA's copy state and the parity of its barrier's next phase
template <bool PLANAR, bool BULK>
__device__ __forceinline__ void dual3_tile(const StepArgs &a, int apply_bcs, int *node_epoch, int tile,
                                           BulkState *bs, unsigned &phase) {
  using W = Dual3;
  using T = TileDims<3>;
  constexpr int NT = W::NT;
  constexpr int NN = T::N;  // nodes per tile
  constexpr int CAP = W::cap(PLANAR, BULK);
  constexpr int R4 = W::rec4(PLANAR);
  const DevGrid &g = a.g;

  __shared__ int pairs_x[W::MAXPAIR], pairs_y[W::MAXPAIR];
  __shared__ int npair[2];
  // every layer's source cells: first sorted position and running prefix
  __shared__ int cell_k0[W::NL * W::NCELL], cell_pref[W::NL * W::NCELL + 1];
  __shared__ int warp_tmp[33];
  extern __shared__ __align__(16) float dyn_smem[];
  float *acc = dyn_smem;                                           // [7][NN]
  float2(*st_wx)[CAP] = (float2(*)[CAP])(acc + 7 * NN);            // [3] x weights (N, dN) per offset
  float2(*st_wy)[CAP] = st_wx + 3;                                 // [3]
  float4 *st_p = (float4 *)(st_wy + 3);                            // (m, m v)
  float4 *st_s0 = st_p + CAP;                                      // (Sxx, Sxy, Sxy, Syy)
  float4 *st_s1 = st_s0 + CAP;                                     // (Sxz, Syz, Szz, Nz2)
  float4 *st_z = st_s1 + CAP;                                      // (Nz0, Nz1, dNz0, dNz1)
  float4 *st_f = st_z + CAP;                                       // PLANAR: (f, 0)
  float4 *raw = (float4 *)((char *)acc + 7 * NN * 4 + CAP * W::slot_bytes(PLANAR));  // BULK: [CAP][R4] records

  const int tid = threadIdx.x;
  const int t0[3] = {(tile % g.tdim[0]) * T::X, ((tile / g.tdim[0]) % g.tdim[1]) * T::Y,
                     (tile / (g.tdim[0] * g.tdim[1])) * T::Z};
  for (int k = tid; k < 7 * NN; k += NT) acc[k] = 0.0f;
  if (tid == 0) {
    node_epoch[tile] = a.epoch;
    npair[0] = build_dual_pairs(t0[0], g.n[0], pairs_x);
  } else if (tid == 32) {
    npair[1] = build_dual_pairs(t0[1], g.n[1], pairs_y);
  }
  __syncthreads();
  const int nx = npair[0], ny = npair[1];
  const int nitems = nx * ny;
  const int dz_lo = max(t0[2] - 1, 0), dz_hi = min(t0[2] + T::Z, g.n[2]);
  const int kd0 = a.B.kd[0];
  const long long kd01 = (long long)a.B.kd[0] * a.B.kd[1];

  // ---- all layers' dual source cells -> sorted ranges, one prefix ----
  const int ntab = (dz_hi - dz_lo + 1) * W::NCELL;
  {
    constexpr int PER = (W::NL * W::NCELL + NT - 1) / NT;
    int cnt[PER];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < PER; k++) {
      const int idx = tid * PER + k;
      cnt[k] = 0;
      if (idx < ntab) {
        const int layer = idx / W::NCELL, vc = idx % W::NCELL;
        const int sx = t0[0] - 1 + vc % W::NS, sy = t0[1] - 1 + vc / W::NS;
        int k0 = 0;
        if (sx >= 0 && sx <= g.n[0] && sy >= 0 && sy <= g.n[1]) {
          const long long f = sx + (long long)sy * kd0 + (long long)(dz_lo + layer) * kd01;
          k0 = a.B.offset[f];
          cnt[k] = a.B.offset[f + 1] - k0;
        }
        cell_k0[idx] = k0;
        sum += cnt[k];
      }
    }
    int total;
    int ex = block_exclusive_scan(sum, warp_tmp, total);
#pragma unroll
    for (int k = 0; k < PER; k++) {
      const int idx = tid * PER + k;
      if (idx < ntab) cell_pref[idx] = ex;
      ex += cnt[k];
    }
    if (tid == 0) cell_pref[ntab] = total;
  }
  __syncthreads();

  // one round of items covers a tile of up to 24 pairs per axis; grids whose
  // face tiles have 27 (a node count divisible by 8 along x or y) run the
  // cell-row scatter instead (the host's dual_pairs_max)
  static_assert(T::X * 3 * T::Y * 3 <= NT * W::IPT, "one round of items covers a tile");
  int item_cell[W::IPT], item_tl[W::IPT], item_ix[W::IPT], item_iy[W::IPT];
  bool item_ok[W::IPT];
  // window of three z nodes per item: (m, m vx), (m vy, m vz), (fx, fy), fz
  float2 wa[W::IPT][3], wb[W::IPT][3], wc[W::IPT][3];
  float wz[W::IPT][3];
#pragma unroll
  for (int q = 0; q < W::IPT; q++) {
    const int it = q * NT + tid;
    item_ok[q] = it < nitems;
    const int px = item_ok[q] ? pairs_x[it % nx] : 0;
    const int py = item_ok[q] ? pairs_y[it / nx] : 0;
    item_cell[q] = pair_src(py) * W::NS + pair_src(px);
    item_tl[q] = pair_tgt(px) + T::X * pair_tgt(py);
    item_ix[q] = pair_off(px);
    item_iy[q] = pair_off(py);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      wa[q][k] = wb[q][k] = wc[q][k] = make_float2(0.0f, 0.0f);
      wz[q][k] = 0.0f;
    }
  }

  // The tile's particles, all layers in z order, are positions
  // 0 .. cell_pref[ntab] of the table; they are staged in pieces of CAP
  // positions regardless of layer boundaries.  Table cell of position j:
  auto locate = [&](int j) {
    int lo = 0, hi = ntab;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (cell_pref[mid] <= j) lo = mid; else hi = mid;
    }
    return lo;
  };
  // ---- node dz_lo + L - 1 gets nothing from layers after L: flush, shift ----
  auto flush_shift = [&](int L) {
#pragma unroll
    for (int q = 0; q < W::IPT; q++) {
      if (item_ok[q]) {
        const int tz = max(dz_lo + L - 1, 0);
        const int lz = tz - t0[2];
        if (lz >= 0 && lz < T::Z && tz < g.n[2]) {
          const int ln = item_tl[q] + T::X * T::Y * lz;
          atomicAdd(&acc[ln], wa[q][0].x);
          atomicAdd(&acc[NN + ln], wa[q][0].y);
          atomicAdd(&acc[2 * NN + ln], wb[q][0].x);
          atomicAdd(&acc[3 * NN + ln], wb[q][0].y);
          atomicAdd(&acc[4 * NN + ln], wc[q][0].x);
          atomicAdd(&acc[5 * NN + ln], wc[q][0].y);
          atomicAdd(&acc[6 * NN + ln], wz[q][0]);
        }
      }
#pragma unroll
      for (int k = 0; k < 2; k++) {
        wa[q][k] = wa[q][k + 1];
        wb[q][k] = wb[q][k + 1];
        wc[q][k] = wc[q][k + 1];
        wz[q][k] = wz[q][k + 1];
      }
      wa[q][2] = wb[q][2] = wc[q][2] = make_float2(0.0f, 0.0f);
      wz[q][2] = 0.0f;
    }
  };

  const int nlayers = dz_hi - dz_lo + 1;
  const int total = cell_pref[ntab];
  const int nrows = nlayers * W::NS;
  // table cells of positions tid + r NT of the next piece, found while the
  // current piece's items run; the next piece's records are copied in then
  constexpr int R = (CAP + NT - 1) / NT;
  int pf_lo[R], pf_s[R];
  // storage slot of list position j (table cell lo), for the gathered staging
  auto slot_of = [&](int j, int lo) { return a.B.order[cell_k0[lo] + (j - cell_pref[lo])]; };
  int L = 0;  // layer whose particles the items add next
  if (BULK && total > 0)
    issue_piece<W::NS, R4>(a.B.rec, cell_k0, cell_pref, nrows, 0, min(CAP, total), raw, bs);
  for (int p0 = 0; p0 < total; p0 += CAP) {
    const int p1 = min(p0 + CAP, total);
    if (BULK) {
      mbar_wait(bs, phase, a.fault);
      phase ^= 1u;
    }
    // ---- stage positions [p0, p1) from their records ----
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int j = p0 + tid + r * NT;
      if (j < p1) {
        const int lo = p0 > 0 ? pf_lo[r] : locate(j);
        float4 own[5];
        const float4 *rc = own;
        if (BULK)
          rc = raw + (size_t)(j - p0) * R4;
        else
          make_record<PMPM_SHAPE_QUADRATIC, true, PLANAR>(a, p0 > 0 ? pf_s[r] : slot_of(j, lo), own);
        const int jj = dual_slot(j - p0);
        // the particle's dual cell: its nodes are d - 1 .. d + 1 per axis
        const int layer = lo / W::NCELL, vc = lo - layer * W::NCELL;
        const int dz = dz_lo + layer;
        const int sx = t0[0] - 1 + vc % W::NS, sy = t0[1] - 1 + vc / W::NS;
        const float4 xp = rc[3];
        const float ux = scaled_coord(xp.x, g.origin[0], g.inv_h);
        const float uy = scaled_coord(xp.y, g.origin[1], g.inv_h);
        const float uz = scaled_coord(xp.z, g.origin[2], g.inv_h);
#pragma unroll
        for (int i = 0; i < 3; i++) {
          float N, dN;
          axis_weight<PMPM_SHAPE_QUADRATIC>(ux - (float)(sx - 1 + i), g.inv_h, 0, N, dN);
          st_wx[i][jj] = make_float2(N, dN);
          axis_weight<PMPM_SHAPE_QUADRATIC>(uy - (float)(sy - 1 + i), g.inv_h, 0, N, dN);
          st_wy[i][jj] = make_float2(N, dN);
        }
        float Nz[3], dNz[3];
#pragma unroll
        for (int k = 0; k < 3; k++) axis_weight<PMPM_SHAPE_QUADRATIC>(uz - (float)(dz - 1 + k), g.inv_h, 0, Nz[k], dNz[k]);
        // (m, m v), -V sigma as (xx, xy, xy, yy) (xz, yz, zz, -), f_ext: k_records
        st_p[jj] = rc[0];
        st_s0[jj] = rc[1];
        const float4 s1 = rc[2];
        st_s1[jj] = make_float4(s1.x, s1.y, s1.z, Nz[2]);
        st_z[jj] = make_float4(Nz[0], Nz[1], dNz[0], dNz[1]);
        if (PLANAR) st_f[jj] = rc[4];
      }
    }
    __syncthreads();
    if (p1 < total) {
      const int n1 = min(p1 + CAP, total);
      if (BULK) issue_piece<W::NS, R4>(a.B.rec, cell_k0, cell_pref, nrows, p1, n1, raw, bs);
#pragma unroll
      for (int r = 0; r < R; r++) {
        const int j = p1 + tid + r * NT;
        if (j < n1) {
          pf_lo[r] = locate(j);
          if (!BULK) pf_s[r] = slot_of(j, pf_lo[r]);
        }
      }
    }
    // ---- items: layers with particles before p1 add their part of the piece;
    // layers that end in it (empty ones included) are complete ----
    while (L < nlayers) {
      const int ls = cell_pref[L * W::NCELL], le = cell_pref[(L + 1) * W::NCELL];
      if (ls < p1) {
        const int *pref = cell_pref + L * W::NCELL;
#pragma unroll
        for (int q = 0; q < W::IPT; q++) {
          if (!item_ok[q]) continue;
          const int vc = item_cell[q];
          const int j0 = max(pref[vc], p0) - p0, j1 = min(pref[vc + 1], p1) - p0;
          const float2 *wxp = st_wx[item_ix[q]], *wyp = st_wy[item_iy[q]];
          auto add = [&](int jp) {
            const int j = dual_slot(jp);
            const float2 wx = wxp[j], wy = wyp[j];
            const float4 pm = st_p[j], s0 = st_s0[j], s1 = st_s1[j], zw = st_z[j];
            const float nn = wx.x * wy.x, gx = wx.y * wy.x, gy = wx.x * wy.y;
            const float2 nn2 = make_float2(nn, nn), gx2 = make_float2(gx, gx), gy2 = make_float2(gy, gy);
            const float2 mm = __fmul2_rn(make_float2(pm.x, pm.y), nn2);
            const float2 mv = __fmul2_rn(make_float2(pm.z, pm.w), nn2);
            // f = Nz (f_ext nn + S_c0 gx + S_c1 gy) + dNz (S_c2 nn)
            float2 A = __ffma2_rn(make_float2(s0.z, s0.w), gy2, __fmul2_rn(make_float2(s0.x, s0.y), gx2));
            float Az = fmaf(s1.y, gy, s1.x * gx);
            if (PLANAR) {
              const float4 fe = st_f[j];
              A = __ffma2_rn(make_float2(fe.x, fe.y), nn2, A);
              Az = fmaf(fe.z, nn, Az);
            }
            const float2 B = __fmul2_rn(make_float2(s1.x, s1.y), nn2);
            const float Bz = s1.z * nn;
            const float Nz[3] = {zw.x, zw.y, s1.w};
            const float dNz[3] = {zw.z, zw.w, -zw.z - zw.w};  // the three derivatives sum to zero
#pragma unroll
            for (int k = 0; k < 3; k++) {
              const float2 n2 = make_float2(Nz[k], Nz[k]), d2 = make_float2(dNz[k], dNz[k]);
              wa[q][k] = __ffma2_rn(mm, n2, wa[q][k]);
              wb[q][k] = __ffma2_rn(mv, n2, wb[q][k]);
              wc[q][k] = __ffma2_rn(B, d2, __ffma2_rn(A, n2, wc[q][k]));
              wz[q][k] = fmaf(Bz, dNz[k], fmaf(Az, Nz[k], wz[q][k]));
            }
          };
          // four particles per pass: their shared-memory loads overlap the arithmetic
          int j = j0;
          for (; j + 3 < j1; j += 4) {
            add(j);
            add(j + 1);
            add(j + 2);
            add(j + 3);
          }
          for (; j < j1; j++) add(j);
        }
      }
      if (le > p1) break;  // the layer goes on in the next piece
      flush_shift(L);
      L++;
    }
    __syncthreads();
  }
  for (; L < nlayers; L++) flush_shift(L);  // layers after the last particle
#pragma unroll
  for (int q = 0; q < W::IPT; q++) {
    if (!item_ok[q]) continue;
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const int tz = min(dz_hi + k, g.n[2] - 1);
      const int lz = tz - t0[2];
      if (lz >= 0 && lz < T::Z) {
        const int ln = item_tl[q] + T::X * T::Y * lz;
        atomicAdd(&acc[ln], wa[q][k].x);
        atomicAdd(&acc[NN + ln], wa[q][k].y);
        atomicAdd(&acc[2 * NN + ln], wb[q][k].x);
        atomicAdd(&acc[3 * NN + ln], wb[q][k].y);
        atomicAdd(&acc[4 * NN + ln], wc[q][k].x);
        atomicAdd(&acc[5 * NN + ln], wc[q][k].y);
        atomicAdd(&acc[6 * NN + ln], wz[q][k]);
      }
    }
  }
  __syncthreads();
  tile_epilogue3(a, apply_bcs, t0, acc, tid, NT);
}
// One persistent CTA pass over the active-tile queue (grid: 1 CTA per SM).
template <bool PLANAR, bool BULK>
__global__ void __launch_bounds__(Dual3::NT, 1) k_p2g_dual3(StepArgs a, int apply_bcs, int *node_epoch) {
  __shared__ int cur;
  __shared__ BulkState bs;
  if (blockIdx.x == 0 && threadIdx.x == 0) a.N.tile_queue[2 + (a.p2g_par ^ 1)] = 0;  // the next launch's counter
  if (binning_failed_cta(a.fault)) return;
  if (threadIdx.x == 0) bulk_init(&bs);
  __syncthreads();
  unsigned phase = 0;
  for (int tile = next_tile(a, &cur); tile >= 0; tile = next_tile(a, &cur))
    dual3_tile<PLANAR, BULK>(a, apply_bcs, node_epoch, tile, &bs, phase);
}

// --------------------------------------------------------------------------
// P2G, 3D quadratic: warp per row of dual cells, scatter into brick boxes
// --------------------------------------------------------------------------
//
// All particles of dual cell d reach the same 27 nodes d-1 .. d+1 (clamped
// onto the grid).  One CTA per brick of 8^3 dual cells that holds particles.
// A warp takes a row of 8 cells along x (consecutive keys, so the row's
// particles are one contiguous sorted range), stages them in its own
// shared-memory area (per-axis weights and derivatives, m, m v, -V sigma,
// f_ext; up to 64 at a time), then sums three cells at a time: lane
// (cell, i, j) adds the cell's particles to the three nodes
// d - 1 + (i, j, 0..2) in registers, reading the staged values as
// near-broadcasts.  The sums go into the brick's shared 10^3-node box, which
// is added once per node to the global accumulators; the node epilogue
// (k_node_epilogue) finishes the nodes and clears the accumulators.  No
// block barrier inside the row loop.
struct Cells3 {
  static constexpr int NW = 8;      // warps per CTA
  static constexpr int NT = NW * 32;
  static constexpr int B = 8;       // brick edge (dual cells)
  static constexpr int BOX = B + 2; // node box edge
  static constexpr int NBOX = BOX * BOX * BOX;
  static constexpr int NF = 31;     // staged floats per particle
  static constexpr int CAPW = 64;   // staged particles per warp
};

constexpr int cells3_smem_bytes() { return (7 * Cells3::NBOX + Cells3::NW * Cells3::NF * Cells3::CAPW) * 4; }

__global__ void __launch_bounds__(Cells3::NT, 2) k_p2g_cells3(StepArgs a) {
  using W = Cells3;
  const DevGrid &g = a.g;
  const int brick = blockIdx.x;
  if (a.B.brick_epoch[brick] != a.epoch || binning_failed(a.fault)) return;
  extern __shared__ __align__(16) float csm[];
  float *box = csm;  // [7][NBOX]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float(*stg)[W::CAPW] = (float(*)[W::CAPW])(box + 7 * W::NBOX + warp * W::NF * W::CAPW);  // [NF][CAPW]
  for (int k = threadIdx.x; k < 7 * W::NBOX; k += W::NT) box[k] = 0.0f;
  const int kb0 = a.B.kb[0], kb1 = a.B.kb[1];
  const int b0[3] = {(brick % kb0) * W::B, ((brick / kb0) % kb1) * W::B, (brick / (kb0 * kb1)) * W::B};
  __syncthreads();
  const DevParticles &P = a.P;
  const int st = P.stride;
  const int kd0 = a.B.kd[0];
  const long long kd01 = (long long)a.B.kd[0] * a.B.kd[1];
  const int ncx = min(W::B, kd0 - b0[0]);  // cells of the brick along x
  const int lc = lane / 9, lij = lane % 9, li = lij % 3, lj = lij / 3;
  const bool has_f = a.has_planar && !a.remap;
  for (int row = warp; row < W::B * W::B; row += W::NW) {
    const int dy = b0[1] + row % W::B, dz = b0[2] + row / W::B;
    if (dy >= a.B.kd[1] || dz >= a.B.kd[2]) continue;
    const long long key0 = b0[0] + (long long)dy * kd0 + (long long)dz * kd01;
    const int offv = lane <= ncx ? a.B.offset[key0 + lane] : 0;  // lane c: start of cell c
    const int rs = __shfl_sync(0xffffffffu, offv, 0), re = __shfl_sync(0xffffffffu, offv, ncx);
    if (rs == re) continue;
    for (int c0 = rs; c0 < re; c0 += W::CAPW) {
      const int c1 = min(c0 + W::CAPW, re);
      // ---- stage the chunk's particles ----
      for (int j = lane; j < c1 - c0; j += 32) {
        const int s = a.B.order[c0 + j];
        float u[3];
#pragma unroll
        for (int c = 0; c < 3; c++) u[c] = scaled_coord(P.x[c * st + s], g.origin[c], g.inv_h);
        const int dxc = dual_coord(u[0], (int)u[0]);
        const int dd[3] = {dxc, dy, dz};
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
          for (int i = 0; i < 3; i++) {
            float N, dN;
            axis_weight<PMPM_SHAPE_QUADRATIC>(u[c] - (float)(dd[c] - 1 + i), g.inv_h, 0, N, dN);
            stg[c * 3 + i][j] = N;
            stg[9 + c * 3 + i][j] = dN;
          }
        const float pm = P.m[s];
        stg[18][j] = pm;
#pragma unroll
        for (int c = 0; c < 3; c++) {
          stg[19 + c][j] = pm * P.v[c * st + s];
          stg[22 + c][j] = has_f ? P.fext[c * st + s] : 0.0f;
        }
        const float nv = a.remap ? 0.0f : -P.V[s];
#pragma unroll
        for (int k = 0; k < 6; k++) stg[25 + k][j] = nv * P.sig[k * st + s];
      }
      __syncwarp();
      // ---- three cells at a time: lane (cell, i, j) sums nodes (i, j, 0..2) ----
      for (int pass = 0; pass < ncx; pass += 3) {
        const int cell = pass + lc;
        const int cs_ = __shfl_sync(0xffffffffu, offv, min(cell, ncx));
        const int ce_ = __shfl_sync(0xffffffffu, offv, min(cell + 1, ncx));
        if (lane >= 27 || cell >= ncx) continue;
        const int q0 = max(cs_, c0) - c0, q1 = min(ce_, c1) - c0;
        if (q0 >= q1) continue;
        float acc[3][7];
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
          for (int c = 0; c < 7; c++) acc[k][c] = 0.0f;
        for (int q = q0; q < q1; q++) {
          const float nx = stg[li][q], ny = stg[3 + lj][q];
          const float dnx = stg[9 + li][q], dny = stg[12 + lj][q];
          const float nn = nx * ny, gx = dnx * ny, gy = nx * dny;
          const float Sxx = stg[25][q], Syy = stg[26][q], Szz = stg[27][q];
          const float Sxy = stg[28][q], Sxz = stg[29][q], Syz = stg[30][q];
          float Ax = Sxx * gx + Sxy * gy, Ay = Sxy * gx + Syy * gy, Az = Sxz * gx + Syz * gy;
          if (has_f) {
            Ax += stg[22][q] * nn;
            Ay += stg[23][q] * nn;
            Az += stg[24][q] * nn;
          }
          const float Bx = Sxz * nn, By = Syz * nn, Bz = Szz * nn;
          const float mn = stg[18][q] * nn, mvx = stg[19][q] * nn, mvy = stg[20][q] * nn, mvz = stg[21][q] * nn;
#pragma unroll
          for (int k = 0; k < 3; k++) {
            const float Nz = stg[6 + k][q], dNz = stg[15 + k][q];
            acc[k][0] += mn * Nz;
            acc[k][1] += mvx * Nz;
            acc[k][2] += mvy * Nz;
            acc[k][3] += mvz * Nz;
            acc[k][4] += Ax * Nz + Bx * dNz;
            acc[k][5] += Ay * Nz + By * dNz;
            acc[k][6] += Az * Nz + Bz * dNz;
          }
        }
        const int d0 = b0[0] + cell;
        const int nx = min(max(d0 - 1 + li, 0), g.n[0] - 1) - (b0[0] - 1);
        const int ny = min(max(dy - 1 + lj, 0), g.n[1] - 1) - (b0[1] - 1);
#pragma unroll
        for (int k = 0; k < 3; k++) {
          const int nz = min(max(dz - 1 + k, 0), g.n[2] - 1) - (b0[2] - 1);
          const int bl = nx + W::BOX * (ny + W::BOX * nz);
#pragma unroll
          for (int c = 0; c < 7; c++) atomicAdd(&box[c * W::NBOX + bl], acc[k][c]);
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();
  for (int bl = threadIdx.x; bl < W::NBOX; bl += W::NT) {
    const float m = box[bl];
    if (m == 0.0f) continue;
    const int x = b0[0] - 1 + bl % W::BOX, y = b0[1] - 1 + (bl / W::BOX) % W::BOX,
              z = b0[2] - 1 + bl / (W::BOX * W::BOX);
    if (x < 0 || y < 0 || z < 0 || x >= g.n[0] || y >= g.n[1] || z >= g.n[2]) continue;
    float *dst = a.N.acc + 8 * (size_t)flat_index(g, x, y, z);
#pragma unroll
    for (int c = 0; c < 7; c++) atomicAdd(dst + c, box[c * W::NBOX + bl]);
  }
}

// Node epilogue of the scatter P2G, one thread per node of the active tiles:
// p_nt = p + f dt for m above the cutoff (the reference leaves lighter nodes
// at 0), the node conditions, v = p/m; the accumulators are cleared.
template <int D>
__global__ void __launch_bounds__(TileDims<D>::N) k_node_epilogue(StepArgs a, int apply_bcs, int *node_epoch) {
  using T = TileDims<D>;
  const DevGrid &g = a.g;
  const int tile = blockIdx.x;
  if (a.N.tile_epoch[tile] != a.epoch) return;
  if (threadIdx.x == 0) node_epoch[tile] = a.epoch;
  const int tx = tile % g.tdim[0], ty = (tile / g.tdim[0]) % g.tdim[1], tz = tile / (g.tdim[0] * g.tdim[1]);
  const int lx = threadIdx.x % T::X, ly = (threadIdx.x / T::X) % T::Y, lz = threadIdx.x / (T::X * T::Y);
  const int nc[3] = {tx * T::X + lx, ty * T::Y + ly, D == 3 ? tz * T::Z + lz : 0};
  if (nc[0] >= g.n[0] || nc[1] >= g.n[1] || nc[2] >= g.n[2]) return;
  const int node = flat_index(g, nc[0], nc[1], nc[2]);
  float4 *ac = reinterpret_cast<float4 *>(a.N.acc + 8 * (size_t)node);
  const float4 q0 = ac[0], q1 = ac[1];
  ac[0] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  ac[1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  float mass = q0.x;
  const float mom[3] = {q0.y, q0.z, q0.w}, force[3] = {q1.x, q1.y, q1.z};
  float p[3] = {0.0f, 0.0f, 0.0f}, pnt[3] = {0.0f, 0.0f, 0.0f};
  const bool live = mass > a.cutoff;
  if (live) {
#pragma unroll
    for (int c = 0; c < D; c++) {
      p[c] = mom[c];
      pnt[c] = mom[c] + force[c] * a.dt;
    }
  } else {
    mass = 0.0f;
  }
  if (apply_bcs) node_bcs<D>(a, node, nc, mass, p, pnt);
  write_node<D>(a, node, mass, p, pnt, live);
}

// --------------------------------------------------------------------------
// G2P + deformation update + stress update
// --------------------------------------------------------------------------

template <int D>
__device__ __forceinline__ float det_rows(const float *A) {
  if (D == 2) return A[0] * A[3] - A[2] * A[1];
  const float c0 = A[4] * A[8] - A[5] * A[7];
  const float c1 = A[3] * A[8] - A[5] * A[6];
  const float c2 = A[3] * A[7] - A[4] * A[6];
  return (A[0] * c0 - A[1] * c1) + A[2] * c2;
}

// Material update of storage slot s from velocity gradient L
// (Solver::stress_update, src/solver/solver.cpp:110-121; materials by colour).
// FULL = false leaves out the iterative materials (VonMises, Modified Cam
// Clay, Drucker-Prager cap): launches whose handle holds none of them use it,
// so their FP64 Newton code does not raise the register count of the common
// kernels.
template <int D, bool FULL = true>
__device__ __forceinline__ void stress_update_point(const StepArgs &a, int s, const float *L) {
  const DevParticles &P = a.P;
  const int color = P.color[s];
  if (color >= a.nmat) return;
  const DevMaterial &mt = a.mat[color];
  if (mt.type == PMPM_MAT_NONE) return;
  if ((mt.type == PMPM_MAT_LINEAR_ELASTIC || mt.type == PMPM_MAT_NEWTON_FLUID) && !P.active[s]) return;
  const int st = P.stride;
  float S[9];
  if (mt.type == PMPM_MAT_LINEAR_ELASTIC) {
    load_sig3<D>(P, s, S);
    le_update<D>(mt, L, a.dt, S);
  } else if (mt.type == PMPM_MAT_NEWTON_FLUID) {
    nf_update<D>(mt, L, P.m[s], P.V[s], P.V0[s], S);
  } else if (mt.type == PMPM_MAT_VON_MISES) {
    if constexpr (D == 3 && FULL) {  // 3D only (rejected at create)
      float eps[9];
#pragma unroll
      for (int x = 0; x < 3; x++)
#pragma unroll
        for (int y = 0; y < 3; y++) eps[3 * x + y] = P.eps[eps_index<3>(x, y) * st + s];
      float acc = P.acc[s];
      vm_update(mt.p, L, a.dt, eps, acc, S);
#pragma unroll
      for (int x = 0; x < 3; x++)
#pragma unroll
        for (int y = x; y < 3; y++) P.eps[eps_index<3>(x, y) * st + s] = eps[3 * x + y];
      P.acc[s] = acc;
    } else {
      return;
    }
  } else if (mt.type == PMPM_MAT_MODIFIED_CAM_CLAY || mt.type == PMPM_MAT_DRUCKER_PRAGER_CAP) {
    if constexpr (FULL) {
      float eps[9], sref[9];
#pragma unroll
      for (int x = 0; x < D; x++)
#pragma unroll
        for (int y = 0; y < D; y++) eps[x * D + y] = P.eps[eps_index<D>(x, y) * st + s];
#pragma unroll
      for (int x = 0; x < 3; x++)
#pragma unroll
        for (int y = 0; y < 3; y++) {
          const int k = sig_index<D>(x, y);
          sref[3 * x + y] = (k < 0 || !a.has_sref) ? 0.0f : P.sref[k * st + s];
        }
      load_sig3<D>(P, s, S);
      float alpha = P.acc[s], pc = P.pc[s];
      if (mt.type == PMPM_MAT_MODIFIED_CAM_CLAY)
        mcc_update<D>(mt.p, L, a.dt, P.V[s], eps, sref, S, alpha, pc);
      else
        dpc_update<D>(mt.p, L, a.dt, P.V0[s], eps, sref, S, alpha, pc);
#pragma unroll
      for (int x = 0; x < D; x++)
#pragma unroll
        for (int y = x; y < D; y++) P.eps[eps_index<D>(x, y) * st + s] = eps[x * D + y];
      P.acc[s] = alpha;
      P.pc[s] = pc;
    } else {
      return;
    }
  } else {
    float eps[9], sref[9];
#pragma unroll
    for (int x = 0; x < D; x++)
#pragma unroll
      for (int y = 0; y < D; y++) eps[x * D + y] = P.eps[eps_index<D>(x, y) * st + s];
    if (a.has_sref) {
      // the reference stress uses the stress's symmetric layout
#pragma unroll
      for (int x = 0; x < 3; x++)
#pragma unroll
        for (int y = 0; y < 3; y++) {
          int k = sig_index<D>(x, y);
          sref[3 * x + y] = k < 0 ? 0.0f : P.sref[k * st + s];
        }
    } else {
#pragma unroll
      for (int k = 0; k < 9; k++) sref[k] = 0.0f;
    }
    float prm[8];
    const float *pp = mt.p;
    if (P.pE && mt.p[7] >= 0.0f) {
      dp_particle_params(mt, P.pE[s], P.pphi[s], prm);
      pp = prm;
    }
    dp_update<D>(pp, L, a.dt, eps, sref, S, false);
#pragma unroll
    for (int x = 0; x < D; x++)
#pragma unroll
      for (int y = x; y < D; y++) P.eps[eps_index<D>(x, y) * st + s] = eps[x * D + y];
  }
  store_sig3<D>(P, s, S);
}

__device__ __forceinline__ void prefetch_l2(const float *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// A 3D node's packed velocities (v, -), (v_nt, -) (32 bytes, 32-byte aligned:
// two float4 per node from a 256-byte aligned allocation) in one 256-bit
// read-only load (sm_100), where two 128-bit loads took two instructions.
__device__ __forceinline__ void ldg_node8(const float4 *p, float4 &q0, float4 &q1) {
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(q0.x), "=f"(q0.y), "=f"(q0.z), "=f"(q0.w), "=f"(q1.x), "=f"(q1.y), "=f"(q1.z), "=f"(q1.w)
      : "l"(p));
}

template <int D, int SF, bool FULL = true>
__device__ __forceinline__ void g2p_body(const StepArgs &a, int s, int do_stress, int store_L) {
  const DevParticles &P = a.P;
  const DevGrid &g = a.g;
  const int st = P.stride;
  constexpr int K = Stencil<SF>::K;
  float x[3] = {0, 0, 0}, v[3] = {0, 0, 0}, u[3] = {0, 0, 0};
  int b[3] = {0, 0, 0};
  bool inside = true;
#pragma unroll
  for (int c = 0; c < D; c++) {
    x[c] = P.x[c * st + s];
    v[c] = P.v[c * st + s];
    u[c] = scaled_coord(x[c], g.origin[c], g.inv_h);
    b[c] = (int)u[c];
    inside = inside && b[c] >= 0 && b[c] < g.n[c];
  }
  float L[9];
#pragma unroll
  for (int k = 0; k < 9; k++) L[k] = 0.0f;
  // F is loaded before the stencil gather so that its DRAM latency overlaps
  // the node loads; the cubic 3D gather instead requests it into L2 and
  // loads it after the gather (nine registers fewer while the stencil's
  // loads are in flight)
  constexpr bool F_LATE = D == 3 && SF == PMPM_SHAPE_CUBIC;
  float F[9];
  if constexpr (F_LATE) {
#pragma unroll
    for (int k = 0; k < D * D; k++) prefetch_l2(P.F + k * st + s);
  } else {
#pragma unroll
    for (int k = 0; k < D * D; k++) F[k] = P.F[k * st + s];
  }
  // 3D: the state the stress update reads after the gather is requested
  // into L2 now (no registers held), so its DRAM latency overlaps the gather
  // too (column G2P 0.104 -> 0.098 ms; the batched 2D G2P ran 6 % slower
  // with it)
  if constexpr (D == 3) {
    if (do_stress) {
#pragma unroll
      for (int k = 0; k < 6; k++) prefetch_l2(P.sig + k * st + s);
      if (P.eps) {
#pragma unroll
        for (int k = 0; k < 6; k++) prefetch_l2(P.eps + k * st + s);
      }
      if (a.has_sref) {
#pragma unroll
        for (int k = 0; k < 6; k++) prefetch_l2(P.sref + k * st + s);
      }
    }
    prefetch_l2(P.V0 + s);
  }
  if (SF != PMPM_SHAPE_QUADRATIC || inside) {
    // per-axis weights, node indices and validity
    float N[3][K], dN[3][K];
    int idx[3][K];
    bool ok[3][K];
#pragma unroll
    for (int c = 0; c < 3; c++) {
#pragma unroll
      for (int k = 0; k < K; k++) {
        N[c][k] = 1.0f;
        dN[c][k] = 0.0f;
        idx[c][k] = 0;
        ok[c][k] = true;
      }
    }
#pragma unroll
    for (int c = 0; c < D; c++) {
      int w0 = Stencil<SF>::WLO;
      if (SF == PMPM_SHAPE_QUADRATIC) w0 = (u[c] - (float)(b[c] - 1)) < 1.5f ? -1 : 0;
      if (SF == PMPM_SHAPE_CUBIC && b[c] - 1 >= 2 && b[c] + 2 <= g.n[c] - 2) {
        // four interior nodes (type 3): the four weights together
        cubic_interior_weights(u[c] - (float)b[c], g.inv_h, N[c], dN[c]);
#pragma unroll
        for (int k = 0; k < K; k++) {
          idx[c][k] = b[c] - 1 + k;
          ok[c][k] = true;
        }
        continue;
      }
#pragma unroll
      for (int k = 0; k < K; k++) {
        const int sel = b[c] + w0 + k;
        const float rel = u[c] - (float)sel;
        const bool in = sel >= 0 && sel < g.n[c];
        const int type = SF == PMPM_SHAPE_CUBIC ? cubic_node_type(sel, g.n[c]) : 0;
        axis_weight<SF>(rel, g.inv_h, in ? type : 0, N[c][k], dN[c][k]);
        if (SF == PMPM_SHAPE_QUADRATIC) {
          idx[c][k] = min(max(sel, 0), g.n[c] - 1);
          ok[c][k] = true;
        } else {
          idx[c][k] = sel;
          ok[c][k] = in;
        }
      }
    }
    // 3D: the x and y components in packed FP32 pairs (cubic G2P on the bed
    // 0.883 -> 0.783 ms); 2D keeps one FMA per component (the packed form
    // ran the batched 2D G2P 14 % slower)
    float vinc[3] = {0, 0, 0}, dvinc[3] = {0, 0, 0};
    if constexpr (D == 3) {
      // Separable sums: along x first (per (y, z) row of the stencil), then
      // weighted by the row's y/z factors.  v_pic = sum psi v_nt,
      // dv = sum psi (v_nt - v), L = sum grad(psi) v_nt^T.  The x and y
      // components go in packed FP32 pairs (the same roundings as one FMA per
      // component), z alone.
      float2 vinc2 = make_float2(0.0f, 0.0f), dvinc2 = make_float2(0.0f, 0.0f);
      float vincz = 0.0f, dvincz = 0.0f;
      float2 Lr2[3] = {make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f)};  // L[r][0..1]
      float Lrz[3] = {0.0f, 0.0f, 0.0f};                                                               // L[r][2]
      const float2 minus1 = make_float2(-1.0f, -1.0f);
      constexpr int KZ = D == 3 ? K : 1;
      const float4 *vel = reinterpret_cast<const float4 *>(a.N.vel);
#pragma unroll
      for (int kz = 0; kz < KZ; kz++) {
#pragma unroll
        for (int ky = 0; ky < K; ky++) {
          if (!ok[1][ky] || (D == 3 && !ok[2][kz])) continue;
          const int row = idx[1][ky] * g.n[0] + (D == 3 ? idx[2][kz] * g.n[0] * g.n[1] : 0);
          float2 sv2 = make_float2(0.0f, 0.0f), sd2 = make_float2(0.0f, 0.0f), sg2 = make_float2(0.0f, 0.0f);
          float svz = 0.0f, sdz = 0.0f, sgz = 0.0f;
#pragma unroll
          for (int kx = 0; kx < K; kx++) {
            if (!ok[0][kx]) continue;
            const int node = idx[0][kx] + row;
            const float n = N[0][kx], dn = dN[0][kx];
            const float2 n2 = make_float2(n, n), dn2 = make_float2(dn, dn);
            float2 vn2, vnt2;
            if (D == 3) {
              float4 q0, q1;
              ldg_node8(vel + 2 * (size_t)node, q0, q1);
              vn2 = make_float2(q0.x, q0.y);
              vnt2 = make_float2(q1.x, q1.y);
              svz = fmaf(n, q1.z, svz);
              sdz = fmaf(n, q1.z - q0.z, sdz);
              sgz = fmaf(dn, q1.z, sgz);
            } else {
              const float4 q = __ldg(vel + node);
              vn2 = make_float2(q.x, q.y);
              vnt2 = make_float2(q.z, q.w);
            }
            sv2 = __ffma2_rn(n2, vnt2, sv2);
            sd2 = __ffma2_rn(n2, __ffma2_rn(vn2, minus1, vnt2), sd2);  // v_nt - v, rounded once
            sg2 = __ffma2_rn(dn2, vnt2, sg2);
          }
          const float wyz = D == 3 ? N[1][ky] * N[2][kz] : N[1][ky];
          const float gyz = D == 3 ? dN[1][ky] * N[2][kz] : dN[1][ky];
          const float wgz = D == 3 ? N[1][ky] * dN[2][kz] : 0.0f;
          const float2 wyz2 = make_float2(wyz, wyz), gyz2 = make_float2(gyz, gyz);
          vinc2 = __ffma2_rn(wyz2, sv2, vinc2);
          dvinc2 = __ffma2_rn(wyz2, sd2, dvinc2);
          Lr2[0] = __ffma2_rn(wyz2, sg2, Lr2[0]);
          Lr2[1] = __ffma2_rn(gyz2, sv2, Lr2[1]);
          if (D == 3) {
            Lr2[2] = __ffma2_rn(make_float2(wgz, wgz), sv2, Lr2[2]);
            vincz = fmaf(wyz, svz, vincz);
            dvincz = fmaf(wyz, sdz, dvincz);
            Lrz[0] = fmaf(wyz, sgz, Lrz[0]);
            Lrz[1] = fmaf(gyz, svz, Lrz[1]);
            Lrz[2] = fmaf(wgz, svz, Lrz[2]);
          }
        }
      }
      vinc[0] = vinc2.x;
      vinc[1] = vinc2.y;
      vinc[2] = vincz;
      dvinc[0] = dvinc2.x;
      dvinc[1] = dvinc2.y;
      dvinc[2] = dvincz;
#pragma unroll
      for (int r = 0; r < D; r++) {
        L[r * D + 0] = Lr2[r].x;
        L[r * D + 1] = Lr2[r].y;
        if (D == 3) L[r * D + 2] = Lrz[r];
      }
    } else {
      // Separable sums: along x first (per (y, z) row of the stencil), then
      // weighted by the row's y/z factors.  v_pic = sum psi v_nt,
      // dv = sum psi (v_nt - v), L = sum grad(psi) v_nt^T.
      constexpr int KZ = D == 3 ? K : 1;
      const float4 *vel = reinterpret_cast<const float4 *>(a.N.vel);
#pragma unroll
      for (int kz = 0; kz < KZ; kz++) {
#pragma unroll
        for (int ky = 0; ky < K; ky++) {
          if (!ok[1][ky] || (D == 3 && !ok[2][kz])) continue;
          const int row = idx[1][ky] * g.n[0] + (D == 3 ? idx[2][kz] * g.n[0] * g.n[1] : 0);
          float sv[3] = {0, 0, 0}, sd[3] = {0, 0, 0}, sg[3] = {0, 0, 0};
#pragma unroll
          for (int kx = 0; kx < K; kx++) {
            if (!ok[0][kx]) continue;
            const int node = idx[0][kx] + row;
            float vn[3], vnt[3];
            if (D == 3) {
              float4 q0, q1;
              ldg_node8(vel + 2 * (size_t)node, q0, q1);
              vn[0] = q0.x; vn[1] = q0.y; vn[2] = q0.z;
              vnt[0] = q1.x; vnt[1] = q1.y; vnt[2] = q1.z;
            } else {
              const float4 q = __ldg(vel + node);
              vn[0] = q.x; vn[1] = q.y; vn[2] = 0.0f;
              vnt[0] = q.z; vnt[1] = q.w; vnt[2] = 0.0f;
            }
#pragma unroll
            for (int c = 0; c < D; c++) {
              sv[c] += N[0][kx] * vnt[c];
              sd[c] += N[0][kx] * (vnt[c] - vn[c]);
              sg[c] += dN[0][kx] * vnt[c];
            }
          }
          const float wyz = D == 3 ? N[1][ky] * N[2][kz] : N[1][ky];
          const float gyz = D == 3 ? dN[1][ky] * N[2][kz] : dN[1][ky];
          const float wgz = D == 3 ? N[1][ky] * dN[2][kz] : 0.0f;
#pragma unroll
          for (int c = 0; c < D; c++) {
            vinc[c] += wyz * sv[c];
            dvinc[c] += wyz * sd[c];
            L[0 * D + c] += wyz * sg[c];
            L[1 * D + c] += gyz * sv[c];
            if (D == 3) L[2 * D + c] += wgz * sv[c];
          }
        }
      }
    }
    // RigidBodyLevelSet::set_position (rigidbodylevelset.cpp:222-243) moved
    // rigid particles by their set velocity before G2P; their weights above
    // are those of the unmoved position, as the reference's stored psi
    const bool shift = a.rigid_shift && P.rigid[s];
    if (a.musl_pass == 1) {
      // MUSL first mapping: velocities and the new positions (kept aside:
      // the second mappings use this step's start-of-step weights)
      bool finite = true;
#pragma unroll
      for (int c = 0; c < D; c++) {
        const float vnew = a.one_minus_alpha * vinc[c] + a.alpha * (v[c] + dvinc[c]);
        const float x0 = shift ? __fadd_rn(x[c], __fmul_rn(v[c], a.dt)) : x[c];
        const float xnew = x0 + a.dt * vinc[c];
        P.v[c * st + s] = vnew;
        a.musl_x[c * st + s] = xnew;
        finite = finite && isfinite(xnew);
      }
      if (!finite) atomicOr(a.fault, kFaultNonFinite);
      return;
    }
    // v <- (1 - alpha) v_pic + alpha (v + dv); x += dt v_pic; F <- (I + L dt) F; V = det(F) V0
    if constexpr (F_LATE) {
#pragma unroll
      for (int k = 0; k < D * D; k++) F[k] = P.F[k * st + s];
    }
    float A[9], Fn[9];
#pragma unroll
    for (int r = 0; r < D; r++)
#pragma unroll
      for (int c = 0; c < D; c++) A[r * D + c] = (r == c ? 1.0f : 0.0f) + L[r * D + c] * a.dt;
#pragma unroll
    for (int r = 0; r < D; r++)
#pragma unroll
      for (int c = 0; c < D; c++) {
        float acc = A[r * D + 0] * F[0 * D + c];
#pragma unroll
        for (int k = 1; k < D; k++) acc += A[r * D + k] * F[k * D + c];
        Fn[r * D + c] = acc;
      }
    bool finite = true;
    if (a.musl_pass == 2) {
      // MUSL second G2P: L from the remapped velocities; positions from the first mapping
#pragma unroll
      for (int c = 0; c < D; c++) P.x[c * st + s] = a.musl_x[c * st + s];
    } else {
#pragma unroll
      for (int c = 0; c < D; c++) {
        const float vnew = a.one_minus_alpha * vinc[c] + a.alpha * (v[c] + dvinc[c]);
        const float x0 = shift ? __fadd_rn(x[c], __fmul_rn(v[c], a.dt)) : x[c];
        const float xnew = x0 + a.dt * vinc[c];
        P.v[c * st + s] = vnew;
        P.x[c * st + s] = xnew;
        finite = finite && isfinite(xnew);
      }
    }
#pragma unroll
    for (int k = 0; k < D * D; k++) P.F[k * st + s] = Fn[k];
    P.V[s] = det_rows<D>(Fn) * P.V0[s];
    if (!finite) atomicOr(a.fault, kFaultNonFinite);
  }
  if (store_L) {
#pragma unroll
    for (int k = 0; k < D * D; k++) P.L[k * st + s] = L[k];
  }
  if (do_stress) stress_update_point<D, FULL>(a, s, L);
}

// bin_next (quadratic, dual binning): the step's last G2P also bins the
// new positions for the next partition (counts, slots, keys, tile and brick
// marks of epoch + 1), which then skips its binning pass.
// Threads per block and blocks per SM of k_g2p: the 3D cubic gather runs
// 128-thread blocks, five per SM at up to 96 registers (20 warps, no spills;
// F is loaded after the gather).  With the 256-bit node loads, six blocks at
// 80 registers (28 bytes of spills) ran the bed's G2P 1 % slower and seven
// at 72 (96 bytes) 13 % slower; 256-thread blocks fit two at 128 registers.
template <int D, int SF, bool FULL>
struct G2PLaunch {
  static constexpr bool SMALL = D == 3 && SF == PMPM_SHAPE_CUBIC && !FULL;
  static constexpr int NT = SMALL ? 128 : 256;
  static constexpr int MIN_BLOCKS = SMALL ? 5 : (FULL ? 2 : (SF == PMPM_SHAPE_CUBIC ? 2 : 4));
};

template <int D, int SF, bool FULL>
__global__ void __launch_bounds__(G2PLaunch<D, SF, FULL>::NT, G2PLaunch<D, SF, FULL>::MIN_BLOCKS)
    k_g2p(StepArgs a, int do_stress, int store_L) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < a.P.n) g2p_body<D, SF, FULL>(a, s, do_stress, store_L);
  if constexpr (SF == PMPM_SHAPE_QUADRATIC) {
    // the reference hashes of the new positions wait in hash_next until
    // the next partition: the views of this step's partition stay readable
    if (a.bin_next) hash_count_body<D, SF>(a, s, s < a.P.n, a.epoch + 1, a.hash_next);
  }
}

// Stress update alone from the stored velocity gradient.
template <int D>
__global__ void __launch_bounds__(256) k_stress_update(StepArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.P.n) return;
  float L[9];
#pragma unroll
  for (int k = 0; k < D * D; k++) L[k] = a.P.L[k * a.P.stride + s];
  stress_update_point<D>(a, s, L);
}

// --------------------------------------------------------------------------
// shape-function dump (reference psi / dpsi layout, for inspection)
// --------------------------------------------------------------------------

template <int D, int SF>
__global__ void __launch_bounds__(256) k_shape_dump(StepArgs a, float *psi, float *dpsi) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.P.n) return;
  const DevParticles &P = a.P;
  const DevGrid &g = a.g;
  constexpr int NS = IPow<Stencil<SF>::WIN, D>::value;
  const int i = P.id[s];
  float u[3];
  int b[3] = {0, 0, 0};
#pragma unroll
  for (int c = 0; c < D; c++) {
    u[c] = scaled_coord(P.x[c * P.stride + s], g.origin[c], g.inv_h);
    b[c] = (int)u[c];
  }
  for (int sid = 0; sid < NS; sid++) {
    int w[3];
    window_offset<D, SF>(sid, w);
    int t[3] = {b[0] + w[0], b[1] + w[1], D == 3 ? b[2] + w[2] : 0};
    if (SF == PMPM_SHAPE_QUADRATIC)
      for (int c = 0; c < D; c++) t[c] = min(max(t[c], 0), g.n[c] - 1);
    const int f = t[0] + t[1] * g.n[0] + t[2] * g.n[0] * g.n[1];
    float ps = 0.0f, dp[3] = {0.0f, 0.0f, 0.0f};
    if ((unsigned)f < (unsigned)g.ntotal) {
      const int nc[3] = {f % g.n[0], (f / g.n[0]) % g.n[1], f / (g.n[0] * g.n[1])};
      float N[3], dN[3];
      for (int c = 0; c < D; c++) {
        const float rel = u[c] - (float)(b[c] + w[c]);
        const int type = SF == PMPM_SHAPE_CUBIC ? cubic_node_type(nc[c], g.n[c]) : 0;
        axis_weight<SF>(rel, g.inv_h, type, N[c], dN[c]);
      }
      if (D == 2) {
        ps = N[0] * N[1];
        dp[0] = dN[0] * N[1];
        dp[1] = dN[1] * N[0];
      } else {
        ps = N[0] * N[1] * N[2];
        dp[0] = dN[0] * N[1] * N[2];
        dp[1] = dN[1] * N[0] * N[2];
        dp[2] = dN[2] * N[0] * N[1];
      }
    }
    psi[(size_t)i * NS + sid] = ps;
    for (int c = 0; c < D; c++) dpsi[((size_t)i * NS + sid) * D + c] = dp[c];
  }
}

// --------------------------------------------------------------------------
// single-point material update (standalone material binding)
// --------------------------------------------------------------------------

template <int D>
__global__ void __launch_bounds__(256) k_point_update(DevMaterial mt, int n, float dt, const float *L, float *S,
                                                      float *eps, const float *sref, const float *m, const float *V,
                                                      const float *V0, int velgrad_is_increment) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float Li[9], Si[9];
#pragma unroll
  for (int k = 0; k < D * D; k++) Li[k] = L[(size_t)i * D * D + k];
#pragma unroll
  for (int k = 0; k < 9; k++) Si[k] = S[(size_t)i * 9 + k];
  if (mt.type == PMPM_MAT_LINEAR_ELASTIC) {
    le_update<D>(mt, Li, dt, Si);
  } else if (mt.type == PMPM_MAT_NEWTON_FLUID) {
    nf_update<D>(mt, Li, m[i], V[i], V0[i], Si);
  } else if (mt.type == PMPM_MAT_DRUCKER_PRAGER) {
    float e[9], r[9];
#pragma unroll
    for (int k = 0; k < D * D; k++) e[k] = eps[(size_t)i * D * D + k];
#pragma unroll
    for (int k = 0; k < 9; k++) r[k] = sref[(size_t)i * 9 + k];
    dp_update<D>(mt.p, Li, dt, e, r, Si, velgrad_is_increment != 0);
#pragma unroll
    for (int k = 0; k < D * D; k++) eps[(size_t)i * D * D + k] = e[k];
  }
#pragma unroll
  for (int k = 0; k < 9; k++) S[(size_t)i * 9 + k] = Si[k];
}

// --------------------------------------------------------------------------
// batched ensembles: one launch per phase for all instances
// --------------------------------------------------------------------------
//
// Each CTA works inside one instance.  The instance's StepArgs view (grid,
// node and key sub-arrays, materials, boundary conditions, dt) is copied
// from device memory into shared memory, and the single-instance bodies run
// on it unchanged.  Particle arrays are shared: instance i owns storage
// slots [first_i, first_i + n_i), an invariant of the instance-major key
// space (instance i's keys precede instance i+1's, and a particle outside
// its grid takes its instance's sentinel key).

struct BatchBlock {
  int inst, first, end;  // particle block: storage slots [first, end) of instance inst
};
struct BatchTile {
  int inst, tile, global_tile;  // node tile `tile` of instance inst
};

// nwords: how much of the view to copy (the whole of it unless the kernel
// reads nothing past a known member)
__device__ __forceinline__ void load_view(StepArgs &sa, const StepArgs *views, int inst, const DevParticles &P,
                                          int epoch, int nwords = (int)(sizeof(StepArgs) / sizeof(int))) {
  const int *src = reinterpret_cast<const int *>(views + inst);
  int *dst = reinterpret_cast<int *>(&sa);
  for (int k = threadIdx.x; k < nwords; k += blockDim.x) dst[k] = __ldg(src + k);
  __syncthreads();
  if (threadIdx.x == 0) {
    sa.P = P;
    sa.epoch = epoch;
  }
  __syncthreads();
}

template <int D, int SF>
__global__ void __launch_bounds__(256) kb_hash_count(const StepArgs *views, const BatchBlock *blocks, DevParticles P,
                                                     int epoch) {
  __shared__ StepArgs sa;
  const BatchBlock b = blocks[blockIdx.x];
  load_view(sa, views, b.inst, P, epoch);
  const int s = b.first + (int)threadIdx.x;
  hash_count_body<D, SF>(sa, s, s < b.end, sa.epoch, sa.P.hash);
}

// Persistent CTAs over the batch's active-tile queue (tile_list[0 ..
// tile_queue[epoch & 1]) are global tile indices; tile_queue[2 + par] is this
// launch's fetch counter, the other one is reset for the next launch).
template <int D, int SF>
__global__ void __launch_bounds__(TileDims<D>::N, D == 2 ? 3 : 1) kb_p2g(const StepArgs *views, const BatchTile *tiles,
                                                         const int *tile_list, int *tile_queue, int par,
                                                         int ntiles, DevParticles P, int epoch, int apply_bcs,
                                                         int *node_epoch, int gather) {
  __shared__ StepArgs sa;
  __shared__ int cur;
  if (blockIdx.x == 0 && threadIdx.x == 0) tile_queue[2 + (par ^ 1)] = 0;
  if (binning_failed(views[0].fault)) return;
  const int count = min(tile_queue[epoch & 1], ntiles);
  for (;;) {
    if (threadIdx.x == 0) cur = atomicAdd(&tile_queue[2 + par], 1);
    __syncthreads();
    const int idx = cur;
    __syncthreads();
    if (idx >= count) break;
    const BatchTile t = tiles[tile_list[idx]];
    load_view(sa, views, t.inst, P, epoch);
    int *ne = node_epoch + (t.global_tile - t.tile);
    if (gather)
      p2g_gather_body<D, SF>(sa, t.tile, apply_bcs, ne);
    else
      p2g_tile_body<D, SF>(sa, t.tile, apply_bcs, ne);
  }
}

// bin_next: also bin the new positions for the next partition (as k_g2p),
// their reference hashes into hash_next.  view_words: the part of the
// instance view to copy (G2P and the stress update read nothing of the node
// conditions; the binning reads them only for a PlanarDomain)
template <int D, int SF>
__global__ void __launch_bounds__(256) kb_g2p(const StepArgs *views, const BatchBlock *blocks, DevParticles P,
                                              int epoch, int do_stress, int store_L, int bin_next,
                                              unsigned *hash_next, int view_words) {
  __shared__ StepArgs sa;
  const BatchBlock b = blocks[blockIdx.x];
  load_view(sa, views, b.inst, P, epoch, view_words);
  const int s = b.first + (int)threadIdx.x;
  if (s < b.end) g2p_body<D, SF, false>(sa, s, do_stress, store_L);  // batches hold no iterative material
  if (bin_next) hash_count_body<D, SF>(sa, s, s < b.end, epoch + 1, hash_next);
}

}  // namespace pmpm
