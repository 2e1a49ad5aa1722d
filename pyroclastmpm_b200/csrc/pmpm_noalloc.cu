// Spatial partition without any device allocation (pmpm_partition_noalloc).
//
// Some callers cannot allocate device memory at the point where they need a
// partition: host code that runs inside a memory pool's or a framework's
// allocation callback, or plug-ins that live under a fixed device-memory
// budget handed to them by a host application.  This
// entry point serves them: the caller provides the inputs and the outputs,
// and the temporary arrays live in one file-scope device array of fixed size
// that every GPU which loads this library holds until the process exits.
//
// Limits: at most kNoAllocMaxParticles particles and kNoAllocMaxCells cells.
// All calls share the one scratch array, so calls that run at the same time
// on the GPU (different streams, different host threads) race with each
// other; serialise them.  The scratch keeps the previous call's contents;
// everything that must start at zero is cleared by each call.
#include <cuda_runtime.h>

#include <cstdio>

#include "pmpm.h"
#include "pmpm_device.cuh"

namespace {

constexpr int kNoAllocMaxParticles = 1 << 17;
constexpr int kNoAllocMaxCells = 1 << 17;
constexpr int kNaThreads = 1024;
constexpr int kNaPer = 4;
constexpr int kNaChunk = kNaThreads * kNaPer;
constexpr int kNaBlocks = (kNoAllocMaxCells + kNaChunk - 1) / kNaChunk;

constexpr int kNaSmallCell = 32;   // cells up to this size are sorted in registers
constexpr int kNaBigCell = 2048;   // larger cells: bitonic sort in shared memory

// scratch layout (ints): count[cells] | offset[cells + 1] | block_sums[blocks]
// | slot[particles] | order[particles] | big_cells[cells] | flags[4]
// flags: [0] a particle lies outside the grid, [1] big-cell counter,
// [2] a cell holds more than kNaBigCell particles
constexpr int kOffCount = 0;
constexpr int kOffOffset = kOffCount + kNoAllocMaxCells;
constexpr int kOffBlock = kOffOffset + kNoAllocMaxCells + 1;
constexpr int kOffSlot = kOffBlock + kNaBlocks;
constexpr int kOffOrder = kOffSlot + kNoAllocMaxParticles;
constexpr int kOffBig = kOffOrder + kNoAllocMaxParticles;
constexpr int kOffFlags = kOffBig + kNoAllocMaxCells;
constexpr int kScratchInts = kOffFlags + 4;

static __device__ __align__(256) int g_partition_scratch[kScratchInts];

// Device address of g_partition_scratch per device, looked up once.  Two
// host threads making a first call on the same device at once may both
// look it up; they store the same address, so the unsynchronised write is
// harmless.
int *g_scratch_ptr[64] = {nullptr};

struct NaGrid {
  int dim;
  float origin[3];
  float inv_h;
  int n[3];
  int ntotal;
};

__device__ __forceinline__ int na_block_scan(int v, int *sw, int &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) sw[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const int wv = lane < (int)(blockDim.x >> 5) ? sw[lane] : 0;
    int wi = wv;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    sw[lane] = wi - wv;
    if (lane == 31) sw[32] = wi;
  }
  __syncthreads();
  total = sw[32];
  const int r = sw[warp] + incl - v;
  __syncthreads();
  return r;
}

// hash = NODE_MEM_INDEX((int)((x - origin) * inv_h)) and per-cell counts.
// Binning follows the reference's flat index (a particle past a face whose
// flat index stays inside the grid lands in the cell it points at); the
// out-of-domain flag is raised per axis and for non-finite coordinates.
__global__ void na_hash_count(NaGrid g, const float *x, int n, unsigned *hash_out, int *scratch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b[3] = {0, 0, 0};
  bool inside = true;
  for (int c = 0; c < g.dim; c++) {
    const float xc = x[(size_t)i * g.dim + c];
    b[c] = (int)__fmul_rn(__fsub_rn(xc, g.origin[c]), g.inv_h);
    inside = inside && isfinite(xc) && b[c] >= 0 && b[c] < g.n[c];
  }
  const unsigned h = (unsigned)(b[0] + b[1] * g.n[0] + b[2] * g.n[0] * g.n[1]);
  hash_out[i] = h;
  if (h < (unsigned)g.ntotal) {
    scratch[kOffSlot + i] = atomicAdd(&scratch[kOffCount + h], 1);
  } else {
    scratch[kOffSlot + i] = -1;
    inside = false;
  }
  if (!inside) atomicOr(&scratch[kOffFlags + 0], 1);
}

__global__ void __launch_bounds__(kNaThreads) na_scan_reduce(int ncells, int *scratch) {
  __shared__ int sw[33];
  const int base = blockIdx.x * kNaChunk + threadIdx.x * kNaPer;
  int sum = 0;
  for (int k = 0; k < kNaPer; k++)
    if (base + k < ncells) sum += scratch[kOffCount + base + k];
  int total;
  na_block_scan(sum, sw, total);
  if (threadIdx.x == 0) scratch[kOffBlock + blockIdx.x] = total;
}

__global__ void __launch_bounds__(kNaThreads) na_scan_top(int nblocks, int *scratch) {
  __shared__ int sw[33];
  int carry = 0;
  for (int base = 0; base < nblocks; base += kNaThreads) {
    const int i = base + threadIdx.x;
    const int v = i < nblocks ? scratch[kOffBlock + i] : 0;
    int total;
    const int ex = na_block_scan(v, sw, total);
    if (i < nblocks) scratch[kOffBlock + i] = carry + ex;
    carry += total;
  }
}

__global__ void __launch_bounds__(kNaThreads) na_scan_apply(int ncells, int *scratch) {
  __shared__ int sw[33];
  const int base = blockIdx.x * kNaChunk + threadIdx.x * kNaPer;
  int v[kNaPer];
  int sum = 0;
  for (int k = 0; k < kNaPer; k++) {
    v[k] = base + k < ncells ? scratch[kOffCount + base + k] : 0;
    sum += v[k];
  }
  int total;
  int ex = na_block_scan(sum, sw, total) + scratch[kOffBlock + blockIdx.x];
  for (int k = 0; k < kNaPer; k++) {
    if (base + k < ncells) scratch[kOffOffset + base + k] = ex;
    ex += v[k];
  }
  if (base <= ncells - 1 && ncells - 1 < base + kNaPer) scratch[kOffOffset + ncells] = ex;
}

__global__ void na_scatter(int n, const unsigned *hash, int *scratch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int slot = scratch[kOffSlot + i];
  if (slot >= 0) scratch[kOffOrder + scratch[kOffOffset + hash[i]] + slot] = i;
}

// Stable order inside each cell (ascending particle index): small cells by
// insertion sort here, larger ones are listed for na_sort_big.
__global__ void na_sort_small(int ncells, int *scratch) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  const int lo = scratch[kOffOffset + c], hi = scratch[kOffOffset + c + 1];
  if (hi - lo < 2) return;
  if (hi - lo > kNaSmallCell) {
    scratch[kOffBig + atomicAdd(&scratch[kOffFlags + 1], 1)] = c;
    return;
  }
  int *ord = scratch + kOffOrder;
  for (int i = lo + 1; i < hi; i++) {
    const int v = ord[i];
    int j = i - 1;
    while (j >= lo && ord[j] > v) {
      ord[j + 1] = ord[j];
      j--;
    }
    ord[j + 1] = v;
  }
}

__global__ void __launch_bounds__(1024) na_sort_big(int *scratch) {
  __shared__ int key[kNaBigCell];
  const int nbig = scratch[kOffFlags + 1];
  int *ord = scratch + kOffOrder;
  for (int bi = blockIdx.x; bi < nbig; bi += gridDim.x) {
    const int c = scratch[kOffBig + bi];
    const int lo = scratch[kOffOffset + c], cnt = scratch[kOffOffset + c + 1] - lo;
    if (cnt > kNaBigCell) {
      if (threadIdx.x == 0) atomicOr(&scratch[kOffFlags + 2], 1);
      continue;
    }
    int p2 = 1;
    while (p2 < cnt) p2 <<= 1;
    for (int i = threadIdx.x; i < p2; i += blockDim.x) key[i] = i < cnt ? ord[lo + i] : 0x7fffffff;
    __syncthreads();
    for (int k = 2; k <= p2; k <<= 1)
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int i = threadIdx.x; i < p2; i += blockDim.x) {
          const int ixj = i ^ j;
          if (ixj > i && ((key[i] > key[ixj]) == ((i & k) == 0))) {
            const int t = key[i];
            key[i] = key[ixj];
            key[ixj] = t;
          }
        }
        __syncthreads();
      }
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) ord[lo + i] = key[i];
    __syncthreads();
  }
}

// Outputs in the reference layout: sorted_index over the binned particles,
// cell_start / cell_end with 0 for empty cells.
__global__ void na_outputs(int ncells, const int *scratch, int *sorted_index, int *cell_start, int *cell_end) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  const int lo = scratch[kOffOffset + c], hi = scratch[kOffOffset + c + 1];
  for (int i = lo; i < hi; i++) sorted_index[i] = scratch[kOffOrder + i];
  cell_start[c] = hi > lo ? lo : 0;
  cell_end[c] = hi > lo ? hi : 0;
}

int scratch_for_current_device(int **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return PMPM_ERR_CUDA;
  if (!g_scratch_ptr[dev]) {
    int *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void **)&p, g_partition_scratch);
    if (e != cudaSuccess || !p) {
      fprintf(stderr, "pmpm: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
      return PMPM_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return PMPM_OK;
}

}  // namespace

extern "C" int pmpm_partition_noalloc(int dim, const float *origin, float cell_size, const int *num_cells,
                                      const float *positions, int num_particles, unsigned *hash_unsorted,
                                      int *sorted_index, int *cell_start, int *cell_end, void *stream) {
  if ((dim != 2 && dim != 3) || !origin || !num_cells || !(cell_size > 0.0f) || num_particles < 0 ||
      (num_particles > 0 && (!positions || !hash_unsorted || !sorted_index)) || !cell_start || !cell_end)
    return PMPM_ERR_INVALID_ARGUMENT;
  NaGrid g;
  g.dim = dim;
  g.inv_h = 1.0f / cell_size;  // Grid::inv_cell_size, FP32
  long long total = 1;
  for (int c = 0; c < 3; c++) {
    g.origin[c] = c < dim ? origin[c] : 0.0f;
    g.n[c] = c < dim ? num_cells[c] : 1;
    if (g.n[c] < 1) return PMPM_ERR_INVALID_ARGUMENT;
    total *= g.n[c];
  }
  if (total > kNoAllocMaxCells || num_particles > kNoAllocMaxParticles) {
    fprintf(stderr,
            "pmpm_partition_noalloc: %lld cells / %d particles exceed the fixed scratch "
            "(at most %d cells and %d particles)\n",
            total, num_particles, kNoAllocMaxCells, kNoAllocMaxParticles);
    return PMPM_ERR_INVALID_ARGUMENT;
  }
  g.ntotal = (int)total;
  int *scratch = nullptr;
  const int st = scratch_for_current_device(&scratch);
  if (st != PMPM_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const int nblocks = (g.ntotal + kNaChunk - 1) / kNaChunk;
  // per-cell counts and the fault flag must start at zero on every call
  if (cudaMemsetAsync(scratch + kOffCount, 0, sizeof(int) * g.ntotal, s) != cudaSuccess ||
      cudaMemsetAsync(scratch + kOffFlags, 0, sizeof(int) * 4, s) != cudaSuccess)
    return PMPM_ERR_CUDA;
  if (num_particles > 0) {
    na_hash_count<<<(num_particles + 255) / 256, 256, 0, s>>>(g, positions, num_particles, hash_unsorted, scratch);
  }
  na_scan_reduce<<<nblocks, kNaThreads, 0, s>>>(g.ntotal, scratch);
  na_scan_top<<<1, kNaThreads, 0, s>>>(nblocks, scratch);
  na_scan_apply<<<nblocks, kNaThreads, 0, s>>>(g.ntotal, scratch);
  if (num_particles > 0) na_scatter<<<(num_particles + 255) / 256, 256, 0, s>>>(num_particles, hash_unsorted, scratch);
  na_sort_small<<<(g.ntotal + 255) / 256, 256, 0, s>>>(g.ntotal, scratch);
  na_sort_big<<<64, 1024, 0, s>>>(scratch);
  na_outputs<<<(g.ntotal + 255) / 256, 256, 0, s>>>(g.ntotal, scratch, sorted_index, cell_start, cell_end);
  if (cudaGetLastError() != cudaSuccess) return PMPM_ERR_CUDA;
  int flags[4] = {0, 0, 0, 0};
  if (cudaMemcpyAsync(flags, scratch + kOffFlags, sizeof(flags), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return PMPM_ERR_CUDA;
  if (flags[2]) return PMPM_ERR_CELL_OVERFLOW;
  return flags[0] ? PMPM_ERR_OUT_OF_DOMAIN : PMPM_OK;
}
