// Block-neighbour detection that allocates no device memory.
//
// Who needs this: callers that are not allowed to allocate GPU memory once
// they are running, for example code embedded in a host application that
// hands it a fixed memory pool (and forbids cudaMalloc after start-up), or a
// real-time loop that must never block in the allocator.  They still want the
// bounding-sphere block-neighbour matrix that the scoring path computes (the
// reference's detect_block_neighbors, tmol/score/common/sphere_overlap.impl.hh:
// 287-351), for example to drive their own per-block-pair work.  The scoring
// entry points cannot serve them, because a plan owns allocated scratch.
//
// Here the only scratch, the per-block bounding spheres, lives in a
// file-scope device array of fixed size (kMaxBlocks spheres, 4 MiB).  Every
// GPU that loads this library keeps that array until the process exits.
// The caller passes inputs and the output; the entry point calls no
// cudaMalloc, cudaFree or allocating library routine.

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/tmol_b200_ljlk.h"

namespace {

// Largest n_poses * max_n_blocks the entry point accepts.
constexpr int64_t kMaxBlocks = int64_t(1) << 18;  // 262,144 blocks
constexpr int kMaxDevices = 64;

// centroid x, y, z and radius of every block of the last call
static __device__ __align__(256) float g_noalloc_spheres[kMaxBlocks * 4];

// Device address of g_noalloc_spheres, looked up once per device: in host
// code the array's name is a host-side stand-in, not a device address.
// Under CUDA's lazy module loading, the first lookup on a device also loads
// this module there, which takes device memory (the array and the code):
// callers make their first call at start-up.  The cached address is only
// valid while the device's primary context lives (no cudaDeviceReset).
float* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

int scratch_for_current_device(float** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return TMOL_B200_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return TMOL_B200_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_spheres) != cudaSuccess || !ptr)
      return TMOL_B200_ERR_CUDA;
    g_scratch_addr[dev] = static_cast<float*>(ptr);
  }
  *out = g_scratch_addr[dev];
  return TMOL_B200_OK;
}

// Sphere of every block slot: centroid = (sum of its atoms, in order) / n,
// radius = largest centroid distance, in the reference CPU order without
// contraction, so that the result is bit-identical to the scoring path's.
// Slots without a (valid) block get a zero sphere and are never neighbours.
__global__ void noalloc_spheres_kernel(const float* coords, int64_t n_atoms,
                                       const int32_t* block_type,
                                       const int32_t* block_coord_offset,
                                       const int32_t* bt_n_atoms, int nbt,
                                       int64_t n_blocks, float* spheres) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_blocks;
       i += (int64_t)gridDim.x * blockDim.x) {
    float* out = spheres + 4 * i;
    int bt = block_type[i];
    int n = (bt >= 0 && bt < nbt) ? bt_n_atoms[bt] : -1;
    int64_t off = block_coord_offset[i];
    if (n < 0 || off < 0 || off + n > n_atoms) {
      out[0] = out[1] = out[2] = out[3] = 0.0f;
      continue;
    }
    const float* x = coords + 3 * off;
    float cx = 0, cy = 0, cz = 0;
    for (int k = 0; k < n; ++k) {
      cx = __fadd_rn(cx, x[3 * k + 0]);
      cy = __fadd_rn(cy, x[3 * k + 1]);
      cz = __fadd_rn(cz, x[3 * k + 2]);
    }
    float rn = float(n);
    cx = __fdiv_rn(cx, rn);
    cy = __fdiv_rn(cy, rn);
    cz = __fdiv_rn(cz, rn);
    float d2max = 0;
    for (int k = 0; k < n; ++k) {
      float dx = __fsub_rn(x[3 * k + 0], cx);
      float dy = __fsub_rn(x[3 * k + 1], cy);
      float dz = __fsub_rn(x[3 * k + 2], cz);
      float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
      if (d2 > d2max) d2max = d2;
    }
    out[0] = cx;
    out[1] = cy;
    out[2] = cz;
    out[3] = __fsqrt_rn(d2max);
  }
}

// One thread per cell of the [P, B, B] output: 1 iff b1 <= b2, both blocks
// exist and |c1 - c2| < r1 + r2 + reach; every cell is written.
__global__ void noalloc_neighbors_kernel(const float* spheres,
                                         const int32_t* block_type,
                                         const int32_t* bt_n_atoms, int nbt,
                                         int P, int B, float reach,
                                         int32_t* nbr) {
  int64_t n_cells = (int64_t)P * B * B;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n_cells;
       c += (int64_t)gridDim.x * blockDim.x) {
    int64_t p = c / ((int64_t)B * B);
    int64_t rem = c - p * B * B;
    int b1 = (int)(rem / B), b2 = (int)(rem - (int64_t)b1 * B);
    int64_t i1 = p * B + b1, i2 = p * B + b2;
    int bt1 = block_type[i1], bt2 = block_type[i2];
    int hit = 0;
    if (b1 <= b2 && bt1 >= 0 && bt1 < nbt && bt2 >= 0 && bt2 < nbt) {
      const float* s1 = spheres + 4 * i1;
      const float* s2 = spheres + 4 * i2;
      float dx = __fsub_rn(s1[0], s2[0]);
      float dy = __fsub_rn(s1[1], s2[1]);
      float dz = __fsub_rn(s1[2], s2[2]);
      float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
      float thr = __fadd_rn(__fadd_rn(s1[3], s2[3]), reach);
      hit = d2 < __fmul_rn(thr, thr) ? 1 : 0;
    }
    nbr[c] = hit;
  }
}

}  // namespace

extern "C" int tmol_b200_ljlk_block_neighbors_noalloc(
    const float* coords, int64_t n_atoms, const int32_t* block_type,
    const int32_t* block_coord_offset, const int32_t* bt_n_atoms,
    int32_t n_block_types, int32_t n_poses, int32_t max_n_blocks,
    double max_dis, int32_t* block_neighbors, void* stream) {
  if (n_poses < 0 || max_n_blocks < 0 || n_atoms < 0 || n_block_types < 0)
    return TMOL_B200_ERR_SHAPE;
  const int64_t n_blocks = (int64_t)n_poses * max_n_blocks;
  if (n_blocks > kMaxBlocks) return TMOL_B200_ERR_CAPACITY;
  if (n_blocks == 0) return TMOL_B200_OK;
  if (!block_type || !block_coord_offset || !block_neighbors ||
      (n_block_types > 0 && !bt_n_atoms) || (n_atoms > 0 && !coords))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  float* spheres = nullptr;
  int rc = scratch_for_current_device(&spheres);
  if (rc != TMOL_B200_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  int threads = 256;
  int grid_s = (int)((n_blocks + threads - 1) / threads);
  if (grid_s > 65535) grid_s = 65535;
  noalloc_spheres_kernel<<<grid_s, threads, 0, st>>>(
      coords, n_atoms, block_type, block_coord_offset, bt_n_atoms, n_block_types,
      n_blocks, spheres);
  if (cudaGetLastError() != cudaSuccess) return TMOL_B200_ERR_CUDA;
  int64_t n_cells = n_blocks * max_n_blocks;
  int grid_n = (int)((n_cells + threads - 1) / threads);
  if (grid_n > 65535 * 8) grid_n = 65535 * 8;
  noalloc_neighbors_kernel<<<grid_n, threads, 0, st>>>(
      spheres, block_type, bt_n_atoms, n_block_types, n_poses, max_n_blocks,
      (float)max_dis, block_neighbors);
  if (cudaGetLastError() != cudaSuccess) return TMOL_B200_ERR_CUDA;
  return TMOL_B200_OK;
}
