// PoseStack construction on B200: inter-block bond separation from the
// connection graph, and tmol's stacked all-pairs-shortest-paths op; the C
// ABI is include/tmol_b200_pose.h.
//
// Bond separation (tmol_b200_pose_bondsep): one thread per connection point
// runs the bounded search of bondsep.cuh and writes its row of the dense
// [P, B, B, C, C] tensor (pre-filled with 6 by a vectorised fill) and the
// minimum per block pair with an integer atomicMin.  The fill is the
// HBM-bound part (P * B^2 * C^2 * 4 bytes); the searches touch a few nodes
// each.
//
// Stacked APSP (tmol_b200_apsp_stacked): blocked Floyd-Warshall with 32 x 32
// tiles in shared memory (the pivot tile, then its row and column, then every
// other tile from the two final panels), with the reference CPU op's cutoff
// rule applied before and after.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/tmol_b200_ljlk.h"
#include "../../include/tmol_b200_pose.h"
#include "bondsep.cuh"

namespace tmol_b200 {

// ---------------------------------------------------------------------------
// bond separation

__global__ void fill_i32_kernel(int32_t* out, int64_t n, int32_t v) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // 16-byte stores over the aligned middle, scalars at the ends
  const int64_t lead = (int64_t)((16 - ((uintptr_t)out & 15)) & 15) / 4;
  const int64_t head = lead < n ? lead : n;
  const int64_t n4 = (n - head) / 4;
  int4* mid = reinterpret_cast<int4*>(out + head);
  const int4 v4 = make_int4(v, v, v, v);
  for (int64_t k = i; k < n4; k += stride) mid[k] = v4;
  for (int64_t k = i; k < head; k += stride) out[k] = v;
  for (int64_t k = head + 4 * n4 + i; k < n; k += stride) out[k] = v;
}

// One thread per (pose, block, connection); sources in (p, b, c) order.
__global__ void bondsep_sources_kernel(PoseConn g, int32_t* ibb, int32_t* minsep, int* status) {
  const int64_t n_src = (int64_t)g.P * g.B * g.C;
  int reach[BONDSEP_MAX_REACH], dist[BONDSEP_MAX_REACH];
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n_src;
       s += (int64_t)gridDim.x * blockDim.x) {
    const int c0 = (int)(s % g.C);
    const int64_t pb = s / g.C;
    const int p = (int)(pb / g.B), b0 = (int)(pb - (int64_t)p * g.B);
    const int nc = block_n_conn(g, p, b0);
    if (nc < 0) {
      if (c0 == 0) atomicOr(status, kBsIndex);
      continue;
    }
    if (c0 >= nc) continue;
    int st = 0;
    const int n = bounded_paths(g, p, b0, c0, reach, dist, st);
    if (st) atomicOr(status, st);
    for (int k = 0; k < n; ++k) {
      const int b2 = reach[k] >> 3, c2 = reach[k] & 7;
      const int64_t bp = ((int64_t)p * g.B + b0) * g.B + b2;
      if (ibb) ibb[(bp * g.C + c0) * g.C + c2] = dist[k];
      if (minsep) atomicMin(&minsep[bp], dist[k]);
    }
  }
}

// status bits -> a tmol_b200_status code, in the plan builders' priority
__global__ void bondsep_status_kernel(int* status) {
  const int b = *status;
  *status = (b & kBsIndex) ? TMOL_B200_ERR_INDEX_RANGE
            : (b & kBsShape) ? TMOL_B200_ERR_SHAPE
            : (b & kBsCapacity) ? TMOL_B200_ERR_CAPACITY
                                : TMOL_B200_OK;
}

// ---------------------------------------------------------------------------
// stacked all-pairs shortest paths

constexpr int APSP_T = 32;

// min-plus relaxation with -1 as "no path" (apsp.cuda.cu's rule)
__device__ __forceinline__ int32_t relax(int32_t cur, int32_t a, int32_t b) {
  if (a >= 0 && b >= 0) {
    const int32_t s = a + b;
    if (cur < 0 || s < cur) return s;
  }
  return cur;
}

// cutoff rule, before: symmetrised edges below the cutoff, diagonal 0 (one
// thread per unordered pair)
__global__ void apsp_prepare_kernel(int32_t* w, int n, int cutoff) {
  const int g = blockIdx.z;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || j >= n || j < i) return;
  int32_t* m = w + (int64_t)g * n * n;
  if (i == j) {
    m[(int64_t)i * n + i] = 0;
    return;
  }
  const int32_t a = m[(int64_t)j * n + i], b = m[(int64_t)i * n + j];
  int32_t e = (a == -1 || b == -1) ? max(a, b) : min(a, b);
  if (e < 0 || e >= cutoff) e = -1;
  m[(int64_t)i * n + j] = e;
  m[(int64_t)j * n + i] = e;
}

// cutoff rule, after: every pair at or beyond the cutoff, or unreachable,
// at the cutoff
__global__ void apsp_finish_kernel(int32_t* w, int64_t total, int cutoff) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = w[k];
    if (v < 0 || v >= cutoff) w[k] = cutoff;
  }
}

__device__ __forceinline__ int32_t tile_get(const int32_t* m, int n, int i, int j) {
  return (i < n && j < n) ? m[(int64_t)i * n + j] : -1;
}

// phase 1: the pivot tile (kb, kb), 32 x 32 threads
__global__ void __launch_bounds__(1024) apsp_phase1_kernel(int32_t* w, int n, int kb) {
  __shared__ int32_t t[APSP_T][APSP_T + 1];
  int32_t* m = w + (int64_t)blockIdx.x * n * n;
  const int x = threadIdx.y, y = threadIdx.x;
  const int i = kb * APSP_T + x, j = kb * APSP_T + y;
  int32_t cur = tile_get(m, n, i, j);
  t[x][y] = cur;
  for (int k = 0; k < APSP_T; ++k) {
    __syncthreads();
    const int32_t a = t[x][k], b = t[k][y];
    __syncthreads();
    const int32_t nv = relax(cur, a, b);
    if (nv != cur) {
      cur = nv;
      t[x][y] = cur;
    }
  }
  if (i < n && j < n) m[(int64_t)i * n + j] = cur;
}

// phase 2: the pivot row (z = 1) and column (z = 0) tiles
__global__ void __launch_bounds__(1024) apsp_phase2_kernel(int32_t* w, int n, int kb) {
  __shared__ int32_t piv[APSP_T][APSP_T + 1];
  __shared__ int32_t t[APSP_T][APSP_T + 1];
  int32_t* m = w + (int64_t)blockIdx.x * n * n;
  const int other = blockIdx.y + (blockIdx.y >= kb ? 1 : 0);
  const int row = blockIdx.z == 1;
  const int x = threadIdx.y, y = threadIdx.x;
  const int i = (row ? kb : other) * APSP_T + x;
  const int j = (row ? other : kb) * APSP_T + y;
  piv[x][y] = tile_get(m, n, kb * APSP_T + x, kb * APSP_T + y);
  int32_t cur = tile_get(m, n, i, j);
  t[x][y] = cur;
  for (int k = 0; k < APSP_T; ++k) {
    __syncthreads();
    const int32_t a = row ? piv[x][k] : t[x][k];
    const int32_t b = row ? t[k][y] : piv[k][y];
    __syncthreads();
    const int32_t nv = relax(cur, a, b);
    if (nv != cur) {
      cur = nv;
      t[x][y] = cur;
    }
  }
  if (i < n && j < n) m[(int64_t)i * n + j] = cur;
}

// phase 3: every other tile from the final panels; 32 x 8 threads, four
// rows each
__global__ void __launch_bounds__(256) apsp_phase3_kernel(int32_t* w, int n, int kb) {
  __shared__ int32_t colp[APSP_T][APSP_T + 1];  // (i-tile, kb)
  __shared__ int32_t rowp[APSP_T][APSP_T + 1];  // (kb, j-tile)
  int32_t* m = w + (int64_t)blockIdx.x * n * n;
  const int ti = blockIdx.y + (blockIdx.y >= kb ? 1 : 0);
  const int tj = blockIdx.z + (blockIdx.z >= kb ? 1 : 0);
  const int y = threadIdx.x;
  for (int r = threadIdx.y; r < APSP_T; r += 8) {
    colp[r][y] = tile_get(m, n, ti * APSP_T + r, kb * APSP_T + y);
    rowp[r][y] = tile_get(m, n, kb * APSP_T + r, tj * APSP_T + y);
  }
  __syncthreads();
  const int j = tj * APSP_T + y;
  int32_t cur[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) cur[q] = tile_get(m, n, ti * APSP_T + threadIdx.y + 8 * q, j);
  for (int k = 0; k < APSP_T; ++k) {
    const int32_t b = rowp[k][y];
#pragma unroll
    for (int q = 0; q < 4; ++q) cur[q] = relax(cur[q], colp[threadIdx.y + 8 * q][k], b);
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = ti * APSP_T + threadIdx.y + 8 * q;
    if (i < n && j < n) m[(int64_t)i * n + j] = cur[q];
  }
}

}  // namespace tmol_b200

using namespace tmol_b200;

#define BS_CK(x)                                        \
  do {                                                  \
    if ((x) != cudaSuccess) return TMOL_B200_ERR_CUDA;  \
  } while (0)

extern "C" {

int tmol_b200_pose_bondsep(const tmol_b200_pose_connectivity* conn, int32_t* inter_block_bondsep,
                           int32_t* min_bondsep, int32_t* status, void* stream) {
  if (!conn || !status) return TMOL_B200_ERR_INVALID_ARGUMENT;
  const tmol_b200_pose_connectivity& c = *conn;
  if (c.n_poses < 0 || c.max_n_blocks < 0 || c.n_block_types < 0 || c.max_n_conn < 1 || c.max_n_conn > 8)
    return TMOL_B200_ERR_SHAPE;
  if (c.max_n_blocks >= (1 << 27)) return TMOL_B200_ERR_SHAPE;
  const int64_t PB = (int64_t)c.n_poses * c.max_n_blocks;
  if (PB > 0 && (!c.block_type_ind || !c.inter_residue_connections || !c.bt_n_conn || !c.bt_conn_sep))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n_pair = PB * c.max_n_blocks;
  const int64_t n_ibb = n_pair * c.max_n_conn * c.max_n_conn;
  int dev = 0, n_sm = 148;
  BS_CK(cudaGetDevice(&dev));
  BS_CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  BS_CK(cudaMemsetAsync(status, 0, sizeof(int32_t), st));
  const int fill_grid = n_sm * 8;
  if (inter_block_bondsep && n_ibb > 0) {
    fill_i32_kernel<<<fill_grid, 256, 0, st>>>(inter_block_bondsep, n_ibb, MAX_SIG_SEP);
    BS_CK(cudaGetLastError());
  }
  if (min_bondsep && n_pair > 0) {
    fill_i32_kernel<<<fill_grid, 256, 0, st>>>(min_bondsep, n_pair, MAX_SIG_SEP);
    BS_CK(cudaGetLastError());
  }
  if (PB == 0) return TMOL_B200_OK;
  const int64_t n_src = PB * c.max_n_conn;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n_src + 127) / 128, (int64_t)n_sm * 16));
  bondsep_sources_kernel<<<grid, 128, 0, st>>>(pose_conn(c), inter_block_bondsep, min_bondsep, status);
  BS_CK(cudaGetLastError());
  bondsep_status_kernel<<<1, 1, 0, st>>>(status);
  BS_CK(cudaGetLastError());
  return TMOL_B200_OK;
}

int tmol_b200_apsp_stacked(int32_t* weights, int32_t n_graphs, int32_t n_nodes, int32_t cutoff,
                           void* stream) {
  if (n_graphs < 0 || n_nodes < 0 || cutoff < -1) return TMOL_B200_ERR_SHAPE;
  if (n_graphs > 65535) return TMOL_B200_ERR_SHAPE;  // graphs index the grid's x
  if (n_graphs == 0 || n_nodes == 0) return TMOL_B200_OK;
  if (!weights) return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = (n_nodes + APSP_T - 1) / APSP_T;
  if (nb - 1 > 65535) return TMOL_B200_ERR_SHAPE;
  if (cutoff >= 0) {
    dim3 blk(32, 8), grd(nb, (n_nodes + 7) / 8, n_graphs);
    if ((n_nodes + 7) / 8 > 65535) return TMOL_B200_ERR_SHAPE;
    apsp_prepare_kernel<<<grd, blk, 0, st>>>(weights, n_nodes, cutoff);
    BS_CK(cudaGetLastError());
  }
  for (int kb = 0; kb < nb; ++kb) {
    apsp_phase1_kernel<<<n_graphs, dim3(APSP_T, APSP_T), 0, st>>>(weights, n_nodes, kb);
    BS_CK(cudaGetLastError());
    if (nb > 1) {
      apsp_phase2_kernel<<<dim3(n_graphs, nb - 1, 2), dim3(APSP_T, APSP_T), 0, st>>>(weights, n_nodes, kb);
      BS_CK(cudaGetLastError());
      apsp_phase3_kernel<<<dim3(n_graphs, nb - 1, nb - 1), dim3(APSP_T, 8), 0, st>>>(weights, n_nodes, kb);
      BS_CK(cudaGetLastError());
    }
  }
  if (cutoff >= 0) {
    const int64_t total = (int64_t)n_graphs * n_nodes * n_nodes;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 16));
    apsp_finish_kernel<<<grid, 256, 0, st>>>(weights, total, cutoff);
    BS_CK(cudaGetLastError());
  }
  return TMOL_B200_OK;
}

}  // extern "C"
