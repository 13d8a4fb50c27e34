// Learned block-pair screen: BF16-in / FP32-accumulate kernels for training
// and inference of a small MLP (32 -> 128 -> 128 -> 128 -> 1), and the
// pass that turns its predictions into a skip mask for the scoring kernel.
//
// The MLP predicts an upper quantile of log10(|E_atr| + |E_rep| + |E_lk|)
// of a neighbouring block pair from block-pair features (sphere gap,
// centroid distance, radii, sequence separation, first-atom distances,
// sub-sphere gaps and learned block-type embeddings); block pairs predicted
// below a threshold are skipped.  Intra-block pairs and pairs within count-pair reach (bond
// separation <= 4) are never candidates, so the screen never changes the
// count-pair structure.
//
// Training GEMM: C[M, N] = sum_k A(m, k) B(k, n), A and B bf16 addressed
// through (row stride, column stride) so that transposed operands cost
// nothing; 64 x 64 x 32 tiles, four warps of 32 x 32, mma.sync.m16n8k16
// with fp32 accumulators; the epilogue adds a bias, applies ReLU and writes
// fp32 and/or bf16, or accumulates atomically (split-K over a long K).
//
// Inference: one fused kernel per batch of candidate pairs; the weights sit
// in shared memory, each warp carries 16 pairs through all four layers with
// the activations in registers (an m16n8 accumulator pair is exactly the
// next layer's m16k16 operand), and the last layer sets the skip bits.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>

#include "../../include/tmol_b200_screen.h"

namespace tmol_b200 {
namespace screen {

constexpr int BM = 64, BN = 64, BK = 32;
constexpr int PAD = 8;
constexpr int F_IN = 32, HID = 128, EMB = 10, N_SCAL = 12;

struct GemmArgs {
  const __nv_bfloat16* A;
  int64_t a_rs, a_cs;
  const __nv_bfloat16* B;
  int64_t b_rs, b_cs;
  float* C;  // fp32 out (row stride c_rs) or null
  int64_t c_rs;
  __nv_bfloat16* Cb;  // bf16 out (row stride cb_rs) or null
  int64_t cb_rs;
  const float* bias;  // [N] or null
  int M, N, K;
  int relu;
  int accumulate;  // atomicAdd into C (split-K)
  int k_chunk;     // K range per blockIdx.z
};

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ uint32_t pack2f(float lo, float hi) {
  return pack2(__float2bfloat16(lo), __float2bfloat16(hi));
}

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4],
                                         const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(128) gemm_bf16_kernel(GemmArgs g) {
  __shared__ __align__(16) __nv_bfloat16 As[BM][BK + PAD];  // [m][k]
  __shared__ __align__(16) __nv_bfloat16 Bs[BN][BK + PAD];  // [n][k]
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int wm = warp >> 1, wn = warp & 1;  // 2 x 2 warps of 32 x 32
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int k_begin = blockIdx.z * g.k_chunk;
  const int k_end = min(g.K, k_begin + g.k_chunk);
  const int gid = lane >> 2, tig = lane & 3;
  float acc[2][4][4] = {};
  const __nv_bfloat16 zero = __float2bfloat16(0.0f);
  for (int k0 = k_begin; k0 < k_end; k0 += BK) {
    for (int e = tid; e < BM * BK; e += blockDim.x) {
      int r = e / BK, c = e - r * BK;
      int m = m0 + r, k = k0 + c;
      As[r][c] = (m < g.M && k < k_end) ? g.A[m * g.a_rs + (int64_t)k * g.a_cs] : zero;
    }
    for (int e = tid; e < BN * BK; e += blockDim.x) {
      int r = e / BK, c = e - r * BK;
      int n = n0 + r, k = k0 + c;
      Bs[r][c] = (n < g.N && k < k_end) ? g.B[(int64_t)k * g.b_rs + n * g.b_cs] : zero;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      uint32_t af[2][4], bf[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        int r = wm * 32 + i * 16 + gid;
        af[i][0] = pack2(As[r][kk + 2 * tig], As[r][kk + 2 * tig + 1]);
        af[i][1] = pack2(As[r + 8][kk + 2 * tig], As[r + 8][kk + 2 * tig + 1]);
        af[i][2] = pack2(As[r][kk + 2 * tig + 8], As[r][kk + 2 * tig + 9]);
        af[i][3] = pack2(As[r + 8][kk + 2 * tig + 8], As[r + 8][kk + 2 * tig + 9]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int n = wn * 32 + j * 8 + gid;
        bf[j][0] = pack2(Bs[n][kk + 2 * tig], Bs[n][kk + 2 * tig + 1]);
        bf[j][1] = pack2(Bs[n][kk + 2 * tig + 8], Bs[n][kk + 2 * tig + 9]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bf[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        int m = m0 + wm * 32 + i * 16 + gid + (q >= 2 ? 8 : 0);
        int n = n0 + wn * 32 + j * 8 + 2 * tig + (q & 1);
        if (m >= g.M || n >= g.N) continue;
        float v = acc[i][j][q];
        if (g.accumulate) {
          atomicAdd(&g.C[m * g.c_rs + n], v);
          continue;
        }
        if (g.bias) v += g.bias[n];
        if (g.relu) v = v > 0.0f ? v : 0.0f;
        if (g.C) g.C[m * g.c_rs + n] = v;
        if (g.Cb) g.Cb[m * g.cb_rs + n] = __float2bfloat16(v);
      }
}

// dZ = dH * (H > 0) for a ReLU layer, written as bf16 (and fp32 if given).
__global__ void relu_backward_kernel(const float* dH, const __nv_bfloat16* H,
                                     __nv_bfloat16* dZb, float* dZ, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float v = __bfloat162float(H[i]) > 0.0f ? dH[i] : 0.0f;
    dZb[i] = __float2bfloat16(v);
    if (dZ) dZ[i] = v;
  }
}

// Column sums of an [N, M] fp32 matrix, added into db[M] (atomic across
// blocks; db must start at zero).
__global__ void col_sum_kernel(const float* X, int64_t N, int M, float* db) {
  int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= M) return;
  float s = 0;
  for (int64_t r = blockIdx.y; r < N; r += gridDim.y) s += X[r * M + col];
  atomicAdd(&db[col], s);
}

// Pinball (quantile) loss of prediction p against target y at quantile tau,
// averaged over n: loss_i = max(tau (y - p), (tau - 1)(y - p)),
// dloss/dp_i = (-tau or 1 - tau) / n; the mean loss is added to loss[0].
__global__ void pinball_kernel(const float* pred, const float* y, int64_t n,
                               float tau, float* dpred, __nv_bfloat16* dpred_b,
                               float* loss) {
  float local = 0;
  float inv_n = 1.0f / (float)n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float r = y[i] - pred[i];
    float l = r >= 0 ? tau * r : (tau - 1.0f) * r;
    float d = (r >= 0 ? -tau : (1.0f - tau)) * inv_n;
    local += l;
    dpred[i] = d;
    dpred_b[i] = __float2bfloat16(d);
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, local * inv_n);
}

// Adam on fp32 master weights; refreshes the bf16 copy used by the GEMMs.
__global__ void adam_kernel(float* w, const float* grad, float* m, float* v,
                            __nv_bfloat16* wb, int64_t n, float lr, float b1,
                            float b2, float eps, float c1, float c2,
                            float weight_decay) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float gi = grad[i] + weight_decay * w[i];
    float mi = b1 * m[i] + (1.0f - b1) * gi;
    float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
  }
}

// Rows of X [N, 32] (bf16): 12 scalar features, then the embeddings of the
// two block types (10 values each).
__global__ void assemble_features_kernel(const float* scal, const int32_t* bt,
                                         const float* emb, int64_t n,
                                         __nv_bfloat16* X) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * F_IN;
       e += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = e >> 5;
    int c = (int)(e & 31);
    float v;
    if (c < N_SCAL)
      v = scal[r * N_SCAL + c];
    else if (c < N_SCAL + EMB)
      v = emb[(int64_t)bt[2 * r] * EMB + (c - N_SCAL)];
    else
      v = emb[(int64_t)bt[2 * r + 1] * EMB + (c - N_SCAL - EMB)];
    X[e] = __float2bfloat16(v);
  }
}

// Embedding gradient: scatter-add the embedding columns of dX [N, 32].
__global__ void embedding_backward_kernel(const float* dX, const int32_t* bt,
                                          int64_t n, float* demb) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * 2 * EMB;
       e += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = e / (2 * EMB);
    int c = (int)(e - r * 2 * EMB);
    float v = dX[r * F_IN + N_SCAL + c];
    if (c < EMB)
      atomicAdd(&demb[(int64_t)bt[2 * r] * EMB + c], v);
    else
      atomicAdd(&demb[(int64_t)bt[2 * r + 1] * EMB + (c - EMB)], v);
  }
}

// ---------------------------------------------------------------------------
// fused inference

constexpr int INF_WARPS = 4;
constexpr int W1_LD = F_IN + 8;  // padded rows: conflict-free fragment loads
constexpr int WH_LD = HID + 8;

struct InferSmem {
  __nv_bfloat16 w1[HID][W1_LD];
  __nv_bfloat16 w2[HID][WH_LD];
  __nv_bfloat16 w3[HID][WH_LD];
  float w4[HID];
  float b1[HID], b2[HID], b3[HID];
  float b4;
  __nv_bfloat16 x[INF_WARPS][16][W1_LD];
};

struct InferArgs {
  tmol_b200_screen_weights w;
  const float* feats;
  const int32_t* pair_bt;
  const int32_t* pair_row;
  const int32_t* pair_b2;
  const int32_t* count;
  int capacity;
  float threshold;
  uint32_t* mask;
  int words_per_row;
  float* pred;
};

// acc[16][4] = A (16 x K, fragments a[K/16][4]) times W^T (W is [128][K] in
// shared memory with leading dimension ld).
template <int KSTEPS>
__device__ __forceinline__ void layer_mma(float acc[16][4], const uint32_t (*a)[4],
                                          const __nv_bfloat16* W, int ld, int lane) {
  const int gid = lane >> 2, tig = lane & 3;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
  }
#pragma unroll
  for (int ks = 0; ks < KSTEPS; ++ks) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const __nv_bfloat16* wr = W + (j * 8 + gid) * ld + ks * 16 + 2 * tig;
      uint32_t b[2];
      b[0] = *reinterpret_cast<const uint32_t*>(wr);
      b[1] = *reinterpret_cast<const uint32_t*>(wr + 8);
      mma_bf16(acc[j], a[ks], b);
    }
  }
}

// bias + ReLU, rounded to bf16 and repacked as the next layer's A operand
// (n-tiles 2s and 2s+1 of the accumulator form k-step s).
__device__ __forceinline__ void relu_to_operand(const float acc[16][4], const float* bias,
                                                uint32_t a[8][4], int lane) {
  const int tig = lane & 3;
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const int n0 = s * 16 + 2 * tig, n1 = n0 + 8;
    const float* lo = acc[2 * s];
    const float* hi = acc[2 * s + 1];
    a[s][0] = pack2f(fmaxf(lo[0] + bias[n0], 0.f), fmaxf(lo[1] + bias[n0 + 1], 0.f));
    a[s][1] = pack2f(fmaxf(lo[2] + bias[n0], 0.f), fmaxf(lo[3] + bias[n0 + 1], 0.f));
    a[s][2] = pack2f(fmaxf(hi[0] + bias[n1], 0.f), fmaxf(hi[1] + bias[n1 + 1], 0.f));
    a[s][3] = pack2f(fmaxf(hi[2] + bias[n1], 0.f), fmaxf(hi[3] + bias[n1 + 1], 0.f));
  }
}

__global__ void __launch_bounds__(INF_WARPS * 32) infer_kernel(InferArgs g) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  InferSmem& sm = *reinterpret_cast<InferSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const __nv_bfloat16* w1 = (const __nv_bfloat16*)g.w.w1;
  const __nv_bfloat16* w2 = (const __nv_bfloat16*)g.w.w2;
  const __nv_bfloat16* w3 = (const __nv_bfloat16*)g.w.w3;
  for (int e = tid; e < HID * F_IN; e += blockDim.x) sm.w1[e / F_IN][e % F_IN] = w1[e];
  for (int e = tid; e < HID * HID; e += blockDim.x) {
    sm.w2[e / HID][e % HID] = w2[e];
    sm.w3[e / HID][e % HID] = w3[e];
  }
  for (int e = tid; e < HID; e += blockDim.x) {
    sm.w4[e] = __bfloat162float(((const __nv_bfloat16*)g.w.w4)[e]);
    sm.b1[e] = g.w.b1[e];
    sm.b2[e] = g.w.b2[e];
    sm.b3[e] = g.w.b3[e];
  }
  if (tid == 0) sm.b4 = g.w.b4[0];
  __syncthreads();

  const int n = min(*g.count, g.capacity);
  const int n_tiles = (n + 15) / 16;
  const int gid = lane >> 2, tig = lane & 3;
  for (int t = blockIdx.x * INF_WARPS + warp; t < n_tiles; t += gridDim.x * INF_WARPS) {
    const int r0 = t * 16;
    // stage 16 input rows: lane handles row lane & 15, columns
    // [16 * (lane >> 4), 16 * (lane >> 4) + 16)
    {
      const int rr = lane & 15, c0 = (lane >> 4) * 16;
      const int row = r0 + rr;
      __nv_bfloat16* xr = sm.x[warp][rr];
      if (row < n) {
        const float* f = g.feats + (int64_t)row * N_SCAL;
        const float* e1 = g.w.emb + (int64_t)g.pair_bt[2 * row] * EMB;
        const float* e2 = g.w.emb + (int64_t)g.pair_bt[2 * row + 1] * EMB;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const int c = c0 + k;
          const float v = c < N_SCAL ? f[c] : (c < N_SCAL + EMB ? e1[c - N_SCAL] : e2[c - N_SCAL - EMB]);
          xr[c] = __float2bfloat16(v);
        }
      } else {
#pragma unroll
        for (int k = 0; k < 16; ++k) xr[c0 + k] = __float2bfloat16(0.0f);
      }
    }
    __syncwarp();
    uint32_t a[8][4];
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
      const __nv_bfloat16* x0 = &sm.x[warp][gid][ks * 16 + 2 * tig];
      const __nv_bfloat16* x8 = &sm.x[warp][gid + 8][ks * 16 + 2 * tig];
      a[ks][0] = *reinterpret_cast<const uint32_t*>(x0);
      a[ks][1] = *reinterpret_cast<const uint32_t*>(x8);
      a[ks][2] = *reinterpret_cast<const uint32_t*>(x0 + 8);
      a[ks][3] = *reinterpret_cast<const uint32_t*>(x8 + 8);
    }
    __syncwarp();
    float acc[16][4];
    layer_mma<2>(acc, a, &sm.w1[0][0], W1_LD, lane);
    relu_to_operand(acc, sm.b1, a, lane);
    layer_mma<8>(acc, a, &sm.w2[0][0], WH_LD, lane);
    relu_to_operand(acc, sm.b2, a, lane);
    layer_mma<8>(acc, a, &sm.w3[0][0], WH_LD, lane);
    // layer 4: bias + ReLU of layer 3 (rounded to bf16 like the training
    // path's stored activation), dotted with w4 over this lane's columns
    float s0 = 0.f, s8 = 0.f;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int c0 = j * 8 + 2 * tig;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int c = c0 + q;
        float h0 = __bfloat162float(__float2bfloat16(fmaxf(acc[j][q] + sm.b3[c], 0.f)));
        float h8 = __bfloat162float(__float2bfloat16(fmaxf(acc[j][2 + q] + sm.b3[c], 0.f)));
        s0 += h0 * sm.w4[c];
        s8 += h8 * sm.w4[c];
      }
    }
    s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
    s0 += __shfl_xor_sync(0xffffffffu, s0, 2);
    s8 += __shfl_xor_sync(0xffffffffu, s8, 1);
    s8 += __shfl_xor_sync(0xffffffffu, s8, 2);
    if (tig == 0) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = r0 + gid + 8 * h;
        if (row >= n) continue;
        const float p = (h ? s8 : s0) + sm.b4;
        if (g.pred) g.pred[row] = p;
        if (g.mask && p < g.threshold) {
          const int b2 = g.pair_b2[row];
          atomicOr(&g.mask[(int64_t)g.pair_row[row] * g.words_per_row + (b2 >> 5)],
                   1u << (b2 & 31));
        }
      }
    }
  }
}

}  // namespace screen
}  // namespace tmol_b200

using namespace tmol_b200::screen;

namespace {
constexpr int kMaxDevices = 64;
int g_infer_n_sm[kMaxDevices] = {};
std::mutex g_infer_mutex;

inline int grid_for(int64_t work, int cap) {
  int64_t g = (work + 255) / 256;
  return (int)(g < cap ? (g < 1 ? 1 : g) : cap);
}
}  // namespace

extern "C" {

int tmol_b200_screen_gemm(const void* A, int64_t a_rs, int64_t a_cs,
                          const void* B, int64_t b_rs, int64_t b_cs, float* C,
                          int64_t c_rs, void* Cb, int64_t cb_rs,
                          const float* bias, int32_t M, int32_t N, int32_t K,
                          int32_t relu, int32_t accumulate, int32_t k_split,
                          void* stream) {
  if (!A || !B || (!C && !Cb) || M < 0 || N < 0 || K < 0)
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (accumulate && !C) return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (M == 0 || N == 0) return TMOL_B200_OK;
  if (k_split < 1) k_split = 1;
  GemmArgs g;
  g.A = (const __nv_bfloat16*)A;
  g.a_rs = a_rs;
  g.a_cs = a_cs;
  g.B = (const __nv_bfloat16*)B;
  g.b_rs = b_rs;
  g.b_cs = b_cs;
  g.C = C;
  g.c_rs = c_rs;
  g.Cb = (__nv_bfloat16*)Cb;
  g.cb_rs = cb_rs;
  g.bias = bias;
  g.M = M;
  g.N = N;
  g.K = K;
  g.relu = relu;
  g.accumulate = accumulate;
  int chunk = (K + k_split - 1) / k_split;
  chunk = ((chunk + BK - 1) / BK) * BK;
  if (chunk == 0) chunk = BK;
  g.k_chunk = chunk;
  int kz = (K + chunk - 1) / chunk;
  if (kz < 1) kz = 1;
  if (!accumulate && kz > 1) return TMOL_B200_ERR_INVALID_ARGUMENT;
  if ((N + BN - 1) / BN > 65535 * 32 || (M + BM - 1) / BM > 65535 || kz > 65535)
    return TMOL_B200_ERR_SHAPE;
  dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM, kz);
  gemm_bf16_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(g);
  return cudaGetLastError() == cudaSuccess ? TMOL_B200_OK : TMOL_B200_ERR_CUDA;
}

int tmol_b200_screen_relu_backward(const float* dH, const void* H, void* dZb,
                                   float* dZ, int64_t n, void* stream) {
  if (!dH || !H || !dZb || n < 0) return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (n == 0) return TMOL_B200_OK;
  relu_backward_kernel<<<grid_for(n, 4096), 256, 0, (cudaStream_t)stream>>>(
      dH, (const __nv_bfloat16*)H, (__nv_bfloat16*)dZb, dZ, n);
  return cudaGetLastError() == cudaSuccess ? TMOL_B200_OK : TMOL_B200_ERR_CUDA;
}

int tmol_b200_screen_col_sum(const float* X, int64_t N, int32_t M, float* db,
                             void* stream) {
  if (!X || !db || N < 0 || M < 0) return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (N == 0 || M == 0) return TMOL_B200_OK;
  dim3 grid((M + 127) / 128, (unsigned)(N < 1024 ? N : 1024));
  col_sum_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(X, N, M, db);
  return cudaGetLastError() == cudaSuccess ? TMOL_B200_OK : TMOL_B200_ERR_CUDA;
}

int tmol_b200_screen_pinball(const float* pred, const float* y, int64_t n,
                             float tau, float* dpred, void* dpred_b,
                             float* loss, void* stream) {
  if (!pred || !y || !dpred || !dpred_b || !loss || n < 0)
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (n == 0) return TMOL_B200_OK;
  pinball_kernel<<<grid_for(n, 2048), 256, 0, (cudaStream_t)stream>>>(
      pred, y, n, tau, dpred, (__nv_bfloat16*)dpred_b, loss);
  return cudaGetLastError() == cudaSuccess ? TMOL_B200_OK : TMOL_B200_ERR_CUDA;
}

int tmol_b200_screen_adam(float* w, const float* grad, float* m, float* v,
                          void* wb, int64_t n, float lr, float b1, float b2,
                          float eps, int32_t step, float weight_decay,
                          void* stream) {
  if (!w || !grad || !m || !v || step < 1 || n < 0) return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (n == 0) return TMOL_B200_OK;
  // bias corrections, in double on the host
  float c1 = (float)(1.0 - std::pow((double)b1, (double)step));
  float c2 = (float)(1.0 - std::pow((double)b2, (double)step));
  adam_kernel<<<grid_for(n, 2048), 256, 0, (cudaStream_t)stream>>>(
      w, grad, m, v, (__nv_bfloat16*)wb, n, lr, b1, b2, eps, c1, c2, weight_decay);
  return cudaGetLastError() == cudaSuccess ? TMOL_B200_OK : TMOL_B200_ERR_CUDA;
}

int tmol_b200_screen_assemble_features(const float* features,
                                       const int32_t* pair_bt,
                                       const float* emb, int64_t n, void* X,
                                       void* stream) {
  if (!features || !pair_bt || !emb || !X || n < 0) return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (n == 0) return TMOL_B200_OK;
  assemble_features_kernel<<<grid_for(n * F_IN, 4096), 256, 0, (cudaStream_t)stream>>>(
      features, pair_bt, emb, n, (__nv_bfloat16*)X);
  return cudaGetLastError() == cudaSuccess ? TMOL_B200_OK : TMOL_B200_ERR_CUDA;
}

int tmol_b200_screen_embedding_backward(const float* dX, const int32_t* pair_bt,
                                        int64_t n, float* demb, void* stream) {
  if (!dX || !pair_bt || !demb || n < 0) return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (n == 0) return TMOL_B200_OK;
  embedding_backward_kernel<<<grid_for(n * 2 * EMB, 4096), 256, 0, (cudaStream_t)stream>>>(
      dX, pair_bt, n, demb);
  return cudaGetLastError() == cudaSuccess ? TMOL_B200_OK : TMOL_B200_ERR_CUDA;
}

int tmol_b200_screen_infer(const tmol_b200_screen_weights* weights,
                           const float* features, const int32_t* pair_bt,
                           const int32_t* pair_row, const int32_t* pair_b2,
                           const int32_t* count, int32_t capacity,
                           float threshold, uint32_t* mask,
                           int32_t words_per_row, int64_t mask_words,
                           float* pred, void* stream) {
  if (!weights || !features || !pair_bt || !count || capacity < 0)
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  const tmol_b200_screen_weights& w = *weights;
  if (!w.w1 || !w.w2 || !w.w3 || !w.w4 || !w.b1 || !w.b2 || !w.b3 || !w.b4 || !w.emb)
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (mask && (!pair_row || !pair_b2 || words_per_row <= 0 || mask_words < 0))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (!mask && !pred) return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (mask && mask_words > 0 &&
      cudaMemsetAsync(mask, 0, (size_t)mask_words * sizeof(uint32_t), st) != cudaSuccess)
    return TMOL_B200_ERR_CUDA;
  if (capacity == 0) return TMOL_B200_OK;
  const int smem = (int)sizeof(InferSmem);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TMOL_B200_ERR_CUDA;
  int n_sm = 0;
  {
    // the shared-memory opt-in is set once per device, so that calls made
    // while a stream is being captured issue no attribute changes
    std::lock_guard<std::mutex> lock(g_infer_mutex);
    if (!g_infer_n_sm[dev]) {
      int v = 0;
      if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
          cudaFuncSetAttribute(infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
              cudaSuccess)
        return TMOL_B200_ERR_CUDA;
      g_infer_n_sm[dev] = v;
    }
    n_sm = g_infer_n_sm[dev];
  }
  InferArgs g;
  g.w = w;
  g.feats = features;
  g.pair_bt = pair_bt;
  g.pair_row = pair_row;
  g.pair_b2 = pair_b2;
  g.count = count;
  g.capacity = capacity;
  g.threshold = threshold;
  g.mask = mask;
  g.words_per_row = words_per_row;
  g.pred = pred;
  int tiles = (capacity + 15) / 16;
  int grid = (tiles + INF_WARPS - 1) / INF_WARPS;
  if (grid > 2 * n_sm) grid = 2 * n_sm;
  infer_kernel<<<grid, INF_WARPS * 32, smem, st>>>(g);
  return cudaGetLastError() == cudaSuccess ? TMOL_B200_OK : TMOL_B200_ERR_CUDA;
}

}  // extern "C"
