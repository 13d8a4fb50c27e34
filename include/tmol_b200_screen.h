/*
 * tmol_b200_screen: learned block-pair screen for the LJ + LK scoring path.
 *
 * No counterpart in the reference: tmol scores every block pair whose
 * bounding spheres come within the interaction reach
 * (tmol/score/common/sphere_overlap.impl.hh:287-351).  The screen is a small
 * MLP (32 -> 128 -> 128 -> 128 -> 1, ReLU, bf16 weights and activations,
 * fp32 accumulation) that predicts an upper quantile of
 * log10(|E_atr| + |E_rep| + |E_lk| + 1e-6) of a candidate block pair; pairs
 * predicted below a threshold are skipped by the scoring kernel through a
 * per-row bit mask.  Intra-block pairs and count-pair partners (bond
 * separation <= 4) are never candidates and are never skipped.
 *
 * Candidate features (12 fp32 per pair), from the block spheres (centroid
 * c, radius r), d = |c1 - c2|, each block's first atom a and its two
 * sub-spheres u0 (atoms 0-3: N, CA, C, O of an amino acid) and u1 (the
 * other atoms; u0 again for blocks of <= 4 atoms):
 *   d/10, (d - r1 - r2)/6, r1/5, r2/5, log2(b2 - b1)/10,
 *   (|a1 - a2| - d)/5, (|a1 - c2| - d)/5, (|a2 - c1| - d)/5,
 *   sub-sphere gaps (|u1_i - u2_j| - r - r)/6 for (i, j) = (0,0), (0,1),
 *   (1,0), (1,1)
 * followed in the network input by the 10-value embeddings of both block
 * types.
 *
 * All pointers are device pointers; every call enqueues work on `stream`
 * and returns a tmol_b200_status code.
 */
#ifndef TMOL_B200_SCREEN_H
#define TMOL_B200_SCREEN_H

#include "tmol_b200_ljlk.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Network parameters (torch Linear layout: weight [out, in] row-major).
 *   w1 bf16 [128, 32], w2 bf16 [128, 128], w3 bf16 [128, 128], w4 bf16 [128]
 *   b1, b2, b3 fp32 [128], b4 fp32 [1], emb fp32 [n_block_types, 10] */
typedef struct {
  const void* w1;
  const void* w2;
  const void* w3;
  const void* w4;
  const float* b1;
  const float* b2;
  const float* b3;
  const float* b4;
  const float* emb;
} tmol_b200_screen_weights;

/* Install (mask != NULL) or remove (mask == NULL) a skip mask for every
 * later scoring call of the plan: bit (b2 & 31) of word
 * mask[(p * B + b1) * words_per_row + (b2 >> 5)] set = do not score block
 * pair (b1, b2), b1 < b2, of pose p.  words_per_row >= ceil(B / 32).  Bits of
 * the diagonal and of count-pair partners are ignored.  The mask stays
 * owned by the caller and must outlive its use. */
int tmol_b200_ljlk_plan_set_skip_mask(tmol_b200_ljlk_plan* plan,
                                      const uint32_t* mask,
                                      int32_t words_per_row);

/* Screen candidates of the plan's PoseStack at `coords`: every block pair
 * b1 < b2 that passes the scoring kernel's sphere test and is not a
 * count-pair partner.  Writes pair_row[i] = p * B + b1, pair_b2[i] = b2,
 * pair_bt[2 i], pair_bt[2 i + 1] = the block types and features[12 i ..
 * 12 i + 11] for i < min(*count, capacity); *count (device) ends as the number of
 * candidates, which may exceed capacity.  float32 plans only. */
int tmol_b200_ljlk_screen_candidates(tmol_b200_ljlk_plan* plan,
                                     const void* coords, int32_t capacity,
                                     int32_t* pair_row, int32_t* pair_b2,
                                     int32_t* pair_bt, float* features,
                                     int32_t* count, void* stream);

/* Fused inference: predictions for the first min(*count, capacity)
 * candidates; writes pred[i] when pred != NULL and, when mask != NULL,
 * clears mask[0 .. mask_words) and sets the bit of every candidate with
 * pred < threshold. */
int tmol_b200_screen_infer(const tmol_b200_screen_weights* weights,
                           const float* features, const int32_t* pair_bt,
                           const int32_t* pair_row, const int32_t* pair_b2,
                           const int32_t* count, int32_t capacity,
                           float threshold, uint32_t* mask,
                           int32_t words_per_row, int64_t mask_words,
                           float* pred, void* stream);

/* Training building blocks. */

/* C[m, n] (+)= sum_k A(m, k) B(k, n) with A(m, k) = A[m a_rs + k a_cs] and
 * B(k, n) = B[k b_rs + n b_cs] (bf16).  Unless `accumulate`, the epilogue
 * adds bias[n] (if given), applies ReLU (if relu) and writes C (fp32, row
 * stride c_rs) and/or Cb (bf16, row stride cb_rs).  With `accumulate` the
 * product is atomically added to C and K may be split over k_split CTAs. */
int tmol_b200_screen_gemm(const void* A, int64_t a_rs, int64_t a_cs,
                          const void* B, int64_t b_rs, int64_t b_cs, float* C,
                          int64_t c_rs, void* Cb, int64_t cb_rs,
                          const float* bias, int32_t M, int32_t N, int32_t K,
                          int32_t relu, int32_t accumulate, int32_t k_split,
                          void* stream);

/* dZ = dH * (H > 0): bf16 into dZb and, if dZ != NULL, fp32 into dZ. */
int tmol_b200_screen_relu_backward(const float* dH, const void* H, void* dZb,
                                   float* dZ, int64_t n, void* stream);

/* db[m] += sum_r X[r, m] for X [N, M] fp32. */
int tmol_b200_screen_col_sum(const float* X, int64_t N, int32_t M, float* db,
                             void* stream);

/* Mean pinball loss at quantile tau (added to *loss) and its gradient
 * dpred (fp32) / dpred_b (bf16). */
int tmol_b200_screen_pinball(const float* pred, const float* y, int64_t n,
                             float tau, float* dpred, void* dpred_b,
                             float* loss, void* stream);

/* One Adam step (bias-corrected for `step` >= 1, L2 weight decay added to
 * the gradient) on fp32 weights w, refreshing the bf16 copy wb if given. */
int tmol_b200_screen_adam(float* w, const float* grad, float* m, float* v,
                          void* wb, int64_t n, float lr, float b1, float b2,
                          float eps, int32_t step, float weight_decay,
                          void* stream);

/* X [n, 32] bf16 = [features (12), emb[pair_bt[2 i]] (10),
 * emb[pair_bt[2 i + 1]] (10)]. */
int tmol_b200_screen_assemble_features(const float* features,
                                       const int32_t* pair_bt,
                                       const float* emb, int64_t n, void* X,
                                       void* stream);

/* demb[bt] += the embedding columns of dX [n, 32] (fp32) for each pair. */
int tmol_b200_screen_embedding_backward(const float* dX, const int32_t* pair_bt,
                                        int64_t n, float* demb, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TMOL_B200_SCREEN_H */
