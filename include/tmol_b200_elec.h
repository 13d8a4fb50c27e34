/*
 * tmol_b200_elec: B200 (sm_100a) elec (fa_elec) scoring behind a C ABI.
 *
 * The inputs are the tensors of tmol's elec ops
 * ``torch.ops.tmol_elec.elec_pose_scores`` and ``elec_rotamer_scores``
 * (tmol/score/elec/potentials/compiled.ops.cpp:25-523, registered at
 * :650-654), passed as device pointers with their sizes.  Integer tables are
 * int32, row-major and contiguous; real tables (partial charges, global
 * parameters) are float32, or float64 for a plan created with real_bytes 8.
 *
 * An elec plan is a tmol_b200_ljlk_plan of the elec kind: it shares the LJ/LK
 * library's neighbour detection, count-pair tables, launch shape,
 * rebalancing and profiling (tmol_b200_ljlk_plan_set_launch,
 * _plan_rebalance, _profile, _profile_read, _last_counts,
 * _plan_device_bytes accept either kind), while the scoring entry points
 * below take elec plans only (and the LJ/LK ones reject them with
 * TMOL_B200_ERR_INVALID_ARGUMENT).  Energies have one term: [1, P],
 * [1, P, B, B] or [1, n_pairs].  Status codes, stream and allocation rules
 * are those of tmol_b200_ljlk.h.
 */
#ifndef TMOL_B200_ELEC_H
#define TMOL_B200_ELEC_H

#include <stddef.h>
#include <stdint.h>

#include "tmol_b200_ljlk.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tmol_b200_ljlk_plan tmol_b200_elec_plan;

/* Device pointers and sizes of the elec op's static arguments, in the
 * reference op's order (compiled.ops.cpp:28-59):
 *   n_poses = P, max_n_blocks = B, n_rots (P * B for the pose op, the
 *   rotamer count for the rotamer op), n_block_types = nbt,
 *   max_n_block_atoms = A, max_n_conn = C. */
typedef struct {
  int64_t n_atoms; /* rows of rot_coords */
  int32_t n_poses, max_n_blocks, n_rots;
  int32_t n_block_types, max_n_block_atoms, max_n_conn;

  const int32_t* rot_coord_offset;       /* [n_rots] */
  const int32_t* pose_ind_for_atom;      /* [n_atoms] (validated, unused) */
  const int32_t* first_rot_for_block;    /* [P, B] */
  const int32_t* first_rot_block_type;   /* [P, B], -1 = no block */
  const int32_t* block_ind_for_rot;      /* [n_rots] */
  const int32_t* pose_ind_for_rot;       /* [n_rots] */
  const int32_t* block_type_ind_for_rot; /* [n_rots] */
  const int32_t* n_rots_for_pose;        /* [P] */
  const int32_t* rot_offset_for_pose;    /* [P] */
  const int32_t* n_rots_for_block;       /* [P, B] */
  const int32_t* rot_offset_for_block;   /* [P, B] */
  int32_t max_n_rots_per_pose;

  const int32_t* min_bondsep;               /* [P, B, B] */
  const int32_t* inter_block_bondsep;       /* [P, B, B, C, C] */
  const int32_t* bt_n_atoms;                /* [nbt] */
  const void* bt_partial_charge;            /* [nbt, A] real */
  const int32_t* bt_n_conn;                 /* [nbt] */
  const int32_t* bt_conn_atom;              /* [nbt, C] */
  const int32_t* bt_inter_repr_path_distance; /* [nbt, A, A] */
  const int32_t* bt_intra_repr_path_distance; /* [nbt, A, A] */
  const int32_t* bt_is_ligand_fragment;     /* [nbt] */
  const void* global_params; /* [1, 5] real: D, D0, S, min_dis, max_dis */
  double max_dis;            /* neighbour-detection reach */
} tmol_b200_elec_inputs;

/* Replaces the per-call setup of ElecPoseScoreDispatch::forward
 * (tmol/score/elec/potentials/elec_pose_score.impl.hh:385-560): derives the
 * count-pair tables and the potential's constants once.  `real_bytes` is 4
 * (float32) or 8 (float64). */
int tmol_b200_elec_plan_create(const tmol_b200_elec_inputs* inputs, int real_bytes,
                               const tmol_b200_ljlk_launch* launch, void* stream,
                               tmol_b200_elec_plan** plan_out);

/* The plan of the rotamer op (any number of rotamers per block; the
 * elec_rotamer_scores setup, compiled.ops.cpp:275-399, 588-647). */
int tmol_b200_elec_rotamer_plan_create(const tmol_b200_elec_inputs* inputs, int real_bytes,
                                       const tmol_b200_ljlk_launch* launch, void* stream,
                                       tmol_b200_elec_plan** plan_out);

int tmol_b200_elec_plan_destroy(tmol_b200_elec_plan* plan);

/* Replaces ElecPoseScoreOp::forward (compiled.ops.cpp:28-149;
 * elec_pose_score.impl.hh:385-856):
 *   energies        [1, P] (block_pair == 0) or [1, P, B, B]; overwritten
 *   block_neighbors [P, B, B] int32 or NULL; overwritten when given */
int tmol_b200_elec_forward(tmol_b200_elec_plan* plan, const void* coords, int block_pair,
                           void* energies, int32_t* block_neighbors, void* stream);

/* Replaces ElecPoseScoreOp::backward (compiled.ops.cpp:150-271) with a
 * recompute adjoint (the reference's block-pair backward,
 * elec_pose_score.impl.hh:858-1125, for per-pose weights too):
 *   dTdV     [1, P] (block_pair == 0) or [1, P, B, B]
 *   dcoords  [n_atoms, 3]; overwritten */
int tmol_b200_elec_backward(tmol_b200_elec_plan* plan, const void* coords, int block_pair,
                            const void* dTdV, void* dcoords, void* stream);

/* The elec pose op's autograd pair with a speculative gradient, as
 * tmol_b200_ljlk_forward_speculative / _backward_speculative (no
 * counterpart in the reference). */
int tmol_b200_elec_forward_speculative(tmol_b200_elec_plan* plan, const void* coords,
                                       void* energies, int32_t* block_neighbors, void* stream);
int tmol_b200_elec_backward_speculative(tmol_b200_elec_plan* plan, const void* coords,
                                        const void* dTdV, void* dcoords, int speculated,
                                        void* stream);

/* Energies [1, P] and weights[0, pose] * dE/dcoords in one pass. */
int tmol_b200_elec_energy_and_gradient(tmol_b200_elec_plan* plan, const void* coords,
                                       const void* weights, void* energies, void* dcoords,
                                       void* stream);

/* Rotamer scoring (elec_rotamer_scores; ElecRotamerScoreDispatch,
 * elec_pose_score.impl.hh:1127-1699),
 * as tmol_b200_ljlk_rotamer_count / _fill / _forward / _backward with one
 * energy term: energies and dTdV are [1, n_pairs]. */
int tmol_b200_elec_rotamer_count(tmol_b200_elec_plan* plan, const void* coords,
                                 int64_t* n_pairs, int64_t* n_items, void* stream);
int tmol_b200_elec_rotamer_fill(tmol_b200_elec_plan* plan, int32_t* indices, int32_t* items,
                                void* stream);
int tmol_b200_elec_rotamer_forward(tmol_b200_elec_plan* plan, const void* coords,
                                   const int32_t* items, int64_t n_items, int64_t n_pairs,
                                   void* energies, void* stream);
int tmol_b200_elec_rotamer_backward(tmol_b200_elec_plan* plan, const void* coords,
                                    const int32_t* items, int64_t n_items, int64_t n_pairs,
                                    const void* dTdV, void* dcoords, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TMOL_B200_ELEC_H */
