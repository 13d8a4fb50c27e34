/*
 * tmol_b200_lkball: B200 (sm_100a) LK-ball scoring behind a C ABI: water
 * generation and the four-term score (lk_ball_iso, lk_ball, lk_bridge,
 * lk_bridge_uncpl).
 *
 * The inputs are the tensors of tmol's LK-ball ops
 * ``torch.ops.tmol_lk_ball.gen_pose_waters`` and ``lk_ball_pose_score``
 * (tmol/score/lk_ball/potentials/compiled.ops.cpp:25-987, registered at
 * :978-982), as device pointers with their sizes: int32 tables row-major;
 * reals float32, or float64 for a plan created with real_bytes 8.  A plan
 * is a tmol_b200_ljlk_plan of the LK-ball kind (the launch, rebalance,
 * profiling and counter helpers of tmol_b200_ljlk.h accept it); the entry
 * points below take LK-ball plans only.  Status codes, stream and
 * allocation rules are those of tmol_b200_ljlk.h.
 *
 * Waters are [n_atoms, 4, 3]: up to four per polar atom (NaN in unused
 * slots), as the reference lays them out.
 */
#ifndef TMOL_B200_LKBALL_H
#define TMOL_B200_LKBALL_H

#include <stddef.h>
#include <stdint.h>

#include "tmol_b200_ljlk.h"
#include "tmol_b200_pose.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tmol_b200_ljlk_plan tmol_b200_lkball_plan;

/* The static arguments of both ops (compiled.ops.cpp:27-64, 363-398):
 *   P = n_poses, B = max_n_blocks, nbt = n_block_types,
 *   A = max_n_block_atoms, C = max_n_conn, NT = max_n_tiles (ceil(A/32)),
 *   NB = max_n_all_bonds. */
typedef struct {
  int64_t n_atoms;
  int32_t n_poses, max_n_blocks, n_rots;
  int32_t n_block_types, max_n_block_atoms, max_n_conn, max_n_tiles, max_n_all_bonds;

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

  const int32_t* inter_residue_connections; /* [P, B, C, 2] */
  const int32_t* min_bondsep;               /* [P, B, B] */
  const int32_t* inter_block_bondsep;       /* [P, B, B, C, C] */
  const int32_t* bt_n_atoms;                /* [nbt] */
  const int32_t* bt_n_conn;                 /* [nbt] */
  const int32_t* bt_conn_atom;              /* [nbt, C] */

  /* water generation (gen_pose_waters) */
  const int32_t* bt_n_all_bonds;            /* [nbt] */
  const int32_t* bt_all_bonds;              /* [nbt, NB, 3] */
  const int32_t* bt_atom_all_bond_ranges;   /* [nbt, A, 2] */
  const int32_t* bt_tile_n_donH;            /* [nbt, NT] */
  const int32_t* bt_tile_n_acc;             /* [nbt, NT] */
  const int32_t* bt_tile_donH_inds;         /* [nbt, NT, 32] */
  const int32_t* bt_tile_donH_hvy_inds;     /* [nbt, NT, 32] */
  const int32_t* bt_tile_which_donH_for_hvy;/* [nbt, NT, 32] */
  const int32_t* bt_tile_acc_inds;          /* [nbt, NT, 32] */
  const int32_t* bt_tile_hybridization;     /* [nbt, NT, 32] */
  const int32_t* bt_tile_acc_n_attached_H;  /* [nbt, NT, 32] */
  const int32_t* bt_atom_is_hydrogen;       /* [nbt, A] */
  const void* water_gen_global_params;      /* [1, 4] real: distance, sp2 / sp3 / ring angles */
  const void* sp2_water_tors;               /* [n_sp2] real */
  const void* sp3_water_tors;               /* [n_sp3] real */
  const void* ring_water_tors;              /* [n_ring] real */
  int32_t n_sp2_tors, n_sp3_tors, n_ring_tors;

  /* scoring (lk_ball_pose_score) */
  const int32_t* bt_tile_n_polar_atoms;     /* [nbt, NT] */
  const int32_t* bt_tile_n_occluder_atoms;  /* [nbt, NT] */
  const int32_t* bt_tile_pol_occ_inds;      /* [nbt, NT, 32] */
  const void* bt_tile_lk_ball_params;       /* [nbt, NT, 32, 9] real */
  const int32_t* bt_path_distance;          /* [nbt, A, A] */
  const void* global_params;                /* [1, 5] real: hbond, OH-donor, H distances, water distance, max_dis */
  double max_dis;                           /* neighbour-detection reach */
} tmol_b200_lkball_inputs;

/* Replaces the per-call setup of both dispatches (gen_pose_waters.impl.hh:
 * 35-130, lk_ball_pose_score.impl.hh:362-470): validates the tables and
 * resolves every water's building atoms (acceptor bases across block
 * connections, tmol/score/hbond/identification.hh:26-168) once.
 *
 * A plan serves water generation when bt_all_bonds is given (with the other
 * water-generation tables), scoring when bt_tile_pol_occ_inds is given
 * (with the other scoring tables, the bond separations and global_params),
 * or both; the tables of the part left out may be NULL, and its entry
 * points then return TMOL_B200_ERR_INVALID_ARGUMENT.  This is how the two
 * reference ops, which take different argument lists, map onto plans. */
int tmol_b200_lkball_plan_create(const tmol_b200_lkball_inputs* inputs, int real_bytes,
                                 const tmol_b200_ljlk_launch* launch, void* stream,
                                 tmol_b200_lkball_plan** plan_out);
int tmol_b200_lkball_plan_destroy(tmol_b200_lkball_plan* plan);

/* The same plan built from the PoseStack's connectivity
 * (include/tmol_b200_pose.h) instead of the dense min_bondsep /
 * inter_block_bondsep tensors, which may then be NULL (the count-pair
 * tables come straight from the connectivity, as for the LJ/LK and elec
 * plans); `rotamers` selects a rotamer plan. */
int tmol_b200_lkball_plan_create_from_connectivity(const tmol_b200_lkball_inputs* inputs,
                                                   const tmol_b200_pose_connectivity* conn, int real_bytes,
                                                   const tmol_b200_ljlk_launch* launch, void* stream, int rotamers,
                                                   tmol_b200_lkball_plan** plan_out);

/* gen_pose_waters forward (GeneratePoseWaters::forward,
 * gen_pose_waters.impl.hh:35-230): waters [n_atoms, 4, 3], overwritten. */
int tmol_b200_lkball_waters(tmol_b200_lkball_plan* plan, const void* coords, void* waters, void* stream);

/* gen_pose_waters backward (GeneratePoseWaters::backward,
 * gen_pose_waters.impl.hh:231-440): dcoords
 * [n_atoms, 3] += the adjoint of dL/dwaters [n_atoms, 4, 3] (accumulated,
 * not overwritten). */
int tmol_b200_lkball_waters_backward(tmol_b200_lkball_plan* plan, const void* coords,
                                     const void* dwaters, void* dcoords, void* stream);

/* lk_ball_pose_score forward (LKBallPoseScoreDispatch::forward,
 * lk_ball_pose_score.impl.hh:362-681): energies [4, P] (block_pair == 0)
 * or [4, P, B, B], overwritten; block_neighbors [P, B, B] or NULL. */
int tmol_b200_lkball_forward(tmol_b200_lkball_plan* plan, const void* coords, const void* waters,
                             int block_pair, void* energies, int32_t* block_neighbors, void* stream);

/* lk_ball_pose_score backward as a recompute adjoint (the reference's
 * backward, lk_ball_pose_score.impl.hh:682-1004): with
 * dTdV [4, P] or [4, P, B, B], dcoords [n_atoms, 3] and dwaters
 * [n_atoms, 4, 3] are overwritten with the gradients of sum dTdV * E with
 * respect to the coordinates (directly) and the waters. */
int tmol_b200_lkball_backward(tmol_b200_lkball_plan* plan, const void* coords, const void* waters,
                              int block_pair, const void* dTdV, void* dcoords, void* dwaters,
                              void* stream);

/* lk_ball_pose_score's forward / backward pair with a speculative gradient
 * (whole-pose mode; no counterpart in the reference, whose backward always
 * recomputes): as tmol_b200_ljlk_forward_speculative /
 * _backward_speculative, the kept gradient being both the coordinates'
 * direct part and the waters' part. */
int tmol_b200_lkball_forward_speculative(tmol_b200_lkball_plan* plan, const void* coords, const void* waters,
                                         void* energies, int32_t* block_neighbors, void* stream);
int tmol_b200_lkball_backward_speculative(tmol_b200_lkball_plan* plan, const void* coords, const void* waters,
                                          const void* dTdV, void* dcoords, void* dwaters, int speculated,
                                          void* stream);

/* Whole-pose energies and gradient in one call (a plan with both parts):
 * the waters, the four energies [4, P] (overwritten) and dcoords [n_atoms,
 * 3] (overwritten) = d(sum_t,p weights[t, p] * E[t, p]) / dcoords through
 * the waters, weights [4, P].  Equivalent to gen_pose_waters forward,
 * lk_ball_pose_score forward and backward, and gen_pose_waters backward
 * (lk_ball_energy_term.py:240-300 composes them so), with the waters and
 * their adjoint kept in the plan's scratch and one scoring pass. */
int tmol_b200_lkball_energy_and_gradient(tmol_b200_lkball_plan* plan, const void* coords, const void* weights,
                                         void* energies, void* dcoords, void* stream);

/* The rotamer op, lk_ball_rotamer_score (LKBallRotamerScoreDispatch,
 * lk_ball_pose_score.impl.hh:1005-1380; compiled.ops.cpp:604-842): a plan
 * over a rotamer set (the inputs' indexing is the set's, n_rots its
 * rotamers, coordinates and waters its atoms).  Water generation on such a
 * plan builds every rotamer's waters (gen_pose_waters on the rotamers'
 * coordinates, as tmol's rotamer scoring calls it), with atoms of other
 * blocks from those blocks' first rotamers.  count / fill give the
 * dispatched rotamer pairs (pose, rot1, rot2) and work items as
 * tmol_b200_ljlk_rotamer_count / _fill do (count synchronises the stream);
 * forward writes energies [4, n_pairs]; backward overwrites dcoords
 * [n_atoms, 3] and dwaters [n_atoms, 4, 3] with the gradients of
 * sum dTdV * E, dTdV [4, n_pairs]. */
int tmol_b200_lkball_rotamer_plan_create(const tmol_b200_lkball_inputs* inputs, int real_bytes,
                                         const tmol_b200_ljlk_launch* launch, void* stream,
                                         tmol_b200_lkball_plan** plan_out);
int tmol_b200_lkball_rotamer_count(tmol_b200_lkball_plan* plan, const void* coords, int64_t* n_pairs,
                                   int64_t* n_items, void* stream);
int tmol_b200_lkball_rotamer_fill(tmol_b200_lkball_plan* plan, int32_t* indices, int32_t* items, void* stream);
int tmol_b200_lkball_rotamer_forward(tmol_b200_lkball_plan* plan, const void* coords, const void* waters,
                                     const int32_t* items, int64_t n_items, int64_t n_pairs, void* energies,
                                     void* stream);
int tmol_b200_lkball_rotamer_backward(tmol_b200_lkball_plan* plan, const void* coords, const void* waters,
                                      const int32_t* items, int64_t n_items, int64_t n_pairs, const void* dTdV,
                                      void* dcoords, void* dwaters, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TMOL_B200_LKBALL_H */
