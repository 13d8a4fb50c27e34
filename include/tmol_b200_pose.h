/*
 * tmol_b200_pose: B200 (sm_100a) PoseStack construction steps behind a C ABI:
 * inter-block bond separation and tmol's stacked all-pairs-shortest-paths op.
 *
 * tmol builds inter_block_bondsep [P, B, B, C, C] by filling a dense
 * connection-point matrix per pose and running all-pairs shortest paths over
 * it (tmol/pose/pose_stack_builder.py:436-599, 1230-1343;
 * tmol/pose/compiled/apsp.cuda.cu, apsp.cpu.cpp).  Here the separations come
 * from a bounded search per connection point (separations are capped at 6),
 * written straight into the dense outputs or, for a scoring plan, into its
 * compact count-pair tables without any [P, B, B, C, C] tensor.
 *
 * Integer tables are int32, row-major, on the device.  Functions return a
 * tmol_b200_status (tmol_b200_ljlk.h).
 */
#ifndef TMOL_B200_POSE_H
#define TMOL_B200_POSE_H

#include <stddef.h>
#include <stdint.h>

#include "tmol_b200_elec.h"
#include "tmol_b200_ljlk.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A PoseStack's connectivity (tmol's PoseStack.block_type_ind,
 * inter_residue_connections, PackedBlockTypes.n_conn and
 * conn_at_intrablock_bond_sep). */
typedef struct {
  int32_t n_poses, max_n_blocks, n_block_types, max_n_conn; /* P, B, nbt, C (C <= 8) */
  const int32_t* block_type_ind;            /* [P, B], -1 = no block */
  const int32_t* inter_residue_connections; /* [P, B, C, 2]: (block, connection) bonded to, or -1 */
  const int32_t* bt_n_conn;                 /* [nbt] */
  const int32_t* bt_conn_sep;               /* [nbt, C, C]: bonds between connection atoms */
} tmol_b200_pose_connectivity;

/* Replaces PoseStackBuilder._calculate_interblock_bondsep_from_connectivity_graph
 * and the connection-matrix steps before it (pose_stack_builder.py:459-599,
 * 1230-1343), and BondDependentTerm's min_block_bondsep
 * (tmol/score/bond_dependent_term.py:91-100):
 *   inter_block_bondsep [P, B, B, C, C] or NULL: shortest bond count between
 *                       connection c1 of block b1 and c2 of b2, capped at 6
 *                       (6 where a slot does not exist); overwritten
 *   min_bondsep         [P, B, B] or NULL: the minimum over (c1, c2);
 *                       overwritten
 *   status              one int32 on the device, required: set, once the
 *                       enqueued work has run, to TMOL_B200_OK or to the
 *                       error the connectivity shows (TMOL_B200_ERR_INDEX_RANGE
 *                       for an index out of range, TMOL_B200_ERR_SHAPE for a
 *                       bond recorded in one direction only,
 *                       TMOL_B200_ERR_CAPACITY for more than 64 connection
 *                       points within 5 bonds of one); the outputs are
 *                       meaningful only when it reads TMOL_B200_OK
 * Enqueued on `stream`; allocates nothing, does not synchronise.  The return
 * value reports invalid arguments and launch failures only. */
int tmol_b200_pose_bondsep(const tmol_b200_pose_connectivity* conn, int32_t* inter_block_bondsep,
                           int32_t* min_bondsep, int32_t* status, void* stream);

/* Replaces tmol's stacked_apsp / tmol_apsp::apsp_op
 * (tmol/pose/compiled/apsp_ops.py:16-33, apsp.cuda.cu, apsp.cpu.cpp), in place
 * on weights [n_graphs, n_nodes, n_nodes] (-1 = no edge, other weights
 * non-negative):
 *   cutoff == -1  exact shortest paths over the directed weights (-1 where
 *                 unreachable)
 *   cutoff >= 0   the reference CPU rule: edges are symmetrised (the lighter
 *                 of w[i][j], w[j][i] where both exist) and kept only below
 *                 the cutoff; the diagonal is 0, every pair at or beyond the
 *                 cutoff (or unreachable) is set to the cutoff.
 * Enqueued on `stream`; allocates nothing, does not synchronise. */
int tmol_b200_apsp_stacked(int32_t* weights, int32_t n_graphs, int32_t n_nodes, int32_t cutoff,
                           void* stream);

/* Scoring plans whose count-pair tables come from the connectivity instead
 * of the dense min_bondsep / inter_block_bondsep arguments (which are then
 * not read and may be NULL): the same plan as tmol_b200_ljlk_plan_create /
 * tmol_b200_ljlk_rotamer_plan_create (rotamers != 0) and the elec
 * counterparts, without any [P, B, B, C, C] tensor.  conn's sizes must equal
 * the inputs' (n_poses, max_n_blocks, n_block_types, max_n_conn). */
int tmol_b200_ljlk_plan_create_from_connectivity(const tmol_b200_ljlk_inputs* inputs,
                                                 const tmol_b200_pose_connectivity* conn, int real_bytes,
                                                 const tmol_b200_ljlk_launch* launch, void* stream,
                                                 int rotamers, tmol_b200_ljlk_plan** plan_out);
int tmol_b200_elec_plan_create_from_connectivity(const tmol_b200_elec_inputs* inputs,
                                                 const tmol_b200_pose_connectivity* conn, int real_bytes,
                                                 const tmol_b200_ljlk_launch* launch, void* stream,
                                                 int rotamers, tmol_b200_elec_plan** plan_out);

#ifdef __cplusplus
}
#endif

#endif /* TMOL_B200_POSE_H */
