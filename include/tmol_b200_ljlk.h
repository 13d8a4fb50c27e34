/*
 * tmol_b200_ljlk: B200 (sm_100a) LJ + LK pose scoring behind a C ABI.
 *
 * The inputs are the tensors of tmol's pose-score op
 * ``torch.ops.tmol_ljlk.ljlk_pose_scores``
 * (tmol/score/ljlk/potentials/compiled.ops.cpp:533-597, registered at :667-670),
 * passed as device pointers with their sizes.  All integer tables are int32,
 * row-major and contiguous; real tables are float32 (or float64 through the
 * *_f64 entry points).
 *
 * Life cycle:
 *   tmol_b200_ljlk_plan_create   once per PoseStack (reads the static tables,
 *                                derives compact count-pair / parameter
 *                                tables, allocates scratch; synchronises the
 *                                stream once to validate indices)
 *   tmol_b200_ljlk_forward       energies (whole-pose [3, P] or block-pair
 *                                [3, P, B, B]) and, optionally, the dense
 *                                block-neighbour matrix [P, B, B]
 *   tmol_b200_ljlk_backward      recompute adjoint: dL/dcoords [N, 3] from
 *                                dL/dE ([3, P] or [3, P, B, B])
 *   tmol_b200_ljlk_plan_destroy
 *
 * forward/backward enqueue work on `stream`, allocate nothing and never
 * synchronise; a plan owns scratch memory, so one plan must not be used by
 * two streams at once.  Every function returns a tmol_b200_status code.
 */
#ifndef TMOL_B200_LJLK_H
#define TMOL_B200_LJLK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  TMOL_B200_OK = 0,
  TMOL_B200_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad flag */
  TMOL_B200_ERR_SHAPE = 2,            /* inconsistent or unsupported sizes */
  TMOL_B200_ERR_INDEX_RANGE = 3,      /* a table holds an out-of-range index */
  TMOL_B200_ERR_CAPACITY = 4,         /* a fixed-capacity table overflowed */
  TMOL_B200_ERR_CUDA = 5,             /* a CUDA runtime call failed */
  TMOL_B200_ERR_DTYPE = 6             /* plan and call disagree on float width */
} tmol_b200_status;

/* Device pointers and sizes of the op's static arguments (everything but
 * the coordinates and the output-mode flag).  Names and meanings follow the
 * reference op (compiled.ops.cpp:33-60):
 *   n_poses = P, max_n_blocks = B, n_rots = P * B (one rotamer per block),
 *   n_block_types = nbt, max_n_block_atoms = A, max_n_conn = C,
 *   max_n_tiles = ceil(A / 32), n_atom_types = T. */
typedef struct {
  int64_t n_atoms; /* rows of rot_coords */
  int32_t n_poses, max_n_blocks, n_rots;
  int32_t n_block_types, max_n_block_atoms, max_n_conn, max_n_tiles;
  int32_t n_atom_types;

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

  const int32_t* min_bondsep;         /* [P, B, B] */
  const int32_t* inter_block_bondsep; /* [P, B, B, C, C] */
  const int32_t* bt_n_atoms;          /* [nbt] */
  const int32_t* bt_n_heavy_atoms_in_tile; /* [nbt, max_n_tiles] */
  const int32_t* bt_heavy_atoms_in_tile;   /* [nbt, 32 * max_n_tiles] */
  const int32_t* bt_atom_types;       /* [nbt, A] */
  const int32_t* bt_n_conn;           /* [nbt] */
  const int32_t* bt_conn_atom;        /* [nbt, C] */
  const int32_t* bt_path_distance;    /* [nbt, A, A] */
  const int32_t* bt_is_ligand_fragment; /* [nbt] */
  const void* type_params;   /* [T, 10] float or double */
  const void* global_params; /* [1, 5] float or double */
  double max_dis;            /* neighbour-detection reach */
} tmol_b200_ljlk_inputs;

/* Launch shape of the scoring kernel; zeros select the built-in defaults.
 * A work item is (pose, block b1, a range of later blocks b2 >= b1).
 *   rows_per_item        work items a warp takes per atomic ticket
 *   warps_per_cta        warps per CTA (at most 16; 8 for float64 plans and
 *                        the rotamer and LK-ball kernels); every warp works
 *                        alone
 *   ctas_per_sm          resident CTAs per SM of the persistent grid
 *                        (defaults: 16 x 1 for float pose plans of LJ/LK
 *                        and elec, else 8 x 2)
 *   candidates_per_item  candidate blocks b2 per work item (at most 1024)
 *   slots_per_group      neighbouring blocks whose atoms share one pass of
 *                        the warp's 32 lanes (1-12, default 12): how many
 *                        block pairs a warp screens at once */
typedef struct {
  int32_t rows_per_item;
  int32_t warps_per_cta;
  int32_t ctas_per_sm;
  int32_t candidates_per_item;
  int32_t slots_per_group;
} tmol_b200_ljlk_launch;

typedef struct tmol_b200_ljlk_plan tmol_b200_ljlk_plan;

/* Replaces the per-call setup of LJLKPoseScoreDispatch::forward
 * (tmol/score/ljlk/potentials/ljlk_pose_score.impl.hh:628-778): derives the
 * compact tables once.  `real_bytes` is 4 (float32) or 8 (float64). */
int tmol_b200_ljlk_plan_create(const tmol_b200_ljlk_inputs* inputs,
                               int real_bytes,
                               const tmol_b200_ljlk_launch* launch,
                               void* stream, tmol_b200_ljlk_plan** plan_out);

int tmol_b200_ljlk_plan_destroy(tmol_b200_ljlk_plan* plan);

/* Reorders the plan's work items longest-first by the cost each item took
 * in the last scoring call made with counting on (the counting kernels time
 * each item; see tmol_b200_ljlk_plan_set_counting) (synchronises the
 * stream).  Coordinates change
 * little between calls in minimisation or trajectory replay, so the order
 * keeps the tail of the next launches short.  An item costlier than half a
 * warp's share of the call is first split over the halves of its candidate
 * range (up to half again as many items as the plan started with); the
 * kernels read the item count from plan memory, so a CUDA graph captured
 * before a rebalance stays valid (one captured before set_launch does
 * not).  Items that ran in the tail of the measured call look cheaper than
 * they are beside other heavy items: a second call and rebalance measure
 * them again in longest-first order. */
int tmol_b200_ljlk_plan_rebalance(tmol_b200_ljlk_plan* plan, void* stream);

/* Changes the launch shape of an existing plan (autotuning). */
int tmol_b200_ljlk_plan_set_launch(tmol_b200_ljlk_plan* plan,
                                   const tmol_b200_ljlk_launch* launch);

/* Replaces LJLKPoseScoreOp::forward / LJLKPoseScoreDispatch::forward
 * (compiled.ops.cpp:33-155; ljlk_pose_score.impl.hh:628-1158):
 *   coords         [n_atoms, 3] device
 *   energies       [3, P] (block_pair == 0) or [3, P, B, B] (block_pair != 0);
 *                  overwritten
 *   block_neighbors [P, B, B] int32 or NULL; overwritten when given */
int tmol_b200_ljlk_forward(tmol_b200_ljlk_plan* plan, const void* coords,
                           int block_pair, void* energies,
                           int32_t* block_neighbors, void* stream);

/* Replaces LJLKPoseScoreOp::backward (compiled.ops.cpp:157-278) with a
 * recompute adjoint (the reference's block-pair backward,
 * ljlk_pose_score.impl.hh:1160-1477, generalised to per-pose weights):
 *   dTdV       [3, P] (block_pair == 0) or [3, P, B, B] (block_pair != 0)
 *   dcoords    [n_atoms, 3]; overwritten with sum_t dTdV_t * dE_t/dcoords */
int tmol_b200_ljlk_backward(tmol_b200_ljlk_plan* plan, const void* coords,
                            int block_pair, const void* dTdV, void* dcoords,
                            void* stream);

/* The drop-in op's autograd pair with a speculative gradient (no counterpart
 * in the reference, whose backward always recomputes).  Whole-pose mode only.
 * forward_speculative returns what tmol_b200_ljlk_forward returns; once the
 * plan has seen a backward_speculative call, the same fused pass also takes
 * the gradient with that call's dTdV and keeps it in the plan.
 * backward_speculative writes sum_t dTdV_t * dE_t/dcoords into dcoords:
 * when `speculated` is nonzero (the caller's last forward_speculative on
 * this plan was the forward of these coordinates) and dTdV equals the
 * weights that forward used, the kept gradient is copied on the device and
 * the scoring launch does no work; otherwise the gradient is recomputed.
 * Minimisation, which calls forward then backward with the same weights
 * every step, pays one scoring pass per step instead of two.  The calls
 * keep state in the plan: make them in order on one stream. */
int tmol_b200_ljlk_forward_speculative(tmol_b200_ljlk_plan* plan, const void* coords,
                                       void* energies, int32_t* block_neighbors, void* stream);
int tmol_b200_ljlk_backward_speculative(tmol_b200_ljlk_plan* plan, const void* coords,
                                        const void* dTdV, void* dcoords, int speculated,
                                        void* stream);

/* Energies and weighted gradient in one pass, the work of the reference's
 * whole-pose forward when coords require grad (ljlk_pose_score.impl.hh:
 * 953-1119) followed by its elementwise backward (compiled.ops.cpp:164-173):
 *   weights    [3, P]: dL/dE per term and pose
 *   energies   [3, P]; overwritten
 *   dcoords    [n_atoms, 3]; overwritten with sum_t weights_t * dE_t/dcoords */
int tmol_b200_ljlk_energy_and_gradient(tmol_b200_ljlk_plan* plan,
                                       const void* coords, const void* weights,
                                       void* energies, void* dcoords,
                                       void* stream);

/* Work counting, off by default: while enabled, the LJ/LK, elec and
 * LK-ball scoring calls (pose and rotamer ops) run a kernel instantiation
 * that also counts its work (slower: the counters take registers and
 * instructions in its item loop).  No counterpart in the reference. */
int tmol_b200_ljlk_plan_set_counting(tmol_b200_ljlk_plan* plan, int enable);

/* Work counters of the last forward / energy_and_gradient call (all zero
 * when that call ran with counting off), the units of the throughput and
 * roofline figures (synchronises the stream):
 *   counts[0] neighbouring block pairs (incl. each block with itself)
 *   counts[1] atom pairs they hold (inter: n1 * n2, intra: n (n - 1) / 2)
 *   counts[2] heavy-atom pairs they hold (same rule)
 *   counts[3] atom pairs closer than max_dis with non-zero count-pair weight
 *   counts[4] heavy-atom pairs among counts[3] */
int tmol_b200_ljlk_last_counts(tmol_b200_ljlk_plan* plan, void* stream,
                               int64_t* counts);

/* Kernel timing: while enabled, CUDA events bracket each scoring-kernel
 * launch (up to 4096); profile_read sums their durations (synchronising). */
int tmol_b200_ljlk_profile(tmol_b200_ljlk_plan* plan, int enable);
int tmol_b200_ljlk_profile_read(tmol_b200_ljlk_plan* plan, double* total_ms,
                                int32_t* n_launches);

/* Measurement helper with no counterpart in the reference: times a
 * register-resident FMA loop over every SM and returns the device's FP32
 * throughput in TFLOP/s, the denominator of the scoring kernel's roofline.
 * Allocates 4 bytes and synchronises the stream. */
int tmol_b200_measure_fp32_peak(void* stream, double* tflops);

/* Sizes of the plan's device allocations in bytes. */
int64_t tmol_b200_ljlk_plan_device_bytes(const tmol_b200_ljlk_plan* plan);

/* Block-neighbour matrix without any device allocation.  No counterpart in
 * the reference: it exists for callers that may not allocate GPU memory
 * while running (code living inside a memory pool it does not own, or a
 * loop that must never enter the allocator) but need the same bounding-
 * sphere neighbour matrix as tmol_b200_ljlk_forward returns.
 *   coords              [n_atoms, 3] float32, device
 *   block_type          [n_poses * max_n_blocks] int32 (the op's
 *                       first_rot_block_type; -1 or out of range = no block)
 *   block_coord_offset  [n_poses * max_n_blocks] int32 (the op's
 *                       rot_coord_offset: first atom of each block)
 *   bt_n_atoms          [n_block_types] int32
 *   block_neighbors     [n_poses, max_n_blocks, max_n_blocks] int32 out;
 *                       every cell is written (1 iff b1 <= b2 are neighbours)
 * Scratch (the block spheres) is a fixed array in the library's device
 * memory: at most 262,144 blocks (n_poses * max_n_blocks), 4 MiB, kept by
 * every GPU that loads the library until the process exits; larger inputs
 * return TMOL_B200_ERR_CAPACITY before any GPU work.  The first call on a
 * device looks up that array's device address (cudaGetSymbolAddress).  With
 * CUDA's default lazy module loading that lookup is also what loads this
 * library's device code onto the device, and the load itself takes device
 * memory: the 4 MiB array plus the kernels' code.  So make the first call on
 * each device at start-up, before the host's own pool reserves the free
 * memory and before any stream capture; later calls allocate nothing.  The
 * looked-up address is kept for the life of the process: do not use this
 * entry point across a cudaDeviceReset (or any teardown of the device's
 * primary context), after which that address is no longer valid.  Every call
 * shares the one array and overwrites it, so calls that overlap on the GPU
 * (different streams, or different host threads on one device) race; order
 * them on one stream.  Calls no cudaMalloc, cudaFree or allocating routine. */
int tmol_b200_ljlk_block_neighbors_noalloc(
    const float* coords, int64_t n_atoms, const int32_t* block_type,
    const int32_t* block_coord_offset, const int32_t* bt_n_atoms,
    int32_t n_block_types, int32_t n_poses, int32_t max_n_blocks,
    double max_dis, int32_t* block_neighbors, void* stream);

/* ---- Rotamer scoring (tmol's ljlk_rotamer_scores, the packer's op) ----
 *
 * The inputs are those of torch.ops.tmol_ljlk.ljlk_rotamer_scores
 * (compiled.ops.cpp:599-662): the same struct, where block (p, b) owns
 * rotamers rot_offset_for_block[p, b] .. + n_rots_for_block[p, b] - 1
 * (n_rots is the total; a block with no rotamers takes no part), each with
 * its own block type and coordinates.  One call scores every rotamer pair
 * of neighbouring blocks and every rotamer with itself:
 *   count    -> number of pairs n and of work items (synchronises `stream`)
 *   fill     -> indices [3, n] int32 (pose, rot1, rot2) in the reference's
 *               order, and the work items [n_items, 4] int32
 *   forward  -> energies [3, n]; backward -> dL/dcoords [n_atoms, 3] from
 *               dL/dE [3, n]
 * A rotamer plan only serves these calls (the pose entry points reject it). */

/* Replaces the per-call set-up of LJLKRotamerScoreDispatch::forward
 * (ljlk_pose_score.impl.hh:1479-1630): validates every rotamer table. */
int tmol_b200_ljlk_rotamer_plan_create(const tmol_b200_ljlk_inputs* inputs,
                                       int real_bytes,
                                       const tmol_b200_ljlk_launch* launch,
                                       void* stream,
                                       tmol_b200_ljlk_plan** plan_out);

/* Rotamer spheres, block spheres enclosing each block's rotamers and the
 * block-neighbour rule, bit-exact with compute_rot_spheres,
 * compute_block_spheres_from_rot_spheres and detect_block_neighbors
 * (sphere_overlap.impl.hh:23-107, 455-510, 287-351), and the pair counts of
 * rot_neighbor_indices_from_block_neighbors (:512-610). */
int tmol_b200_ljlk_rotamer_count(tmol_b200_ljlk_plan* plan, const void* coords,
                                  int64_t* n_pairs, int64_t* n_items,
                                  void* stream);

/* The dispatch indices of the last count (rot_neighbor_indices_from_block_
 * neighbors, sphere_overlap.impl.hh:512-610) and the work items. */
int tmol_b200_ljlk_rotamer_fill(tmol_b200_ljlk_plan* plan, int32_t* indices,
                                int32_t* items, void* stream);

/* Energies of the dispatched pairs: LJLKRotamerScoreOp::forward
 * (compiled.ops.cpp:282-406, ljlk_pose_score.impl.hh:1632-1819). */
int tmol_b200_ljlk_rotamer_forward(tmol_b200_ljlk_plan* plan,
                                    const void* coords, const int32_t* items,
                                    int64_t n_items, int64_t n_pairs,
                                    void* energies, void* stream);

/* Recompute adjoint: LJLKRotamerScoreOp::backward (compiled.ops.cpp:408-529,
 * ljlk_pose_score.impl.hh:1826-2126). */
int tmol_b200_ljlk_rotamer_backward(tmol_b200_ljlk_plan* plan,
                                     const void* coords, const int32_t* items,
                                     int64_t n_items, int64_t n_pairs,
                                     const void* dTdV, void* dcoords,
                                     void* stream);

/* Human-readable text of a status code. */
const char* tmol_b200_status_string(int status);

#ifdef __cplusplus
}
#endif

#endif /* TMOL_B200_LJLK_H */
