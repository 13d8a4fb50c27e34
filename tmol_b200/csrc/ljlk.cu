// B200 LJ + LK pose scoring: plan creation, block spheres and the fused
// neighbour-detection + atom-pair kernel (forward energies and recompute
// adjoint), behind the C ABI declared in include/tmol_b200_ljlk.h.
//
// Layout in HBM (per PoseStack, built once by tmol_b200_ljlk_plan_create):
//   blk_bt[P*B], blk_off[P*B]      block type and first-atom offset per block
//   pose_last[P]                   1 + index of each pose's last real block
//   bt_tf[nbt*A]                   per block-type atom: compact atom type | heavy
//   ljtab, lktab[ntp*ntp]          per atom-type-pair LJ / LK constants
//   bt_pd[nbt][A][A] (u8)          intra-block bond separation
//   bt_conn_pd[nbt][C][A] (u8)     bond separation from each connection atom
//   cp_*[P*B][CP_CAP]              per block: the later blocks within
//                                  count-pair reach (min bond separation <= 4)
//                                  with their connection-pair separations;
//                                  replaces the dense [P,B,B,C,C] tensor
//   work[n_work] (int4)            rows: (pose, b1) for every block slot up
//                                  to each pose's last real block
//   spheres[P*B][4]                centroid + radius, rebuilt every call
//
// Scoring (one persistent launch per call, after the sphere kernel): every
// warp is an independent worker taking rows from an atomic ticket.  For row
// (p, b1) it stages b1's atoms (a tile of 32) in its shared-memory slab,
// tests b1 against all later blocks of the pose with the bounding-sphere rule
// (32 candidates per ballot) and evaluates each neighbouring block pair at
// once, in two phases: a screening pass over all atom pairs (distance and
// count-pair weight) compacts the pairs that contribute into a per-warp
// queue, split into LJ-only and heavy-atom (LJ + LK) pairs, and a dense pass
// evaluates the queue with every lane busy.  Energies stay in registers for
// the whole row; gradients accumulate in the slab (b1's across the whole
// row) and are flushed to global memory once per block pair (b2) or row (b1).

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/tmol_b200_elec.h"
#include "../../include/tmol_b200_ljlk.h"
#include "../../include/tmol_b200_lkball.h"
#include "../../include/tmol_b200_pose.h"
#include "../../include/tmol_b200_screen.h"
#include "bondsep.cuh"
#include "elec_potentials.cuh"
#include "ljlk_potentials.cuh"

namespace tmol_b200 {

constexpr int TILE = 32;
constexpr int MAX_CONN = 4;
// Work counters (units of the throughput and roofline figures):
//   [0] block pairs, [1] atom pairs (inter n1*n2, intra n(n-1)/2),
//   [2] heavy-atom pairs (same rule), [3] atom pairs inside max_dis with a
//   non-zero count-pair weight, [4] heavy-atom pairs among those.
// Per warp they are warp-uniform.
constexpr int N_COUNTS = 5;
constexpr int CP_CAP = 16;
constexpr int MAX_ROWS_PER_ITEM = 64;
constexpr int MAX_WARPS = 16;

// The energy term a plan scores: LJ + LK (fa_ljatr, fa_ljrep, fa_lk) or
// elec (fa_elec).  Both share the neighbour detection, count-pair tables,
// staging and screening; they differ in the per-atom record (atom type and
// heavy flag, or partial charge) and the pair potential.
enum TermKind : int { kTermLJLK = 0, kTermElec = 1, kTermLKBall = 2 };

__host__ __device__ constexpr int n_terms(int term) {
  return term == kTermElec ? 1 : (term == kTermLKBall ? 4 : 3);
}

enum StatusBits : int {
  kStIndex = 1,
  kStCapacity = 2,
  kStShape = 4,
};

// ---------------------------------------------------------------------------
// rounding-exact helpers (no contraction) so that spheres and neighbour tests
// reproduce the reference's CPU arithmetic bit for bit

__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float sqrt_rn(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// 1 / sqrt(x) (x > 0): the hardware estimate in fp32, correctly rounded
// operations in fp64
__device__ __forceinline__ float inv_sqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double inv_sqrt(double x) { return 1.0 / sqrt(x); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double sqrt_rn(double a) { return __dsqrt_rn(a); }

// ---------------------------------------------------------------------------
// plan-building kernels

struct PlanBuildArgs {
  tmol_b200_ljlk_inputs in;
  int* blk_bt;
  int* blk_off;
  int* pose_last;
  uint8_t* bt_pd;
  uint8_t* bt_conn_pd;
  int* bt_flags;  // heavy flag per bt-atom (before type flags are merged)
  int* cp_count;
  int* cp_b2;
  int* cp_minsep;
  uint8_t* cp_seps;
  int* status;
  int rotamers;  // rotamer plan: blocks may own any number of rotamers
  int* rot_bt;   // rotamer plan: per-rotamer copies (validated)
  int* rot_off;
  int* rot_block;
  int* rot_pose;
  int term;
  // elec: bond separations from each connection atom come from the
  // representative table (the intra-block table is in.bt_path_distance)
  const int32_t* bt_inter_pd;
  // plans built from the pose's connectivity instead of the dense
  // min_bondsep / inter_block_bondsep tensors
  int use_conn;
  PoseConn conn;
};

__global__ void plan_blocks_kernel(PlanBuildArgs a) {
  const tmol_b200_ljlk_inputs& in = a.in;
  int P = in.n_poses, B = in.max_n_blocks;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P * B;
       i += gridDim.x * blockDim.x) {
    int p = i / B, b = i - p * B;
    int bt_first = in.first_rot_block_type[i];
    int rot = in.rot_offset_for_block[i];
    int bt = -1, off = 0;
    if (a.rotamers) {
      // a block without rotamers takes no part in rotamer scoring
      const int nr = in.n_rots_for_block[i];
      if (nr < 0) atomicOr(a.status, kStIndex);
      if (nr <= 0) {
        if (bt_first >= 0) atomicOr(a.status, kStShape);
        a.blk_bt[i] = -1;
        a.blk_off[i] = 0;
        continue;
      }
      if (rot < 0 || (int64_t)rot + nr > in.n_rots) {
        atomicOr(a.status, kStIndex);
        a.blk_bt[i] = -1;
        a.blk_off[i] = 0;
        continue;
      }
    }
    if (rot < 0 || rot >= in.n_rots) {
      if (bt_first >= 0) atomicOr(a.status, kStIndex);
    } else {
      if (in.pose_ind_for_rot[rot] != p || in.block_ind_for_rot[rot] != b)
        atomicOr(a.status, kStShape);
      bt = in.block_type_ind_for_rot[rot];
      off = in.rot_coord_offset[rot];
      if (bt >= in.n_block_types) {
        atomicOr(a.status, kStIndex);
        bt = -1;
      }
      if ((bt >= 0) != (bt_first >= 0) || (bt >= 0 && bt != bt_first))
        atomicOr(a.status, kStShape);
      if (bt >= 0) {
        int n = in.bt_n_atoms[bt];
        if (off < 0 || (int64_t)off + n > in.n_atoms) {
          atomicOr(a.status, kStIndex);
          bt = -1;
        }
      }
    }
    a.blk_bt[i] = bt;
    a.blk_off[i] = off;
    if (bt >= 0) atomicMax(&a.pose_last[p], b + 1);
  }
}

// Rotamer plan: per rotamer, its pose, block, block type and coordinates
// must be in range and the rotamer must lie in its block's range.
// One record per block slot for the scoring kernel's row and neighbour
// loads: {block type or -1, first atom, atom count, connections | ligand
// flag << 8}, from the validated block tables.
__global__ void plan_block_info_kernel(int64_t n, const int* blk_bt, const int* blk_off, const int* bt_n_atoms,
                                       const int* bt_n_conn, const int* bt_is_ligand, int4* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int bt = blk_bt[i];
    int4 r = make_int4(bt, blk_off[i], 0, 0);
    if (bt >= 0) {
      r.z = bt_n_atoms[bt];
      r.w = (bt_n_conn[bt] & 0xff) | ((bt_is_ligand[bt] ? 1 : 0) << 8);
    }
    out[i] = r;
  }
}

__global__ void plan_rotamers_kernel(PlanBuildArgs a) {
  const tmol_b200_ljlk_inputs& in = a.in;
  const int P = in.n_poses, B = in.max_n_blocks;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < in.n_rots; r += gridDim.x * blockDim.x) {
    const int p = in.pose_ind_for_rot[r], b = in.block_ind_for_rot[r];
    int bt = in.block_type_ind_for_rot[r];
    const int off = in.rot_coord_offset[r];
    if (p < 0 || p >= P || b < 0 || b >= B) {
      atomicOr(a.status, kStIndex);
    } else {
      const int i = p * B + b;
      const int r0 = in.rot_offset_for_block[i], nr = in.n_rots_for_block[i];
      if (r < r0 || r >= r0 + nr) atomicOr(a.status, kStShape);
    }
    if (bt < 0 || bt >= in.n_block_types) {
      atomicOr(a.status, kStIndex);
      bt = 0;
    } else if (off < 0 || (int64_t)off + in.bt_n_atoms[bt] > in.n_atoms) {
      atomicOr(a.status, kStIndex);
    }
    a.rot_bt[r] = bt;
    a.rot_off[r] = off < 0 ? 0 : off;
    a.rot_block[r] = b < 0 || b >= B ? 0 : b;
    a.rot_pose[r] = p < 0 || p >= P ? 0 : p;
  }
}

// Per block-type atom: compact type index | heavy flag, byte copies of the
// bond-separation tables, and index validation.
__global__ void plan_block_types_kernel(PlanBuildArgs a, const int* type_map,
                                        uint16_t* bt_tf) {
  const tmol_b200_ljlk_inputs& in = a.in;
  int nbt = in.n_block_types, A = in.max_n_block_atoms, C = in.max_n_conn;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nbt * A;
       i += gridDim.x * blockDim.x) {
    int bt = i / A, at = i - bt * A;
    int n = in.bt_n_atoms[bt];
    if (n < 0 || n > A) {
      if (at == 0) atomicOr(a.status, kStIndex);
      continue;
    }
    uint16_t tf = 0;
    if (at < n) {
      if (a.term == kTermLJLK) {
        int t = in.bt_atom_types[i];
        if (t < 0 || t >= in.n_atom_types || type_map[t] < 0) {
          atomicOr(a.status, kStIndex);
        } else {
          tf = (uint16_t)(type_map[t] | (a.bt_flags[i] == kHeavy ? 256 : 0));
        }
      }
      for (int at2 = 0; at2 < A; ++at2) {
        int v = in.bt_path_distance[(int64_t)i * A + at2];
        a.bt_pd[(int64_t)i * A + at2] = (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
      }
    }
    bt_tf[i] = tf;
    const int32_t* cpd_src = a.bt_inter_pd ? a.bt_inter_pd : in.bt_path_distance;
    int nc = in.bt_n_conn[bt];
    if (at == 0 && (nc < 0 || nc > C)) atomicOr(a.status, kStIndex);
    for (int c = 0; c < C; ++c) {
      uint8_t v = 6;
      if (c < nc && at < n) {
        int ca = in.bt_conn_atom[bt * C + c];
        if (ca < 0 || ca >= n) {
          atomicOr(a.status, kStIndex);
        } else {
          int d = cpd_src[((int64_t)bt * A + ca) * A + at];
          v = (uint8_t)(d < 0 ? 0 : (d > 255 ? 255 : d));
        }
      }
      a.bt_conn_pd[((int64_t)bt * C + c) * A + at] = v;
    }
  }
}

// Type-pair tables for every ordered pair of the compact atom types.
template <typename Real>
__global__ void plan_tables_kernel(const Real* type_params, const Real* gp,
                                   const int* compact_types, int ntp,
                                   LJRecord<Real>* ljtab, LKRecord<Real>* lktab) {
  GlobalParams<Real> g = {gp[0], gp[1], gp[2], gp[3], gp[4]};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntp * ntp;
       i += gridDim.x * blockDim.x) {
    AtomParams<Real> pr[2];
    int ts[2] = {compact_types[i / ntp], compact_types[i % ntp]};
    for (int k = 0; k < 2; ++k) {
      const Real* r = type_params + 10 * (int64_t)ts[k];
      pr[k].lj_radius = r[0];
      pr[k].lj_wdepth = r[1];
      pr[k].lk_dgfree = r[2];
      pr[k].lk_lambda = r[3];
      pr[k].lk_volume = r[4];
      int f = 0;
      if (r[5] != 0) f |= kDonor;
      if (r[6] != 0) f |= kHydroxyl;
      if (r[7] != 0) f |= kPolarH;
      if (r[8] != 0) f |= kAcceptor;
      if (r[9] != 0) f |= kCarbonLK;
      pr[k].flags = f;
    }
    build_records(pr[0], pr[1], g, ljtab[i], lktab[i]);
  }
}

__global__ void plan_heavy_kernel(PlanBuildArgs a) {
  const tmol_b200_ljlk_inputs& in = a.in;
  int nbt = in.n_block_types, nt = in.max_n_tiles, A = in.max_n_block_atoms;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nbt * nt * TILE;
       i += gridDim.x * blockDim.x) {
    int bt = i / (nt * TILE);
    int rem = i - bt * nt * TILE;
    int t = rem / TILE, k = rem - t * TILE;
    int nh = in.bt_n_heavy_atoms_in_tile[bt * nt + t];
    if (k < nh) {
      int loc = in.bt_heavy_atoms_in_tile[(int64_t)bt * nt * TILE + t * TILE + k];
      int at = t * TILE + loc;
      if (loc < 0 || loc >= TILE || at >= A) {
        atomicOr(a.status, kStIndex);
      } else {
        a.bt_flags[bt * A + at] = kHeavy;
      }
    }
  }
}

// One warp per (pose, b1): later blocks b2 with min_bondsep <= 4.
__global__ void plan_count_pair_kernel(PlanBuildArgs a) {
  const tmol_b200_ljlk_inputs& in = a.in;
  int P = in.n_poses, B = in.max_n_blocks, C = in.max_n_conn;
  int lane = threadIdx.x & 31;
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int n_warps = (gridDim.x * blockDim.x) >> 5;
  for (int row = warp; row < P * B; row += n_warps) {
    int p = row / B, b1 = row - p * B;
    int cnt = 0;
    if (a.blk_bt[row] >= 0) {
      const int32_t* mrow = in.min_bondsep + (int64_t)row * B;
      for (int base = b1 + 1; base < B; base += 32) {
        int b2 = base + lane;
        bool hit = false;
        int ms = 0;
        if (b2 < B && a.blk_bt[p * B + b2] >= 0) {
          ms = mrow[b2];
          hit = ms <= 4;
        }
        unsigned m = __ballot_sync(0xffffffffu, hit);
        if (hit) {
          int slot = cnt + __popc(m & ((1u << lane) - 1));
          if (slot < CP_CAP) {
            int64_t e = (int64_t)row * CP_CAP + slot;
            a.cp_b2[e] = b2;
            a.cp_minsep[e] = ms;
            const int32_t* s =
                in.inter_block_bondsep + (((int64_t)p * B + b1) * B + b2) * C * C;
            for (int c1 = 0; c1 < MAX_CONN; ++c1)
              for (int c2 = 0; c2 < MAX_CONN; ++c2) {
                int v = (c1 < C && c2 < C) ? s[c1 * C + c2] : 6;
                a.cp_seps[e * 16 + c1 * 4 + c2] =
                    (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
              }
          } else {
            atomicOr(a.status, kStCapacity);
          }
        }
        cnt += __popc(m);
      }
    }
    if (lane == 0) a.cp_count[row] = cnt < CP_CAP ? cnt : CP_CAP;
  }
}

// The same partner table from the pose's connectivity, without the dense
// tensors: one thread per row (pose, b1) runs the bounded search from each of
// b1's connection points (bondsep.cuh) and keeps the later blocks whose
// minimum separation is <= 4, in increasing b2, with their connection-pair
// separations (6 where unreached).
constexpr int CONN_ROW_CAP = 48;  // distinct later blocks within the cap

__global__ void plan_count_pair_conn_kernel(PlanBuildArgs a) {
  const int P = a.in.n_poses, B = a.in.max_n_blocks;
  const PoseConn& g = a.conn;
  int reach[BONDSEP_MAX_REACH], dist[BONDSEP_MAX_REACH];
  int part_b2[CONN_ROW_CAP], part_min[CONN_ROW_CAP];
  uint8_t part_sep[CONN_ROW_CAP][16];
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < P * B; row += gridDim.x * blockDim.x) {
    const int p = row / B, b1 = row - p * B;
    int cnt = 0;
    if (a.blk_bt[row] >= 0) {
      const int nc = block_n_conn(g, p, b1);
      if (nc < 0 || nc > MAX_CONN) atomicOr(a.status, kStIndex);
      int n_part = 0, st = 0;
      for (int c1 = 0; c1 < nc && c1 < MAX_CONN; ++c1) {
        const int n = bounded_paths(g, p, b1, c1, reach, dist, st);
        for (int k = 0; k < n; ++k) {
          const int b2 = reach[k] >> 3, c2 = reach[k] & 7;
          if (b2 <= b1) continue;
          int q = 0;
          while (q < n_part && part_b2[q] != b2) ++q;
          if (q == n_part) {
            if (n_part == CONN_ROW_CAP) {
              st |= kBsCapacity;
              continue;
            }
            part_b2[q] = b2;
            part_min[q] = MAX_SIG_SEP;
            for (int e = 0; e < 16; ++e) part_sep[q][e] = MAX_SIG_SEP;
            ++n_part;
          }
          if (c2 < MAX_CONN) part_sep[q][c1 * 4 + c2] = (uint8_t)dist[k];
          part_min[q] = min(part_min[q], dist[k]);
        }
      }
      if (st & kBsIndex) atomicOr(a.status, kStIndex);
      if (st & kBsShape) atomicOr(a.status, kStShape);
      if (st & kBsCapacity) atomicOr(a.status, kStCapacity);
      // partners in increasing b2 (the dense route's order)
      for (;;) {
        int best = -1;
        for (int q = 0; q < n_part; ++q)
          if (part_min[q] <= 4 && a.blk_bt[p * B + part_b2[q]] >= 0 && (best < 0 || part_b2[q] < part_b2[best]))
            best = q;
        if (best < 0) break;
        if (cnt < CP_CAP) {
          const int64_t e = (int64_t)row * CP_CAP + cnt;
          a.cp_b2[e] = part_b2[best];
          a.cp_minsep[e] = part_min[best];
          for (int k = 0; k < 16; ++k) a.cp_seps[e * 16 + k] = part_sep[best][k];
        } else {
          atomicOr(a.status, kStCapacity);
        }
        ++cnt;
        part_min[best] = MAX_SIG_SEP + 1;  // taken
      }
    }
    a.cp_count[row] = cnt < CP_CAP ? cnt : CP_CAP;
  }
}

// ---------------------------------------------------------------------------
// per-call kernels

template <typename Real>
struct AtomRec;

template <typename Real>
struct ScoreArgs {
  const Real* coords;
  // when set and nonzero, the launch has nothing to do: the gradient was
  // taken from a speculative pass (pose_backward_speculative)
  const int* done;
  // what the sphere pass zeroes before the scoring launch adds to it (no
  // separate memsets in a step): reals of dcoords, of energies and of
  // zero_aux (LK-ball: the waters' gradient), and the work counters
  int64_t zero_dcoords, zero_energies, zero_aux_n;
  Real* zero_aux;
  int zero_counts;
  // pose plans of the LJ/LK and elec terms: per block {block type, first
  // atom, atom count, connections | ligand << 8} and every atom as a
  // staged record (coordinates with its type or charge), written by the
  // sphere kernel each call; null elsewhere (the staging then gathers)
  const int4* blk_info;
  AtomRec<Real>* packed;
  const int* blk_bt;
  const int* blk_off;
  const int* pose_last;
  const uint16_t* bt_tf;  // per block-type atom: compact type | heavy << 8
  const LJRecord<Real>* ljtab;
  const LKRecord<Real>* lktab;
  int ntp;  // compact atom types (tables are ntp x ntp)
  const uint8_t* bt_pd;
  const uint8_t* bt_conn_pd;
  const int* bt_n_atoms;
  const int* bt_n_conn;
  const int* bt_is_ligand;
  const int* cp_count;
  const int* cp_b2;
  const int* cp_minsep;
  const uint8_t* cp_seps;
  Real* spheres;
  GlobalParams<Real> g;
  Real reach;
  const int4* work;
  int* item_cost;  // measured cost of each work item (clock cycles / 16)
  int P, B, A, C;
  Real* energies;
  int32_t* nbr;
  const Real* dTdV;
  Real* dcoords;
  int* ticket;
  unsigned long long* counts;
  // optional skip mask: bit b2 of row (p, b1) set = do not score the block
  // pair (never honoured for b1 == b2 or count-pair partners)
  const uint32_t* skip;
  int skip_words;  // 32-bit words per row
  int max_slots;   // neighbouring blocks packed per screening group
  // elec plans: partial charge per block-type atom [nbt * A] and the
  // potential's per-unit-charge constants (ElecK layout)
  const Real* bt_q;
  const Real* elec_k;
};

// Bounding sphere per block: centroid (sum of atoms in order, then divided
// by the atom count) and largest centroid distance, as
// sphere_overlap.impl.hh:109-196 computes them on the CPU.  One warp per
// block: lanes load 32 atoms at a time, lane 0 adds them in atom order
// (shuffled to it one by one, no contraction) so that the sums are
// bit-identical to the sequential CPU loop; the maximum is order-free.
template <typename Real>
__device__ __forceinline__ void warp_sphere(const Real* coords, const int* bt_n_atoms, int bt,
                                            int off, int lane, Real* out) {
  if (bt < 0) {
    if (lane < 4) out[lane] = Real(0);
    return;
  }
  int n = bt_n_atoms[bt];
  const Real* x = coords + 3 * (int64_t)off;
  Real cx = 0, cy = 0, cz = 0;
  for (int base = 0; base < n; base += 32) {
    int k = base + lane;
    Real ax = 0, ay = 0, az = 0;
    if (k < n) {
      ax = x[3 * k + 0];
      ay = x[3 * k + 1];
      az = x[3 * k + 2];
    }
    int cnt = min(32, n - base);
    for (int q = 0; q < cnt; ++q) {
      Real vx = __shfl_sync(0xffffffffu, ax, q);
      Real vy = __shfl_sync(0xffffffffu, ay, q);
      Real vz = __shfl_sync(0xffffffffu, az, q);
      cx = add_rn(cx, vx);
      cy = add_rn(cy, vy);
      cz = add_rn(cz, vz);
    }
  }
  Real rn = Real(n);
  cx = div_rn(cx, rn);
  cy = div_rn(cy, rn);
  cz = div_rn(cz, rn);
  Real d2max = 0;
  for (int k = lane; k < n; k += 32) {
    Real dx = sub_rn(x[3 * k + 0], cx);
    Real dy = sub_rn(x[3 * k + 1], cy);
    Real dz = sub_rn(x[3 * k + 2], cz);
    Real d2 = add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
    if (d2 > d2max) d2max = d2;
  }
  for (int o = 16; o > 0; o >>= 1) {
    Real v = __shfl_xor_sync(0xffffffffu, d2max, o);
    d2max = v > d2max ? v : d2max;
  }
  if (lane == 0) {
    out[0] = cx;
    out[1] = cy;
    out[2] = cz;
    out[3] = sqrt_rn(d2max);
  }
}

template <typename Real>
__device__ __forceinline__ void pack_block(const ScoreArgs<Real>& s, int bt, int off, int lane);

template <typename Real>
__global__ void spheres_kernel(ScoreArgs<Real> s) {
  if (s.done && *s.done) return;  // the scoring launch that follows does no work
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t n_threads = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = tid; i < s.zero_dcoords; i += n_threads) s.dcoords[i] = Real(0);
  for (int64_t i = tid; i < s.zero_energies; i += n_threads) s.energies[i] = Real(0);
  for (int64_t i = tid; i < s.zero_aux_n; i += n_threads) s.zero_aux[i] = Real(0);
  if (s.zero_counts && s.counts && tid < N_COUNTS) s.counts[tid] = 0;
  if (tid == 0 && s.ticket) *s.ticket = 0;  // the scoring launch's work ticket
  const int lane = threadIdx.x & 31;
  const int n_blocks = s.P * s.B;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n_blocks; i += warps) {
    warp_sphere(s.coords, s.bt_n_atoms, s.blk_bt[i], s.blk_off[i], lane, s.spheres + 4 * (int64_t)i);
    if (s.packed) pack_block(s, s.blk_bt[i], s.blk_off[i], lane);
  }
}

// ---------------------------------------------------------------------------
// Per-warp shared-memory slab.
//
// Side 0 holds a tile (<= 32 atoms) of the row block b1; side 1 packs the
// atoms of up to MAX_SLOTS neighbouring blocks b2 (at most M1 atoms), so that
// one screening pass covers several block pairs with every lane busy.  The
// pair queue collects the atom pairs that contribute (inside max_dis with a
// non-zero count-pair weight): LJ-only pairs from the front, heavy-atom
// (LJ + LK) pairs from the back.  Both sides live in one atom array (side 0
// at [0, TILE), side 1 at [TILE, TILE + M1)), each atom one 16-byte record
// (x, y, z, type) so that a pair costs two vector loads; an entry packs
// a (5 bits: a side-0 atom) | k (7 bits: an index into the atom array) |
// count-pair-weight-0.2 flag (bit 12).  Entries come in runs that share k:
// screening emits each side-1 atom's pairs together, the intra-tile pass
// each row's.  One screening chunk (32 side-1 atoms x 32 rows) emits at
// most 1024 entries, so a queue of QCAP >= 1024 takes any chunk whole.

constexpr int M1 = 96;
constexpr int MAX_SLOTS = 12;
// copies of the side-0 force accumulators: lane l adds an entry's force on
// its side-0 atom into copy l % A_COPIES, so that at most four lanes of a
// step can meet at one address (shared atomics serialise on a conflict)
constexpr int A_COPIES = 8;
constexpr int QCAP = 1024;
constexpr int kTfHeavy = 256;

enum SlotKind : int {
  kSlotFar = 0,       // bond separation > 4 everywhere: weight 1
  kSlotStriking = 1,  // count pair through the connection atoms
  kSlotIntra = 2,     // another tile of block b1: intra-block separation table
};

// One staged atom: coordinates and either per block-type atom flags
// (LJ/LK: compact atom type | heavy << 8) or the partial charge (elec).
template <typename Real>
struct alignas(16) AtomRec {
  Real x, y, z;
  union {
    int tf;
    Real q;
  };
};

constexpr int N_ATOMS = TILE + M1;

// Writes block (bt, off)'s atoms as staged records: coordinates and the
// block-type atom's compact type | heavy flag (LJ/LK) or partial charge
// (elec), so that staging a block costs one vector load per atom.
template <typename Real>
__device__ __forceinline__ void pack_block(const ScoreArgs<Real>& s, int bt, int off, int lane) {
  if (bt < 0) return;
  const int n = s.bt_n_atoms[bt];
  for (int k = lane; k < n; k += 32) {
    const Real* c = s.coords + 3 * ((int64_t)off + k);
    AtomRec<Real> a;
    a.x = c[0];
    a.y = c[1];
    a.z = c[2];
    if (s.bt_q)
      a.q = s.bt_q[(int64_t)bt * s.A + k];
    else
      a.tf = s.bt_tf[(int64_t)bt * s.A + k];
    s.packed[(int64_t)off + k] = a;
  }
}

template <typename Real>
struct Slab {
  AtomRec<Real> at[N_ATOMS];            // side 0, then side 1
  Real gx[N_ATOMS], gy[N_ATOMS], gz[N_ATOMS];  // gradient accumulators
  Real ga[A_COPIES][3][TILE];  // side-0 forces of entries' a atoms, by copy
  uint32_t cpd0[TILE];  // bond separation to each connection atom, a byte each
  uint32_t cpd1[M1];
  int gidx1[M1];  // global atom index
  uint8_t slot1[M1];   // slot of the packed atom
  uint8_t local1[M1];  // atom index within its block
  uint8_t seps[MAX_SLOTS][16];
  int slot_kind[MAX_SLOTS], slot_nc[MAX_SLOTS], slot_lig[MAX_SLOTS];
  Real slot_sph[MAX_SLOTS][4];  // bounding sphere of each slot's block
  unsigned long long counts[8];
  uint16_t queue[QCAP];
};

struct RowInfo {
  int p, b1, i1, bt1, off1, n1, nc1, lig1;
  int st1, c1;  // tile of b1 in side 0
};



template <typename Real>
__device__ __forceinline__ Real warp_sum(Real v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename Real>
__device__ __forceinline__ uint32_t load_cpd(const ScoreArgs<Real>& s, int bt,
                                             int nconn, int at) {
  uint32_t v = 0x06060606u;
  for (int k = 0; k < nconn; ++k) {
    uint32_t d = s.bt_conn_pd[((int64_t)bt * s.C + k) * s.A + at];
    v = (v & ~(0xffu << (8 * k))) | (d << (8 * k));
  }
  return v;
}

// Stage atoms [start, start + cnt) of block (bt, off) into side 0.
template <typename Real, int TERM = kTermLJLK>
__device__ __forceinline__ void stage_side0(const ScoreArgs<Real>& s,
                                            Slab<Real>& w, int bt, int off,
                                            int start, int cnt, int nconn,
                                            int lane) {
  if (lane < cnt) {
    int at = start + lane;
    AtomRec<Real> a;
    if (s.packed) {
      a = s.packed[(int64_t)off + at];
    } else {
      const Real* c = s.coords + 3 * ((int64_t)off + at);
      a.x = c[0];
      a.y = c[1];
      a.z = c[2];
      if (TERM == kTermElec)
        a.q = s.bt_q[(int64_t)bt * s.A + at];
      else
        a.tf = s.bt_tf[(int64_t)bt * s.A + at];
    }
    w.at[lane] = a;
    w.cpd0[lane] = load_cpd(s, bt, nconn, at);
    w.gx[lane] = 0;
    w.gy[lane] = 0;
    w.gz[lane] = 0;
  }
#pragma unroll
  for (int k = 0; k < A_COPIES; ++k) {
    w.ga[k][0][lane] = 0;
    w.ga[k][1][lane] = 0;
    w.ga[k][2][lane] = 0;
  }
}

// Append the atoms of [start, start + cnt) of block (bt, off) that can reach
// block b1 to side 1 at j0: an atom farther than r1 + max_dis from b1's
// centroid is farther than max_dis from every b1 atom, and every term is zero
// there.  Returns the number of atoms kept; with `heavy`, also the number of
// heavy atoms among all cnt (a work counter).
template <typename Real, int TERM = kTermLJLK>
__device__ __forceinline__ int stage_side1(const ScoreArgs<Real>& s,
                                           Slab<Real>& w, int j0, int slot,
                                           int bt, int off, int start,
                                           int cnt, int nconn, Real cx,
                                           Real cy, Real cz, Real reach2,
                                           int lane, int* heavy = nullptr) {
  bool keep = false;
  AtomRec<Real> a;
  a.x = a.y = a.z = Real(0);
  a.tf = 0;
  int at = start + lane;
  if (lane < cnt) {
    if (s.packed) {
      a = s.packed[(int64_t)off + at];
    } else {
      const Real* c = s.coords + 3 * ((int64_t)off + at);
      a.x = c[0];
      a.y = c[1];
      a.z = c[2];
      if (TERM == kTermElec)
        a.q = s.bt_q[(int64_t)bt * s.A + at];
      else
        a.tf = s.bt_tf[(int64_t)bt * s.A + at];
    }
    Real dx = a.x - cx, dy = a.y - cy, dz = a.z - cz;
    keep = dx * dx + dy * dy + dz * dz < reach2;
  }
  if (heavy)
    *heavy = TERM == kTermLJLK ? __popc(__ballot_sync(0xffffffffu, lane < cnt && (a.tf & kTfHeavy))) : 0;
  unsigned km = __ballot_sync(0xffffffffu, keep);
  if (keep) {
    int j = j0 + __popc(km & ((1u << lane) - 1));
    w.at[TILE + j] = a;
    w.cpd1[j] = load_cpd(s, bt, nconn, at);
    w.gidx1[j] = off + at;
    w.slot1[j] = (uint8_t)slot;
    w.local1[j] = (uint8_t)at;
    w.gx[TILE + j] = 0;
    w.gy[TILE + j] = 0;
    w.gz[TILE + j] = 0;
  }
  return __popc(km);
}

template <typename Real>
__device__ __forceinline__ void flush_side0(const ScoreArgs<Real>& s,
                                            Slab<Real>& w, int off, int start,
                                            int cnt, int lane) {
  if (lane < cnt) {
    Real* d = s.dcoords + 3 * ((int64_t)off + start + lane);
    Real gx = w.gx[lane], gy = w.gy[lane], gz = w.gz[lane];
#pragma unroll
    for (int k = 0; k < A_COPIES; ++k) {
      gx += w.ga[k][0][lane];
      gy += w.ga[k][1][lane];
      gz += w.ga[k][2][lane];
    }
    if (gx != 0) atomicAdd(d + 0, gx);
    if (gy != 0) atomicAdd(d + 1, gy);
    if (gz != 0) atomicAdd(d + 2, gz);
  }
}

template <typename Real>
__device__ __forceinline__ void flush_side1(const ScoreArgs<Real>& s,
                                            Slab<Real>& w, int m, int lane) {
  for (int j = lane; j < m; j += 32) {
    Real* d = s.dcoords + 3 * (int64_t)w.gidx1[j];
    Real gx = w.gx[TILE + j], gy = w.gy[TILE + j], gz = w.gz[TILE + j];
    if (gx != 0) atomicAdd(d + 0, gx);
    if (gy != 0) atomicAdd(d + 1, gy);
    if (gz != 0) atomicAdd(d + 2, gz);
  }
}

// What the out-of-line screening and evaluation functions need, by value.
template <typename Real>
struct EvalCtx {
  union {
    const LJRecord<Real>* ljtab;  // LJ/LK
    const Real* elec_k;           // elec: ElecK constants
  };
  const LKRecord<Real>* lktab;
  const uint8_t* pd;  // intra-block separations of b1, row st1 (tile start)
  int ntp, A;
  Real max_dis;
  Real wt0, wt1, wt2;  // gradient weights of the three terms (elec: wt0)
};

template <typename Real>
struct E3 {
  Real atr, rep, lk;
};

__device__ __forceinline__ void cnt_add(unsigned long long* c, int k, long long v, int lane) {
  if (lane == 0) c[k] += (unsigned long long)v;
}

// The pair-evaluation helpers below are out of line by default (one copy
// each: the kernel's code footprint and register budget stay small).
#ifndef TMOL_B200_LJLK_OUTLINE
#define TMOL_B200_LJLK_OUTLINE __noinline__
#endif

// Dense evaluation of one queue (HEAVY: LJ + LK, else LJ only; elec: the
// elec energy in .atr); returns the lane's energy sums.  Entries come in
// screening order, so lanes sharing a1 are mostly contiguous: their a1
// forces are summed with a segmented shuffle reduction and added once per
// segment.
template <typename Real, bool GRAD, int TERM = kTermLJLK>
__device__ TMOL_B200_LJLK_OUTLINE E3<Real> eval_queue(EvalCtx<Real> c, Slab<Real>* wp,
                                            int nl, int nh, int lane) {
  Slab<Real>& w = *wp;
  E3<Real> acc = {0, 0, 0};
  const Real dmax = c.max_dis;
  const Real far_dmin = c.max_dis - Real(1.5);
  const Real far_first = far_dmin > Real(4.5) ? far_dmin : Real(4.5);
  const Real inv_hf = Real(1) / (dmax - far_dmin);
  ElecK<Real> K;
  if (TERM == kTermElec) K = load_elec_k(c.elec_k);
  // one pass over the LJ-only entries, then the heavy-atom ones: only the
  // step holding both has lanes on different paths
  const int n = nl + nh;
  for (int base = 0; base < n; base += 32) {
    int i = base + lane;
    bool act = i < n;
    const bool heavy = TERM == kTermLJLK && i >= nl;
    int e = act ? (int)w.queue[heavy ? QCAP - 1 - (i - nl) : i] : 0;
    // j: the entry's k (runs of equal k are consecutive), a1: its a
    int a1 = e & 31, j = (e >> 5) & 127;
    Real wcp = (e >> 12) & 1 ? Real(0.2) : Real(1);
    Real fx = 0, fy = 0, fz = 0;
    if (act && TERM == kTermElec) {
      const AtomRec<Real> p1 = w.at[a1];
      const AtomRec<Real> p2 = w.at[j];
      const Real dx = p1.x - p2.x;
      const Real dy = p1.y - p2.y;
      const Real dz = p1.z - p2.z;
      const Real d2 = dx * dx + dy * dy + dz * dz;
      // coincident atoms take the flat region and add no force
      const Real inv_d = inv_sqrt(d2);
      const Real d = d2 > Real(0) ? d2 * inv_d : Real(0);
      Real f, df = 0;
      elec_eval<Real, GRAD>(d, K, f, df);
      const Real wq = wcp * p1.q * p2.q;
      acc.atr += wq * f;
      if (GRAD && d != Real(0)) {
        const Real g = wq * c.wt0 * df * inv_d;
        fx = g * dx;
        fy = g * dy;
        fz = g * dz;
      }
    } else if (act) {
      const AtomRec<Real> p1 = w.at[a1];
      const AtomRec<Real> p2 = w.at[j];
      int t1 = p1.tf & 0xff, t2 = p2.tf & 0xff;
      // records are symmetric in the two types (LJ by construction, LK as
      // sums of both directions), so only the upper triangle is read (lower
      // type first): half the tables' footprint in L1
      Real dx = p1.x - p2.x;
      Real dy = p1.y - p2.y;
      Real dz = p1.z - p2.z;
      const Real d2 = dx * dx + dy * dy + dz * dz;
      // coincident atoms (d2 = 0) take the linear LJ and flat LK regions,
      // which never use inv_d, and add no force
      const Real inv_d = inv_sqrt(d2);
      const Real d = d2 > Real(0) ? d2 * inv_d : Real(0);
      int tp = t1 < t2 ? t1 * c.ntp + t2 : t2 * c.ntp + t1;
      Real atr, rep, datr, drep;
      lj_eval<Real, GRAD>(d, inv_d, c.ljtab + tp, atr, rep, datr, drep);
      acc.atr += wcp * atr;
      acc.rep += wcp * rep;
      Real dE = c.wt0 * datr + c.wt1 * drep;
      if (heavy) {
        Real lk, dlk;
        lk_eval<Real, GRAD>(d, inv_d, c.lktab + tp, far_dmin, far_first, inv_hf, lk, dlk);
        acc.lk += wcp * lk;
        dE += c.wt2 * dlk;
      }
      if (GRAD && d != Real(0)) {
        Real f = wcp * dE * inv_d;
        fx = f * dx;
        fy = f * dy;
        fz = f * dz;
      }
    }
    if (GRAD) {
      // segments: maximal runs of lanes with equal j (the entry's k); a
      // run only merges lanes before the next segment head, so j values that
      // recur later in the warp form separate segments
      int key = act ? j : -1 - lane;
      int kprev = __shfl_up_sync(0xffffffffu, key, 1);
      bool head = lane == 0 || kprev != key;
      unsigned heads = __ballot_sync(0xffffffffu, head);
      unsigned after = heads & ~((2u << lane) - 1u);
      int seg_end = after ? __ffs(after) - 1 : 32;
      Real sx = fx, sy = fy, sz = fz;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        Real tx = __shfl_down_sync(0xffffffffu, sx, o);
        Real ty = __shfl_down_sync(0xffffffffu, sy, o);
        Real tz = __shfl_down_sync(0xffffffffu, sz, o);
        if (lane + o < seg_end) {
          sx += tx;
          sy += ty;
          sz += tz;
        }
      }
      // segment heads and a targets add with shared-memory atomics: the
      // same j can head two segments and the same a1 sit in two runs'
      // entries of one step (cheaper than finding the unique targets)
      const bool add0 = act && head;
      if (add0) {
        atomicAdd(&w.gx[j], -sx);
        atomicAdd(&w.gy[j], -sy);
        atomicAdd(&w.gz[j], -sz);
      }
      __syncwarp();
      if (act) {
        Real(*ga)[TILE] = w.ga[lane & (A_COPIES - 1)];
        atomicAdd(&ga[0][a1], fx);
        atomicAdd(&ga[1][a1], fy);
        atomicAdd(&ga[2][a1], fz);
      }
      __syncwarp();  // the next step's adds may touch the same atoms
    }
  }
  return acc;
}

template <typename Real, bool GRAD, int TERM = kTermLJLK, bool COUNT = true>
__device__ __forceinline__ void drain_queue(const EvalCtx<Real>& c,
                                            Slab<Real>* wp, int& nl, int& nh,
                                            int lane, E3<Real>& acc) {
  __syncwarp();
  if (COUNT) {
    cnt_add(wp->counts, 3, nl + nh, lane);
    cnt_add(wp->counts, 4, nh, lane);
  }
  if (nl + nh) {
    E3<Real> e = eval_queue<Real, GRAD, TERM>(c, wp, nl, nh, lane);
    acc.atr += e.atr;
    acc.rep += e.rep;
    acc.lk += e.lk;
  }
  __syncwarp();
  nl = 0;
  nh = 0;
}

__device__ __forceinline__ void queue_push(uint16_t* queue, bool in, bool hv,
                                           int entry, int lane, int& nl,
                                           int& nh) {
  unsigned lt = (1u << lane) - 1;
  unsigned mh = __ballot_sync(0xffffffffu, hv);
  unsigned ml = __ballot_sync(0xffffffffu, in && !hv);
  if ((mh | ml) == 0) return;
  if (hv) queue[QCAP - 1 - (nh + __popc(mh & lt))] = (uint16_t)entry;
  if (in && !hv) queue[nl + __popc(ml & lt)] = (uint16_t)entry;
  nh += __popc(mh);
  nl += __popc(ml);
}

// Pairs inside the side-0 tile of c1 atoms (a1 < a2), weights from the
// intra-block separation table (ljlk_pose_score.impl.hh:115-134; the ligand
// 3/4 -> 5 rule is already folded into that table and is not applied again).
template <typename Real, bool GRAD, int TERM = kTermLJLK, bool COUNT = true>
__device__ TMOL_B200_LJLK_OUTLINE E3<Real> intra_tile(EvalCtx<Real> c, Slab<Real>* wp,
                                            int st1, int c1, int lane) {
  Slab<Real>& w = *wp;
  E3<Real> acc = {0, 0, 0};
  const Real maxd2 = c.max_dis * c.max_dis;
  int nl = 0, nh = 0;
  int npairs = c1 * c1;
  int qq = TILE / c1, rr = TILE - qq * c1;
  int a1 = lane / c1, a2 = lane - a1 * c1;
  for (int base = 0; base < npairs; base += 32) {
    bool in = false, hv = false;
    int wbit = 0;
    if (base + lane < npairs && a1 < a2) {
      const AtomRec<Real> p1 = w.at[a1], p2 = w.at[a2];
      Real dx = p1.x - p2.x;
      Real dy = p1.y - p2.y;
      Real dz = p1.z - p2.z;
      Real d2 = dx * dx + dy * dy + dz * dz;
      if (d2 < maxd2) {
        int sep = c.pd[a1 * c.A + st1 + a2];
        in = sep >= 4;
        wbit = sep == 4;
        hv = TERM == kTermLJLK && in && (p1.tf & p2.tf & kTfHeavy);
      }
    }
    // the row a1 is the entry's k (a row's entries are consecutive)
    queue_push(w.queue, in, hv, a2 | (a1 << 5) | (wbit << 12), lane, nl, nh);
    a1 += qq;
    a2 += rr;
    if (a2 >= c1) {
      a2 -= c1;
      a1 += 1;
    }
  }
  drain_queue<Real, GRAD, TERM, COUNT>(c, wp, nl, nh, lane, acc);
  return acc;
}

// Screen side 0 (c1 atoms, nc1 connections) against the m packed side-1
// atoms of `ns` slots, draining the queue whenever it could overflow.  Lanes
// walk the packed atoms (32 per chunk); side-0 atoms are broadcast one per
// step, skipping those farther than r_k + max_dis from every slot block's
// centroid.  Returns the lane's energy sums.
template <typename Real, bool GRAD, int TERM = kTermLJLK, bool COUNT = true>
__device__ TMOL_B200_LJLK_OUTLINE E3<Real> screen_slots(EvalCtx<Real> c, Slab<Real>* wp,
                                              int c1, int nc1, int m, int ns,
                                              int lane) {
  Slab<Real>& w = *wp;
  E3<Real> acc = {0, 0, 0};
  const Real maxd2 = c.max_dis * c.max_dis;
  bool act0 = false;
  if (lane < c1) {
    const AtomRec<Real> p0 = w.at[lane];
    for (int k = 0; k < ns; ++k) {
      Real dx = p0.x - w.slot_sph[k][0];
      Real dy = p0.y - w.slot_sph[k][1];
      Real dz = p0.z - w.slot_sph[k][2];
      Real rr = w.slot_sph[k][3] + c.max_dis;
      act0 |= dx * dx + dy * dy + dz * dz < rr * rr * Real(1.0001);
    }
  }
  const unsigned rows = __ballot_sync(0xffffffffu, act0);
  const unsigned heavy_rows =
      TERM == kTermLJLK ? __ballot_sync(0xffffffffu, lane < c1 && (w.at[lane].tf & kTfHeavy)) : 0u;
  int nl = 0, nh = 0;
  for (int cbase = 0; cbase < m; cbase += 32) {
    const int j = cbase + lane;
    const bool valid = j < m;
    const int jj = valid ? j : 0;
    const AtomRec<Real> pj = w.at[TILE + jj];
    const Real xj = pj.x, yj = pj.y, zj = pj.z;
    const int heavy_j = TERM == kTermLJLK && valid ? (pj.tf & kTfHeavy) : 0;
    const int slot = w.slot1[jj];
    const int kind = w.slot_kind[slot];
    // count-pair classes of this lane's pairs with the active rows, once per
    // chunk: excl (separation < 4, weight 0) and w02 (separation 4, 0.2)
    unsigned excl = 0, w02 = 0;
    if (valid && kind != kSlotFar) {
      const bool lig = w.slot_lig[slot];
      if (kind == kSlotStriking) {
        // separation through the connections: min over (u, v) of
        // pd1[a1][u] + seps[u][v] + pd2[j][v], capped at 5; the minimum
        // over v depends on this lane only
        const int nc2 = w.slot_nc[slot];
        const uint32_t cpdj = w.cpd1[jj];
        const uint8_t* seps = w.seps[slot];
        int best[MAX_CONN];
#pragma unroll
        for (int u = 0; u < MAX_CONN; ++u) {
          best[u] = 255;
          if (u < nc1)
            for (int v = 0; v < nc2; ++v) {
              const int t = seps[u * 4 + v] + ((cpdj >> (8 * v)) & 0xff);
              best[u] = t < best[u] ? t : best[u];
            }
        }
        for (unsigned rm = rows; rm; rm &= rm - 1) {
          const int a1 = __ffs(rm) - 1;
          const uint32_t c0 = w.cpd0[a1];
          int sep = 5;
#pragma unroll
          for (int u = 0; u < MAX_CONN; ++u) {
            const int t = (int)((c0 >> (8 * u)) & 0xff) + best[u];
            sep = t < sep ? t : sep;
          }
          if (lig && (sep == 3 || sep == 4)) sep = 5;
          excl |= (unsigned)(sep < 4) << a1;
          w02 |= (unsigned)(sep == 4) << a1;
        }
      } else {
        // another tile of block b1: the intra-block separation table
        const uint8_t* pd = c.pd + w.local1[jj];
        for (unsigned rm = rows; rm; rm &= rm - 1) {
          const int a1 = __ffs(rm) - 1;
          int sep = pd[a1 * c.A];
          if (lig && (sep == 3 || sep == 4)) sep = 5;
          excl |= (unsigned)(sep < 4) << a1;
          w02 |= (unsigned)(sep == 4) << a1;
        }
      }
    }
    const unsigned live = valid ? rows & ~excl : 0u;
    // distance tests of this lane's atom against every active row, as a
    // row mask (no per-pair ballots)
    unsigned inm = 0;
    for (unsigned rm = rows; rm; rm &= rm - 1) {
      const int a1 = __ffs(rm) - 1;
      const AtomRec<Real> pa = w.at[a1];
      const Real dx = pa.x - xj;
      const Real dy = pa.y - yj;
      const Real dz = pa.z - zj;
      const Real d2 = dx * dx + dy * dy + dz * dz;
      inm |= (d2 < maxd2 ? 1u : 0u) << a1;
    }
    inm &= live;
    const unsigned hm = heavy_j ? inm & heavy_rows : 0u;
    const unsigned lm = inm & ~hm;
    // each lane's entries go out together (a run of equal k), at offsets
    // from a warp scan of the counts (LJ-only low half-word, heavy high)
    const int cnt = __popc(lm) | (__popc(hm) << 16);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    const int tot = __shfl_sync(0xffffffffu, incl, 31);
    const int tl = tot & 0xffff, th = tot >> 16;
    if (tl + th == 0) continue;
    if (nl + nh + tl + th > QCAP) drain_queue<Real, GRAD, TERM, COUNT>(c, wp, nl, nh, lane, acc);
    const int before = incl - cnt;
    int ql = nl + (before & 0xffff);
    int qh = nh + (before >> 16);
    const int kbits = (TILE + j) << 5;
    for (unsigned b = lm; b; b &= b - 1) {
      const int a1 = __ffs(b) - 1;
      w.queue[ql++] = (uint16_t)(a1 | kbits | (int)(((w02 >> a1) & 1u) << 12));
    }
    for (unsigned b = hm; b; b &= b - 1) {
      const int a1 = __ffs(b) - 1;
      w.queue[QCAP - 1 - qh++] = (uint16_t)(a1 | kbits | (int)(((w02 >> a1) & 1u) << 12));
    }
    nl += tl;
    nh += th;
  }
  drain_queue<Real, GRAD, TERM, COUNT>(c, wp, nl, nh, lane, acc);
  return acc;
}

// Count-pair lookup for (row block, b2): lanes hold the row's partner list.
struct RowPartners {
  int b2;      // this lane's partner block, or -1
  int minsep;  // its minimum bond separation
  int entry;   // its cp table entry
};

// Adds a warp's block-pair energies to entry `o` of the [n_terms, stride]
// output (the warp owns the entry).
template <typename Real, int TERM>
__device__ __forceinline__ void add_pair_energies(Real* out, int64_t stride, int64_t o,
                                                  const E3<Real>& e, int lane) {
  const Real v0 = warp_sum(e.atr);
  if (TERM == kTermElec) {
    if (lane == 0) out[o] += v0;
    return;
  }
  const Real v1 = warp_sum(e.rep), v2 = warp_sum(e.lk);
  if (lane == 0) {
    out[o] += v0;
    out[stride + o] += v1;
    out[2 * stride + o] += v2;
  }
}

// Scores the staged slots against side 0 and flushes their gradients.
template <typename Real, bool GRAD, bool BLOCK_PAIR, int TERM, bool COUNT>
__device__ __forceinline__ void score_group(const ScoreArgs<Real>& s,
                                            Slab<Real>& w, const EvalCtx<Real>& c,
                                            const RowInfo& r, int& m, int& ns,
                                            int lane, E3<Real>& acc,
                                            int64_t pair_o, bool want_E) {
  __syncwarp();
  if (m > 0) {
    E3<Real> e = screen_slots<Real, GRAD, TERM, COUNT>(c, &w, r.c1, r.nc1, m, ns, lane);
    if (GRAD) flush_side1(s, w, m, lane);
    if (BLOCK_PAIR) {
      if (want_E) add_pair_energies<Real, TERM>(s.energies, (int64_t)s.P * s.B * s.B, pair_o, e, lane);
    } else {
      acc.atr += e.atr;
      acc.rep += e.rep;
      acc.lk += e.lk;
    }
  }
  __syncwarp();
  m = 0;
  ns = 0;
}

// The fused kernel.  A work item is (pose p, block b1, candidate range
// [c0, c1) of later blocks b2 >= b1).  Every warp takes items from a global
// ticket, tests b1 against each candidate with the bounding-sphere rule of
// tmol/score/common/sphere_overlap.impl.hh:287-351 (32 per ballot) and
// scores the hits: b1 with itself when b1 is in the range, the other
// neighbours packed into side 1.  GRAD selects the adjoint (which also
// yields the energies when s.energies is set); BLOCK_PAIR selects
// per-block-pair energies / weights instead of per-pose ones (one block pair
// per group).
#ifndef TMOL_B200_FLOAT_MIN_CTAS
#define TMOL_B200_FLOAT_MIN_CTAS 2
#endif

// float: up to 16 warps per CTA (one CTA of 16 warps per SM measured best),
// 128 registers; double: up to 8 warps
template <typename Real, bool GRAD, bool BLOCK_PAIR, int TERM, bool COUNT>
__global__ void __launch_bounds__(sizeof(Real) == 4 ? 512 : 256, 1)
    score_kernel(ScoreArgs<Real> s, int items_per_ticket) {
  if (s.done && *s.done) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Slab<Real>& w = reinterpret_cast<Slab<Real>*>(smem_raw)[warp];
  if (lane < N_COUNTS) w.counts[lane] = 0;
  __syncwarp();
  const bool want_E = !GRAD || s.energies != nullptr;
  const int64_t stride = (int64_t)s.P * s.B * s.B;
  const int max_slots = BLOCK_PAIR ? 1 : s.max_slots;
  const Real reach_atoms = s.g.max_dis;

  const int n_work = s.ticket[2];
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(s.ticket, 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    int it0 = t * items_per_ticket;
    if (it0 >= n_work) break;
    int it1 = min(it0 + items_per_ticket, n_work);
    for (int item = it0; item < it1; ++item) {
      // item costs for plan_rebalance: measured by the counting instantiation
      const long long t_item = COUNT ? clock64() : 0;
      int4 wi = s.work[item];
      RowInfo r;
      r.p = wi.x;
      r.b1 = wi.y;
      int cand0 = wi.z, cand1 = wi.w;
      r.i1 = r.p * s.B + r.b1;
      if (s.blk_info) {
        const int4 bi1 = s.blk_info[r.i1];
        r.bt1 = bi1.x;
        if (r.bt1 < 0) continue;
        r.off1 = bi1.y;
        r.n1 = bi1.z;
        r.nc1 = bi1.w & 0xff;
        r.lig1 = bi1.w >> 8;
      } else {
        r.bt1 = s.blk_bt[r.i1];
        if (r.bt1 < 0) continue;
        r.off1 = s.blk_off[r.i1];
        r.n1 = s.bt_n_atoms[r.bt1];
        r.nc1 = s.bt_n_conn[r.bt1];
        r.lig1 = s.bt_is_ligand[r.bt1];
      }
      E3<Real> acc = {0, 0, 0};
      EvalCtx<Real> ec;
      if (TERM == kTermElec)
        ec.elec_k = s.elec_k;
      else
        ec.ljtab = s.ljtab;
      ec.lktab = s.lktab;
      ec.ntp = s.ntp;
      ec.A = s.A;
      ec.max_dis = s.g.max_dis;
      ec.wt0 = ec.wt1 = ec.wt2 = 0;
      if (GRAD && !BLOCK_PAIR) {
        ec.wt0 = s.dTdV[r.p];
        if (TERM == kTermLJLK) {
          ec.wt1 = s.dTdV[s.P + r.p];
          ec.wt2 = s.dTdV[2 * s.P + r.p];
        }
      }
      const Quad<Real> sph1 = reinterpret_cast<const Quad<Real>*>(s.spheres)[r.i1];
      const Real c1x = sph1.a, c1y = sph1.b, c1z = sph1.c, rad1 = sph1.d;
      const Real reach1 = rad1 + reach_atoms;
      const Real reach1_2 = reach1 * reach1 * Real(1.0001);

      // with a skip mask: the row's count-pair partners, which it never skips
      int skip_ncp = 0, skip_cp = -1;
      if (s.skip) {
        skip_ncp = s.cp_count[r.i1];
        if (lane < skip_ncp) skip_cp = s.cp_b2[r.i1 * CP_CAP + lane];
      }

      // neighbour tests of the whole range first: one ballot mask per 32
      // candidates, kept in registers (lane k holds the mask of batch k)
      unsigned my_mask = 0;
      int n_batches = (cand1 - cand0 + 31) / 32;
      for (int bi = 0; bi < n_batches; ++bi) {
        int b2 = cand0 + bi * 32 + lane;
        bool hit = false;
        if (b2 < cand1) {
          int i2 = r.p * s.B + b2;
          if (s.blk_bt[i2] >= 0) {
            const Quad<Real> s2 = reinterpret_cast<const Quad<Real>*>(s.spheres)[i2];
            Real dx = sub_rn(c1x, s2.a);
            Real dy = sub_rn(c1y, s2.b);
            Real dz = sub_rn(c1z, s2.c);
            Real d2 = add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
            Real thr = add_rn(add_rn(rad1, s2.d), s.reach);
            hit = d2 < mul_rn(thr, thr);
          }
          if (s.nbr) s.nbr[(int64_t)r.i1 * s.B + b2] = hit ? 1 : 0;
        }
        if (s.skip) {
          // a screened-out pair is dropped unless it is b1 itself or one of
          // b1's count-pair partners (bond separation <= 4)
          bool drop = hit && b2 != r.b1 &&
                      ((s.skip[(int64_t)r.i1 * s.skip_words + (b2 >> 5)] >> (b2 & 31)) & 1u);
          for (int k = 0; k < skip_ncp; ++k)
            if (__shfl_sync(0xffffffffu, skip_cp, k) == b2) drop = false;
          if (drop) hit = false;
        }
        unsigned mk = __ballot_sync(0xffffffffu, hit);
        if (lane == bi) my_mask = mk;
      }
      bool any = __any_sync(0xffffffffu, my_mask != 0);
      if (!any) {
        if (COUNT && s.item_cost && lane == 0)
          s.item_cost[item] = (int)min((clock64() - t_item) >> 4, (long long)0x7fffffff);
        continue;
      }

      // the row's count-pair partners, one per lane
      RowPartners rp;
      {
        int ncp = s.cp_count[r.i1];
        rp.b2 = -1;
        rp.minsep = 6;
        rp.entry = r.i1 * CP_CAP + lane;
        if (lane < ncp) {
          rp.b2 = s.cp_b2[rp.entry];
          rp.minsep = s.cp_minsep[rp.entry];
        }
      }
      int nt1 = (r.n1 + TILE - 1) / TILE;
      for (int ti = 0; ti < nt1; ++ti) {
        r.st1 = ti * TILE;
        r.c1 = min(TILE, r.n1 - r.st1);
        stage_side0<Real, TERM>(s, w, r.bt1, r.off1, r.st1, r.c1, r.nc1, lane);
        ec.pd = s.bt_pd + ((int64_t)r.bt1 * s.A + r.st1) * s.A;
        __syncwarp();
        int h1 = COUNT && TERM == kTermLJLK
                     ? __popc(__ballot_sync(0xffffffffu, lane < r.c1 && (w.at[lane].tf & kTfHeavy)))
                     : 0;
        int m = 0, ns = 0;
        int64_t pair_o = 0;
        for (int bi = 0; bi < n_batches; ++bi) {
          unsigned mask = __shfl_sync(0xffffffffu, my_mask, bi);
          while (mask) {
            int k = __ffs(mask) - 1;
            mask &= mask - 1;
            int bb2 = cand0 + bi * 32 + k;
            if (bb2 == r.b1) {
              // b1 with itself: this tile with itself, then with b1's later tiles
              score_group<Real, GRAD, BLOCK_PAIR, TERM, COUNT>(s, w, ec, r, m, ns, lane, acc, pair_o, want_E);
              pair_o = (int64_t)r.i1 * s.B + r.b1;
              if (BLOCK_PAIR && GRAD) {
                ec.wt0 = s.dTdV[pair_o];
                if (TERM == kTermLJLK) {
                  ec.wt1 = s.dTdV[stride + pair_o];
                  ec.wt2 = s.dTdV[2 * stride + pair_o];
                }
              }
              if (COUNT) {
                if (ti == 0) {
                  cnt_add(w.counts, 0, 1, lane);
                  cnt_add(w.counts, 1, (long long)r.n1 * (r.n1 - 1) / 2, lane);
                }
                cnt_add(w.counts, 2, (long long)h1 * (h1 - 1) / 2, lane);
              }
              {
                E3<Real> e = intra_tile<Real, GRAD, TERM, COUNT>(ec, &w, r.st1, r.c1, lane);
                if (BLOCK_PAIR) {
                  if (want_E) add_pair_energies<Real, TERM>(s.energies, stride, pair_o, e, lane);
                } else {
                  acc.atr += e.atr;
                  acc.rep += e.rep;
                  acc.lk += e.lk;
                }
              }
              for (int tj = ti + 1; tj < nt1; ++tj) {
                int st2 = tj * TILE, c2 = min(TILE, r.n1 - st2);
                if (lane == 0) {
                  w.slot_kind[0] = kSlotIntra;
                  w.slot_nc[0] = 0;
                  w.slot_lig[0] = 0;
                  w.slot_sph[0][0] = c1x;
                  w.slot_sph[0][1] = c1y;
                  w.slot_sph[0][2] = c1z;
                  w.slot_sph[0][3] = rad1;
                }
                int h2 = 0;
                m = stage_side1<Real, TERM>(s, w, 0, 0, r.bt1, r.off1, st2, c2, 0, c1x, c1y, c1z, reach1_2, lane,
                                            COUNT ? &h2 : nullptr);
                if (COUNT) cnt_add(w.counts, 2, (long long)h1 * h2, lane);
                ns = 1;
                score_group<Real, GRAD, BLOCK_PAIR, TERM, COUNT>(s, w, ec, r, m, ns, lane, acc, pair_o, want_E);
              }
              continue;
            }
            int i2 = r.p * s.B + bb2;
            int bt2, off2, n2, nc2_all, lig2;
            if (s.blk_info) {
              const int4 bi2 = s.blk_info[i2];
              bt2 = bi2.x;
              off2 = bi2.y;
              n2 = bi2.z;
              nc2_all = bi2.w & 0xff;
              lig2 = bi2.w >> 8;
            } else {
              bt2 = s.blk_bt[i2];
              off2 = s.blk_off[i2];
              n2 = s.bt_n_atoms[bt2];
              nc2_all = s.bt_n_conn[bt2];
              lig2 = s.bt_is_ligand[bt2];
            }
            int nt2 = (n2 + TILE - 1) / TILE;
            unsigned pm = __ballot_sync(0xffffffffu, rp.b2 == bb2);
            int kind = kSlotFar, nc2 = 0, e = 0;
            if (pm) {
              int src = __ffs(pm) - 1;
              int msep = __shfl_sync(0xffffffffu, rp.minsep, src);
              e = __shfl_sync(0xffffffffu, rp.entry, src);
              kind = msep <= 4 ? kSlotStriking : kSlotFar;
            }
            if (kind == kSlotStriking) nc2 = nc2_all;
            int lig = r.lig1 && lig2;
            const Real* s2 = s.spheres + 4 * (int64_t)i2;
            if (COUNT && ti == 0) {
              cnt_add(w.counts, 0, 1, lane);
              cnt_add(w.counts, 1, (long long)r.n1 * n2, lane);
            }
            for (int tj = 0; tj < nt2; ++tj) {
              int st2 = tj * TILE, c2 = min(TILE, n2 - st2);
              if (m + c2 > M1 || ns == max_slots)
                score_group<Real, GRAD, BLOCK_PAIR, TERM, COUNT>(s, w, ec, r, m, ns, lane, acc, pair_o, want_E);
              if (lane == 0) {
                w.slot_kind[ns] = kind;
                w.slot_nc[ns] = nc2;
                w.slot_lig[ns] = lig;
              }
              if (lane < 4) w.slot_sph[ns][lane] = s2[lane];
              if (kind == kSlotStriking && lane < 16) w.seps[ns][lane] = s.cp_seps[(int64_t)e * 16 + lane];
              int h2 = 0;
              int kept = stage_side1<Real, TERM>(s, w, m, ns, bt2, off2, st2, c2, nc2, c1x, c1y, c1z, reach1_2, lane,
                                                 COUNT ? &h2 : nullptr);
              if (COUNT) cnt_add(w.counts, 2, (long long)h1 * h2, lane);
              if (kept > 0) {
                m += kept;
                ns += 1;
              }
              if (BLOCK_PAIR) {
                pair_o = (int64_t)r.i1 * s.B + bb2;
                if (GRAD) {
                  ec.wt0 = s.dTdV[pair_o];
                  if (TERM == kTermLJLK) {
                    ec.wt1 = s.dTdV[stride + pair_o];
                    ec.wt2 = s.dTdV[2 * stride + pair_o];
                  }
                }
              }
            }
          }
        }
        score_group<Real, GRAD, BLOCK_PAIR, TERM, COUNT>(s, w, ec, r, m, ns, lane, acc, pair_o, want_E);
        if (GRAD) flush_side0(s, w, r.off1, r.st1, r.c1, lane);
        __syncwarp();
      }
      if (!BLOCK_PAIR && want_E) {
        Real v0 = warp_sum(acc.atr);
        Real v1 = TERM == kTermLJLK ? warp_sum(acc.rep) : Real(0);
        Real v2 = TERM == kTermLJLK ? warp_sum(acc.lk) : Real(0);
        if (lane == 0) {
          if (v0 != Real(0)) atomicAdd(&s.energies[r.p], v0);
          if (v1 != Real(0)) atomicAdd(&s.energies[s.P + r.p], v1);
          if (v2 != Real(0)) atomicAdd(&s.energies[2 * s.P + r.p], v2);
        }
      }
      if (COUNT && s.item_cost && lane == 0)
        s.item_cost[item] = (int)min((clock64() - t_item) >> 4, (long long)0x7fffffff);
    }
  }
  __syncwarp();
  if (COUNT && s.counts && lane < N_COUNTS && w.counts[lane])
    atomicAdd(&s.counts[lane], w.counts[lane]);
}

// ---------------------------------------------------------------------------
// Rotamer scoring (tmol's ljlk_rotamer_scores, ljlk_pose_score.impl.hh:
// 1479-2126): every block owns a range of rotamers, each with its own block
// type and coordinates; the energies of every rotamer pair of neighbouring
// blocks (and of each rotamer with itself) are reported separately.

// Rotamer indexing for the rotamer kernels.
struct RotArgs {
  const int* rot_bt;     // [R] block type of each rotamer
  const int* rot_off;    // [R] first coordinate row
  const int* rot_block;  // [R]
  const int* rot_pose;   // [R]
  const int* nrb;        // [P*B] rotamers per block
  const int* rob;        // [P*B] first rotamer of each block
  int R;
  long long* row_pairs;  // [P*B] rotamer pairs per row (then their offsets)
  long long* row_items;  // [P*B] work items per row (then their offsets)
  int4* items;           // (rot1, first rot2, n rot2, first pair)
  long long n_items;
  int32_t* indices;      // [3, n_pairs] (pose, rot1, rot2)
  long long n_pairs;
};

// Bounding sphere of each rotamer, as spheres_kernel (the reference's
// compute_rot_spheres on the CPU, sphere_overlap.impl.hh:23-107).
template <typename Real>
__global__ void rot_spheres_kernel(ScoreArgs<Real> s, RotArgs ra, Real* rs) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < ra.R; r += warps)
    warp_sphere(s.coords, s.bt_n_atoms, ra.rot_bt[r], ra.rot_off[r], lane, rs + 4 * (int64_t)r);
}

// Block spheres enclosing all rotamers of each block: the mean of the
// rotamer centres and the largest centre distance plus rotamer radius
// (compute_block_spheres_from_rot_spheres, sphere_overlap.impl.hh:455-510),
// in the reference's order.
template <typename Real>
__global__ void block_spheres_from_rots_kernel(ScoreArgs<Real> s, RotArgs ra, const Real* rs) {
  const int n_blocks = s.P * s.B;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_blocks; i += gridDim.x * blockDim.x) {
    Real* out = s.spheres + 4 * (int64_t)i;
    const int n = ra.nrb[i], r0 = ra.rob[i];
    if (s.blk_bt[i] < 0 || n <= 0 || r0 < 0) {
      out[0] = out[1] = out[2] = out[3] = Real(0);
      continue;
    }
    Real cx = 0, cy = 0, cz = 0;
    for (int r = 0; r < n; ++r) {
      const Real* q = rs + 4 * (int64_t)(r0 + r);
      cx = add_rn(cx, q[0]);
      cy = add_rn(cy, q[1]);
      cz = add_rn(cz, q[2]);
    }
    const Real rn = Real(n);
    cx = div_rn(cx, rn);
    cy = div_rn(cy, rn);
    cz = div_rn(cz, rn);
    Real rmax = 0;
    for (int r = 0; r < n; ++r) {
      const Real* q = rs + 4 * (int64_t)(r0 + r);
      Real dx = sub_rn(q[0], cx), dy = sub_rn(q[1], cy), dz = sub_rn(q[2], cz);
      Real d = add_rn(sqrt_rn(add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz))), q[3]);
      if (d > rmax) rmax = d;
    }
    out[0] = cx;
    out[1] = cy;
    out[2] = cz;
    out[3] = rmax;
  }
}

// The reference neighbour rule between blocks i1 and i2 (bit-exact).
template <typename Real>
__device__ __forceinline__ bool block_hit(const ScoreArgs<Real>& s, int i1, int i2) {
  if (s.blk_bt[i2] < 0) return false;
  const Real* s1 = s.spheres + 4 * (int64_t)i1;
  const Real* s2 = s.spheres + 4 * (int64_t)i2;
  Real dx = sub_rn(s1[0], s2[0]);
  Real dy = sub_rn(s1[1], s2[1]);
  Real dz = sub_rn(s1[2], s2[2]);
  Real d2 = add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
  Real thr = add_rn(add_rn(s1[3], s2[3]), s.reach);
  return d2 < mul_rn(thr, thr);
}

// Per row (p, b1): how many rotamer pairs and work items its neighbouring
// blocks b2 >= b1 dispatch (n(b1) on the diagonal, n(b1) * n(b2) off it;
// one item per rotamer of b1 and neighbour).
template <typename Real>
__global__ void rot_row_count_kernel(ScoreArgs<Real> s, RotArgs ra) {
  const int lane = threadIdx.x & 31;
  const int n_rows = s.P * s.B;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n_rows; row += warps) {
    long long pairs = 0, items = 0;
    if (s.blk_bt[row] >= 0) {
      const int p = row / s.B, b1 = row - p * s.B;
      const long long n1 = ra.nrb[row];
      for (int b2 = b1 + lane; b2 < s.pose_last[p]; b2 += 32) {
        const int i2 = p * s.B + b2;
        if (!block_hit(s, row, i2)) continue;
        pairs += b2 == b1 ? n1 : n1 * ra.nrb[i2];
        items += n1;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
      items += __shfl_xor_sync(0xffffffffu, items, o);
    }
    if (lane == 0) {
      ra.row_pairs[row] = pairs;
      ra.row_items[row] = items;
    }
  }
}

// Exclusive scans of a[0..n) and b[0..n) in place, totals into t[0], t[1];
// one CTA of 1024 threads, each scanning a contiguous chunk.
__global__ void __launch_bounds__(1024) scan2_kernel(long long* a, long long* b, int n,
                                                     long long* t) {
  __shared__ long long sa[1024], sb[1024];
  const int tid = threadIdx.x;
  const int chunk = (n + 1023) / 1024;
  const int lo = min(n, tid * chunk), hi = min(n, lo + chunk);
  long long va = 0, vb = 0;
  for (int i = lo; i < hi; ++i) {
    va += a[i];
    vb += b[i];
  }
  sa[tid] = va;
  sb[tid] = vb;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    long long xa = tid >= o ? sa[tid - o] : 0, xb = tid >= o ? sb[tid - o] : 0;
    __syncthreads();
    sa[tid] += xa;
    sb[tid] += xb;
    __syncthreads();
  }
  long long ra_ = sa[tid] - va, rb_ = sb[tid] - vb;
  for (int i = lo; i < hi; ++i) {
    const long long xa = a[i], xb = b[i];
    a[i] = ra_;
    b[i] = rb_;
    ra_ += xa;
    rb_ += xb;
  }
  if (tid == 1023) {
    t[0] = sa[1023];
    t[1] = sb[1023];
  }
}

// Writes the dispatch indices (pose, rot1, rot2) in the reference's order
// (pose, b1, b2, rotamer of b1, rotamer of b2) and the work items, row by
// row from the scanned offsets.
template <typename Real>
__global__ void rot_row_fill_kernel(ScoreArgs<Real> s, RotArgs ra) {
  const int lane = threadIdx.x & 31;
  const int n_rows = s.P * s.B;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const long long np = ra.n_pairs;
  for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n_rows; row += warps) {
    if (s.blk_bt[row] < 0) continue;
    const int p = row / s.B, b1 = row - p * s.B;
    const int n1 = ra.nrb[row], o1 = ra.rob[row];
    long long pair_off = ra.row_pairs[row], item_off = ra.row_items[row];
    for (int base = b1; base < s.pose_last[p]; base += 32) {
      const int b2l = base + lane;
      const bool hit = b2l < s.pose_last[p] && block_hit(s, row, p * s.B + b2l);
      unsigned m = __ballot_sync(0xffffffffu, hit);
      while (m) {
        const int k = __ffs(m) - 1;
        m &= m - 1;
        const int b2 = base + k;
        const int i2 = p * s.B + b2;
        const bool diag = b2 == b1;
        const int n2 = diag ? 1 : ra.nrb[i2];
        const int o2 = ra.rob[i2];
        for (int i = lane; i < n1; i += 32) {
          const long long first = pair_off + (long long)i * n2;
          if (item_off + i < ra.n_items)
            ra.items[item_off + i] = make_int4(o1 + i, diag ? o1 + i : o2, n2, (int)first);
        }
        const long long cnt = (long long)n1 * n2;
        for (long long q = lane; q < cnt; q += 32) {
          const long long d = pair_off + q;
          if (d >= np) break;
          const int i = (int)(q / n2), j = (int)(q - (long long)i * n2);
          ra.indices[d] = p;
          ra.indices[np + d] = o1 + i;
          ra.indices[2 * np + d] = diag ? o1 + i : o2 + j;
        }
        pair_off += cnt;
        item_off += n1;
      }
    }
  }
}

// Scoring of work items: rotamer rot1 (side 0, tile by tile) against the
// rotamers rot2 of one neighbouring block (side 1, one rotamer tile per
// group), or against itself on the diagonal.  Energies go to the item's
// pairs (energies[t * n_pairs + d]; the warp owns them), the adjoint
// weights come from dTdV[t * n_pairs + d].
template <typename Real, bool GRAD, int TERM, bool COUNT>
__global__ void __launch_bounds__(256, sizeof(Real) == 4 ? TMOL_B200_FLOAT_MIN_CTAS : 1)
    rotamer_kernel(ScoreArgs<Real> s, RotArgs ra, const Real* rs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Slab<Real>& w = reinterpret_cast<Slab<Real>*>(smem_raw)[warp];
  if (lane < N_COUNTS) w.counts[lane] = 0;
  __syncwarp();
  const long long np = ra.n_pairs;
  const bool want_E = s.energies != nullptr;
  const Real reach_atoms = s.g.max_dis;
  for (;;) {
    int it = 0;
    if (lane == 0) it = atomicAdd(s.ticket, 1);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= ra.n_items) break;
    const int4 item = ra.items[it];
    const int rot1 = item.x, rot2_first = item.y, n_rot2 = item.z;
    const long long pair_first = item.w;
    RowInfo r;
    r.p = ra.rot_pose[rot1];
    r.b1 = ra.rot_block[rot1];
    r.i1 = r.p * s.B + r.b1;
    r.bt1 = ra.rot_bt[rot1];
    r.off1 = ra.rot_off[rot1];
    r.n1 = s.bt_n_atoms[r.bt1];
    r.nc1 = s.bt_n_conn[r.bt1];
    r.lig1 = s.bt_is_ligand[r.bt1];
    EvalCtx<Real> ec;
    if (TERM == kTermElec)
      ec.elec_k = s.elec_k;
    else
      ec.ljtab = s.ljtab;
    ec.lktab = s.lktab;
    ec.ntp = s.ntp;
    ec.A = s.A;
    ec.max_dis = s.g.max_dis;
    ec.wt0 = ec.wt1 = ec.wt2 = 0;
    const Real* sph1 = rs + 4 * (int64_t)rot1;
    const Real c1x = sph1[0], c1y = sph1[1], c1z = sph1[2], rad1 = sph1[3];
    const Real reach1 = rad1 + reach_atoms;
    const Real reach1_2 = reach1 * reach1 * Real(1.0001);
    const bool diag = rot2_first == rot1;
    // block-level count pair of (b1, b2): kind and connection separations
    int kind = kSlotFar, cp_entry = 0, b2 = diag ? r.b1 : ra.rot_block[rot2_first];
    if (!diag) {
      const int ncp = s.cp_count[r.i1];
      const int e = r.i1 * CP_CAP + lane;
      const bool match = lane < ncp && s.cp_b2[e] == b2;
      const unsigned pm = __ballot_sync(0xffffffffu, match);
      if (pm) {
        const int src = __ffs(pm) - 1;
        const int msep = __shfl_sync(0xffffffffu, lane < ncp ? s.cp_minsep[e] : 6, src);
        cp_entry = r.i1 * CP_CAP + src;
        kind = msep <= 4 ? kSlotStriking : kSlotFar;
      }
    }
    const int nt1 = (r.n1 + TILE - 1) / TILE;
    for (int ti = 0; ti < nt1; ++ti) {
      r.st1 = ti * TILE;
      r.c1 = min(TILE, r.n1 - r.st1);
      stage_side0<Real, TERM>(s, w, r.bt1, r.off1, r.st1, r.c1, r.nc1, lane);
      ec.pd = s.bt_pd + ((int64_t)r.bt1 * s.A + r.st1) * s.A;
      __syncwarp();
      for (int k = 0; k < n_rot2; ++k) {
        const long long d = pair_first + k;
        if (GRAD) {
          ec.wt0 = s.dTdV[d];
          if (TERM == kTermLJLK) {
            ec.wt1 = s.dTdV[np + d];
            ec.wt2 = s.dTdV[2 * np + d];
          }
        }
        E3<Real> e = {0, 0, 0};
        if (ti == 0) {
          const long long n2a = diag ? 0 : s.bt_n_atoms[ra.rot_bt[rot2_first + k]];
          if (COUNT) {
            cnt_add(w.counts, 0, 1, lane);
            cnt_add(w.counts, 1, diag ? (long long)r.n1 * (r.n1 - 1) / 2 : (long long)r.n1 * n2a, lane);
          }
        }
        if (diag) {
          // this tile with itself, then with the rotamer's later tiles
          E3<Real> t = intra_tile<Real, GRAD, TERM, COUNT>(ec, &w, r.st1, r.c1, lane);
          e.atr += t.atr;
          e.rep += t.rep;
          e.lk += t.lk;
          for (int tj = ti + 1; tj < nt1; ++tj) {
            const int st2 = tj * TILE, c2 = min(TILE, r.n1 - st2);
            if (lane == 0) {
              w.slot_kind[0] = kSlotIntra;
              w.slot_nc[0] = 0;
              w.slot_lig[0] = 0;
              w.slot_sph[0][0] = c1x;
              w.slot_sph[0][1] = c1y;
              w.slot_sph[0][2] = c1z;
              w.slot_sph[0][3] = rad1;
            }
            const int m = stage_side1<Real, TERM>(s, w, 0, 0, r.bt1, r.off1, st2, c2, 0, c1x, c1y, c1z, reach1_2, lane);
            __syncwarp();
            if (m > 0) {
              E3<Real> g = screen_slots<Real, GRAD, TERM, COUNT>(ec, &w, r.c1, r.nc1, m, 1, lane);
              if (GRAD) flush_side1(s, w, m, lane);
              e.atr += g.atr;
              e.rep += g.rep;
              e.lk += g.lk;
            }
            __syncwarp();
          }
        } else {
          const int rot2 = rot2_first + k;
          const int bt2 = ra.rot_bt[rot2], off2 = ra.rot_off[rot2];
          const int nc2 = kind == kSlotStriking ? s.bt_n_conn[bt2] : 0;
          const int lig = r.lig1 && s.bt_is_ligand[bt2];
          const Real* sph2 = rs + 4 * (int64_t)rot2;
          // every atom of rot2 lies within its radius of its centre: when the
          // spheres are farther apart than both radii plus the reach, the
          // atom cull would drop them all, so the pair is left at zero
          const Real sx = sph2[0] - c1x, sy = sph2[1] - c1y, sz = sph2[2] - c1z;
          const Real lim = reach1 + sph2[3];
          const int n2 = sx * sx + sy * sy + sz * sz < lim * lim * Real(1.0001) ? s.bt_n_atoms[bt2] : 0;
          for (int st2 = 0; st2 < n2; st2 += TILE) {
            const int c2 = min(TILE, n2 - st2);
            if (lane == 0) {
              w.slot_kind[0] = kind;
              w.slot_nc[0] = nc2;
              w.slot_lig[0] = lig;
            }
            if (lane < 4) w.slot_sph[0][lane] = sph2[lane];
            if (kind == kSlotStriking && lane < 16) w.seps[0][lane] = s.cp_seps[(int64_t)cp_entry * 16 + lane];
            const int m = stage_side1<Real, TERM>(s, w, 0, 0, bt2, off2, st2, c2, nc2, c1x, c1y, c1z, reach1_2, lane);
            __syncwarp();
            if (m > 0) {
              E3<Real> g = screen_slots<Real, GRAD, TERM, COUNT>(ec, &w, r.c1, r.nc1, m, 1, lane);
              if (GRAD) flush_side1(s, w, m, lane);
              e.atr += g.atr;
              e.rep += g.rep;
              e.lk += g.lk;
            }
            __syncwarp();
          }
        }
        if (want_E) add_pair_energies<Real, TERM>(s.energies, np, d, e, lane);
      }
      if (GRAD) flush_side0(s, w, r.off1, r.st1, r.c1, lane);
      __syncwarp();
    }
  }
  __syncwarp();
  if (COUNT && s.counts && lane < N_COUNTS && w.counts[lane])
    atomicAdd(&s.counts[lane], w.counts[lane]);
}

#include "lkball.cuh"

// Sub-spheres of every block for the screen's features: atoms [0, 4) (the
// backbone N, CA, C, O of an amino acid) and atoms [4, n) (the rest; the
// first part again when n <= 4), each as centroid + largest centroid
// distance.  Plain fp32: these are network inputs, not neighbour tests.
__global__ void sub_spheres_kernel(ScoreArgs<float> s, float* sub) {
  const int n_blocks = s.P * s.B;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_blocks; i += gridDim.x * blockDim.x) {
    float* out = sub + 8 * (int64_t)i;
    const int bt = s.blk_bt[i];
    if (bt < 0) {
      for (int k = 0; k < 8; ++k) out[k] = 0.0f;
      continue;
    }
    const int n = s.bt_n_atoms[bt];
    const float* x = s.coords + 3 * (int64_t)s.blk_off[i];
    for (int part = 0; part < 2; ++part) {
      int a0 = 0, a1 = n < 4 ? n : 4;
      if (part == 1 && n > 4) {
        a0 = 4;
        a1 = n;
      }
      float cx = 0, cy = 0, cz = 0;
      for (int k = a0; k < a1; ++k) {
        cx += x[3 * k];
        cy += x[3 * k + 1];
        cz += x[3 * k + 2];
      }
      const float inv = a1 > a0 ? 1.0f / (float)(a1 - a0) : 0.0f;
      cx *= inv;
      cy *= inv;
      cz *= inv;
      float r2 = 0;
      for (int k = a0; k < a1; ++k) {
        float dx = x[3 * k] - cx, dy = x[3 * k + 1] - cy, dz = x[3 * k + 2] - cz;
        r2 = fmaxf(r2, dx * dx + dy * dy + dz * dz);
      }
      out[4 * part + 0] = cx;
      out[4 * part + 1] = cy;
      out[4 * part + 2] = cz;
      out[4 * part + 3] = sqrtf(r2);
    }
  }
}

__device__ __forceinline__ float dist3(float ax, float ay, float az, float bx, float by, float bz) {
  return sqrtf((ax - bx) * (ax - bx) + (ay - by) * (ay - by) + (az - bz) * (az - bz));
}

// Block-pair screen candidates: every later block b2 of row (p, b1) that
// passes the scoring kernel's sphere test (same arithmetic, so the same
// pairs) and is not a count-pair partner (bond separation <= 4).  Appends
// (row, b2), both block types and 12 features per pair in warp-aggregated
// chunks; *count ends as the total, entries past `capacity` are not written.
// Features (fp32), with c, r the block spheres, d = |c1 - c2|, a a block's
// first atom and (u, v) the sub-spheres of sub_spheres_kernel:
//   d/10, (d - r1 - r2)/6, r1/5, r2/5, log2(b2 - b1)/10,
//   (|a1 - a2| - d)/5, (|a1 - c2| - d)/5, (|a2 - c1| - d)/5,
//   then (|u1 - u2| - r_u1 - r_u2)/6 for (u1, u2) = (0,0), (0,1), (1,0), (1,1).
__global__ void screen_candidates_kernel(ScoreArgs<float> s, const float* sub,
                                         int capacity, int32_t* pair_row,
                                         int32_t* pair_b2, int32_t* pair_bt,
                                         float* feats, int32_t* count) {
  const int lane = threadIdx.x & 31;
  const int n_rows = s.P * s.B;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n_rows; row += warps) {
    const int bt1 = s.blk_bt[row];
    if (bt1 < 0) continue;
    const int p = row / s.B, b1 = row - p * s.B;
    const int last = s.pose_last[p];
    const float* sph1 = s.spheres + 4 * (int64_t)row;
    const float c1x = sph1[0], c1y = sph1[1], c1z = sph1[2], rad1 = sph1[3];
    const float* a1 = s.coords + 3 * (int64_t)s.blk_off[row];
    const float a1x = a1[0], a1y = a1[1], a1z = a1[2];
    const float* u1 = sub + 8 * (int64_t)row;
    const int ncp = s.cp_count[row];
    const int my_cp = lane < ncp ? s.cp_b2[row * CP_CAP + lane] : -1;
    for (int base = b1 + 1; base < last; base += 32) {
      const int b2 = base + lane;
      const int i2 = p * s.B + b2;
      bool take = false;
      int bt2 = -1;
      if (b2 < last) {
        bt2 = s.blk_bt[i2];
        if (bt2 >= 0) {
          const float* s2 = s.spheres + 4 * (int64_t)i2;
          float dx = sub_rn(c1x, s2[0]);
          float dy = sub_rn(c1y, s2[1]);
          float dz = sub_rn(c1z, s2[2]);
          float d2 = add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
          float thr = add_rn(add_rn(rad1, s2[3]), s.reach);
          take = d2 < mul_rn(thr, thr);
        }
      }
      for (int k = 0; k < ncp; ++k)
        if (__shfl_sync(0xffffffffu, my_cp, k) == b2) take = false;
      const unsigned m = __ballot_sync(0xffffffffu, take);
      if (!m) continue;
      int first = 0;
      if (lane == 0) first = atomicAdd(count, __popc(m));
      first = __shfl_sync(0xffffffffu, first, 0);
      if (!take) continue;
      const int idx = first + __popc(m & ((1u << lane) - 1u));
      if (idx >= capacity) continue;
      const float* s2 = s.spheres + 4 * (int64_t)i2;
      const float* a2 = s.coords + 3 * (int64_t)s.blk_off[i2];
      const float* u2 = sub + 8 * (int64_t)i2;
      const float c2x = s2[0], c2y = s2[1], c2z = s2[2], rad2 = s2[3];
      const float a2x = a2[0], a2y = a2[1], a2z = a2[2];
      const float d = dist3(c1x, c1y, c1z, c2x, c2y, c2z);
      float* f = feats + 12 * (int64_t)idx;
      f[0] = d * 0.1f;
      f[1] = (d - rad1 - rad2) * (1.0f / 6.0f);
      f[2] = rad1 * 0.2f;
      f[3] = rad2 * 0.2f;
      f[4] = log2f((float)(b2 - b1)) * 0.1f;
      f[5] = (dist3(a1x, a1y, a1z, a2x, a2y, a2z) - d) * 0.2f;
      f[6] = (dist3(a1x, a1y, a1z, c2x, c2y, c2z) - d) * 0.2f;
      f[7] = (dist3(a2x, a2y, a2z, c1x, c1y, c1z) - d) * 0.2f;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float* x1 = u1 + 4 * (q >> 1);
        const float* x2 = u2 + 4 * (q & 1);
        f[8 + q] = (dist3(x1[0], x1[1], x1[2], x2[0], x2[1], x2[2]) - x1[3] - x2[3]) * (1.0f / 6.0f);
      }
      pair_row[idx] = row;
      pair_b2[idx] = b2;
      pair_bt[2 * idx] = bt1;
      pair_bt[2 * idx + 1] = bt2;
    }
  }
}

// FP32 issue-rate probe: 8 independent FMA chains per thread, so that the
// FMA pipe, not latency, bounds it.  2 FLOP per FMA.
__global__ void fp32_peak_kernel(float* out, int iters, float a, float b) {
  float x[8];
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-3f + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = fmaf(x[k], a, b);
  }
  float acc = 0;
  for (int k = 0; k < 8; ++k) acc += x[k];
  if (acc == 1234.5f) out[0] = acc;  // keeps the chains live
}

}  // namespace tmol_b200

// ---------------------------------------------------------------------------
// host side

using namespace tmol_b200;

struct tmol_b200_ljlk_plan {
  int real_bytes;
  int term = kTermLJLK;
  void* bt_q = nullptr;    // elec: partial charges [nbt * A] reals
  void* elec_k = nullptr;  // elec: ElecK constants [N_ELEC_K] reals
  unsigned char elec_k_host[N_ELEC_K * sizeof(double)];
  // LK-ball plans: water sites [N * 4], per block type polar / occluder
  // atom lists and per-atom parameters [nbt * A * 9] reals
  void* lkb_sites = nullptr;
  int* lkb_pol = nullptr;
  int* lkb_npol = nullptr;
  int* lkb_occ = nullptr;
  int* lkb_nocc = nullptr;
  int* lkb_nbocc = nullptr;
  int lkb_maxpol = 0, lkb_maxocc = 0;
  void* lkb_par = nullptr;
  double lkb_water_dist = 0;
  int* lkb_active = nullptr;    // occupied water sites, ascending
  int64_t lkb_n_active = 0;
  void* lkb_waters = nullptr;   // [N, 4, 3] scratch of the one-call energy + gradient (NaN in empty slots)
  void* lkb_dwaters = nullptr;
  tmol_b200_ljlk_inputs dims;  // sizes only; pointers are not kept
  int P, B, nbt, A, C, ntiles, T;
  int64_t N;
  double reach;
  int* blk_bt = nullptr;
  int* blk_off = nullptr;
  int4* blk_info = nullptr;  // pose plans of LJ/LK and elec: {bt, off, n_atoms, n_conn | ligand << 8}
  void* packed = nullptr;    // and their atoms as staged records [n_atoms], rewritten every call
  int* pose_last = nullptr;
  uint16_t* bt_tf = nullptr;
  int* type_map = nullptr;
  int* compact_types = nullptr;
  void* ljtab = nullptr;
  void* lktab = nullptr;
  int ntp = 0;
  uint8_t* bt_pd = nullptr;
  uint8_t* bt_conn_pd = nullptr;
  int* bt_flags = nullptr;
  int* bt_n_atoms = nullptr;
  int* bt_n_conn = nullptr;
  int* bt_is_ligand = nullptr;
  int* cp_count = nullptr;
  int* cp_b2 = nullptr;
  int* cp_minsep = nullptr;
  uint8_t* cp_seps = nullptr;
  int4* work = nullptr;
  int* item_cost = nullptr;
  int n_work = 0;
  int work_cap = 0;  // capacity of work / item_cost
  void* spheres = nullptr;
  int* counters = nullptr;  // [0] ticket, [1] status, [2] work items
  unsigned long long* counts = nullptr;  // [N_COUNTS] of the last forward
  bool counting = false;  // whole-pose LJ/LK and elec kernels fill `counts`
  // speculative gradient of the pose ops: the weights of the last
  // backward (for the next speculative forward), the weights the last
  // speculative forward used and the gradient it took with them, and the
  // device flag a backward sets when its weights match those
  void* spec_next = nullptr;  // [n_terms, P]
  void* spec_used = nullptr;  // [n_terms, P]
  void* spec_g = nullptr;     // [N, 3]
  void* spec_dw = nullptr;    // LK-ball: [N, 4, 3], the waters' gradient
  int* spec_flag = nullptr;
  bool spec_ready = false;  // spec_next holds a backward's weights
  bool spec_taken = false;  // the last speculative forward took a gradient
  unsigned char global_params[5 * sizeof(double)];
  // kernel timing: event pairs around each scoring-kernel launch
  bool profiling = false;
  std::vector<cudaEvent_t> prof_events;
  int prof_n = 0;
  tmol_b200_ljlk_launch launch;
  int n_sm = 148;
  int64_t device_bytes = 0;
  std::vector<int> host_pose_last;
  const uint32_t* skip = nullptr;  // caller-owned screen mask, or null
  int skip_words = 0;
  float* sub_spheres = nullptr;  // screen features: [P*B][2][4] (float plans)
  // rotamer plans
  bool rotamers = false;
  int R = 0;
  int* rot_bt = nullptr;
  int* rot_off = nullptr;
  int* rot_block = nullptr;
  int* rot_pose = nullptr;
  int* nrb = nullptr;  // rotamers per block [P*B]
  int* rob = nullptr;  // first rotamer of each block [P*B]
  void* rot_spheres = nullptr;   // [R][4] reals
  long long* row_pairs = nullptr;  // [P*B] + 2 totals
  long long* row_items = nullptr;  // [P*B]
  long long n_pairs = -1, n_items = -1;  // of the last rotamer_count
};

namespace {

#define CK(x)                                   \
  do {                                          \
    cudaError_t e_ = (x);                       \
    if (e_ != cudaSuccess) return TMOL_B200_ERR_CUDA; \
  } while (0)

template <typename T>
cudaError_t dalloc(tmol_b200_ljlk_plan* pl, T** p, size_t n) {
  size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
  pl->device_bytes += bytes;
  return cudaMalloc((void**)p, bytes);
}

int status_from_bits(int bits) {
  if (bits & kStIndex) return TMOL_B200_ERR_INDEX_RANGE;
  if (bits & kStShape) return TMOL_B200_ERR_SHAPE;
  if (bits & kStCapacity) return TMOL_B200_ERR_CAPACITY;
  return TMOL_B200_OK;
}

void free_plan(tmol_b200_ljlk_plan* pl) {
  void* ptrs[] = {pl->blk_bt,    pl->blk_off,    pl->pose_last,  pl->bt_tf,
                  pl->type_map,  pl->compact_types, pl->ljtab,   pl->lktab,
                  pl->bt_pd,     pl->bt_conn_pd, pl->bt_flags,   pl->bt_n_atoms,
                  pl->bt_n_conn, pl->bt_is_ligand, pl->cp_count, pl->cp_b2,
                  pl->cp_minsep, pl->cp_seps,    pl->work,       pl->spheres,
                  pl->item_cost,
                  pl->counters,  pl->counts,     pl->sub_spheres, pl->rot_bt,
                  pl->rot_off,   pl->rot_block,  pl->rot_pose,    pl->nrb,
                  pl->rob,       pl->rot_spheres, pl->row_pairs,  pl->row_items,
                  pl->bt_q,      pl->elec_k,      pl->lkb_sites,   pl->lkb_pol,
                  pl->lkb_npol,  pl->lkb_occ,     pl->lkb_nocc,    pl->lkb_par,
                  pl->lkb_waters, pl->lkb_dwaters, pl->lkb_nbocc, pl->lkb_active,
                  pl->blk_info,  pl->packed,      pl->spec_next,   pl->spec_used, pl->spec_g,
                  pl->spec_dw,   pl->spec_flag};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (cudaEvent_t e : pl->prof_events) cudaEventDestroy(e);
  delete pl;
}

void default_launch(tmol_b200_ljlk_launch& l) {
  if (l.rows_per_item <= 0) l.rows_per_item = 1;
  if (l.warps_per_cta <= 0) l.warps_per_cta = 8;
  if (l.ctas_per_sm <= 0) l.ctas_per_sm = 2;
  if (l.candidates_per_item <= 0) l.candidates_per_item = 64;
  if (l.slots_per_group <= 0) l.slots_per_group = MAX_SLOTS;
  l.slots_per_group = std::min(l.slots_per_group, MAX_SLOTS);
  l.rows_per_item = std::min(l.rows_per_item, MAX_ROWS_PER_ITEM);
  l.warps_per_cta = std::min(l.warps_per_cta, MAX_WARPS);
  l.candidates_per_item = std::min(l.candidates_per_item, 32 * 32);
}

template <typename Real, int TERM>
cudaError_t set_smem_limits_term() {
  const int smem = (int)std::min<size_t>(MAX_WARPS * sizeof(Slab<Real>), 227 * 1024);
  const void* kernels[] = {
      (const void*)score_kernel<Real, false, false, TERM, false>,
      (const void*)score_kernel<Real, false, true, TERM, false>,
      (const void*)score_kernel<Real, true, false, TERM, false>,
      (const void*)score_kernel<Real, true, true, TERM, false>,
      (const void*)score_kernel<Real, false, false, TERM, true>,
      (const void*)score_kernel<Real, false, true, TERM, true>,
      (const void*)score_kernel<Real, true, false, TERM, true>,
      (const void*)score_kernel<Real, true, true, TERM, true>,
      (const void*)rotamer_kernel<Real, false, TERM, false>,
      (const void*)rotamer_kernel<Real, true, TERM, false>,
      (const void*)rotamer_kernel<Real, false, TERM, true>,
      (const void*)rotamer_kernel<Real, true, TERM, true>};
  for (const void* k : kernels) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <typename Real>
cudaError_t set_smem_limits(int term) {
  return term == kTermElec ? set_smem_limits_term<Real, kTermElec>() : set_smem_limits_term<Real, kTermLJLK>();
}

int build_work(tmol_b200_ljlk_plan* pl, cudaStream_t st) {
  // items (pose, b1, [c0, c1)): the later blocks of each row in ranges of
  // CAND_CHUNK candidates
  std::vector<int4> work;
  for (int p = 0; p < pl->P; ++p) {
    int nb = pl->host_pose_last[p];
    for (int r = 0; r < nb; ++r)
      for (int c = r; c < nb; c += pl->launch.candidates_per_item)
        work.push_back(make_int4(p, r, c, std::min(nb, c + pl->launch.candidates_per_item)));
  }
  if (pl->work) cudaFree(pl->work);
  if (pl->item_cost) cudaFree(pl->item_cost);
  pl->work = nullptr;
  pl->item_cost = nullptr;
  pl->n_work = (int)work.size();
  // room for the items plan_rebalance splits off the heaviest ones
  pl->work_cap = pl->n_work + pl->n_work / 2 + 64;
  CK(cudaMalloc((void**)&pl->work, (size_t)pl->work_cap * sizeof(int4)));
  CK(cudaMalloc((void**)&pl->item_cost, (size_t)pl->work_cap * sizeof(int)));
  CK(cudaMemsetAsync(pl->item_cost, 0, (size_t)pl->work_cap * sizeof(int), st));
  if (!work.empty())
    CK(cudaMemcpyAsync(pl->work, work.data(), work.size() * sizeof(int4),
                       cudaMemcpyHostToDevice, st));
  // the kernels read the item count from here, so that a graph captured
  // before a rebalance still walks every item
  CK(cudaMemcpyAsync(pl->counters + 2, &pl->n_work, sizeof(int), cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
  return TMOL_B200_OK;
}

template <typename Real>
ScoreArgs<Real> score_args(tmol_b200_ljlk_plan* pl, const void* coords) {
  ScoreArgs<Real> s = {};
  s.coords = (const Real*)coords;
  s.blk_bt = pl->blk_bt;
  s.blk_off = pl->blk_off;
  s.blk_info = pl->blk_info;
  s.packed = (AtomRec<Real>*)pl->packed;
  s.pose_last = pl->pose_last;
  s.bt_tf = pl->bt_tf;
  s.ljtab = (const LJRecord<Real>*)pl->ljtab;
  s.lktab = (const LKRecord<Real>*)pl->lktab;
  s.ntp = pl->ntp;
  s.bt_pd = pl->bt_pd;
  s.bt_conn_pd = pl->bt_conn_pd;
  s.bt_n_atoms = pl->bt_n_atoms;
  s.bt_n_conn = pl->bt_n_conn;
  s.bt_is_ligand = pl->bt_is_ligand;
  s.cp_count = pl->cp_count;
  s.cp_b2 = pl->cp_b2;
  s.cp_minsep = pl->cp_minsep;
  s.cp_seps = pl->cp_seps;
  s.spheres = (Real*)pl->spheres;
  const Real* gp = (const Real*)pl->global_params;
  if (pl->term == kTermElec) {
    // elec global parameters: D, D0, S, min_dis, max_dis
    s.g.max_dis = gp[4];
    s.bt_q = (const Real*)pl->bt_q;
    s.elec_k = (const Real*)pl->elec_k;
  } else if (pl->term == kTermLKBall) {
    // LK-ball global parameters: hbond, OH-donor, H distances, water
    // distance, max_dis
    s.g.max_dis = gp[4];
    s.g.lj_hbond_dis = gp[0];
    s.g.lj_hbond_OH_donor_dis = gp[1];
    s.g.lj_hbond_hdis = gp[2];
  } else {
    s.g.max_dis = gp[0];
    s.g.lj_dlin_sigma_factor = gp[1];
    s.g.lj_hbond_dis = gp[2];
    s.g.lj_hbond_OH_donor_dis = gp[3];
    s.g.lj_hbond_hdis = gp[4];
  }
  s.reach = (Real)pl->reach;
  s.work = pl->work;
  s.item_cost = pl->item_cost;
  s.P = pl->P;
  s.B = pl->B;
  s.A = pl->A;
  s.C = pl->C;
  s.ticket = pl->counters;
  s.counts = pl->counts;
  s.skip = pl->skip;
  s.skip_words = pl->skip_words;
  s.max_slots = pl->launch.slots_per_group > 0 ? pl->launch.slots_per_group : MAX_SLOTS;
  return s;
}

template <typename Real, bool GRAD, bool BLOCK_PAIR>
int launch_score(tmol_b200_ljlk_plan* pl, ScoreArgs<Real> s, cudaStream_t st) {
  int n_blocks = pl->P * pl->B;
  int threads = 256;
  int grid_s = std::max(1, std::min((n_blocks + 7) / 8, pl->n_sm * 16));
  spheres_kernel<Real><<<grid_s, threads, 0, st>>>(s);  // also resets the work ticket
  CK(cudaGetLastError());
  if (pl->n_work == 0) return TMOL_B200_OK;
  int warps = pl->launch.warps_per_cta;
  if (sizeof(Real) == 8) warps = std::min(warps, 8);  // the float64 kernel: at most 256 threads
  size_t smem = warps * sizeof(Slab<Real>);
  // the work counters cost registers and instructions in the item loop:
  // they are compiled into a separate instantiation, used on request
  auto kern = pl->term == kTermElec
                  ? (pl->counting ? score_kernel<Real, GRAD, BLOCK_PAIR, kTermElec, true>
                                  : score_kernel<Real, GRAD, BLOCK_PAIR, kTermElec, false>)
                  : (pl->counting ? score_kernel<Real, GRAD, BLOCK_PAIR, kTermLJLK, true>
                                  : score_kernel<Real, GRAD, BLOCK_PAIR, kTermLJLK, false>);
  int R = pl->launch.rows_per_item;
  int n_tickets = (pl->n_work + R - 1) / R;
  int grid = std::max(1, std::min((n_tickets + warps - 1) / warps, pl->n_sm * pl->launch.ctas_per_sm));
  bool prof = pl->profiling && 2 * (size_t)pl->prof_n + 1 < pl->prof_events.size();
  if (prof) CK(cudaEventRecord(pl->prof_events[2 * pl->prof_n], st));
  kern<<<grid, 32 * warps, smem, st>>>(s, pl->launch.rows_per_item);
  CK(cudaGetLastError());
  if (prof) {
    CK(cudaEventRecord(pl->prof_events[2 * pl->prof_n + 1], st));
    ++pl->prof_n;
  }
  return TMOL_B200_OK;
}

template <typename Real>
int forward_impl(tmol_b200_ljlk_plan* pl, const void* coords, int block_pair,
                 void* energies, int32_t* nbr, cudaStream_t st) {
  ScoreArgs<Real> s = score_args<Real>(pl, coords);
  s.energies = (Real*)energies;
  s.nbr = nbr;
  const size_t nt = n_terms(pl->term);
  size_t n_e = block_pair ? nt * pl->P * pl->B * pl->B : nt * pl->P;
  if (block_pair)
    CK(cudaMemsetAsync(energies, 0, n_e * sizeof(Real), st));
  else
    s.zero_energies = (int64_t)n_e;  // by the sphere pass
  if (nbr) CK(cudaMemsetAsync(nbr, 0, (size_t)pl->P * pl->B * pl->B * sizeof(int32_t), st));
  s.zero_counts = 1;
  if (block_pair) return launch_score<Real, false, true>(pl, s, st);
  return launch_score<Real, false, false>(pl, s, st);
}

template <typename Real>
int backward_impl(tmol_b200_ljlk_plan* pl, const void* coords, int block_pair,
                  const void* dTdV, void* dcoords, cudaStream_t st) {
  ScoreArgs<Real> s = score_args<Real>(pl, coords);
  s.dTdV = (const Real*)dTdV;
  s.dcoords = (Real*)dcoords;
  s.counts = nullptr;
  s.zero_dcoords = (int64_t)pl->N * 3;  // by the sphere pass
  if (block_pair) return launch_score<Real, true, true>(pl, s, st);
  return launch_score<Real, true, false>(pl, s, st);
}

template <typename Real>
int energy_and_gradient_impl(tmol_b200_ljlk_plan* pl, const void* coords,
                             const void* weights, void* energies, void* dcoords,
                             cudaStream_t st) {
  ScoreArgs<Real> s = score_args<Real>(pl, coords);
  s.dTdV = (const Real*)weights;
  s.dcoords = (Real*)dcoords;
  s.energies = (Real*)energies;
  // the sphere pass zeroes the outputs before the scoring launch adds to them
  s.zero_dcoords = (int64_t)pl->N * 3;
  s.zero_energies = (int64_t)n_terms(pl->term) * pl->P;
  s.zero_counts = 1;
  return launch_score<Real, true, false>(pl, s, st);
}

// Sets *flag to 1 when a[0, n) and b[0, n) are equal element by element
// (one block).
template <typename Real>
__global__ void __launch_bounds__(1024) spec_match_kernel(const Real* a, const Real* b, int n, int* flag) {
  int differ = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) differ |= !(a[i] == b[i]);
  differ = __syncthreads_or(differ);
  if (threadIdx.x == 0) *flag = differ ? 0 : 1;
}

// dst[0, n) = src[0, n) when *flag is set.
template <typename Real>
__global__ void spec_copy_kernel(const int* flag, const Real* src, Real* dst, int64_t n) {
  if (!*flag) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

// The pose op's forward that also takes the gradient with the weights of
// the last backward (kept in the plan), in one fused pass: an autograd
// backward that follows with the same weights then needs no second pass.
template <typename Real>
int forward_speculative_impl(tmol_b200_ljlk_plan* pl, const void* coords, void* energies, int32_t* nbr,
                             cudaStream_t st) {
  pl->spec_taken = false;
  if (!pl->spec_ready) return forward_impl<Real>(pl, coords, 0, energies, nbr, st);
  pl->spec_taken = true;
  const size_t w_bytes = (size_t)n_terms(pl->term) * pl->P * sizeof(Real);
  if (w_bytes) CK(cudaMemcpyAsync(pl->spec_used, pl->spec_next, w_bytes, cudaMemcpyDeviceToDevice, st));
  ScoreArgs<Real> s = score_args<Real>(pl, coords);
  s.energies = (Real*)energies;
  s.nbr = nbr;
  s.dTdV = (const Real*)pl->spec_used;
  s.dcoords = (Real*)pl->spec_g;
  if (nbr) CK(cudaMemsetAsync(nbr, 0, (size_t)pl->P * pl->B * pl->B * sizeof(int32_t), st));
  // energies, the kept gradient and the counters: by the sphere pass
  s.zero_energies = (int64_t)n_terms(pl->term) * pl->P;
  s.zero_dcoords = (int64_t)pl->N * 3;
  s.zero_counts = 1;
  return launch_score<Real, true, false>(pl, s, st);
}

// The pose op's backward: when `speculated` (the plan's last speculative
// forward was the forward of these coordinates, and took a gradient) and
// dTdV equals the weights that forward used, the gradient is that pass's
// (copied on the device; the scoring launch exits at once); otherwise it
// is recomputed.  Either way dTdV becomes the weights of the next
// speculative forward.  No host synchronisation.
template <typename Real>
int backward_speculative_impl(tmol_b200_ljlk_plan* pl, const void* coords, const void* dTdV, void* dcoords,
                              int speculated, cudaStream_t st) {
  const int n_w = n_terms(pl->term) * pl->P;
  const int64_t n_g = (int64_t)pl->N * 3;
  if (speculated && pl->spec_taken && n_w > 0) {
    spec_match_kernel<Real><<<1, 1024, 0, st>>>((const Real*)dTdV, (const Real*)pl->spec_used, n_w, pl->spec_flag);
    CK(cudaGetLastError());
  } else {
    CK(cudaMemsetAsync(pl->spec_flag, 0, sizeof(int), st));
  }
  // a hit copies the kept gradient whole; a miss zeroes dcoords in the
  // sphere pass (which a hit skips) before the scoring launch
  if (n_g > 0) {
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n_g + 255) / 256, (int64_t)pl->n_sm * 8));
    spec_copy_kernel<Real><<<grid, 256, 0, st>>>(pl->spec_flag, (const Real*)pl->spec_g, (Real*)dcoords, n_g);
    CK(cudaGetLastError());
  }
  ScoreArgs<Real> s = score_args<Real>(pl, coords);
  s.dTdV = (const Real*)dTdV;
  s.dcoords = (Real*)dcoords;
  s.counts = nullptr;
  s.done = pl->spec_flag;
  s.zero_dcoords = n_g;
  const int rc = launch_score<Real, true, false>(pl, s, st);
  if (rc != TMOL_B200_OK) return rc;
  if (n_w > 0) CK(cudaMemcpyAsync(pl->spec_next, dTdV, (size_t)n_w * sizeof(Real), cudaMemcpyDeviceToDevice, st));
  pl->spec_ready = true;
  return TMOL_B200_OK;
}

RotArgs rot_args(tmol_b200_ljlk_plan* pl) {
  RotArgs ra = {};
  ra.rot_bt = pl->rot_bt;
  ra.rot_off = pl->rot_off;
  ra.rot_block = pl->rot_block;
  ra.rot_pose = pl->rot_pose;
  ra.nrb = pl->nrb;
  ra.rob = pl->rob;
  ra.R = pl->R;
  ra.row_pairs = pl->row_pairs;
  ra.row_items = pl->row_items;
  return ra;
}

template <typename Real>
int rotamer_count_impl(tmol_b200_ljlk_plan* pl, const void* coords, int64_t* n_pairs,
                       int64_t* n_items, cudaStream_t st) {
  ScoreArgs<Real> s = score_args<Real>(pl, coords);
  RotArgs ra = rot_args(pl);
  const int n_rows = pl->P * pl->B;
  long long totals[2] = {0, 0};
  if (n_rows > 0) {
    if (pl->R > 0) {
      int gr = std::max(1, std::min((pl->R + 7) / 8, pl->n_sm * 16));
      rot_spheres_kernel<Real><<<gr, 256, 0, st>>>(s, ra, (Real*)pl->rot_spheres);
      CK(cudaGetLastError());
    }
    int gb = std::max(1, std::min((n_rows + 255) / 256, pl->n_sm * 8));
    block_spheres_from_rots_kernel<Real><<<gb, 256, 0, st>>>(s, ra, (const Real*)pl->rot_spheres);
    CK(cudaGetLastError());
    int gw = std::max(1, std::min((n_rows + 7) / 8, pl->n_sm * 16));
    rot_row_count_kernel<Real><<<gw, 256, 0, st>>>(s, ra);
    CK(cudaGetLastError());
    scan2_kernel<<<1, 1024, 0, st>>>(pl->row_pairs, pl->row_items, n_rows, pl->row_pairs + n_rows);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(totals, pl->row_pairs + n_rows, sizeof(totals), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }
  // pair indices are int32 in the op's output, and work items address pairs
  // with an int
  if (totals[0] >= ((long long)1 << 31) || totals[1] >= ((long long)1 << 31)) {
    pl->n_pairs = pl->n_items = -1;
    return TMOL_B200_ERR_CAPACITY;
  }
  pl->n_pairs = totals[0];
  pl->n_items = totals[1];
  *n_pairs = totals[0];
  *n_items = totals[1];
  return TMOL_B200_OK;
}

template <typename Real>
int rotamer_fill_impl(tmol_b200_ljlk_plan* pl, int32_t* indices, int32_t* items, cudaStream_t st) {
  ScoreArgs<Real> s = score_args<Real>(pl, nullptr);
  RotArgs ra = rot_args(pl);
  ra.items = (int4*)items;
  ra.n_items = pl->n_items;
  ra.indices = indices;
  ra.n_pairs = pl->n_pairs;
  const int n_rows = pl->P * pl->B;
  if (n_rows == 0 || (pl->n_pairs == 0 && pl->n_items == 0)) return TMOL_B200_OK;
  int gw = std::max(1, std::min((n_rows + 7) / 8, pl->n_sm * 16));
  rot_row_fill_kernel<Real><<<gw, 256, 0, st>>>(s, ra);
  CK(cudaGetLastError());
  return TMOL_B200_OK;
}

template <typename Real, bool GRAD>
int rotamer_score_impl(tmol_b200_ljlk_plan* pl, const void* coords, const int32_t* items,
                       int64_t n_items, int64_t n_pairs, void* energies, const void* dTdV,
                       void* dcoords, cudaStream_t st) {
  ScoreArgs<Real> s = score_args<Real>(pl, coords);
  RotArgs ra = rot_args(pl);
  ra.items = (int4*)items;
  ra.n_items = n_items;
  ra.n_pairs = n_pairs;
  s.energies = (Real*)energies;
  s.dTdV = (const Real*)dTdV;
  s.dcoords = (Real*)dcoords;
  s.counts = GRAD ? nullptr : pl->counts;
  if (!GRAD) CK(cudaMemsetAsync(pl->counts, 0, N_COUNTS * sizeof(unsigned long long), st));
  if (energies) CK(cudaMemsetAsync(energies, 0, (size_t)n_terms(pl->term) * n_pairs * sizeof(Real), st));
  if (dcoords) CK(cudaMemsetAsync(dcoords, 0, (size_t)pl->N * 3 * sizeof(Real), st));
  if (n_items == 0) return TMOL_B200_OK;
  if (pl->R > 0) {
    int gr = std::max(1, std::min((pl->R + 7) / 8, pl->n_sm * 16));
    rot_spheres_kernel<Real><<<gr, 256, 0, st>>>(s, ra, (Real*)pl->rot_spheres);
    CK(cudaGetLastError());
  }
  CK(cudaMemsetAsync(pl->counters, 0, sizeof(int), st));
  const int warps = std::min(pl->launch.warps_per_cta, 8);  // a kernel of at most 256 threads
  const size_t smem = warps * sizeof(Slab<Real>);
  int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n_items + warps - 1) / warps,
                                                         (int64_t)pl->n_sm * pl->launch.ctas_per_sm));
  auto kern = pl->term == kTermElec
                  ? (pl->counting ? rotamer_kernel<Real, GRAD, kTermElec, true> : rotamer_kernel<Real, GRAD, kTermElec, false>)
                  : (pl->counting ? rotamer_kernel<Real, GRAD, kTermLJLK, true> : rotamer_kernel<Real, GRAD, kTermLJLK, false>);
  kern<<<grid, 32 * warps, smem, st>>>(s, ra, (const Real*)pl->rot_spheres);
  CK(cudaGetLastError());
  return TMOL_B200_OK;
}

template <typename Real>
LkbArgs<Real> lkb_args(tmol_b200_ljlk_plan* pl) {
  LkbArgs<Real> k = {};
  k.sites = (const LkbSite<Real>*)pl->lkb_sites;
  k.n_sites = pl->N * LKB_NW;
  k.active = pl->lkb_active;
  k.n_active = pl->lkb_n_active;
  k.pol = pl->lkb_pol;
  k.npol = pl->lkb_npol;
  k.occ = pl->lkb_occ;
  k.nocc = pl->lkb_nocc;
  k.nbocc = pl->lkb_nbocc;
  k.maxpol = pl->lkb_maxpol;
  k.maxocc = pl->lkb_maxocc;
  k.par = (const Real*)pl->lkb_par;
  const Real* gp = (const Real*)pl->global_params;
  k.hbond_dis = gp[0];
  k.hbond_oh = gp[1];
  k.hbond_h = gp[2];
  k.water_dist = (Real)pl->lkb_water_dist;
  k.max_dis = gp[4];
  return k;
}

// `prefilled`: the empty slots of `waters` already hold NaN (the plan's
// scratch, filled once)
template <typename Real>
int lkb_waters_impl(tmol_b200_ljlk_plan* pl, const void* coords, void* waters, cudaStream_t st,
                    bool prefilled = false) {
  LkbArgs<Real> k = lkb_args<Real>(pl);
  k.waters_out = (Real*)waters;
  if (k.n_sites == 0) return TMOL_B200_OK;
  // all-ones bytes are a NaN in float and double
  if (!prefilled) CK(cudaMemsetAsync(waters, 0xff, sizeof(Real) * 3 * (size_t)k.n_sites, st));
  if (k.n_active == 0) return TMOL_B200_OK;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((k.n_active + 255) / 256, (int64_t)pl->n_sm * 16));
  lkb_waters_kernel<Real><<<grid, 256, 0, st>>>(k, (const Real*)coords);
  CK(cudaGetLastError());
  return TMOL_B200_OK;
}

template <typename Real>
int lkb_waters_backward_impl(tmol_b200_ljlk_plan* pl, const void* coords, const void* dwaters, void* dcoords,
                             cudaStream_t st) {
  LkbArgs<Real> k = lkb_args<Real>(pl);
  k.dwaters = (const Real*)dwaters;
  if (k.n_active == 0) return TMOL_B200_OK;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((k.n_active + 255) / 256, (int64_t)pl->n_sm * 16));
  lkb_waters_backward_kernel<Real><<<grid, 256, 0, st>>>(k, (const Real*)coords, (Real*)dcoords);
  CK(cudaGetLastError());
  return TMOL_B200_OK;
}

template <typename Real, bool GRAD, bool BLOCK_PAIR>
int lkb_score_impl(tmol_b200_ljlk_plan* pl, const void* coords, const void* waters, void* energies, int32_t* nbr,
                   const void* dTdV, void* dcoords, void* dwaters, cudaStream_t st, const int* done = nullptr) {
  ScoreArgs<Real> s = score_args<Real>(pl, coords);
  s.done = done;
  LkbArgs<Real> k = lkb_args<Real>(pl);
  k.water_dist = ((const Real*)pl->global_params)[3];  // the score op's own copy
  k.waters = (const Real*)waters;
  k.dwaters_out = (Real*)dwaters;
  s.energies = (Real*)energies;
  s.nbr = nbr;
  s.dTdV = (const Real*)dTdV;
  s.dcoords = (Real*)dcoords;
  const size_t PBB = (size_t)pl->P * pl->B * pl->B;
  // block-pair energies and weights are addressed by an int block-pair index
  if (BLOCK_PAIR && PBB >= ((size_t)1 << 31)) return TMOL_B200_ERR_CAPACITY;
  if (energies && BLOCK_PAIR) CK(cudaMemsetAsync(energies, 0, PBB * 4 * sizeof(Real), st));
  if (nbr) CK(cudaMemsetAsync(nbr, 0, PBB * sizeof(int32_t), st));
  // the whole-pose energies, the gradients, the counters and the work
  // ticket: by the sphere pass (which a taken speculative gradient skips:
  // its outputs are then copied whole)
  if (energies && !BLOCK_PAIR) s.zero_energies = (int64_t)pl->P * 4;
  if (dcoords) s.zero_dcoords = (int64_t)pl->N * 3;
  if (dwaters) {
    s.zero_aux = (Real*)dwaters;
    s.zero_aux_n = (int64_t)pl->N * LKB_NW * 3;
  }
  s.zero_counts = 1;
  const int n_blocks = pl->P * pl->B;
  const int grid_s = std::max(1, std::min((n_blocks + 7) / 8, pl->n_sm * 16));
  spheres_kernel<Real><<<grid_s, 256, 0, st>>>(s);
  CK(cudaGetLastError());
  if (pl->n_work == 0) return TMOL_B200_OK;
  const int warps = std::min(pl->launch.warps_per_cta, 8);  // a kernel of at most 256 threads
  const int R = pl->launch.rows_per_item;
  const int n_tickets = (pl->n_work + R - 1) / R;
  const int grid = std::max(1, std::min((n_tickets + warps - 1) / warps, pl->n_sm * pl->launch.ctas_per_sm));
  const bool prof = pl->profiling && 2 * (size_t)pl->prof_n + 1 < pl->prof_events.size();
  if (prof) CK(cudaEventRecord(pl->prof_events[2 * pl->prof_n], st));
  if (pl->counting)
    lkb_score_kernel<Real, GRAD, BLOCK_PAIR, true><<<grid, 32 * warps, 0, st>>>(s, k, R);
  else
    lkb_score_kernel<Real, GRAD, BLOCK_PAIR, false><<<grid, 32 * warps, 0, st>>>(s, k, R);
  CK(cudaGetLastError());
  if (prof) {
    CK(cudaEventRecord(pl->prof_events[2 * pl->prof_n + 1], st));
    ++pl->prof_n;
  }
  return TMOL_B200_OK;
}

// LK-ball's score op with a speculative gradient, as
// forward_speculative_impl / backward_speculative_impl: the kept gradient
// is the coordinates' direct part and the waters' part.
template <typename Real>
int lkb_forward_speculative_impl(tmol_b200_ljlk_plan* pl, const void* coords, const void* waters, void* energies,
                                 int32_t* nbr, cudaStream_t st) {
  pl->spec_taken = false;
  if (!pl->spec_ready)
    return lkb_score_impl<Real, false, false>(pl, coords, waters, energies, nbr, nullptr, nullptr, nullptr, st);
  pl->spec_taken = true;
  const size_t w_bytes = (size_t)4 * pl->P * sizeof(Real);
  if (w_bytes) CK(cudaMemcpyAsync(pl->spec_used, pl->spec_next, w_bytes, cudaMemcpyDeviceToDevice, st));
  return lkb_score_impl<Real, true, false>(pl, coords, waters, energies, nbr, pl->spec_used, pl->spec_g,
                                           pl->spec_dw, st);
}

template <typename Real>
int lkb_backward_speculative_impl(tmol_b200_ljlk_plan* pl, const void* coords, const void* waters,
                                  const void* dTdV, void* dcoords, void* dwaters, int speculated,
                                  cudaStream_t st) {
  const int n_w = 4 * pl->P;
  if (speculated && pl->spec_taken && n_w > 0) {
    spec_match_kernel<Real><<<1, 1024, 0, st>>>((const Real*)dTdV, (const Real*)pl->spec_used, n_w, pl->spec_flag);
    CK(cudaGetLastError());
  } else {
    CK(cudaMemsetAsync(pl->spec_flag, 0, sizeof(int), st));
  }
  // zeroes the outputs; its scoring launch does no work when the flag is set
  const int rc = lkb_score_impl<Real, true, false>(pl, coords, waters, nullptr, nullptr, dTdV, dcoords, dwaters,
                                                   st, pl->spec_flag);
  if (rc != TMOL_B200_OK) return rc;
  const int64_t n_g = (int64_t)pl->N * 3, n_dw = (int64_t)pl->N * LKB_NW * 3;
  if (n_g > 0) {
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n_dw + 255) / 256, (int64_t)pl->n_sm * 8));
    spec_copy_kernel<Real><<<grid, 256, 0, st>>>(pl->spec_flag, (const Real*)pl->spec_g, (Real*)dcoords, n_g);
    CK(cudaGetLastError());
    spec_copy_kernel<Real><<<grid, 256, 0, st>>>(pl->spec_flag, (const Real*)pl->spec_dw, (Real*)dwaters, n_dw);
    CK(cudaGetLastError());
  }
  if (n_w > 0) CK(cudaMemcpyAsync(pl->spec_next, dTdV, (size_t)n_w * sizeof(Real), cudaMemcpyDeviceToDevice, st));
  pl->spec_ready = true;
  return TMOL_B200_OK;
}

template <typename Real, bool GRAD>
int lkb_rotamer_score_impl(tmol_b200_ljlk_plan* pl, const void* coords, const void* waters, const int32_t* items,
                           int64_t n_items, int64_t n_pairs, void* energies, const void* dTdV, void* dcoords,
                           void* dwaters, cudaStream_t st) {
  ScoreArgs<Real> s = score_args<Real>(pl, coords);
  LkbArgs<Real> k = lkb_args<Real>(pl);
  k.water_dist = ((const Real*)pl->global_params)[3];
  k.waters = (const Real*)waters;
  k.dwaters_out = (Real*)dwaters;
  RotArgs ra = rot_args(pl);
  ra.items = (int4*)items;
  ra.n_items = n_items;
  ra.n_pairs = n_pairs;
  s.energies = (Real*)energies;
  s.dTdV = (const Real*)dTdV;
  s.dcoords = (Real*)dcoords;
  s.nbr = nullptr;
  s.counts = pl->counts;
  CK(cudaMemsetAsync(pl->counts, 0, N_COUNTS * sizeof(unsigned long long), st));
  if (energies) CK(cudaMemsetAsync(energies, 0, (size_t)4 * n_pairs * sizeof(Real), st));
  if (dcoords) CK(cudaMemsetAsync(dcoords, 0, (size_t)pl->N * 3 * sizeof(Real), st));
  if (dwaters) CK(cudaMemsetAsync(dwaters, 0, (size_t)pl->N * LKB_NW * 3 * sizeof(Real), st));
  if (n_items == 0) return TMOL_B200_OK;
  if (pl->R > 0) {
    const int gr = std::max(1, std::min((pl->R + 7) / 8, pl->n_sm * 16));
    rot_spheres_kernel<Real><<<gr, 256, 0, st>>>(s, ra, (Real*)pl->rot_spheres);
    CK(cudaGetLastError());
  }
  CK(cudaMemsetAsync(pl->counters, 0, sizeof(int), st));
  const int warps = std::min(pl->launch.warps_per_cta, 8);  // a kernel of at most 256 threads
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n_items + warps - 1) / warps,
                                                               (int64_t)pl->n_sm * pl->launch.ctas_per_sm));
  if (pl->counting)
    lkb_rotamer_kernel<Real, GRAD, true><<<grid, 32 * warps, 0, st>>>(s, k, ra, (const Real*)pl->rot_spheres);
  else
    lkb_rotamer_kernel<Real, GRAD, false><<<grid, 32 * warps, 0, st>>>(s, k, ra, (const Real*)pl->rot_spheres);
  CK(cudaGetLastError());
  return TMOL_B200_OK;
}

}  // namespace

extern "C" {

const char* tmol_b200_status_string(int status) {
  switch (status) {
    case TMOL_B200_OK: return "ok";
    case TMOL_B200_ERR_INVALID_ARGUMENT: return "invalid argument";
    case TMOL_B200_ERR_SHAPE: return "inconsistent or unsupported tensor sizes";
    case TMOL_B200_ERR_INDEX_RANGE: return "index out of range in an input table";
    case TMOL_B200_ERR_CAPACITY: return "fixed-capacity table overflow";
    case TMOL_B200_ERR_CUDA: return "CUDA runtime error";
    case TMOL_B200_ERR_DTYPE: return "float width mismatch";
  }
  return "unknown status";
}

}  // extern "C"

namespace {

// What an elec plan needs beyond the shared inputs (whose bt_path_distance
// is then the intra-block representative table).
struct ElecExtra {
  const void* partial_charge;      // [nbt, A] reals
  const int32_t* inter_repr_pd;    // [nbt, A, A]
};

// LK-ball plan tables: each block type's polar and occluder atoms (the
// reference's per-tile lists, lk_ball_pose_score.impl.hh:560-640, flattened
// to one list per block type), their nine parameters per atom, and every
// water site of the PoseStack (lkb_sites_kernel).
template <typename Real>
int build_lkball(tmol_b200_ljlk_plan* pl, const tmol_b200_lkball_inputs* k, const std::vector<int>& h_nat,
                 cudaStream_t st) {
  const int nbt = pl->nbt, A = pl->A, NT = k->max_n_tiles;
  const bool waters = k->bt_all_bonds != nullptr, scoring = k->bt_tile_pol_occ_inds != nullptr;
  const size_t ntile = scoring ? (size_t)nbt * NT : 0;
  std::vector<int> npol(ntile), nocc(ntile), inds(ntile * TILE);
  std::vector<Real> tpar(ntile * TILE * LKB_NPAR);
  Real wg[4] = {0, 0, 0, 0};
  if (ntile > 0) {
    CK(cudaMemcpyAsync(npol.data(), k->bt_tile_n_polar_atoms, sizeof(int) * ntile, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(nocc.data(), k->bt_tile_n_occluder_atoms, sizeof(int) * ntile, cudaMemcpyDeviceToHost,
                       st));
    CK(cudaMemcpyAsync(inds.data(), k->bt_tile_pol_occ_inds, sizeof(int) * ntile * TILE, cudaMemcpyDeviceToHost,
                       st));
    CK(cudaMemcpyAsync(tpar.data(), k->bt_tile_lk_ball_params, sizeof(Real) * tpar.size(),
                       cudaMemcpyDeviceToHost, st));
  }
  if (waters && k->water_gen_global_params)
    CK(cudaMemcpyAsync(wg, k->water_gen_global_params, sizeof(wg), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  std::vector<std::vector<int>> pol(nbt), occ(nbt);
  std::vector<Real> par((size_t)std::max(nbt * A, 1) * LKB_NPAR, Real(0));
  for (int bt = 0; scoring && bt < nbt; ++bt)
    for (int t = 0; t < NT; ++t) {
      const size_t tb = (size_t)bt * NT + t;
      if (npol[tb] < 0 || nocc[tb] < npol[tb] || nocc[tb] > TILE) return TMOL_B200_ERR_INDEX_RANGE;
      for (int q = 0; q < nocc[tb]; ++q) {
        const int i = inds[tb * TILE + q];
        const int a = t * TILE + i;
        if (i < 0 || i >= TILE || a >= h_nat[bt] || a >= A) return TMOL_B200_ERR_INDEX_RANGE;
        if (q < npol[tb]) pol[bt].push_back(a);
        occ[bt].push_back(a);
        std::copy_n(&tpar[(tb * TILE + q) * LKB_NPAR], LKB_NPAR, &par[((size_t)bt * A + a) * LKB_NPAR]);
      }
    }
  // occluders that are donors or acceptors (parameters 4 and 7) first: the
  // scoring kernel queues their pairs apart (the water-bridge term)
  std::vector<int> hnbocc(std::max(nbt, 1), 0);
  for (int bt = 0; bt < nbt; ++bt) {
    auto bridges = [&](int a) {
      const Real* q = &par[((size_t)bt * A + a) * LKB_NPAR];
      return q[4] != Real(0) || q[7] != Real(0);
    };
    std::stable_partition(occ[bt].begin(), occ[bt].end(), bridges);
    for (int a : occ[bt]) hnbocc[bt] += bridges(a) ? 1 : 0;
  }
  int maxpol = 1, maxocc = 1;
  for (int bt = 0; bt < nbt; ++bt) {
    maxpol = std::max(maxpol, (int)pol[bt].size());
    maxocc = std::max(maxocc, (int)occ[bt].size());
  }
  std::vector<int> hpol((size_t)std::max(nbt, 1) * maxpol, 0), hocc((size_t)std::max(nbt, 1) * maxocc, 0);
  std::vector<int> hnpol(std::max(nbt, 1), 0), hnocc(std::max(nbt, 1), 0);
  for (int bt = 0; bt < nbt; ++bt) {
    hnpol[bt] = (int)pol[bt].size();
    hnocc[bt] = (int)occ[bt].size();
    std::copy(pol[bt].begin(), pol[bt].end(), &hpol[(size_t)bt * maxpol]);
    std::copy(occ[bt].begin(), occ[bt].end(), &hocc[(size_t)bt * maxocc]);
  }
  pl->lkb_maxpol = maxpol;
  pl->lkb_maxocc = maxocc;
  pl->lkb_water_dist = (double)wg[0];
  if (scoring) {
    CK(dalloc(pl, &pl->lkb_pol, hpol.size()));
    CK(dalloc(pl, &pl->lkb_occ, hocc.size()));
    CK(dalloc(pl, &pl->lkb_npol, hnpol.size()));
    CK(dalloc(pl, &pl->lkb_nocc, hnocc.size()));
    CK(dalloc(pl, &pl->lkb_nbocc, hnbocc.size()));
    CK(cudaMemcpyAsync(pl->lkb_nbocc, hnbocc.data(), sizeof(int) * hnbocc.size(), cudaMemcpyHostToDevice, st));
    CK(dalloc(pl, (Real**)&pl->lkb_par, par.size()));
    CK(cudaMemcpyAsync(pl->lkb_pol, hpol.data(), sizeof(int) * hpol.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(pl->lkb_occ, hocc.data(), sizeof(int) * hocc.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(pl->lkb_npol, hnpol.data(), sizeof(int) * hnpol.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(pl->lkb_nocc, hnocc.data(), sizeof(int) * hnocc.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(pl->lkb_par, par.data(), sizeof(Real) * par.size(), cudaMemcpyHostToDevice, st));
  }
  if (scoring && !pl->rotamers) {
    // the score op's speculative gradient (lkb_backward_speculative)
    CK(dalloc(pl, (Real**)&pl->spec_next, (size_t)4 * std::max(pl->P, 1)));
    CK(dalloc(pl, (Real**)&pl->spec_used, (size_t)4 * std::max(pl->P, 1)));
    CK(dalloc(pl, (Real**)&pl->spec_g, (size_t)std::max<int64_t>(pl->N, 1) * 3));
    CK(dalloc(pl, (Real**)&pl->spec_dw, (size_t)std::max<int64_t>(pl->N, 1) * LKB_NW * 3));
    CK(dalloc(pl, &pl->spec_flag, 1));
  }
  if (!waters) return TMOL_B200_OK;
  const int64_t n_sites = pl->N * LKB_NW;
  if (n_sites >= ((int64_t)1 << 31)) return TMOL_B200_ERR_SHAPE;  // site indices are int
  if (scoring) {
    CK(dalloc(pl, (Real**)&pl->lkb_waters, (size_t)n_sites * 3));
    CK(dalloc(pl, (Real**)&pl->lkb_dwaters, (size_t)n_sites * 3));
  }
  CK(dalloc(pl, (LkbSite<Real>**)&pl->lkb_sites, (size_t)n_sites));
  CK(cudaMemsetAsync(pl->lkb_sites, 0, sizeof(LkbSite<Real>) * std::max<int64_t>(n_sites, 1), st));
  const int64_t PB = (int64_t)pl->P * pl->B;
  if (PB > 0 && nbt > 0 && k->n_rots > 0) {
    LkbRots rs;
    rs.rot_coord_offset = k->rot_coord_offset;
    rs.pose_ind_for_rot = k->pose_ind_for_rot;
    rs.block_ind_for_rot = k->block_ind_for_rot;
    rs.block_type_ind_for_rot = k->block_type_ind_for_rot;
    rs.first_rot_for_block = k->first_rot_for_block;
    rs.first_rot_block_type = k->first_rot_block_type;
    rs.bt_n_atoms = pl->bt_n_atoms;
    rs.R = k->n_rots;
    rs.nbt = nbt;
    rs.N = pl->N;
    LkbTables t;
    t.irc = k->inter_residue_connections;
    t.all_bonds = k->bt_all_bonds;
    t.ranges = k->bt_atom_all_bond_ranges;
    t.NB = k->max_n_all_bonds;
    t.NT = NT;
    t.tile_n_donH = k->bt_tile_n_donH;
    t.tile_n_acc = k->bt_tile_n_acc;
    t.tile_donH = k->bt_tile_donH_inds;
    t.tile_donH_hvy = k->bt_tile_donH_hvy_inds;
    t.tile_which = k->bt_tile_which_donH_for_hvy;
    t.tile_acc = k->bt_tile_acc_inds;
    t.tile_hyb = k->bt_tile_hybridization;
    t.tile_nH = k->bt_tile_acc_n_attached_H;
    t.is_h = k->bt_atom_is_hydrogen;
    t.bt_conn_atom = k->bt_conn_atom;
    const int g = std::max(1, std::min<int>((k->n_rots + 127) / 128, pl->n_sm * 8));
    lkb_sites_kernel<Real><<<g, 128, 0, st>>>(
        rs, pl->P, pl->B, pl->C, A, t, (const Real*)k->sp2_water_tors,
        k->n_sp2_tors, (const Real*)k->sp3_water_tors, k->n_sp3_tors, (const Real*)k->ring_water_tors,
        k->n_ring_tors, wg[1], wg[2], wg[3], (LkbSite<Real>*)pl->lkb_sites, pl->counters + 1);
    CK(cudaGetLastError());
  }
  // the occupied sites, in ascending order (the per-call kernels visit only
  // these); the plan's waters scratch holds NaN in the empty slots for good
  std::vector<LkbSite<Real>> h_sites((size_t)n_sites);
  if (n_sites > 0)
    CK(cudaMemcpyAsync(h_sites.data(), pl->lkb_sites, sizeof(LkbSite<Real>) * n_sites, cudaMemcpyDeviceToHost,
                       st));
  CK(cudaStreamSynchronize(st));
  std::vector<int> active;
  for (int64_t i = 0; i < n_sites; ++i)
    if (h_sites[i].kind != kLkbNone) active.push_back((int)i);
  pl->lkb_n_active = (int64_t)active.size();
  CK(dalloc(pl, &pl->lkb_active, active.size()));
  if (!active.empty())
    CK(cudaMemcpyAsync(pl->lkb_active, active.data(), sizeof(int) * active.size(), cudaMemcpyHostToDevice, st));
  if (scoring && n_sites > 0)
    CK(cudaMemsetAsync(pl->lkb_waters, 0xff, sizeof(Real) * 3 * (size_t)n_sites, st));
  return TMOL_B200_OK;
}

int create_plan(const tmol_b200_ljlk_inputs* in, int real_bytes,
                const tmol_b200_ljlk_launch* launch, void* stream, bool rotamers,
                tmol_b200_ljlk_plan** plan_out, const ElecExtra* elec = nullptr,
                const tmol_b200_pose_connectivity* conn = nullptr,
                const tmol_b200_lkball_inputs* lkb = nullptr) {
  if (!in || !plan_out) return TMOL_B200_ERR_INVALID_ARGUMENT;
  const int term = elec ? kTermElec : (lkb ? kTermLKBall : kTermLJLK);
  // an LK-ball plan serves water generation (its bond and hbond tables
  // given), scoring (its polar / occluder tables given), or both
  const bool lkb_waters = lkb && lkb->bt_all_bonds;
  const bool scoring = !lkb || lkb->bt_tile_pol_occ_inds;
  if (lkb && !lkb_waters && !scoring) return TMOL_B200_ERR_INVALID_ARGUMENT;
  *plan_out = nullptr;
  if (real_bytes != 4 && real_bytes != 8) return TMOL_B200_ERR_DTYPE;
  const int P = in->n_poses, B = in->max_n_blocks, nbt = in->n_block_types;
  const int A = in->max_n_block_atoms, C = in->max_n_conn, nt = in->max_n_tiles;
  const int T = in->n_atom_types;
  if (P < 0 || B < 0 || nbt < 0 || A < 0 || C < 0 || T < 0 || in->n_atoms < 0)
    return TMOL_B200_ERR_SHAPE;
  if (C > MAX_CONN || B >= 65536) return TMOL_B200_ERR_SHAPE;
  // block slots, formed in 64 bits; the kernels index blocks (and their
  // count-pair rows, 16 entries each) in 32-bit ints, so the product is
  // capped far below where those indices could wrap
  const int64_t n_slots = (int64_t)P * B;
  if (n_slots > ((int64_t)1 << 26)) return TMOL_B200_ERR_SHAPE;
  if (rotamers ? in->n_rots < 0 : (int64_t)in->n_rots != n_slots) return TMOL_B200_ERR_SHAPE;
  if (rotamers && n_slots > 0 && !in->n_rots_for_block) return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (nt * TILE < A) return TMOL_B200_ERR_SHAPE;
  if (in->n_atoms >= ((int64_t)1 << 31)) return TMOL_B200_ERR_SHAPE;
  // with the pose's connectivity, the dense bond-separation tensors are not
  // read (and may be null)
  const void* dense_cp[] = {in->min_bondsep, in->inter_block_bondsep};
  const void* conn_req[] = {conn ? conn->block_type_ind : nullptr, conn ? conn->inter_residue_connections : nullptr,
                            conn ? conn->bt_n_conn : nullptr, conn ? conn->bt_conn_sep : nullptr};
  if (conn && (conn->n_poses != P || conn->max_n_blocks != B || conn->n_block_types != nbt ||
               conn->max_n_conn != C))
    return TMOL_B200_ERR_SHAPE;
  if (n_slots > 0 && scoring) {
    if (conn) {
      for (const void* r : conn_req)
        if (!r) return TMOL_B200_ERR_INVALID_ARGUMENT;
    } else {
      for (const void* r : dense_cp)
        if (!r) return TMOL_B200_ERR_INVALID_ARGUMENT;
    }
  }
  const void* req[] = {in->rot_coord_offset, in->first_rot_block_type, in->block_ind_for_rot,
                       in->pose_ind_for_rot, in->block_type_ind_for_rot, in->rot_offset_for_block,
                       in->bt_n_atoms, in->bt_n_conn, in->bt_conn_atom,
                       scoring ? in->bt_path_distance : in->bt_n_atoms,
                       lkb ? in->bt_n_atoms : in->bt_is_ligand_fragment,
                       scoring ? in->global_params : in->bt_n_atoms};
  if (lkb && lkb->max_n_tiles * TILE < A) return TMOL_B200_ERR_SHAPE;
  if (lkb_waters && n_slots > 0 && nbt > 0) {
    const void* lreq[] = {lkb->inter_residue_connections, lkb->first_rot_for_block, lkb->bt_atom_all_bond_ranges,
                          lkb->bt_tile_n_donH,
                          lkb->bt_tile_n_acc, lkb->bt_tile_donH_inds, lkb->bt_tile_donH_hvy_inds,
                          lkb->bt_tile_which_donH_for_hvy, lkb->bt_tile_acc_inds, lkb->bt_tile_hybridization,
                          lkb->bt_tile_acc_n_attached_H, lkb->bt_atom_is_hydrogen, lkb->water_gen_global_params};
    for (const void* r : lreq)
      if (!r) return TMOL_B200_ERR_INVALID_ARGUMENT;
    if (lkb->max_n_all_bonds < 0 || lkb->n_sp2_tors < 0 || lkb->n_sp3_tors < 0 || lkb->n_ring_tors < 0)
      return TMOL_B200_ERR_SHAPE;
    if ((lkb->n_sp2_tors && !lkb->sp2_water_tors) || (lkb->n_sp3_tors && !lkb->sp3_water_tors) ||
        (lkb->n_ring_tors && !lkb->ring_water_tors))
      return TMOL_B200_ERR_INVALID_ARGUMENT;
  }
  if (lkb && scoring && nbt > 0) {
    const void* lreq[] = {lkb->bt_tile_n_polar_atoms, lkb->bt_tile_n_occluder_atoms, lkb->bt_tile_lk_ball_params};
    for (const void* r : lreq)
      if (!r) return TMOL_B200_ERR_INVALID_ARGUMENT;
  }
  const void* req_ljlk[] = {in->bt_n_heavy_atoms_in_tile, in->bt_heavy_atoms_in_tile, in->bt_atom_types,
                            in->type_params};
  const void* req_elec[] = {elec ? elec->partial_charge : nullptr, elec ? elec->inter_repr_pd : nullptr};
  if (n_slots > 0 && nbt > 0) {
    for (const void* r : req)
      if (!r) return TMOL_B200_ERR_INVALID_ARGUMENT;
    if (term == kTermLJLK) {
      for (const void* r : req_ljlk)
        if (!r) return TMOL_B200_ERR_INVALID_ARGUMENT;
    } else if (term == kTermElec) {
      for (const void* r : req_elec)
        if (!r) return TMOL_B200_ERR_INVALID_ARGUMENT;
    }
  }
  if (scoring && !in->global_params) return TMOL_B200_ERR_INVALID_ARGUMENT;

  cudaStream_t st = (cudaStream_t)stream;
  auto* pl = new tmol_b200_ljlk_plan();
  pl->real_bytes = real_bytes;
  pl->term = term;
  pl->dims = *in;
  pl->P = P;
  pl->B = B;
  pl->nbt = nbt;
  pl->A = A;
  pl->C = C;
  pl->ntiles = nt;
  pl->T = T;
  pl->N = in->n_atoms;
  pl->reach = in->max_dis;
  pl->launch = launch ? *launch : tmol_b200_ljlk_launch{0, 0, 0, 0};
  // float pose plans of LJ/LK and elec: one CTA of 16 warps per SM unless
  // the caller chose
  if (real_bytes == 4 && !rotamers && term != kTermLKBall && pl->launch.warps_per_cta <= 0 &&
      pl->launch.ctas_per_sm <= 0) {
    pl->launch.warps_per_cta = 16;
    pl->launch.ctas_per_sm = 1;
  }
  default_launch(pl->launch);
  int dev = 0;
  int rc = TMOL_B200_OK;
#define PCK(x)                         \
  do {                                 \
    if ((x) != cudaSuccess) {          \
      free_plan(pl);                   \
      return TMOL_B200_ERR_CUDA;       \
    }                                  \
  } while (0)
  PCK(cudaGetDevice(&dev));
  PCK(cudaDeviceGetAttribute(&pl->n_sm, cudaDevAttrMultiProcessorCount, dev));
  PCK(real_bytes == 4 ? set_smem_limits<float>(term) : set_smem_limits<double>(term));
  const int64_t PB = (int64_t)P * B;
  PCK(dalloc(pl, &pl->blk_bt, PB));
  PCK(dalloc(pl, &pl->blk_off, PB));
  PCK(dalloc(pl, &pl->pose_last, P));
  PCK(dalloc(pl, &pl->bt_tf, (size_t)nbt * A));
  PCK(dalloc(pl, &pl->type_map, std::max(T, 1)));
  PCK(dalloc(pl, &pl->bt_pd, (size_t)nbt * A * A));
  PCK(dalloc(pl, &pl->bt_conn_pd, (size_t)nbt * C * A));
  PCK(dalloc(pl, &pl->bt_flags, (size_t)nbt * A));
  PCK(dalloc(pl, &pl->bt_n_atoms, nbt));
  PCK(dalloc(pl, &pl->bt_n_conn, nbt));
  PCK(dalloc(pl, &pl->bt_is_ligand, nbt));
  PCK(dalloc(pl, &pl->cp_count, PB));
  PCK(dalloc(pl, &pl->cp_b2, PB * CP_CAP));
  PCK(dalloc(pl, &pl->cp_minsep, PB * CP_CAP));
  PCK(dalloc(pl, &pl->cp_seps, PB * CP_CAP * 16));
  PCK(dalloc(pl, (unsigned char**)&pl->spheres, PB * 4 * real_bytes));
  if (!rotamers && term != kTermLKBall) {
    PCK(dalloc(pl, &pl->blk_info, PB));
    PCK(dalloc(pl, (unsigned char**)&pl->packed,
               std::max<int64_t>(in->n_atoms, 1) * (real_bytes == 4 ? sizeof(AtomRec<float>) : sizeof(AtomRec<double>))));
    PCK(dalloc(pl, (unsigned char**)&pl->spec_next, (size_t)n_terms(term) * std::max(P, 1) * real_bytes));
    PCK(dalloc(pl, (unsigned char**)&pl->spec_used, (size_t)n_terms(term) * std::max(P, 1) * real_bytes));
    PCK(dalloc(pl, (unsigned char**)&pl->spec_g, (size_t)std::max<int64_t>(in->n_atoms, 1) * 3 * real_bytes));
    PCK(dalloc(pl, &pl->spec_flag, 1));
  }
  if (real_bytes == 4) PCK(dalloc(pl, &pl->sub_spheres, PB * 8));
  PCK(dalloc(pl, &pl->counters, 4));
  PCK(dalloc(pl, &pl->counts, N_COUNTS));
  if (term == kTermElec) {
    PCK(dalloc(pl, (unsigned char**)&pl->bt_q, (size_t)nbt * A * real_bytes));
    PCK(dalloc(pl, (unsigned char**)&pl->elec_k, (size_t)N_ELEC_K * real_bytes));
    if (nbt > 0 && A > 0)
      PCK(cudaMemcpyAsync(pl->bt_q, elec->partial_charge, (size_t)nbt * A * real_bytes,
                          cudaMemcpyDeviceToDevice, st));
  }

  PCK(cudaMemsetAsync(pl->pose_last, 0, sizeof(int) * std::max(P, 1), st));
  PCK(cudaMemsetAsync(pl->counters, 0, sizeof(int) * 4, st));
  PCK(cudaMemsetAsync(pl->bt_flags, 0, sizeof(int) * std::max<int64_t>((int64_t)nbt * A, 1), st));
  PCK(cudaMemcpyAsync(pl->bt_n_atoms, in->bt_n_atoms, sizeof(int) * nbt, cudaMemcpyDeviceToDevice, st));
  PCK(cudaMemcpyAsync(pl->bt_n_conn, in->bt_n_conn, sizeof(int) * nbt, cudaMemcpyDeviceToDevice, st));
  if (term == kTermLKBall)
    // LK-ball's inter-block count pair has no ligand rule
    PCK(cudaMemsetAsync(pl->bt_is_ligand, 0, sizeof(int) * std::max(nbt, 1), st));
  else
    PCK(cudaMemcpyAsync(pl->bt_is_ligand, in->bt_is_ligand_fragment, sizeof(int) * nbt,
                        cudaMemcpyDeviceToDevice, st));
  if (scoring)
    PCK(cudaMemcpyAsync(pl->global_params, in->global_params, 5 * real_bytes, cudaMemcpyDeviceToHost, st));

  PlanBuildArgs a;
  a.in = *in;
  a.blk_bt = pl->blk_bt;
  a.blk_off = pl->blk_off;
  a.pose_last = pl->pose_last;
  a.bt_pd = pl->bt_pd;
  a.bt_conn_pd = pl->bt_conn_pd;
  a.bt_flags = pl->bt_flags;
  a.cp_count = pl->cp_count;
  a.cp_b2 = pl->cp_b2;
  a.cp_minsep = pl->cp_minsep;
  a.cp_seps = pl->cp_seps;
  a.status = pl->counters + 1;
  a.term = term;
  a.bt_inter_pd = elec ? elec->inter_repr_pd : nullptr;
  a.use_conn = conn ? 1 : 0;
  a.conn = conn ? pose_conn(*conn) : PoseConn{};
  a.rotamers = rotamers ? 1 : 0;
  a.rot_bt = a.rot_off = a.rot_block = a.rot_pose = nullptr;
  if (rotamers) {
    const int R = in->n_rots;
    pl->rotamers = true;
    pl->R = R;
    PCK(dalloc(pl, &pl->rot_bt, R));
    PCK(dalloc(pl, &pl->rot_off, R));
    PCK(dalloc(pl, &pl->rot_block, R));
    PCK(dalloc(pl, &pl->rot_pose, R));
    PCK(dalloc(pl, &pl->nrb, PB));
    PCK(dalloc(pl, &pl->rob, PB));
    PCK(dalloc(pl, (unsigned char**)&pl->rot_spheres, (size_t)R * 4 * real_bytes));
    PCK(dalloc(pl, &pl->row_pairs, PB + 2));
    PCK(dalloc(pl, &pl->row_items, PB));
    if (PB > 0) {
      PCK(cudaMemcpyAsync(pl->nrb, in->n_rots_for_block, sizeof(int) * PB, cudaMemcpyDeviceToDevice, st));
      PCK(cudaMemcpyAsync(pl->rob, in->rot_offset_for_block, sizeof(int) * PB, cudaMemcpyDeviceToDevice, st));
    }
    a.rot_bt = pl->rot_bt;
    a.rot_off = pl->rot_off;
    a.rot_block = pl->rot_block;
    a.rot_pose = pl->rot_pose;
    if (R > 0) {
      int gr = std::max(1, std::min((R + 255) / 256, pl->n_sm * 8));
      plan_rotamers_kernel<<<gr, 256, 0, st>>>(a);
      PCK(cudaGetLastError());
    }
  }
  int g = std::max(1, std::min<int>((int)((PB + 255) / 256), pl->n_sm * 8));
  if (PB > 0) {
    plan_blocks_kernel<<<g, 256, 0, st>>>(a);
    PCK(cudaGetLastError());
    if (pl->blk_info) {
      plan_block_info_kernel<<<g, 256, 0, st>>>(PB, pl->blk_bt, pl->blk_off, pl->bt_n_atoms, pl->bt_n_conn,
                                                pl->bt_is_ligand, pl->blk_info);
      PCK(cudaGetLastError());
    }
  }
  if (nbt > 0 && term == kTermLJLK) {
    int gh = std::max(1, std::min(((nbt * nt * TILE) + 255) / 256, pl->n_sm * 8));
    plan_heavy_kernel<<<gh, 256, 0, st>>>(a);
    PCK(cudaGetLastError());
  }
  if (PB > 0 && !scoring) {
    // water generation only: no count-pair tables
  } else if (PB > 0 && conn) {
    int gc = std::max(1, std::min<int>((int)((PB + 127) / 128), pl->n_sm * 16));
    plan_count_pair_conn_kernel<<<gc, 128, 0, st>>>(a);
    PCK(cudaGetLastError());
  } else if (PB > 0) {
    int gc = std::max(1, std::min<int>((int)((PB * 32 + 255) / 256), pl->n_sm * 16));
    plan_count_pair_kernel<<<gc, 256, 0, st>>>(a);
    PCK(cudaGetLastError());
  }
  int status_bits = 0;
  pl->host_pose_last.assign(std::max(P, 1), 0);
  PCK(cudaMemcpyAsync(&status_bits, pl->counters + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (P > 0)
    PCK(cudaMemcpyAsync(pl->host_pose_last.data(), pl->pose_last, sizeof(int) * P,
                        cudaMemcpyDeviceToHost, st));
  // compact atom types: the types the block types use, in index order
  std::vector<int> h_types(term == kTermLJLK ? (size_t)nbt * A : 0), h_nat(std::max(nbt, 1));
  if (nbt > 0) {
    if (term == kTermLJLK)
      PCK(cudaMemcpyAsync(h_types.data(), in->bt_atom_types, sizeof(int) * h_types.size(),
                          cudaMemcpyDeviceToHost, st));
    PCK(cudaMemcpyAsync(h_nat.data(), in->bt_n_atoms, sizeof(int) * nbt, cudaMemcpyDeviceToHost, st));
  }
  PCK(cudaStreamSynchronize(st));
  rc = status_from_bits(status_bits);
  if (rc != TMOL_B200_OK) {
    free_plan(pl);
    return rc;
  }
  std::vector<int> type_map(std::max(T, 1), -1), compact;
  for (int bt = 0; term == kTermLJLK && bt < nbt; ++bt) {
    int n = std::min(std::max(h_nat[bt], 0), A);
    for (int k = 0; k < n; ++k) {
      int t = h_types[(size_t)bt * A + k];
      if (t >= 0 && t < T) type_map[t] = 0;
    }
  }
  for (int t = 0; t < T; ++t)
    if (type_map[t] == 0) {
      type_map[t] = (int)compact.size();
      compact.push_back(t);
    }
  pl->ntp = (int)compact.size();
  if (pl->ntp > 255) {
    free_plan(pl);
    return TMOL_B200_ERR_SHAPE;
  }
  size_t ntp2 = (size_t)std::max(pl->ntp, 1) * std::max(pl->ntp, 1);
  PCK(dalloc(pl, &pl->compact_types, std::max(pl->ntp, 1)));
  PCK(dalloc(pl, (unsigned char**)&pl->ljtab,
             ntp2 * (real_bytes == 4 ? sizeof(LJRecord<float>) : sizeof(LJRecord<double>))));
  PCK(dalloc(pl, (unsigned char**)&pl->lktab,
             ntp2 * (real_bytes == 4 ? sizeof(LKRecord<float>) : sizeof(LKRecord<double>))));
  PCK(cudaMemcpyAsync(pl->type_map, type_map.data(), sizeof(int) * std::max(T, 1),
                      cudaMemcpyHostToDevice, st));
  if (pl->ntp > 0)
    PCK(cudaMemcpyAsync(pl->compact_types, compact.data(), sizeof(int) * pl->ntp,
                        cudaMemcpyHostToDevice, st));
  if (nbt > 0 && scoring) {
    int gb = std::max(1, std::min(((nbt * A) + 255) / 256, pl->n_sm * 8));
    plan_block_types_kernel<<<gb, 256, 0, st>>>(a, pl->type_map, pl->bt_tf);
    PCK(cudaGetLastError());
  }
  if (term == kTermElec) {
    // the potential's constants from the five global parameters, which the
    // reference passes to the potential as floats
    double k[N_ELEC_K];
    float gpf[5];
    for (int i = 0; i < 5; ++i)
      gpf[i] = real_bytes == 4 ? ((const float*)pl->global_params)[i]
                               : (float)((const double*)pl->global_params)[i];
    elec_constants(gpf[0], gpf[1], gpf[2], gpf[3], gpf[4], k);
    for (int i = 0; i < N_ELEC_K; ++i) {
      if (real_bytes == 4)
        ((float*)pl->elec_k_host)[i] = (float)k[i];
      else
        ((double*)pl->elec_k_host)[i] = k[i];
    }
    PCK(cudaMemcpyAsync(pl->elec_k, pl->elec_k_host, (size_t)N_ELEC_K * real_bytes, cudaMemcpyHostToDevice,
                        st));
  }
  if (term == kTermLKBall) {
    rc = real_bytes == 4 ? build_lkball<float>(pl, lkb, h_nat, st) : build_lkball<double>(pl, lkb, h_nat, st);
    if (rc != TMOL_B200_OK) {
      free_plan(pl);
      return rc;
    }
  }
  if (pl->ntp > 0) {
    int gt = std::max(1, std::min((int)((ntp2 + 127) / 128), pl->n_sm * 8));
    if (real_bytes == 4)
      plan_tables_kernel<float><<<gt, 128, 0, st>>>(
          (const float*)in->type_params, (const float*)in->global_params, pl->compact_types,
          pl->ntp, (LJRecord<float>*)pl->ljtab, (LKRecord<float>*)pl->lktab);
    else
      plan_tables_kernel<double><<<gt, 128, 0, st>>>(
          (const double*)in->type_params, (const double*)in->global_params, pl->compact_types,
          pl->ntp, (LJRecord<double>*)pl->ljtab, (LKRecord<double>*)pl->lktab);
    PCK(cudaGetLastError());
  }
  PCK(cudaMemcpyAsync(&status_bits, pl->counters + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
  PCK(cudaStreamSynchronize(st));
  rc = status_from_bits(status_bits);
  if (rc != TMOL_B200_OK) {
    free_plan(pl);
    return rc;
  }
  rc = (rotamers || !scoring) ? TMOL_B200_OK : build_work(pl, st);
  if (rc != TMOL_B200_OK) {
    free_plan(pl);
    return rc;
  }
  pl->device_bytes += (int64_t)pl->work_cap * (sizeof(int4) + sizeof(int));
#undef PCK
  *plan_out = pl;
  return TMOL_B200_OK;
}

tmol_b200_ljlk_inputs shared_inputs(const tmol_b200_elec_inputs* e) {
  tmol_b200_ljlk_inputs in = {};
  in.n_atoms = e->n_atoms;
  in.n_poses = e->n_poses;
  in.max_n_blocks = e->max_n_blocks;
  in.n_rots = e->n_rots;
  in.n_block_types = e->n_block_types;
  in.max_n_block_atoms = e->max_n_block_atoms;
  in.max_n_conn = e->max_n_conn;
  in.max_n_tiles = (e->max_n_block_atoms + TILE - 1) / TILE;
  in.n_atom_types = 0;
  in.rot_coord_offset = e->rot_coord_offset;
  in.pose_ind_for_atom = e->pose_ind_for_atom;
  in.first_rot_for_block = e->first_rot_for_block;
  in.first_rot_block_type = e->first_rot_block_type;
  in.block_ind_for_rot = e->block_ind_for_rot;
  in.pose_ind_for_rot = e->pose_ind_for_rot;
  in.block_type_ind_for_rot = e->block_type_ind_for_rot;
  in.n_rots_for_pose = e->n_rots_for_pose;
  in.rot_offset_for_pose = e->rot_offset_for_pose;
  in.n_rots_for_block = e->n_rots_for_block;
  in.rot_offset_for_block = e->rot_offset_for_block;
  in.max_n_rots_per_pose = e->max_n_rots_per_pose;
  in.min_bondsep = e->min_bondsep;
  in.inter_block_bondsep = e->inter_block_bondsep;
  in.bt_n_atoms = e->bt_n_atoms;
  in.bt_n_conn = e->bt_n_conn;
  in.bt_conn_atom = e->bt_conn_atom;
  in.bt_path_distance = e->bt_intra_repr_path_distance;
  in.bt_is_ligand_fragment = e->bt_is_ligand_fragment;
  in.global_params = e->global_params;
  in.max_dis = e->max_dis;
  return in;
}

int create_lkball_plan(const tmol_b200_lkball_inputs* k, int real_bytes, const tmol_b200_ljlk_launch* launch,
                       void* stream, bool rotamers, tmol_b200_ljlk_plan** plan_out,
                       const tmol_b200_pose_connectivity* conn = nullptr) {
  if (!k || !plan_out) return TMOL_B200_ERR_INVALID_ARGUMENT;
  tmol_b200_ljlk_inputs in = {};
  in.n_atoms = k->n_atoms;
  in.n_poses = k->n_poses;
  in.max_n_blocks = k->max_n_blocks;
  in.n_rots = k->n_rots;
  in.n_block_types = k->n_block_types;
  in.max_n_block_atoms = k->max_n_block_atoms;
  in.max_n_conn = k->max_n_conn;
  in.max_n_tiles = k->max_n_tiles;
  in.n_atom_types = 0;
  in.rot_coord_offset = k->rot_coord_offset;
  in.pose_ind_for_atom = k->pose_ind_for_atom;
  in.first_rot_for_block = k->first_rot_for_block;
  in.first_rot_block_type = k->first_rot_block_type;
  in.block_ind_for_rot = k->block_ind_for_rot;
  in.pose_ind_for_rot = k->pose_ind_for_rot;
  in.block_type_ind_for_rot = k->block_type_ind_for_rot;
  in.n_rots_for_pose = k->n_rots_for_pose;
  in.rot_offset_for_pose = k->rot_offset_for_pose;
  in.n_rots_for_block = k->n_rots_for_block;
  in.rot_offset_for_block = k->rot_offset_for_block;
  in.max_n_rots_per_pose = k->max_n_rots_per_pose;
  in.min_bondsep = k->min_bondsep;
  in.inter_block_bondsep = k->inter_block_bondsep;
  in.bt_n_atoms = k->bt_n_atoms;
  in.bt_n_conn = k->bt_n_conn;
  in.bt_conn_atom = k->bt_conn_atom;
  in.bt_path_distance = k->bt_path_distance;
  in.global_params = k->global_params;
  in.max_dis = k->max_dis;
  return create_plan(&in, real_bytes, launch, stream, rotamers, plan_out, nullptr, conn, k);
}

int create_elec_plan(const tmol_b200_elec_inputs* e, int real_bytes, const tmol_b200_ljlk_launch* launch,
                     void* stream, bool rotamers, tmol_b200_ljlk_plan** plan_out,
                     const tmol_b200_pose_connectivity* conn = nullptr) {
  if (!e || !plan_out) return TMOL_B200_ERR_INVALID_ARGUMENT;
  const tmol_b200_ljlk_inputs in = shared_inputs(e);
  const ElecExtra x = {e->bt_partial_charge, e->bt_inter_repr_path_distance};
  return create_plan(&in, real_bytes, launch, stream, rotamers, plan_out, &x, conn);
}

bool pose_plan_of(const tmol_b200_ljlk_plan* plan, int term) {
  return plan && !plan->rotamers && plan->term == term;
}

bool rotamer_plan_of(const tmol_b200_ljlk_plan* plan, int term) {
  return plan && plan->rotamers && plan->term == term;
}

int pose_forward(tmol_b200_ljlk_plan* plan, int term, const void* coords, int block_pair, void* energies,
                 int32_t* block_neighbors, void* stream) {
  if (!pose_plan_of(plan, term) || !energies || (!coords && plan->N > 0))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4)
    return forward_impl<float>(plan, coords, block_pair, energies, block_neighbors, st);
  return forward_impl<double>(plan, coords, block_pair, energies, block_neighbors, st);
}

int pose_backward(tmol_b200_ljlk_plan* plan, int term, const void* coords, int block_pair, const void* dTdV,
                  void* dcoords, void* stream) {
  if (!pose_plan_of(plan, term) || !dTdV || !dcoords || (!coords && plan->N > 0))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4)
    return backward_impl<float>(plan, coords, block_pair, dTdV, dcoords, st);
  return backward_impl<double>(plan, coords, block_pair, dTdV, dcoords, st);
}

int pose_forward_speculative(tmol_b200_ljlk_plan* plan, int term, const void* coords, void* energies,
                             int32_t* block_neighbors, void* stream) {
  if (!pose_plan_of(plan, term) || !plan->spec_g || !energies || (!coords && plan->N > 0))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4) return forward_speculative_impl<float>(plan, coords, energies, block_neighbors, st);
  return forward_speculative_impl<double>(plan, coords, energies, block_neighbors, st);
}

int pose_backward_speculative(tmol_b200_ljlk_plan* plan, int term, const void* coords, const void* dTdV,
                              void* dcoords, int speculated, void* stream) {
  if (!pose_plan_of(plan, term) || !plan->spec_g || !dTdV || !dcoords || (!coords && plan->N > 0))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4) return backward_speculative_impl<float>(plan, coords, dTdV, dcoords, speculated, st);
  return backward_speculative_impl<double>(plan, coords, dTdV, dcoords, speculated, st);
}

int pose_energy_and_gradient(tmol_b200_ljlk_plan* plan, int term, const void* coords, const void* weights,
                             void* energies, void* dcoords, void* stream) {
  if (!pose_plan_of(plan, term) || !weights || !energies || !dcoords || (!coords && plan->N > 0))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4)
    return energy_and_gradient_impl<float>(plan, coords, weights, energies, dcoords, st);
  return energy_and_gradient_impl<double>(plan, coords, weights, energies, dcoords, st);
}

int rotamer_count(tmol_b200_ljlk_plan* plan, int term, const void* coords, int64_t* n_pairs,
                  int64_t* n_items, void* stream) {
  if (!rotamer_plan_of(plan, term) || !n_pairs || !n_items || (!coords && plan->N > 0))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4) return rotamer_count_impl<float>(plan, coords, n_pairs, n_items, st);
  return rotamer_count_impl<double>(plan, coords, n_pairs, n_items, st);
}

int rotamer_fill(tmol_b200_ljlk_plan* plan, int term, int32_t* indices, int32_t* items, void* stream) {
  if (!rotamer_plan_of(plan, term) || plan->n_pairs < 0) return TMOL_B200_ERR_INVALID_ARGUMENT;
  if ((plan->n_pairs > 0 && !indices) || (plan->n_items > 0 && !items))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4) return rotamer_fill_impl<float>(plan, indices, items, st);
  return rotamer_fill_impl<double>(plan, indices, items, st);
}

int rotamer_forward(tmol_b200_ljlk_plan* plan, int term, const void* coords, const int32_t* items,
                    int64_t n_items, int64_t n_pairs, void* energies, void* stream) {
  if (!rotamer_plan_of(plan, term) || !energies || n_items < 0 || n_pairs < 0 || (n_items > 0 && !items) ||
      (!coords && plan->N > 0))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (n_items >= ((int64_t)1 << 31) || n_pairs >= ((int64_t)1 << 31)) return TMOL_B200_ERR_CAPACITY;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4)
    return rotamer_score_impl<float, false>(plan, coords, items, n_items, n_pairs, energies, nullptr, nullptr,
                                            st);
  return rotamer_score_impl<double, false>(plan, coords, items, n_items, n_pairs, energies, nullptr, nullptr,
                                           st);
}

int rotamer_backward(tmol_b200_ljlk_plan* plan, int term, const void* coords, const int32_t* items,
                     int64_t n_items, int64_t n_pairs, const void* dTdV, void* dcoords, void* stream) {
  if (!rotamer_plan_of(plan, term) || !dTdV || !dcoords || n_items < 0 || n_pairs < 0 ||
      (n_items > 0 && !items) || (!coords && plan->N > 0))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (n_items >= ((int64_t)1 << 31) || n_pairs >= ((int64_t)1 << 31)) return TMOL_B200_ERR_CAPACITY;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4)
    return rotamer_score_impl<float, true>(plan, coords, items, n_items, n_pairs, nullptr, dTdV, dcoords, st);
  return rotamer_score_impl<double, true>(plan, coords, items, n_items, n_pairs, nullptr, dTdV, dcoords, st);
}

}  // namespace

extern "C" {

namespace {
// An NVTX range around an entry point's work (named by the entry point), so
// that the scoring calls show up in Nsight Systems timelines; without a tool
// attached a push/pop costs a few nanoseconds.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};
}  // namespace

int tmol_b200_ljlk_plan_create(const tmol_b200_ljlk_inputs* in, int real_bytes,
                               const tmol_b200_ljlk_launch* launch,
                               void* stream, tmol_b200_ljlk_plan** plan_out) {
  NvtxRange nvtx_range("tmol_b200_ljlk_plan_create");
  return create_plan(in, real_bytes, launch, stream, false, plan_out);
}

int tmol_b200_ljlk_rotamer_plan_create(const tmol_b200_ljlk_inputs* in, int real_bytes,
                                       const tmol_b200_ljlk_launch* launch,
                                       void* stream, tmol_b200_ljlk_plan** plan_out) {
  NvtxRange nvtx_range("tmol_b200_ljlk_rotamer_plan_create");
  return create_plan(in, real_bytes, launch, stream, true, plan_out);
}

int tmol_b200_ljlk_plan_create_from_connectivity(const tmol_b200_ljlk_inputs* in,
                                                 const tmol_b200_pose_connectivity* conn, int real_bytes,
                                                 const tmol_b200_ljlk_launch* launch, void* stream,
                                                 int rotamers, tmol_b200_ljlk_plan** plan_out) {
  NvtxRange nvtx_range("tmol_b200_ljlk_plan_create_from_connectivity");
  if (!conn) return TMOL_B200_ERR_INVALID_ARGUMENT;
  return create_plan(in, real_bytes, launch, stream, rotamers != 0, plan_out, nullptr, conn);
}

int tmol_b200_elec_plan_create_from_connectivity(const tmol_b200_elec_inputs* in,
                                                 const tmol_b200_pose_connectivity* conn, int real_bytes,
                                                 const tmol_b200_ljlk_launch* launch, void* stream,
                                                 int rotamers, tmol_b200_elec_plan** plan_out) {
  NvtxRange nvtx_range("tmol_b200_elec_plan_create_from_connectivity");
  if (!conn) return TMOL_B200_ERR_INVALID_ARGUMENT;
  return create_elec_plan(in, real_bytes, launch, stream, rotamers != 0, plan_out, conn);
}

int tmol_b200_ljlk_plan_destroy(tmol_b200_ljlk_plan* plan) {
  if (!plan) return TMOL_B200_ERR_INVALID_ARGUMENT;
  free_plan(plan);
  return TMOL_B200_OK;
}

int tmol_b200_ljlk_plan_set_launch(tmol_b200_ljlk_plan* plan,
                                   const tmol_b200_ljlk_launch* launch) {
  if (!plan || !launch) return TMOL_B200_ERR_INVALID_ARGUMENT;
  int old_cpi = plan->launch.candidates_per_item;
  plan->launch = *launch;
  default_launch(plan->launch);
  if (plan->launch.candidates_per_item != old_cpi) return build_work(plan, 0);
  return TMOL_B200_OK;
}

int tmol_b200_ljlk_forward(tmol_b200_ljlk_plan* plan, const void* coords,
                           int block_pair, void* energies,
                           int32_t* block_neighbors, void* stream) {
  NvtxRange nvtx_range("tmol_b200_ljlk_forward");
  return pose_forward(plan, kTermLJLK, coords, block_pair, energies, block_neighbors, stream);
}

int tmol_b200_ljlk_backward(tmol_b200_ljlk_plan* plan, const void* coords,
                            int block_pair, const void* dTdV, void* dcoords,
                            void* stream) {
  NvtxRange nvtx_range("tmol_b200_ljlk_backward");
  return pose_backward(plan, kTermLJLK, coords, block_pair, dTdV, dcoords, stream);
}

int tmol_b200_ljlk_forward_speculative(tmol_b200_ljlk_plan* plan, const void* coords,
                                       void* energies, int32_t* block_neighbors, void* stream) {
  NvtxRange nvtx_range("tmol_b200_ljlk_forward_speculative");
  return pose_forward_speculative(plan, kTermLJLK, coords, energies, block_neighbors, stream);
}

int tmol_b200_ljlk_backward_speculative(tmol_b200_ljlk_plan* plan, const void* coords,
                                        const void* dTdV, void* dcoords, int speculated,
                                        void* stream) {
  NvtxRange nvtx_range("tmol_b200_ljlk_backward_speculative");
  return pose_backward_speculative(plan, kTermLJLK, coords, dTdV, dcoords, speculated, stream);
}

int tmol_b200_ljlk_energy_and_gradient(tmol_b200_ljlk_plan* plan,
                                       const void* coords, const void* weights,
                                       void* energies, void* dcoords,
                                       void* stream) {
  NvtxRange nvtx_range("tmol_b200_ljlk_energy_and_gradient");
  return pose_energy_and_gradient(plan, kTermLJLK, coords, weights, energies, dcoords, stream);
}

int tmol_b200_ljlk_plan_set_counting(tmol_b200_ljlk_plan* plan, int enable) {
  if (!plan) return TMOL_B200_ERR_INVALID_ARGUMENT;
  plan->counting = enable != 0;
  return TMOL_B200_OK;
}

int tmol_b200_ljlk_last_counts(tmol_b200_ljlk_plan* plan, void* stream,
                               int64_t* counts) {
  if (!plan || !counts) return TMOL_B200_ERR_INVALID_ARGUMENT;
  unsigned long long h[N_COUNTS] = {};
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaMemcpyAsync(h, plan->counts, sizeof(h), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int k = 0; k < N_COUNTS; ++k) counts[k] = (int64_t)h[k];
  return TMOL_B200_OK;
}

int tmol_b200_ljlk_profile(tmol_b200_ljlk_plan* plan, int enable) {
  if (!plan) return TMOL_B200_ERR_INVALID_ARGUMENT;
  plan->profiling = enable != 0;
  plan->prof_n = 0;
  if (plan->profiling && plan->prof_events.empty()) {
    plan->prof_events.resize(2 * 4096);
    for (auto& e : plan->prof_events) CK(cudaEventCreate(&e));
  }
  return TMOL_B200_OK;
}

int tmol_b200_ljlk_profile_read(tmol_b200_ljlk_plan* plan, double* total_ms,
                                int32_t* n_launches) {
  if (!plan || !total_ms || !n_launches) return TMOL_B200_ERR_INVALID_ARGUMENT;
  double tot = 0;
  for (int k = 0; k < plan->prof_n; ++k) {
    CK(cudaEventSynchronize(plan->prof_events[2 * k + 1]));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, plan->prof_events[2 * k], plan->prof_events[2 * k + 1]));
    tot += ms;
  }
  *total_ms = tot;
  *n_launches = plan->prof_n;
  return TMOL_B200_OK;
}

int tmol_b200_measure_fp32_peak(void* stream, double* tflops) {
  if (!tflops) return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0, n_sm = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  float* out = nullptr;
  CK(cudaMallocAsync((void**)&out, sizeof(float), st));
  const int threads = 512, blocks = n_sm * 4, iters = 1 << 16;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  fp32_peak_kernel<<<blocks, threads, 0, st>>>(out, iters / 8, 0.999f, 1e-4f);
  CK(cudaEventRecord(e0, st));
  fp32_peak_kernel<<<blocks, threads, 0, st>>>(out, iters, 0.999f, 1e-4f);
  CK(cudaEventRecord(e1, st));
  CK(cudaEventSynchronize(e1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CK(cudaFreeAsync(out, st));
  CK(cudaStreamSynchronize(st));
  double flops = 2.0 * 8.0 * (double)iters * threads * blocks;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return TMOL_B200_OK;
}

int tmol_b200_ljlk_plan_rebalance(tmol_b200_ljlk_plan* plan, void* stream) {
  NvtxRange nvtx_range("tmol_b200_ljlk_plan_rebalance");
  if (!plan) return TMOL_B200_ERR_INVALID_ARGUMENT;
  int n = plan->n_work;
  if (n == 0) return TMOL_B200_OK;
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<int4> work(n);
  std::vector<int> cost(n);
  CK(cudaMemcpyAsync(work.data(), plan->work, sizeof(int4) * n, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(cost.data(), plan->item_cost, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  // An item costlier than half a warp's share of the whole call would end
  // after every other warp: it is split into two items over the halves of
  // its candidate range (each estimated at half the cost, measured in the
  // next call), until it is cheap enough, holds one candidate, or the
  // buffers are full.
  long long total = 0;
  for (int c : cost) total += c;
  const long long warps =
      std::max(1LL, (long long)plan->n_sm * plan->launch.ctas_per_sm * plan->launch.warps_per_cta);
  const long long limit = std::max(1LL, total / warps / 2);
  for (size_t i = 0; i < work.size(); ++i) {
    while (cost[i] > limit && work[i].w - work[i].z > 1 && (int)work.size() < plan->work_cap) {
      int4 hi = work[i];
      const int mid = (work[i].z + work[i].w) / 2;
      hi.z = mid;
      work[i].w = mid;
      cost[i] /= 2;
      work.push_back(hi);
      cost.push_back(cost[i]);
    }
  }
  n = (int)work.size();
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  // longest items first, so that the last items any warp takes are short
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  std::vector<int4> sorted(n);
  std::vector<int> sorted_cost(n);
  for (int i = 0; i < n; ++i) {
    sorted[i] = work[order[i]];
    sorted_cost[i] = cost[order[i]];
  }
  plan->n_work = n;
  CK(cudaMemcpyAsync(plan->work, sorted.data(), sizeof(int4) * n, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(plan->item_cost, sorted_cost.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(plan->counters + 2, &plan->n_work, sizeof(int), cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
  return TMOL_B200_OK;
}

int tmol_b200_ljlk_plan_set_skip_mask(tmol_b200_ljlk_plan* plan,
                                      const uint32_t* mask,
                                      int32_t words_per_row) {
  if (!plan) return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (mask && words_per_row < (plan->B + 31) / 32) return TMOL_B200_ERR_SHAPE;
  plan->skip = mask;
  plan->skip_words = mask ? words_per_row : 0;
  return TMOL_B200_OK;
}

int tmol_b200_ljlk_screen_candidates(tmol_b200_ljlk_plan* plan,
                                     const void* coords, int32_t capacity,
                                     int32_t* pair_row, int32_t* pair_b2,
                                     int32_t* pair_bt, float* features,
                                     int32_t* count, void* stream) {
  NvtxRange nvtx_range("tmol_b200_ljlk_screen_candidates");
  if (!plan || !count || capacity < 0 || (!coords && plan->N > 0))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (capacity > 0 && (!pair_row || !pair_b2 || !pair_bt || !features))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (plan->real_bytes != 4) return TMOL_B200_ERR_DTYPE;
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaMemsetAsync(count, 0, sizeof(int32_t), st));
  const int n_blocks = plan->P * plan->B;
  if (n_blocks == 0) return TMOL_B200_OK;
  ScoreArgs<float> s = score_args<float>(plan, coords);
  const int threads = 256;
  const int grid = std::max(1, std::min((n_blocks + 7) / 8, plan->n_sm * 16));
  spheres_kernel<float><<<grid, threads, 0, st>>>(s);
  CK(cudaGetLastError());
  const int grid_u = std::max(1, std::min((n_blocks + threads - 1) / threads, plan->n_sm * 8));
  sub_spheres_kernel<<<grid_u, threads, 0, st>>>(s, plan->sub_spheres);
  CK(cudaGetLastError());
  screen_candidates_kernel<<<grid, threads, 0, st>>>(s, plan->sub_spheres, capacity, pair_row,
                                                     pair_b2, pair_bt, features, count);
  CK(cudaGetLastError());
  return TMOL_B200_OK;
}

int tmol_b200_ljlk_rotamer_count(tmol_b200_ljlk_plan* plan, const void* coords,
                                  int64_t* n_pairs, int64_t* n_items, void* stream) {
  NvtxRange nvtx_range("tmol_b200_ljlk_rotamer_count");
  return rotamer_count(plan, kTermLJLK, coords, n_pairs, n_items, stream);
}

int tmol_b200_ljlk_rotamer_fill(tmol_b200_ljlk_plan* plan, int32_t* indices, int32_t* items,
                                void* stream) {
  NvtxRange nvtx_range("tmol_b200_ljlk_rotamer_fill");
  return rotamer_fill(plan, kTermLJLK, indices, items, stream);
}

int tmol_b200_ljlk_rotamer_forward(tmol_b200_ljlk_plan* plan, const void* coords,
                                    const int32_t* items, int64_t n_items, int64_t n_pairs,
                                    void* energies, void* stream) {
  NvtxRange nvtx_range("tmol_b200_ljlk_rotamer_forward");
  return rotamer_forward(plan, kTermLJLK, coords, items, n_items, n_pairs, energies, stream);
}

int tmol_b200_ljlk_rotamer_backward(tmol_b200_ljlk_plan* plan, const void* coords,
                                     const int32_t* items, int64_t n_items, int64_t n_pairs,
                                     const void* dTdV, void* dcoords, void* stream) {
  NvtxRange nvtx_range("tmol_b200_ljlk_rotamer_backward");
  return rotamer_backward(plan, kTermLJLK, coords, items, n_items, n_pairs, dTdV, dcoords, stream);
}

// ---------------------------------------------------------------------------
// elec entry points (include/tmol_b200_elec.h)

int tmol_b200_elec_plan_create(const tmol_b200_elec_inputs* in, int real_bytes,
                               const tmol_b200_ljlk_launch* launch, void* stream,
                               tmol_b200_elec_plan** plan_out) {
  NvtxRange nvtx_range("tmol_b200_elec_plan_create");
  return create_elec_plan(in, real_bytes, launch, stream, false, plan_out);
}

int tmol_b200_elec_rotamer_plan_create(const tmol_b200_elec_inputs* in, int real_bytes,
                                       const tmol_b200_ljlk_launch* launch, void* stream,
                                       tmol_b200_elec_plan** plan_out) {
  NvtxRange nvtx_range("tmol_b200_elec_rotamer_plan_create");
  return create_elec_plan(in, real_bytes, launch, stream, true, plan_out);
}

int tmol_b200_elec_plan_destroy(tmol_b200_elec_plan* plan) {
  if (!plan || plan->term != kTermElec) return TMOL_B200_ERR_INVALID_ARGUMENT;
  free_plan(plan);
  return TMOL_B200_OK;
}

int tmol_b200_elec_forward(tmol_b200_elec_plan* plan, const void* coords, int block_pair,
                           void* energies, int32_t* block_neighbors, void* stream) {
  NvtxRange nvtx_range("tmol_b200_elec_forward");
  return pose_forward(plan, kTermElec, coords, block_pair, energies, block_neighbors, stream);
}

int tmol_b200_elec_backward(tmol_b200_elec_plan* plan, const void* coords, int block_pair,
                            const void* dTdV, void* dcoords, void* stream) {
  NvtxRange nvtx_range("tmol_b200_elec_backward");
  return pose_backward(plan, kTermElec, coords, block_pair, dTdV, dcoords, stream);
}

int tmol_b200_elec_forward_speculative(tmol_b200_elec_plan* plan, const void* coords,
                                       void* energies, int32_t* block_neighbors, void* stream) {
  NvtxRange nvtx_range("tmol_b200_elec_forward_speculative");
  return pose_forward_speculative(plan, kTermElec, coords, energies, block_neighbors, stream);
}

int tmol_b200_elec_backward_speculative(tmol_b200_elec_plan* plan, const void* coords,
                                        const void* dTdV, void* dcoords, int speculated,
                                        void* stream) {
  NvtxRange nvtx_range("tmol_b200_elec_backward_speculative");
  return pose_backward_speculative(plan, kTermElec, coords, dTdV, dcoords, speculated, stream);
}

int tmol_b200_elec_energy_and_gradient(tmol_b200_elec_plan* plan, const void* coords,
                                       const void* weights, void* energies, void* dcoords,
                                       void* stream) {
  NvtxRange nvtx_range("tmol_b200_elec_energy_and_gradient");
  return pose_energy_and_gradient(plan, kTermElec, coords, weights, energies, dcoords, stream);
}

int tmol_b200_elec_rotamer_count(tmol_b200_elec_plan* plan, const void* coords,
                                 int64_t* n_pairs, int64_t* n_items, void* stream) {
  NvtxRange nvtx_range("tmol_b200_elec_rotamer_count");
  return rotamer_count(plan, kTermElec, coords, n_pairs, n_items, stream);
}

int tmol_b200_elec_rotamer_fill(tmol_b200_elec_plan* plan, int32_t* indices, int32_t* items,
                                void* stream) {
  NvtxRange nvtx_range("tmol_b200_elec_rotamer_fill");
  return rotamer_fill(plan, kTermElec, indices, items, stream);
}

int tmol_b200_elec_rotamer_forward(tmol_b200_elec_plan* plan, const void* coords,
                                   const int32_t* items, int64_t n_items, int64_t n_pairs,
                                   void* energies, void* stream) {
  NvtxRange nvtx_range("tmol_b200_elec_rotamer_forward");
  return rotamer_forward(plan, kTermElec, coords, items, n_items, n_pairs, energies, stream);
}

int tmol_b200_elec_rotamer_backward(tmol_b200_elec_plan* plan, const void* coords,
                                    const int32_t* items, int64_t n_items, int64_t n_pairs,
                                    const void* dTdV, void* dcoords, void* stream) {
  NvtxRange nvtx_range("tmol_b200_elec_rotamer_backward");
  return rotamer_backward(plan, kTermElec, coords, items, n_items, n_pairs, dTdV, dcoords, stream);
}

// LK-ball entry points (include/tmol_b200_lkball.h)

int tmol_b200_lkball_plan_create(const tmol_b200_lkball_inputs* inputs, int real_bytes,
                                 const tmol_b200_ljlk_launch* launch, void* stream,
                                 tmol_b200_lkball_plan** plan_out) {
  NvtxRange nvtx_range("tmol_b200_lkball_plan_create");
  return create_lkball_plan(inputs, real_bytes, launch, stream, false, plan_out);
}

int tmol_b200_lkball_plan_create_from_connectivity(const tmol_b200_lkball_inputs* inputs,
                                                   const tmol_b200_pose_connectivity* conn, int real_bytes,
                                                   const tmol_b200_ljlk_launch* launch, void* stream, int rotamers,
                                                   tmol_b200_lkball_plan** plan_out) {
  NvtxRange nvtx_range("tmol_b200_lkball_plan_create_from_connectivity");
  if (!conn) return TMOL_B200_ERR_INVALID_ARGUMENT;
  return create_lkball_plan(inputs, real_bytes, launch, stream, rotamers != 0, plan_out, conn);
}

int tmol_b200_lkball_rotamer_plan_create(const tmol_b200_lkball_inputs* inputs, int real_bytes,
                                         const tmol_b200_ljlk_launch* launch, void* stream,
                                         tmol_b200_lkball_plan** plan_out) {
  NvtxRange nvtx_range("tmol_b200_lkball_rotamer_plan_create");
  return create_lkball_plan(inputs, real_bytes, launch, stream, true, plan_out);
}

int tmol_b200_lkball_rotamer_count(tmol_b200_lkball_plan* plan, const void* coords, int64_t* n_pairs,
                                   int64_t* n_items, void* stream) {
  NvtxRange nvtx_range("tmol_b200_lkball_rotamer_count");
  if (!plan || !plan->lkb_pol) return TMOL_B200_ERR_INVALID_ARGUMENT;
  return rotamer_count(plan, kTermLKBall, coords, n_pairs, n_items, stream);
}

int tmol_b200_lkball_rotamer_fill(tmol_b200_lkball_plan* plan, int32_t* indices, int32_t* items, void* stream) {
  NvtxRange nvtx_range("tmol_b200_lkball_rotamer_fill");
  if (!plan || !plan->lkb_pol) return TMOL_B200_ERR_INVALID_ARGUMENT;
  return rotamer_fill(plan, kTermLKBall, indices, items, stream);
}

int tmol_b200_lkball_rotamer_forward(tmol_b200_lkball_plan* plan, const void* coords, const void* waters,
                                     const int32_t* items, int64_t n_items, int64_t n_pairs, void* energies,
                                     void* stream) {
  NvtxRange nvtx_range("tmol_b200_lkball_rotamer_forward");
  if (!rotamer_plan_of(plan, kTermLKBall) || !plan->lkb_pol || !energies || n_items < 0 || n_pairs < 0 ||
      (n_items > 0 && !items) || (plan->N > 0 && (!coords || !waters)))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (n_items >= ((int64_t)1 << 31) || n_pairs >= ((int64_t)1 << 31)) return TMOL_B200_ERR_CAPACITY;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4)
    return lkb_rotamer_score_impl<float, false>(plan, coords, waters, items, n_items, n_pairs, energies, nullptr,
                                                nullptr, nullptr, st);
  return lkb_rotamer_score_impl<double, false>(plan, coords, waters, items, n_items, n_pairs, energies, nullptr,
                                               nullptr, nullptr, st);
}

int tmol_b200_lkball_rotamer_backward(tmol_b200_lkball_plan* plan, const void* coords, const void* waters,
                                      const int32_t* items, int64_t n_items, int64_t n_pairs, const void* dTdV,
                                      void* dcoords, void* dwaters, void* stream) {
  NvtxRange nvtx_range("tmol_b200_lkball_rotamer_backward");
  if (!rotamer_plan_of(plan, kTermLKBall) || !plan->lkb_pol || !dTdV || !dcoords || !dwaters || n_items < 0 ||
      n_pairs < 0 || (n_items > 0 && !items) || (plan->N > 0 && (!coords || !waters)))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (n_items >= ((int64_t)1 << 31) || n_pairs >= ((int64_t)1 << 31)) return TMOL_B200_ERR_CAPACITY;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4)
    return lkb_rotamer_score_impl<float, true>(plan, coords, waters, items, n_items, n_pairs, nullptr, dTdV,
                                               dcoords, dwaters, st);
  return lkb_rotamer_score_impl<double, true>(plan, coords, waters, items, n_items, n_pairs, nullptr, dTdV,
                                              dcoords, dwaters, st);
}

int tmol_b200_lkball_plan_destroy(tmol_b200_lkball_plan* plan) {
  if (!plan || plan->term != kTermLKBall) return TMOL_B200_ERR_INVALID_ARGUMENT;
  free_plan(plan);
  return TMOL_B200_OK;
}

int tmol_b200_lkball_waters(tmol_b200_lkball_plan* plan, const void* coords, void* waters, void* stream) {
  NvtxRange nvtx_range("tmol_b200_lkball_waters");
  if (!plan || plan->term != kTermLKBall || !plan->lkb_sites) return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (plan->N > 0 && (!coords || !waters)) return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  return plan->real_bytes == 4 ? lkb_waters_impl<float>(plan, coords, waters, st)
                               : lkb_waters_impl<double>(plan, coords, waters, st);
}

int tmol_b200_lkball_waters_backward(tmol_b200_lkball_plan* plan, const void* coords, const void* dwaters,
                                     void* dcoords, void* stream) {
  NvtxRange nvtx_range("tmol_b200_lkball_waters_backward");
  if (!plan || plan->term != kTermLKBall || !plan->lkb_sites) return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (plan->N > 0 && (!coords || !dwaters || !dcoords)) return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  return plan->real_bytes == 4 ? lkb_waters_backward_impl<float>(plan, coords, dwaters, dcoords, st)
                               : lkb_waters_backward_impl<double>(plan, coords, dwaters, dcoords, st);
}

int tmol_b200_lkball_forward(tmol_b200_lkball_plan* plan, const void* coords, const void* waters,
                             int block_pair, void* energies, int32_t* block_neighbors, void* stream) {
  NvtxRange nvtx_range("tmol_b200_lkball_forward");
  if (!plan || plan->term != kTermLKBall || !plan->lkb_pol || !energies) return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (plan->N > 0 && (!coords || !waters)) return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4)
    return block_pair ? lkb_score_impl<float, false, true>(plan, coords, waters, energies, block_neighbors,
                                                           nullptr, nullptr, nullptr, st)
                      : lkb_score_impl<float, false, false>(plan, coords, waters, energies, block_neighbors,
                                                            nullptr, nullptr, nullptr, st);
  return block_pair ? lkb_score_impl<double, false, true>(plan, coords, waters, energies, block_neighbors,
                                                          nullptr, nullptr, nullptr, st)
                    : lkb_score_impl<double, false, false>(plan, coords, waters, energies, block_neighbors,
                                                           nullptr, nullptr, nullptr, st);
}

int tmol_b200_lkball_forward_speculative(tmol_b200_lkball_plan* plan, const void* coords, const void* waters,
                                         void* energies, int32_t* block_neighbors, void* stream) {
  NvtxRange nvtx_range("tmol_b200_lkball_forward_speculative");
  if (!plan || plan->term != kTermLKBall || plan->rotamers || !plan->lkb_pol || !plan->spec_g || !energies)
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (plan->N > 0 && (!coords || !waters)) return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4)
    return lkb_forward_speculative_impl<float>(plan, coords, waters, energies, block_neighbors, st);
  return lkb_forward_speculative_impl<double>(plan, coords, waters, energies, block_neighbors, st);
}

int tmol_b200_lkball_backward_speculative(tmol_b200_lkball_plan* plan, const void* coords, const void* waters,
                                          const void* dTdV, void* dcoords, void* dwaters, int speculated,
                                          void* stream) {
  NvtxRange nvtx_range("tmol_b200_lkball_backward_speculative");
  if (!plan || plan->term != kTermLKBall || plan->rotamers || !plan->lkb_pol || !plan->spec_g || !dTdV)
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (plan->N > 0 && (!coords || !waters || !dcoords || !dwaters)) return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4)
    return lkb_backward_speculative_impl<float>(plan, coords, waters, dTdV, dcoords, dwaters, speculated, st);
  return lkb_backward_speculative_impl<double>(plan, coords, waters, dTdV, dcoords, dwaters, speculated, st);
}

int tmol_b200_lkball_energy_and_gradient(tmol_b200_lkball_plan* plan, const void* coords, const void* weights,
                                         void* energies, void* dcoords, void* stream) {
  NvtxRange nvtx_range("tmol_b200_lkball_energy_and_gradient");
  if (!plan || plan->term != kTermLKBall || !plan->lkb_pol || !plan->lkb_sites || !weights || !energies ||
      !dcoords)
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (plan->N > 0 && !coords) return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if (plan->real_bytes == 4) {
    if ((rc = lkb_waters_impl<float>(plan, coords, plan->lkb_waters, st, true))) return rc;
    if ((rc = lkb_score_impl<float, true, false>(plan, coords, plan->lkb_waters, energies, nullptr, weights,
                                                 dcoords, plan->lkb_dwaters, st)))
      return rc;
    return lkb_waters_backward_impl<float>(plan, coords, plan->lkb_dwaters, dcoords, st);
  }
  if ((rc = lkb_waters_impl<double>(plan, coords, plan->lkb_waters, st, true))) return rc;
  if ((rc = lkb_score_impl<double, true, false>(plan, coords, plan->lkb_waters, energies, nullptr, weights,
                                                dcoords, plan->lkb_dwaters, st)))
    return rc;
  return lkb_waters_backward_impl<double>(plan, coords, plan->lkb_dwaters, dcoords, st);
}

int tmol_b200_lkball_backward(tmol_b200_lkball_plan* plan, const void* coords, const void* waters,
                              int block_pair, const void* dTdV, void* dcoords, void* dwaters,
                              void* stream) {
  NvtxRange nvtx_range("tmol_b200_lkball_backward");
  if (!plan || plan->term != kTermLKBall || !plan->lkb_pol || !dTdV) return TMOL_B200_ERR_INVALID_ARGUMENT;
  if (plan->N > 0 && (!coords || !waters || !dcoords || !dwaters)) return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4)
    return block_pair ? lkb_score_impl<float, true, true>(plan, coords, waters, nullptr, nullptr, dTdV, dcoords,
                                                          dwaters, st)
                      : lkb_score_impl<float, true, false>(plan, coords, waters, nullptr, nullptr, dTdV, dcoords,
                                                           dwaters, st);
  return block_pair ? lkb_score_impl<double, true, true>(plan, coords, waters, nullptr, nullptr, dTdV, dcoords,
                                                         dwaters, st)
                    : lkb_score_impl<double, true, false>(plan, coords, waters, nullptr, nullptr, dTdV, dcoords,
                                                          dwaters, st);
}

int64_t tmol_b200_ljlk_plan_device_bytes(const tmol_b200_ljlk_plan* plan) {
  return plan ? plan->device_bytes : -1;
}

}  // extern "C"
