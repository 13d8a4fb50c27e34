// B200 LJ + LK pose scoring: plan creation, block spheres and the fused
// neighbour-detection + atom-pair kernel (forward energies and recompute
// adjoint), behind the C ABI declared in include/tmol_b200_ljlk.h.
//
// Layout in HBM (per PoseStack, built once by tmol_b200_ljlk_plan_create):
//   blk_bt[P*B], blk_off[P*B]      block type and first-atom offset per block
//   pose_last[P]                   1 + index of each pose's last real block
//   atom_params[nbt*A]             per block-type atom LJ/LK parameters + flags
//   bt_pd[nbt][A][A] (u8)          intra-block bond separation
//   bt_conn_pd[nbt][C][A] (u8)     bond separation from each connection atom
//   cp_*[P*B][CP_CAP]              per block: the later blocks within
//                                  count-pair reach (min bond separation <= 4)
//                                  with their connection-pair separations;
//                                  replaces the dense [P,B,B,C,C] tensor
//   work[n_work] (int4)            (pose, first row, end row) work items
//   spheres[P*B][4]                centroid + radius, rebuilt every call
//
// Scoring (one persistent launch per call, after the sphere kernel):
// CTAs take work items from an atomic ticket.  For item (p, [r0, r1)) the
// CTA tests every candidate pair (b1 in [r0, r1), b2 in [b1, nb)) against the
// bounding-sphere rule of tmol/score/common/sphere_overlap.impl.hh:287-351,
// queues the hits in shared memory, and its warps evaluate the queued block
// pairs, one block pair per warp: the two blocks' atoms (tiles of 32) are
// staged in the warp's shared-memory slab and the warp strides over the atom
// pairs.  Energies stay in registers for the whole item and are reduced once
// per item (whole-pose) or once per block pair (block-pair output).  The
// adjoint accumulates per-atom gradients in the slab with shared-memory
// atomics and flushes each atom once per block pair to global memory.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/tmol_b200_ljlk.h"
#include "ljlk_potentials.cuh"

namespace tmol_b200 {

constexpr int TILE = 32;
constexpr int MAX_CONN = 4;
constexpr int CP_CAP = 16;
constexpr int QUEUE_CAP = 1024;
constexpr int MAX_ROWS_PER_ITEM = 64;
constexpr int MAX_WARPS = 16;

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

template <typename Real>
__global__ void plan_block_types_kernel(PlanBuildArgs a,
                                        AtomParams<Real>* atom_params) {
  const tmol_b200_ljlk_inputs& in = a.in;
  int nbt = in.n_block_types, A = in.max_n_block_atoms, C = in.max_n_conn;
  const Real* tp = (const Real*)in.type_params;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nbt * A;
       i += gridDim.x * blockDim.x) {
    int bt = i / A, at = i - bt * A;
    int n = in.bt_n_atoms[bt];
    if (n < 0 || n > A) {
      if (at == 0) atomicOr(a.status, kStIndex);
      continue;
    }
    AtomParams<Real> prm = {};
    if (at < n) {
      int t = in.bt_atom_types[i];
      if (t < 0 || t >= in.n_atom_types) {
        atomicOr(a.status, kStIndex);
      } else {
        const Real* r = tp + 10 * (int64_t)t;
        prm.lj_radius = r[0];
        prm.lj_wdepth = r[1];
        prm.lk_dgfree = r[2];
        prm.lk_lambda = r[3];
        prm.lk_volume = r[4];
        int f = 0;
        if (r[5] != 0) f |= kDonor;
        if (r[6] != 0) f |= kHydroxyl;
        if (r[7] != 0) f |= kPolarH;
        if (r[8] != 0) f |= kAcceptor;
        if (r[9] != 0) f |= kCarbonLK;
        prm.flags = f | a.bt_flags[i];
      }
      for (int at2 = 0; at2 < A; ++at2) {
        int v = in.bt_path_distance[(int64_t)i * A + at2];
        a.bt_pd[(int64_t)i * A + at2] = (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
      }
    }
    atom_params[i] = prm;
    int nc = in.bt_n_conn[bt];
    if (at == 0 && (nc < 0 || nc > C)) atomicOr(a.status, kStIndex);
    for (int c = 0; c < C; ++c) {
      uint8_t v = 6;
      if (c < nc && at < n) {
        int ca = in.bt_conn_atom[bt * C + c];
        if (ca < 0 || ca >= n) {
          atomicOr(a.status, kStIndex);
        } else {
          int d = in.bt_path_distance[((int64_t)bt * A + ca) * A + at];
          v = (uint8_t)(d < 0 ? 0 : (d > 255 ? 255 : d));
        }
      }
      a.bt_conn_pd[((int64_t)bt * C + c) * A + at] = v;
    }
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

// ---------------------------------------------------------------------------
// per-call kernels

template <typename Real>
struct ScoreArgs {
  const Real* coords;
  const int* blk_bt;
  const int* blk_off;
  const int* pose_last;
  const AtomParams<Real>* atom_params;
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
  int n_work;
  int P, B, A, C;
  Real* energies;
  int32_t* nbr;
  const Real* dTdV;
  Real* dcoords;
  int* ticket;
  unsigned long long* counts;
};

// Bounding sphere per block: centroid (sum of atoms in order, then divided
// by the atom count) and largest centroid distance, as
// sphere_overlap.impl.hh:109-196 computes them on the CPU.
template <typename Real>
__global__ void spheres_kernel(ScoreArgs<Real> s) {
  int n_blocks = s.P * s.B;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_blocks;
       i += gridDim.x * blockDim.x) {
    int bt = s.blk_bt[i];
    Real* out = s.spheres + 4 * (int64_t)i;
    if (bt < 0) {
      out[0] = out[1] = out[2] = out[3] = Real(0);
      continue;
    }
    int n = s.bt_n_atoms[bt];
    const Real* x = s.coords + 3 * (int64_t)s.blk_off[i];
    Real cx = 0, cy = 0, cz = 0;
    for (int k = 0; k < n; ++k) {
      cx = add_rn(cx, x[3 * k + 0]);
      cy = add_rn(cy, x[3 * k + 1]);
      cz = add_rn(cz, x[3 * k + 2]);
    }
    Real rn = Real(n);
    cx = div_rn(cx, rn);
    cy = div_rn(cy, rn);
    cz = div_rn(cz, rn);
    Real d2max = 0;
    for (int k = 0; k < n; ++k) {
      Real dx = sub_rn(x[3 * k + 0], cx);
      Real dy = sub_rn(x[3 * k + 1], cy);
      Real dz = sub_rn(x[3 * k + 2], cz);
      Real d2 = add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
      if (d2 > d2max) d2max = d2;
    }
    out[0] = cx;
    out[1] = cy;
    out[2] = cz;
    out[3] = sqrt_rn(d2max);
  }
}

template <typename Real>
struct WarpSlab {
  Real x[2][TILE], y[2][TILE], z[2][TILE];
  AtomParams<Real> prm[2][TILE];
  Real gx[2][TILE], gy[2][TILE], gz[2][TILE];
  uint8_t cpd[2][MAX_CONN][TILE];
  uint8_t seps[16];
};

template <typename Real>
__device__ __forceinline__ void stage_tile(const ScoreArgs<Real>& s,
                                           WarpSlab<Real>& w, int side, int bt,
                                           int off, int start, int cnt,
                                           int nconn, bool striking, int lane,
                                           bool grad) {
  if (lane < cnt) {
    int at = start + lane;
    const Real* c = s.coords + 3 * ((int64_t)off + at);
    w.x[side][lane] = c[0];
    w.y[side][lane] = c[1];
    w.z[side][lane] = c[2];
    w.prm[side][lane] = s.atom_params[(int64_t)bt * s.A + at];
    if (striking) {
      for (int k = 0; k < nconn; ++k)
        w.cpd[side][k][lane] = s.bt_conn_pd[((int64_t)bt * s.C + k) * s.A + at];
    }
    if (grad) {
      w.gx[side][lane] = 0;
      w.gy[side][lane] = 0;
      w.gz[side][lane] = 0;
    }
  }
}

template <typename Real>
__device__ __forceinline__ void flush_tile(const ScoreArgs<Real>& s,
                                           WarpSlab<Real>& w, int side,
                                           int off, int start, int cnt,
                                           int lane) {
  if (lane < cnt) {
    Real* d = s.dcoords + 3 * ((int64_t)off + start + lane);
    Real gx = w.gx[side][lane], gy = w.gy[side][lane], gz = w.gz[side][lane];
    if (gx != 0) atomicAdd(d + 0, gx);
    if (gy != 0) atomicAdd(d + 1, gy);
    if (gz != 0) atomicAdd(d + 2, gz);
  }
}

// Per-warp work counters (units of the throughput and roofline figures):
//   [0] block pairs, [1] atom pairs (inter n1*n2, intra n(n-1)/2),
//   [2] heavy-atom pairs (same rule), [3] atom pairs inside max_dis with a
//   non-zero count-pair weight, [4] heavy-atom pairs among those.
constexpr int N_COUNTS = 5;

struct WarpCounts {
  long long c[N_COUNTS];
};

// All atom pairs of one block pair.  GRAD: accumulate sum_t wt[t] * dE_t/dx
// into the slab (and the energies into acc); else add the energies to acc.
template <typename Real, bool GRAD>
__device__ void eval_block_pair(const ScoreArgs<Real>& s, WarpSlab<Real>& w,
                                int p, int b1, int b2, int lane, Real acc[3],
                                const Real wt[3], WarpCounts& cnt) {
  int i1 = p * s.B + b1, i2 = p * s.B + b2;
  int bt1 = s.blk_bt[i1], bt2 = s.blk_bt[i2];
  int off1 = s.blk_off[i1], off2 = s.blk_off[i2];
  int n1 = s.bt_n_atoms[bt1], n2 = s.bt_n_atoms[bt2];
  bool intra = b1 == b2;
  bool lig = s.bt_is_ligand[bt1] && s.bt_is_ligand[bt2];
  int minsep = 6;
  bool striking = false;
  int nc1 = 0, nc2 = 0;
  if (!intra) {
    int ncp = s.cp_count[i1];
    for (int k = 0; k < ncp; ++k) {
      int e = i1 * CP_CAP + k;
      if (s.cp_b2[e] == b2) {
        minsep = s.cp_minsep[e];
        striking = true;
        if (lane < 16) w.seps[lane] = s.cp_seps[(int64_t)e * 16 + lane];
        break;
      }
    }
    if (striking) {
      nc1 = s.bt_n_conn[bt1];
      nc2 = s.bt_n_conn[bt2];
    }
  }
  cnt.c[0] += 1;
  cnt.c[1] += intra ? (long long)n1 * (n1 - 1) / 2 : (long long)n1 * n2;
  const Real maxd2 = s.g.max_dis * s.g.max_dis;
  long long h_all = 0;
  int n_in = 0, n_in_heavy = 0;
  int nt1 = (n1 + TILE - 1) / TILE, nt2 = (n2 + TILE - 1) / TILE;
  for (int ti = 0; ti < nt1; ++ti) {
    int st1 = ti * TILE;
    int c1 = min(TILE, n1 - st1);
    stage_tile(s, w, 0, bt1, off1, st1, c1, nc1, striking, lane, GRAD);
    __syncwarp();
    int h1 = __popc(__ballot_sync(0xffffffffu, lane < c1 && (w.prm[0][lane].flags & kHeavy)));
    for (int tj = intra ? ti : 0; tj < nt2; ++tj) {
      int st2 = tj * TILE;
      int c2 = min(TILE, n2 - st2);
      bool same = intra && ti == tj;
      int side2 = same ? 0 : 1;
      if (!same) stage_tile(s, w, 1, bt2, off2, st2, c2, nc2, striking, lane, GRAD);
      __syncwarp();
      int h2 = same ? h1
                    : __popc(__ballot_sync(0xffffffffu,
                                           lane < c2 && (w.prm[1][lane].flags & kHeavy)));
      h_all += same ? (long long)h1 * (h1 - 1) / 2 : (long long)h1 * h2;
      int npairs = c1 * c2;
      for (int k = lane; k < npairs; k += 32) {
        int a1 = k / c2;
        int a2 = k - a1 * c2;
        if (same && a1 >= a2) continue;
        Real dx = w.x[0][a1] - w.x[side2][a2];
        Real dy = w.y[0][a1] - w.y[side2][a2];
        Real dz = w.z[0][a1] - w.z[side2][a2];
        Real d2 = dx * dx + dy * dy + dz * dz;
        if (!(d2 < maxd2)) continue;
        int sep;
        if (intra) {
          sep = s.bt_pd[((int64_t)bt1 * s.A + st1 + a1) * s.A + st2 + a2];
        } else if (striking) {
          sep = 5;
          for (int u = 0; u < nc1; ++u) {
            int pd1 = w.cpd[0][u][a1];
            for (int v = 0; v < nc2; ++v) {
              int t = pd1 + w.seps[u * 4 + v] + w.cpd[1][v][a2];
              sep = t < sep ? t : sep;
            }
          }
        } else {
          sep = minsep;
        }
        if (lig && (sep == 3 || sep == 4)) sep = 5;
        Real wcp = connectivity_weight<Real>(sep);
        if (wcp == Real(0)) continue;
        Real d = sqrt(d2);
        const AtomParams<Real>& pa = w.prm[0][a1];
        const AtomParams<Real>& pb = w.prm[side2][a2];
        LJPair<Real> q = lj_pair(pa, pb, s.g);
        bool heavy = (pa.flags & kHeavy) && (pb.flags & kHeavy);
        ++n_in;
        n_in_heavy += heavy;
        if (!GRAD) {
          Real atr, rep;
          lj_V(d, q, atr, rep);
          acc[0] += wcp * atr;
          acc[1] += wcp * rep;
          if (heavy) acc[2] += wcp * lk_V(d, q.sigma, pa, pb, s.g.max_dis);
        } else {
          Real atr, rep, datr, drep;
          lj_V_dV(d, q, atr, rep, datr, drep);
          acc[0] += wcp * atr;
          acc[1] += wcp * rep;
          Real dE = wt[0] * datr + wt[1] * drep;
          if (heavy) {
            Real lk, dlk;
            lk_V_dV(d, q.sigma, pa, pb, s.g.max_dis, lk, dlk);
            acc[2] += wcp * lk;
            dE += wt[2] * dlk;
          }
          dE *= wcp;
          if (dE != Real(0) && d != Real(0)) {
            Real f = dE / d;
            Real fx = f * dx, fy = f * dy, fz = f * dz;
            atomicAdd(&w.gx[0][a1], fx);
            atomicAdd(&w.gy[0][a1], fy);
            atomicAdd(&w.gz[0][a1], fz);
            atomicAdd(&w.gx[side2][a2], -fx);
            atomicAdd(&w.gy[side2][a2], -fy);
            atomicAdd(&w.gz[side2][a2], -fz);
          }
        }
      }
      __syncwarp();
      if (GRAD && !same) flush_tile(s, w, 1, off2, st2, c2, lane);
      __syncwarp();
    }
    if (GRAD) flush_tile(s, w, 0, off1, st1, c1, lane);
    __syncwarp();
  }
  cnt.c[2] += h_all;
  cnt.c[3] += n_in;
  cnt.c[4] += n_in_heavy;
}

template <typename Real>
__device__ __forceinline__ Real warp_sum(Real v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// The fused per-item kernel.  GRAD selects the adjoint (which also yields
// the energies when s.energies is set); BLOCK_PAIR selects per-block-pair
// energies / weights instead of per-pose ones.
template <typename Real, bool GRAD, bool BLOCK_PAIR>
__global__ void __launch_bounds__(32 * MAX_WARPS)
    score_kernel(ScoreArgs<Real> s, int rows_per_item) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n_warps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSlab<Real>* slabs = reinterpret_cast<WarpSlab<Real>*>(smem_raw);
  WarpSlab<Real>& w = slabs[warp];
  int* queue = reinterpret_cast<int*>(slabs + n_warps);
  __shared__ int s_item, s_qcount;
  __shared__ int s_rowoff[MAX_ROWS_PER_ITEM + 1];
  __shared__ Real s_red[3][MAX_WARPS];
  __shared__ unsigned long long s_cnt[N_COUNTS];
  if (threadIdx.x < N_COUNTS) s_cnt[threadIdx.x] = 0;
  WarpCounts cnt = {};
  const bool want_E = !GRAD || s.energies != nullptr;

  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(s.ticket, 1);
    __syncthreads();
    int item = s_item;
    if (item >= s.n_work) break;
    int4 wi = s.work[item];
    int p = wi.x, r0 = wi.y, r1 = wi.z;
    int nb = s.pose_last[p];
    int nrows = r1 - r0;
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int r = 0; r < nrows; ++r) {
        s_rowoff[r] = acc;
        acc += nb - (r0 + r);
      }
      s_rowoff[nrows] = acc;
    }
    Real acc[3] = {0, 0, 0};
    Real wt[3] = {0, 0, 0};
    if (GRAD && !BLOCK_PAIR) {
      for (int t = 0; t < 3; ++t) wt[t] = s.dTdV[t * s.P + p];
    }
    __syncthreads();
    int n_cand = s_rowoff[nrows];
    for (int base = 0; base < n_cand; base += QUEUE_CAP) {
      if (threadIdx.x == 0) s_qcount = 0;
      __syncthreads();
      int end = min(base + QUEUE_CAP, n_cand);
      for (int c = base + threadIdx.x; c < end; c += blockDim.x) {
        int r = 0;
        while (r + 1 < nrows && s_rowoff[r + 1] <= c) ++r;
        int b1 = r0 + r;
        int b2 = b1 + (c - s_rowoff[r]);
        int i1 = p * s.B + b1, i2 = p * s.B + b2;
        bool hit = false;
        if (s.blk_bt[i1] >= 0 && s.blk_bt[i2] >= 0) {
          const Real* s1 = s.spheres + 4 * (int64_t)i1;
          const Real* s2 = s.spheres + 4 * (int64_t)i2;
          Real dx = sub_rn(s1[0], s2[0]);
          Real dy = sub_rn(s1[1], s2[1]);
          Real dz = sub_rn(s1[2], s2[2]);
          Real d2 = add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
          Real thr = add_rn(add_rn(s1[3], s2[3]), s.reach);
          hit = d2 < mul_rn(thr, thr);
        }
        if (s.nbr) s.nbr[(int64_t)i1 * s.B + b2] = hit ? 1 : 0;
        if (hit) {
          int slot = atomicAdd(&s_qcount, 1);
          queue[slot] = b1 | (b2 << 16);
        }
      }
      __syncthreads();
      int nq = s_qcount;
      for (int e = warp; e < nq; e += n_warps) {
        int pk = queue[e];
        int b1 = pk & 0xffff, b2 = pk >> 16;
        if (BLOCK_PAIR) {
          int64_t o = ((int64_t)p * s.B + b1) * s.B + b2;
          int64_t stride = (int64_t)s.P * s.B * s.B;
          if (GRAD) {
            for (int t = 0; t < 3; ++t) wt[t] = s.dTdV[t * stride + o];
          }
          Real pacc[3] = {0, 0, 0};
          eval_block_pair<Real, GRAD>(s, w, p, b1, b2, lane, pacc, wt, cnt);
          if (want_E) {
            for (int t = 0; t < 3; ++t) {
              Real v = warp_sum(pacc[t]);
              if (lane == 0) s.energies[t * stride + o] = v;
            }
          }
        } else {
          eval_block_pair<Real, GRAD>(s, w, p, b1, b2, lane, acc, wt, cnt);
        }
      }
      __syncthreads();
    }
    if (!BLOCK_PAIR && want_E) {
      for (int t = 0; t < 3; ++t) {
        Real v = warp_sum(acc[t]);
        if (lane == 0) s_red[t][warp] = v;
      }
      __syncthreads();
      if (threadIdx.x < 3) {
        Real v = 0;
        for (int k = 0; k < n_warps; ++k) v += s_red[threadIdx.x][k];
        if (v != Real(0)) atomicAdd(&s.energies[threadIdx.x * s.P + p], v);
      }
    }
  }
  if (s.counts) {
    // counters 0..2 are warp-uniform (lane 0 reports); 3..4 are per lane
    for (int k = 0; k < N_COUNTS; ++k) {
      long long v = cnt.c[k];
      if (k >= 3) {
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      }
      if (lane == 0 && v) atomicAdd(&s_cnt[k], (unsigned long long)v);
    }
    __syncthreads();
    if (threadIdx.x < N_COUNTS && s_cnt[threadIdx.x])
      atomicAdd(&s.counts[threadIdx.x], s_cnt[threadIdx.x]);
  }
}

}  // namespace tmol_b200

// ---------------------------------------------------------------------------
// host side

using namespace tmol_b200;

struct tmol_b200_ljlk_plan {
  int real_bytes;
  tmol_b200_ljlk_inputs dims;  // sizes only; pointers are not kept
  int P, B, nbt, A, C, ntiles, T;
  int64_t N;
  double reach;
  int* blk_bt = nullptr;
  int* blk_off = nullptr;
  int* pose_last = nullptr;
  void* atom_params = nullptr;
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
  int n_work = 0;
  void* spheres = nullptr;
  int* counters = nullptr;  // [0] ticket, [1] status
  unsigned long long* counts = nullptr;  // [N_COUNTS] of the last forward
  unsigned char global_params[5 * sizeof(double)];
  // kernel timing: event pairs around each scoring-kernel launch
  bool profiling = false;
  std::vector<cudaEvent_t> prof_events;
  int prof_n = 0;
  tmol_b200_ljlk_launch launch;
  int n_sm = 148;
  int64_t device_bytes = 0;
  std::vector<int> host_pose_last;
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
  void* ptrs[] = {pl->blk_bt,    pl->blk_off,    pl->pose_last,  pl->atom_params,
                  pl->bt_pd,     pl->bt_conn_pd, pl->bt_flags,   pl->bt_n_atoms,
                  pl->bt_n_conn, pl->bt_is_ligand, pl->cp_count, pl->cp_b2,
                  pl->cp_minsep, pl->cp_seps,    pl->work,       pl->spheres,
                  pl->counters,  pl->counts};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (cudaEvent_t e : pl->prof_events) cudaEventDestroy(e);
  delete pl;
}

void default_launch(tmol_b200_ljlk_launch& l) {
  if (l.rows_per_item <= 0) l.rows_per_item = 4;
  if (l.warps_per_cta <= 0) l.warps_per_cta = 8;
  if (l.ctas_per_sm <= 0) l.ctas_per_sm = 4;
  l.rows_per_item = std::min(l.rows_per_item, MAX_ROWS_PER_ITEM);
  l.warps_per_cta = std::min(l.warps_per_cta, MAX_WARPS);
}

template <typename Real>
cudaError_t set_smem_limits() {
  int smem = (int)(MAX_WARPS * sizeof(WarpSlab<Real>) + QUEUE_CAP * sizeof(int));
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(score_kernel<Real, false, false>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(score_kernel<Real, false, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(score_kernel<Real, true, false>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess)
    return e;
  return cudaFuncSetAttribute(score_kernel<Real, true, true>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

int build_work(tmol_b200_ljlk_plan* pl, cudaStream_t st) {
  std::vector<int4> work;
  int R = pl->launch.rows_per_item;
  for (int p = 0; p < pl->P; ++p) {
    int nb = pl->host_pose_last[p];
    for (int r = 0; r < nb; r += R) work.push_back(make_int4(p, r, std::min(nb, r + R), 0));
  }
  if (pl->work) cudaFree(pl->work);
  pl->work = nullptr;
  pl->n_work = (int)work.size();
  CK(cudaMalloc((void**)&pl->work, std::max<size_t>(work.size(), 1) * sizeof(int4)));
  if (!work.empty())
    CK(cudaMemcpyAsync(pl->work, work.data(), work.size() * sizeof(int4),
                       cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
  return TMOL_B200_OK;
}

template <typename Real>
ScoreArgs<Real> score_args(tmol_b200_ljlk_plan* pl, const void* coords) {
  ScoreArgs<Real> s = {};
  s.coords = (const Real*)coords;
  s.blk_bt = pl->blk_bt;
  s.blk_off = pl->blk_off;
  s.pose_last = pl->pose_last;
  s.atom_params = (const AtomParams<Real>*)pl->atom_params;
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
  s.g.max_dis = gp[0];
  s.g.lj_dlin_sigma_factor = gp[1];
  s.g.lj_hbond_dis = gp[2];
  s.g.lj_hbond_OH_donor_dis = gp[3];
  s.g.lj_hbond_hdis = gp[4];
  s.reach = (Real)pl->reach;
  s.work = pl->work;
  s.n_work = pl->n_work;
  s.P = pl->P;
  s.B = pl->B;
  s.A = pl->A;
  s.C = pl->C;
  s.ticket = pl->counters;
  s.counts = pl->counts;
  return s;
}

template <typename Real, bool GRAD, bool BLOCK_PAIR>
int launch_score(tmol_b200_ljlk_plan* pl, ScoreArgs<Real> s, cudaStream_t st) {
  int n_blocks = pl->P * pl->B;
  int threads = 256;
  int grid_s = std::max(1, std::min((n_blocks + threads - 1) / threads, pl->n_sm * 8));
  spheres_kernel<Real><<<grid_s, threads, 0, st>>>(s);
  CK(cudaGetLastError());
  CK(cudaMemsetAsync(pl->counters, 0, sizeof(int), st));
  if (pl->n_work == 0) return TMOL_B200_OK;
  int warps = pl->launch.warps_per_cta;
  size_t smem = warps * sizeof(WarpSlab<Real>) + QUEUE_CAP * sizeof(int);
  auto kern = score_kernel<Real, GRAD, BLOCK_PAIR>;
  int grid = std::max(1, std::min(pl->n_work, pl->n_sm * pl->launch.ctas_per_sm));
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
  size_t n_e = block_pair ? (size_t)3 * pl->P * pl->B * pl->B : (size_t)3 * pl->P;
  CK(cudaMemsetAsync(energies, 0, n_e * sizeof(Real), st));
  if (nbr) CK(cudaMemsetAsync(nbr, 0, (size_t)pl->P * pl->B * pl->B * sizeof(int32_t), st));
  CK(cudaMemsetAsync(pl->counts, 0, N_COUNTS * sizeof(unsigned long long), st));
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
  CK(cudaMemsetAsync(dcoords, 0, (size_t)pl->N * 3 * sizeof(Real), st));
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
  CK(cudaMemsetAsync(dcoords, 0, (size_t)pl->N * 3 * sizeof(Real), st));
  CK(cudaMemsetAsync(energies, 0, (size_t)3 * pl->P * sizeof(Real), st));
  CK(cudaMemsetAsync(pl->counts, 0, N_COUNTS * sizeof(unsigned long long), st));
  return launch_score<Real, true, false>(pl, s, st);
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

int tmol_b200_ljlk_plan_create(const tmol_b200_ljlk_inputs* in, int real_bytes,
                               const tmol_b200_ljlk_launch* launch,
                               void* stream, tmol_b200_ljlk_plan** plan_out) {
  if (!in || !plan_out) return TMOL_B200_ERR_INVALID_ARGUMENT;
  *plan_out = nullptr;
  if (real_bytes != 4 && real_bytes != 8) return TMOL_B200_ERR_DTYPE;
  const int P = in->n_poses, B = in->max_n_blocks, nbt = in->n_block_types;
  const int A = in->max_n_block_atoms, C = in->max_n_conn, nt = in->max_n_tiles;
  const int T = in->n_atom_types;
  if (P < 0 || B < 0 || nbt < 0 || A < 0 || C < 0 || T < 0 || in->n_atoms < 0)
    return TMOL_B200_ERR_SHAPE;
  if (C > MAX_CONN || B >= 65536 || in->n_rots != P * B) return TMOL_B200_ERR_SHAPE;
  if (nt * TILE < A) return TMOL_B200_ERR_SHAPE;
  if (in->n_atoms >= ((int64_t)1 << 31)) return TMOL_B200_ERR_SHAPE;
  const void* req[] = {in->rot_coord_offset, in->first_rot_block_type, in->block_ind_for_rot,
                       in->pose_ind_for_rot, in->block_type_ind_for_rot, in->rot_offset_for_block,
                       in->min_bondsep, in->inter_block_bondsep, in->bt_n_atoms,
                       in->bt_n_heavy_atoms_in_tile, in->bt_heavy_atoms_in_tile, in->bt_atom_types,
                       in->bt_n_conn, in->bt_conn_atom, in->bt_path_distance,
                       in->bt_is_ligand_fragment, in->type_params, in->global_params};
  if (P * B > 0 && nbt > 0)
    for (const void* r : req)
      if (!r) return TMOL_B200_ERR_INVALID_ARGUMENT;

  cudaStream_t st = (cudaStream_t)stream;
  auto* pl = new tmol_b200_ljlk_plan();
  pl->real_bytes = real_bytes;
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
  pl->launch = launch ? *launch : tmol_b200_ljlk_launch{0, 0, 0};
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
  PCK(real_bytes == 4 ? set_smem_limits<float>() : set_smem_limits<double>());
  const int64_t PB = (int64_t)P * B;
  PCK(dalloc(pl, &pl->blk_bt, PB));
  PCK(dalloc(pl, &pl->blk_off, PB));
  PCK(dalloc(pl, &pl->pose_last, P));
  PCK(dalloc(pl, (unsigned char**)&pl->atom_params,
             (size_t)nbt * A * (real_bytes == 4 ? sizeof(AtomParams<float>) : sizeof(AtomParams<double>))));
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
  PCK(dalloc(pl, &pl->counters, 4));
  PCK(dalloc(pl, &pl->counts, N_COUNTS));

  PCK(cudaMemsetAsync(pl->pose_last, 0, sizeof(int) * std::max(P, 1), st));
  PCK(cudaMemsetAsync(pl->counters, 0, sizeof(int) * 4, st));
  PCK(cudaMemsetAsync(pl->bt_flags, 0, sizeof(int) * std::max<int64_t>((int64_t)nbt * A, 1), st));
  PCK(cudaMemcpyAsync(pl->bt_n_atoms, in->bt_n_atoms, sizeof(int) * nbt, cudaMemcpyDeviceToDevice, st));
  PCK(cudaMemcpyAsync(pl->bt_n_conn, in->bt_n_conn, sizeof(int) * nbt, cudaMemcpyDeviceToDevice, st));
  PCK(cudaMemcpyAsync(pl->bt_is_ligand, in->bt_is_ligand_fragment, sizeof(int) * nbt,
                      cudaMemcpyDeviceToDevice, st));
  PCK(cudaMemcpyAsync(pl->global_params, in->global_params, 5 * real_bytes,
                      cudaMemcpyDeviceToHost, st));

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
  int g = std::max(1, std::min<int>((int)((PB + 255) / 256), pl->n_sm * 8));
  if (PB > 0) {
    plan_blocks_kernel<<<g, 256, 0, st>>>(a);
    PCK(cudaGetLastError());
  }
  if (nbt > 0) {
    int gh = std::max(1, std::min(((nbt * nt * TILE) + 255) / 256, pl->n_sm * 8));
    plan_heavy_kernel<<<gh, 256, 0, st>>>(a);
    PCK(cudaGetLastError());
    int gb = std::max(1, std::min(((nbt * A) + 255) / 256, pl->n_sm * 8));
    if (real_bytes == 4)
      plan_block_types_kernel<float><<<gb, 256, 0, st>>>(a, (AtomParams<float>*)pl->atom_params);
    else
      plan_block_types_kernel<double><<<gb, 256, 0, st>>>(a, (AtomParams<double>*)pl->atom_params);
    PCK(cudaGetLastError());
  }
  if (PB > 0) {
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
  PCK(cudaStreamSynchronize(st));
  rc = status_from_bits(status_bits);
  if (rc != TMOL_B200_OK) {
    free_plan(pl);
    return rc;
  }
  rc = build_work(pl, st);
  if (rc != TMOL_B200_OK) {
    free_plan(pl);
    return rc;
  }
  pl->device_bytes += (int64_t)std::max(pl->n_work, 1) * sizeof(int4);
#undef PCK
  *plan_out = pl;
  return TMOL_B200_OK;
}

int tmol_b200_ljlk_plan_destroy(tmol_b200_ljlk_plan* plan) {
  if (!plan) return TMOL_B200_ERR_INVALID_ARGUMENT;
  free_plan(plan);
  return TMOL_B200_OK;
}

int tmol_b200_ljlk_plan_set_launch(tmol_b200_ljlk_plan* plan,
                                   const tmol_b200_ljlk_launch* launch) {
  if (!plan || !launch) return TMOL_B200_ERR_INVALID_ARGUMENT;
  int old_rows = plan->launch.rows_per_item;
  plan->launch = *launch;
  default_launch(plan->launch);
  if (plan->launch.rows_per_item != old_rows) {
    cudaStream_t st = 0;
    return build_work(plan, st);
  }
  return TMOL_B200_OK;
}

int tmol_b200_ljlk_forward(tmol_b200_ljlk_plan* plan, const void* coords,
                           int block_pair, void* energies,
                           int32_t* block_neighbors, void* stream) {
  if (!plan || !energies || (!coords && plan->N > 0)) return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4)
    return forward_impl<float>(plan, coords, block_pair, energies, block_neighbors, st);
  return forward_impl<double>(plan, coords, block_pair, energies, block_neighbors, st);
}

int tmol_b200_ljlk_backward(tmol_b200_ljlk_plan* plan, const void* coords,
                            int block_pair, const void* dTdV, void* dcoords,
                            void* stream) {
  if (!plan || !dTdV || !dcoords || (!coords && plan->N > 0))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4)
    return backward_impl<float>(plan, coords, block_pair, dTdV, dcoords, st);
  return backward_impl<double>(plan, coords, block_pair, dTdV, dcoords, st);
}

int tmol_b200_ljlk_energy_and_gradient(tmol_b200_ljlk_plan* plan,
                                       const void* coords, const void* weights,
                                       void* energies, void* dcoords,
                                       void* stream) {
  if (!plan || !weights || !energies || !dcoords || (!coords && plan->N > 0))
    return TMOL_B200_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->real_bytes == 4)
    return energy_and_gradient_impl<float>(plan, coords, weights, energies, dcoords, st);
  return energy_and_gradient_impl<double>(plan, coords, weights, energies, dcoords, st);
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

int64_t tmol_b200_ljlk_plan_device_bytes(const tmol_b200_ljlk_plan* plan) {
  return plan ? plan->device_bytes : -1;
}

}  // extern "C"
