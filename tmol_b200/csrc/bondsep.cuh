// Bounded shortest paths over a pose's connection-point graph: the device
// side of inter-block bond separation (tmol's PoseStack builder,
// tmol/pose/pose_stack_builder.py:436-599, 1230-1343).
//
// Nodes are (block, connection) pairs.  Edges join two connections of one
// block, weighted with the bond count between their connection atoms
// (bt_conn_sep), and the two ends of an inter-block bond (weight 1).  Bond
// separations are capped at MAX_SIG_BOND_SEPARATION = 6, and every edge
// weighs at least 0, so the search from one connection point touches only
// the few nodes within 5 bonds; it runs in a thread's local memory instead
// of over the dense [n, n] connection matrix the reference fills before its
// all-pairs pass.
#pragma once

#include <cstdint>

#include "../../include/tmol_b200_pose.h"

namespace tmol_b200 {

constexpr int MAX_SIG_SEP = 6;
constexpr int BONDSEP_MAX_REACH = 64;  // nodes within the cap from one source

enum BondsepStatus : int {
  kBsIndex = 1,     // an index out of range
  kBsShape = 4,     // an inter-block bond recorded in one direction only
  kBsCapacity = 2,  // more than BONDSEP_MAX_REACH nodes within the cap
};

struct PoseConn {
  int P, B, C, nbt;
  const int32_t* bt;         // [P, B]
  const int32_t* irc;        // [P, B, C, 2]
  const int32_t* n_conn;     // [nbt]
  const int32_t* conn_sep;   // [nbt, C, C]
};

__host__ inline PoseConn pose_conn(const tmol_b200_pose_connectivity& c) {
  PoseConn g;
  g.P = c.n_poses;
  g.B = c.max_n_blocks;
  g.C = c.max_n_conn;
  g.nbt = c.n_block_types;
  g.bt = c.block_type_ind;
  g.irc = c.inter_residue_connections;
  g.n_conn = c.bt_n_conn;
  g.conn_sep = c.bt_conn_sep;
  return g;
}

// Connections of block (p, b): 0 for an absent block; -1 for a block type
// out of range.
__device__ __forceinline__ int block_n_conn(const PoseConn& g, int p, int b) {
  const int bt = g.bt[(int64_t)p * g.B + b];
  if (bt < 0) return 0;
  if (bt >= g.nbt) return -1;
  const int n = g.n_conn[bt];
  return (n < 0 || n > g.C) ? -1 : n;
}

// Dijkstra from (p, b0, c0) over the nodes within the cap: reach[k] =
// b << 3 | c, dist[k] its separation (< MAX_SIG_SEP).  Returns the number of
// nodes reached (the source first); status bits on bad input.
__device__ inline int bounded_paths(const PoseConn& g, int p, int b0, int c0, int* reach, int* dist,
                                    int& status) {
  int n = 1;
  uint64_t done = 0;
  reach[0] = (b0 << 3) | c0;
  dist[0] = 0;
  for (;;) {
    int u = -1;
    for (int k = 0; k < n; ++k)
      if (!((done >> k) & 1ull) && (u < 0 || dist[k] < dist[u])) u = k;
    if (u < 0) break;
    done |= 1ull << u;
    const int b = reach[u] >> 3, c = reach[u] & 7, d = dist[u];
    const int bt = g.bt[(int64_t)p * g.B + b];
    const int nc = g.n_conn[bt];
    // candidate edges: the block's other connections, then the bond
    for (int e = 0; e <= nc; ++e) {
      int b2, c2, nd;
      if (e < nc) {
        if (e == c) continue;
        const int w = g.conn_sep[((int64_t)bt * g.C + c) * g.C + e];
        if (w < 0) continue;  // -1: no path inside the block
        b2 = b;
        c2 = e;
        nd = d + w;
      } else {
        const int32_t* t = g.irc + (((int64_t)p * g.B + b) * g.C + c) * 2;
        b2 = t[0];
        c2 = t[1];
        if (b2 < 0) continue;
        const int nc2 = (b2 < g.B) ? block_n_conn(g, p, b2) : -1;
        if (nc2 < 0 || c2 < 0 || c2 >= nc2) {
          status |= kBsIndex;
          continue;
        }
        const int32_t* back = g.irc + (((int64_t)p * g.B + b2) * g.C + c2) * 2;
        if (back[0] != b || back[1] != c) status |= kBsShape;
        nd = d + 1;
      }
      if (nd >= MAX_SIG_SEP || nd < 0) continue;
      const int key = (b2 << 3) | c2;
      int k = 0;
      while (k < n && reach[k] != key) ++k;
      if (k < n) {
        if (!((done >> k) & 1ull) && nd < dist[k]) dist[k] = nd;
      } else if (n < BONDSEP_MAX_REACH) {
        reach[n] = key;
        dist[n] = nd;
        ++n;
      } else {
        status |= kBsCapacity;
      }
    }
  }
  return n;
}

}  // namespace tmol_b200
