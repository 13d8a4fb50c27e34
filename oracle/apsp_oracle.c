/*
 * CPU restatement of tmol's PoseStack bond-separation step, a test oracle
 * (only tests, the smoke check and the benchmark's CPU leg use it):
 *
 *   oracle_apsp_stacked   the stacked all-pairs-shortest-paths op
 *                         (tmol/pose/compiled/apsp.cpu.cpp:9-130): with a
 *                         cutoff, a Dijkstra per source over the symmetrised
 *                         edges lighter than the cutoff, every other pair at
 *                         the cutoff; without one, Floyd-Warshall over the
 *                         directed weights (-1 = no edge).
 *   oracle_pose_bondsep   inter-block bond separation of a PoseStack
 *                         (tmol/pose/pose_stack_builder.py:436-599, 1230-1343):
 *                         a graph whose nodes are the connection points of all
 *                         blocks of a pose, intra-block edges weighted with
 *                         the bond count between the connection atoms, an edge
 *                         of weight 1 per inter-block bond, every other pair at
 *                         MAX_SIG_BOND_SEPARATION (6); shortest paths with
 *                         cutoff 6; scattered to [P, B, B, C, C] (6 where a
 *                         connection slot does not exist), and the minimum
 *                         over the connection pairs, [P, B, B]
 *                         (tmol/score/bond_dependent_term.py:91-100).
 *
 * Weights other than -1 are assumed non-negative, as the reference's inputs
 * are.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MAX_SIG_BOND_SEPARATION 6

/* one graph, cutoff >= 0: the reference's symmetrised edge rule
 * (apsp.cpu.cpp:37-52) into adjacency lists, then a Dijkstra per source that
 * stops at the cutoff (:54-102), choosing the next node by a scan of the
 * nodes reached so far instead of a heap (the distances are the same). */
typedef struct {
  int32_t* deg;   /* [n] */
  int32_t* adj;   /* [n][n]: neighbour */
  int32_t* wgt;   /* [n][n]: edge weight */
  int32_t* seen;  /* [n]: nodes reached from the current source */
  int32_t* dist;  /* [n] */
  int32_t* mark;  /* [n]: 0 unseen, 1 reached, 2 done */
} apsp_scratch;

static void apsp_cutoff(int32_t* w, int n, int cutoff, apsp_scratch* sc) {
  for (int i = 0; i < n; ++i) sc->deg[i] = 0;
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      int32_t wij = w[(size_t)j * n + i], wji = w[(size_t)i * n + j];
      int32_t e = (wij == -1 || wji == -1) ? (wij > wji ? wij : wji) : (wij < wji ? wij : wji);
      if (e != -1 && e < cutoff) {
        sc->adj[(size_t)i * n + sc->deg[i]] = j;
        sc->wgt[(size_t)i * n + sc->deg[i]++] = e;
        sc->adj[(size_t)j * n + sc->deg[j]] = i;
        sc->wgt[(size_t)j * n + sc->deg[j]++] = e;
      }
    }
  for (size_t k = 0; k < (size_t)n * n; ++k) w[k] = cutoff;
  for (int i = 0; i < n; ++i) sc->mark[i] = 0;
  for (int s = 0; s < n; ++s) {
    int ns = 0;
    sc->seen[ns++] = s;
    sc->dist[s] = 0;
    sc->mark[s] = 1;
    for (;;) {
      int u = -1;
      for (int k = 0; k < ns; ++k) {
        int v = sc->seen[k];
        if (sc->mark[v] == 1 && (u < 0 || sc->dist[v] < sc->dist[u])) u = v;
      }
      if (u < 0) break;
      sc->mark[u] = 2;
      w[(size_t)s * n + u] = sc->dist[u];
      for (int k = 0; k < sc->deg[u]; ++k) {
        int v = sc->adj[(size_t)u * n + k];
        int32_t nd = sc->dist[u] + sc->wgt[(size_t)u * n + k];
        if (nd >= cutoff || sc->mark[v] == 2) continue;
        if (sc->mark[v] == 0) {
          sc->mark[v] = 1;
          sc->dist[v] = nd;
          sc->seen[ns++] = v;
        } else if (nd < sc->dist[v]) {
          sc->dist[v] = nd;
        }
      }
    }
    for (int k = 0; k < ns; ++k) sc->mark[sc->seen[k]] = 0;
  }
}

/* one graph, no cutoff: Floyd-Warshall in the reference's loop order
 * (apsp.cpu.cpp:103-127) */
static void apsp_floyd_warshall(int32_t* w, int n) {
  for (int k = 0; k < n; ++k)
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        int32_t ik = w[(size_t)i * n + k], kj = w[(size_t)k * n + j];
        if (ik >= 0 && kj >= 0) {
          int32_t cur = w[(size_t)i * n + j];
          int32_t nw = ik + kj;
          if (cur < 0 || nw < cur) w[(size_t)i * n + j] = nw;
        }
      }
}

int oracle_apsp_stacked(int32_t* weights, int n_graphs, int n_nodes, int cutoff) {
  if (n_graphs < 0 || n_nodes < 0) return 1;
  size_t nn = (size_t)n_nodes * n_nodes;
  apsp_scratch sc = {0};
  if (cutoff != -1 && n_nodes > 0) {
    sc.deg = (int32_t*)malloc((size_t)n_nodes * sizeof(int32_t));
    sc.adj = (int32_t*)malloc(nn * sizeof(int32_t));
    sc.wgt = (int32_t*)malloc(nn * sizeof(int32_t));
    sc.seen = (int32_t*)malloc((size_t)n_nodes * sizeof(int32_t));
    sc.dist = (int32_t*)malloc((size_t)n_nodes * sizeof(int32_t));
    sc.mark = (int32_t*)malloc((size_t)n_nodes * sizeof(int32_t));
  }
  int rc = 0;
  if (cutoff != -1 && n_nodes > 0 && (!sc.deg || !sc.adj || !sc.wgt || !sc.seen || !sc.dist || !sc.mark))
    rc = 2;
  for (int g = 0; g < n_graphs && rc == 0; ++g) {
    int32_t* w = weights + (size_t)g * nn;
    if (cutoff != -1)
      apsp_cutoff(w, n_nodes, cutoff, &sc);
    else
      apsp_floyd_warshall(w, n_nodes);
  }
  free(sc.deg);
  free(sc.adj);
  free(sc.wgt);
  free(sc.seen);
  free(sc.dist);
  free(sc.mark);
  return rc;
}

/* block_type_ind [P, B] (-1 = none), inter_residue_connections
 * [P, B, C, 2] ((block, connection) or -1), bt_n_conn [nbt],
 * bt_conn_sep [nbt, C, C] (bond separation between connection atoms).
 * Outputs inter_block_bondsep [P, B, B, C, C] and min_bondsep [P, B, B]
 * (either may be NULL). */
int oracle_pose_bondsep(int P, int B, int C, int nbt, const int32_t* block_type_ind,
                        const int32_t* irc, const int32_t* bt_n_conn, const int32_t* bt_conn_sep,
                        int32_t* inter_block_bondsep, int32_t* min_bondsep) {
  const int S = MAX_SIG_BOND_SEPARATION;
  int* off = (int*)malloc(sizeof(int) * ((size_t)B + 1));
  int* nconn = (int*)malloc(sizeof(int) * ((size_t)B + 1));
  if (!off || !nconn) return 2;
  if (inter_block_bondsep)
    for (size_t k = 0; k < (size_t)P * B * B * C * C; ++k) inter_block_bondsep[k] = S;
  if (min_bondsep)
    for (size_t k = 0; k < (size_t)P * B * B; ++k) min_bondsep[k] = S;
  int rc = 0;
  for (int p = 0; p < P && rc == 0; ++p) {
    /* the pose's connection points, block by block (exclusive cumsum of
     * n_conn, pose_stack_builder.py:481-486) */
    int n = 0;
    for (int b = 0; b < B; ++b) {
      int bt = block_type_ind[(size_t)p * B + b];
      nconn[b] = (bt >= 0 && bt < nbt) ? bt_n_conn[bt] : 0;
      off[b] = n;
      n += nconn[b];
    }
    if (n == 0) continue;
    int32_t* m = (int32_t*)malloc(sizeof(int32_t) * (size_t)n * n);
    if (!m) {
      rc = 2;
      break;
    }
    for (size_t k = 0; k < (size_t)n * n; ++k) m[k] = S;
    /* same-block pairs, the diagonal included (:520-597) */
    for (int b = 0; b < B; ++b) {
      int bt = block_type_ind[(size_t)p * B + b];
      for (int c1 = 0; c1 < nconn[b]; ++c1)
        for (int c2 = 0; c2 < nconn[b]; ++c2)
          m[(size_t)(off[b] + c1) * n + off[b] + c2] = bt_conn_sep[((size_t)bt * C + c1) * C + c2];
    }
    /* inter-block bonds (:1230-1254) */
    for (int b = 0; b < B; ++b)
      for (int c = 0; c < nconn[b]; ++c) {
        const int32_t* e = irc + (((size_t)p * B + b) * C + c) * 2;
        if (e[0] < 0) continue;
        if (e[0] >= B || e[1] < 0 || e[1] >= nconn[e[0]]) {
          rc = 3;
          continue;
        }
        m[(size_t)(off[b] + c) * n + off[e[0]] + e[1]] = 1;
      }
    oracle_apsp_stacked(m, 1, n, S);
    /* scatter (:1286-1343) and the minimum over connection pairs */
    for (int b1 = 0; b1 < B; ++b1)
      for (int c1 = 0; c1 < nconn[b1]; ++c1)
        for (int b2 = 0; b2 < B; ++b2)
          for (int c2 = 0; c2 < nconn[b2]; ++c2) {
            int32_t d = m[(size_t)(off[b1] + c1) * n + off[b2] + c2];
            if (inter_block_bondsep)
              inter_block_bondsep[((((size_t)p * B + b1) * B + b2) * C + c1) * C + c2] = d;
            if (min_bondsep) {
              int32_t* mb = min_bondsep + ((size_t)p * B + b1) * B + b2;
              if (d < *mb) *mb = d;
            }
          }
    free(m);
  }
  free(off);
  free(nconn);
  return rc;
}
