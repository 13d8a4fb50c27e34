"""The bond-separation oracle (oracle/apsp_oracle.c) against the reference:

- its stacked all-pairs-shortest-paths restatement against the reference's
  compiled apsp op (tmol/pose/compiled/apsp.cpu.cpp) on seeded random graphs
  (directed, disconnected, zero-weight edges; with and without a cutoff), and
  against the known answers of the reference's own APSP tests
  (tmol/tests/pose/compiled/test_all_pairs_shortest_paths.py: path graphs,
  a shortcut edge);
- its PoseStack bond separation against the builder's tensors and against
  the reference route (connection-point matrix as
  tmol/pose/pose_stack_builder.py:459-599, 1230-1254 builds it, the
  reference apsp op with cutoff 6, the scatter of :1271-1343), on 1ubq,
  seeded synthetic batches, a two-chain pose and the exotic blocks (three
  connections, a ring through the side connections).
"""

import numpy
import pytest

from oracle import oracle as O
from tmol_b200.pose.builder import PoseTopology, build_pose_stack, topology_from_sequence
from tmol_b200.pose.synthetic import synthetic_pose_stack

MAX_SEP = 6


def random_graphs(rng, G, N, density, wmax=9):
    w = numpy.full((G, N, N), -1, dtype=numpy.int32)
    m = rng.random((G, N, N)) < density
    w[m] = rng.integers(0, wmax, size=int(m.sum()))
    for g in range(G):
        numpy.fill_diagonal(w[g], 0)
    return w


def path_graph(G, N, fill=-1):
    w = numpy.full((G, N, N), fill, dtype=numpy.int32)
    a = numpy.arange(N)
    w[:, a, a] = 0
    w[:, a[1:], a[:-1]] = 1
    w[:, a[:-1], a[1:]] = 1
    return w


def test_apsp_known_answers():
    for N in (32, 64, 1000):
        G = 5 if N == 1000 else 1
        w = O.apsp_stacked(path_graph(G, N))
        gold = numpy.abs(numpy.arange(N)[None, :] - numpy.arange(N)[:, None])
        assert all(numpy.array_equal(w[g], gold) for g in range(G))
    w = O.apsp_stacked(path_graph(1, 32, fill=6), 6)
    gold = numpy.minimum(numpy.abs(numpy.arange(32)[None, :] - numpy.arange(32)[:, None]), 6)
    assert numpy.array_equal(w[0], gold)
    # a shortcut 10 <-> 20 in a 128-node path: symmetric, with and without cutoff
    for cutoff in (-1, 6):
        g = path_graph(5, 128)
        g[:, 10, 20] = g[:, 20, 10] = 1
        w = O.apsp_stacked(g, cutoff)
        assert numpy.array_equal(w[0], w[0].T)
        assert w[0, 10, 20] == 1 and w[0, 5, 25] == min(11, 6 if cutoff == 6 else 99)


@pytest.mark.skipif(not O.reference_apsp_available(), reason="compiled reference apsp op not built")
def test_apsp_matches_reference_op():
    rng = numpy.random.default_rng(11)
    for trial in range(40):
        G, N = int(rng.integers(1, 4)), int(rng.integers(1, 90))
        w = random_graphs(rng, G, N, rng.uniform(0.01, 0.3))
        if trial % 4 == 0:
            w[:, N // 2:, : N // 2] = -1  # one-way reachability
            w[:, : N // 2, N // 2:] = -1
        for cutoff in (-1, 6, 3, 1):
            assert numpy.array_equal(O.apsp_stacked(w, cutoff), O.reference_apsp(w, cutoff)), (trial, cutoff)


def pconn_route(ps, apsp):
    """The reference builder's route to inter_block_bondsep: the connection
    point matrix, shortest paths with cutoff 6, the scatter."""
    pbt = ps.packed_block_types
    bti = ps.block_type_ind.numpy()
    irc = ps.inter_residue_connections.numpy()
    nconn_bt = pbt.n_conn.numpy()
    sep = pbt.conn_at_intrablock_bond_sep.numpy()
    P, B = bti.shape
    C = pbt.max_n_conn
    nconn = numpy.where(bti >= 0, nconn_bt[numpy.maximum(bti, 0)], 0)
    off = numpy.concatenate([numpy.zeros((P, 1), numpy.int64), numpy.cumsum(nconn, 1)[:, :-1]], 1)
    n_tot = nconn.sum(1)
    M = max(int(n_tot.max()), 1)
    m = numpy.full((P, M, M), MAX_SEP, dtype=numpy.int32)
    for p in range(P):
        for b in range(B):
            k = nconn[p, b]
            o = off[p, b]
            m[p, o:o + k, o:o + k] = sep[bti[p, b], :k, :k]
        for b in range(B):
            for c in range(nconn[p, b]):
                b2, c2 = irc[p, b, c]
                if b2 >= 0:
                    m[p, off[p, b] + c, off[p, b2] + c2] = 1
    m = apsp(m, MAX_SEP)
    ibb = numpy.full((P, B, B, C, C), MAX_SEP, dtype=numpy.int32)
    for p in range(P):
        for b1 in range(B):
            for b2 in range(B):
                k1, k2 = nconn[p, b1], nconn[p, b2]
                if k1 and k2:
                    ibb[p, b1, b2, :k1, :k2] = m[p, off[p, b1]:off[p, b1] + k1, off[p, b2]:off[p, b2] + k2]
    return ibb


def oracle_bondsep(ps):
    pbt = ps.packed_block_types
    return O.pose_bondsep(ps.block_type_ind, ps.inter_residue_connections, pbt.n_conn, pbt.conn_at_intrablock_bond_sep)


def pose_cases(ubq_pose_stack):
    import os
    import sys

    sys.path.insert(0, os.path.dirname(__file__))
    from exotic_blocks import exotic_pose_stack

    two_chains = topology_from_sequence("MKTAYIAK")
    second = topology_from_sequence("GSWEDLV")
    n1 = len(two_chains.block_type_names)
    two = PoseTopology(
        two_chains.block_type_names + second.block_type_names,
        two_chains.bonds + [(n1 + a, ca, n1 + b, cb) for a, ca, b, cb in second.bonds],
    )
    return [
        ("ubq", ubq_pose_stack),
        ("synthetic", synthetic_pose_stack([1, 2, 7, 40, 130], [5, 6, 7, 8, 9])),
        ("two_chains", build_pose_stack([two, topology_from_sequence("AC")])),
        ("exotic", exotic_pose_stack(seed=2)),
    ]


def test_pose_bondsep_matches_builder(ubq_pose_stack):
    for tag, ps in pose_cases(ubq_pose_stack):
        ibb, mb = oracle_bondsep(ps)
        ref = ps.inter_block_bondsep.numpy()
        assert numpy.array_equal(ibb, ref), tag
        assert numpy.array_equal(mb, ref.min(4).min(3)), tag


@pytest.mark.skipif(not O.reference_apsp_available(), reason="compiled reference apsp op not built")
def test_pose_bondsep_matches_reference_route(ubq_pose_stack):
    for tag, ps in pose_cases(ubq_pose_stack):
        ibb, _ = oracle_bondsep(ps)
        assert numpy.array_equal(ibb, pconn_route(ps, O.reference_apsp)), tag
