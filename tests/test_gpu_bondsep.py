"""GPU PoseStack construction steps against the oracle (integer results,
bit-exact):

- inter-block bond separation and its per-block-pair minimum
  (tmol_b200_pose_bondsep) on 1ubq, seeded synthetic batches, a two-chain
  pose and the exotic blocks (three connections, a ring);
- the stacked all-pairs-shortest-paths op (tmol_b200_apsp_stacked) on the
  reference tests' known answers and on seeded random graphs (directed,
  disconnected, zero-weight edges, sizes across tile boundaries), with and
  without a cutoff;
- scoring plans built from the connectivity (no dense bond-separation
  tensors) score like plans built from the dense tensors (LJ/LK pose and
  rotamer plans, elec);
- bad connectivity (a bond recorded one way, an index out of range) is
  rejected.
"""

import numpy
import pytest
import torch

from oracle import oracle as O
from tests.test_bondsep_oracle import path_graph, pose_cases, random_graphs
from tmol_b200 import native
from tmol_b200.pose.bondsep import bondsep_from_connectivity, pose_bondsep, stacked_apsp

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def oracle_case(ps):
    pbt = ps.packed_block_types
    return O.pose_bondsep(ps.block_type_ind, ps.inter_residue_connections, pbt.n_conn, pbt.conn_at_intrablock_bond_sep)


def test_pose_bondsep_matches_oracle(ubq_pose_stack):
    for tag, ps in pose_cases(ubq_pose_stack):
        ibb_o, mb_o = oracle_case(ps)
        ibb, mb = pose_bondsep(ps.to(DEV))
        assert numpy.array_equal(ibb.cpu().numpy(), ibb_o), tag
        assert numpy.array_equal(mb.cpu().numpy(), mb_o), tag
        _, mb2 = pose_bondsep(ps.to(DEV), dense=False)
        assert numpy.array_equal(mb2.cpu().numpy(), mb_o), tag


def test_large_batch_matches_oracle():
    from tmol_b200.pose.synthetic import synthetic_pose_stack

    ps = synthetic_pose_stack([400, 3, 250, 1, 90], [61, 62, 63, 64, 65])
    ibb_o, mb_o = oracle_case(ps)
    ibb, mb = pose_bondsep(ps.to(DEV))
    assert numpy.array_equal(ibb.cpu().numpy(), ibb_o)
    assert numpy.array_equal(mb.cpu().numpy(), mb_o)


def test_bad_connectivity_is_rejected(ubq_pose_stack):
    ps = ubq_pose_stack.to(DEV)
    pbt = ps.packed_block_types
    irc = ps.inter_residue_connections.clone()
    b, c = 5, int(pbt.n_conn[ps.block_type_ind[0, 5]].item()) - 1
    irc[0, b, c] = torch.tensor([7, 0], device=DEV)  # one way only
    with pytest.raises(native.NativeError) as e:
        bondsep_from_connectivity(ps.block_type_ind, irc, pbt.n_conn, pbt.conn_at_intrablock_bond_sep)
    assert e.value.status == 2  # shape
    irc = ps.inter_residue_connections.clone()
    irc[0, 3, 0, 1] = 7  # no such connection
    with pytest.raises(native.NativeError) as e:
        bondsep_from_connectivity(ps.block_type_ind, irc, pbt.n_conn, pbt.conn_at_intrablock_bond_sep)
    assert e.value.status == 3  # index range


def test_apsp_known_answers():
    for N, G in ((32, 1), (64, 1), (1000, 5)):
        w = torch.tensor(path_graph(G, N), device=DEV)
        stacked_apsp(w)
        gold = numpy.abs(numpy.arange(N)[None, :] - numpy.arange(N)[:, None])
        assert all(numpy.array_equal(w[g].cpu().numpy(), gold) for g in range(G))
    w = torch.tensor(path_graph(1, 32, fill=6), device=DEV)
    stacked_apsp(w, 6)
    assert numpy.array_equal(w[0].cpu().numpy(), numpy.minimum(gold[:32, :32], 6))
    for cutoff in (-1, 6):
        g = path_graph(5, 128)
        g[:, 10, 20] = g[:, 20, 10] = 1
        w = torch.tensor(g, device=DEV)
        stacked_apsp(w, cutoff)
        assert numpy.array_equal(w.cpu().numpy(), O.apsp_stacked(g, cutoff))


def test_apsp_random_graphs_match_oracle():
    rng = numpy.random.default_rng(17)
    for trial in range(24):
        G = int(rng.integers(1, 5))
        N = int(rng.choice([1, 5, 31, 32, 33, 64, 95, 130, 257]))
        w = random_graphs(rng, G, N, rng.uniform(0.005, 0.2))
        if trial % 3 == 0:
            w[:, N // 2:, : N // 2] = -1
        for cutoff in (-1, 6, 3):
            d = torch.tensor(w, device=DEV)
            stacked_apsp(d, cutoff)
            assert numpy.array_equal(d.cpu().numpy(), O.apsp_stacked(w, cutoff)), (trial, N, cutoff)


def _energies(plan_cls, args, coords, connectivity, rotamers=False):
    static = [a if i not in (12, 13) or connectivity is None else None for i, a in enumerate(args[:-1])]
    plan = plan_cls(coords, static, rotamers=rotamers, connectivity=connectivity)
    return plan


def test_plans_from_connectivity_score_like_dense_plans(ubq_pose_stack):
    import os
    import sys

    sys.path.insert(0, os.path.dirname(__file__))
    from exotic_blocks import exotic_pose_stack
    from tmol_b200.pose.rotamers import synthetic_rotamer_set
    from tmol_b200.pose.synthetic import synthetic_pose_stack
    from tmol_b200.score.elec_energy_term import ElecEnergyTerm, elec_pose_score_args
    from tmol_b200.score.elec_op import ElecPlan
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args, rotamer_score_args
    from tmol_b200.score.ljlk_op import LJLKPlan

    cases = [ubq_pose_stack.to(DEV), exotic_pose_stack(seed=4).to(DEV), synthetic_pose_stack([120, 8], [3, 4], device=DEV)]
    for ps in cases:
        coords = ps.coords.flatten(0, 1).contiguous()
        for plan_cls, args in (
            (LJLKPlan, pose_score_args(ps, LJLKEnergyTerm(device=DEV))),
            (ElecPlan, elec_pose_score_args(ps, ElecEnergyTerm(device=DEV))),
        ):
            dense = _energies(plan_cls, args, coords, None)
            sparse = _energies(plan_cls, args, coords, ps)
            for bp in (False, True):
                E0, n0 = dense.forward(coords, block_pair=bp)
                E1, n1 = sparse.forward(coords, block_pair=bp)
                numpy.testing.assert_allclose(E1.cpu().numpy(), E0.cpu().numpy(), rtol=1e-6, atol=1e-6)
                assert torch.equal(n0, n1)
            w = torch.rand(dense.N_TERMS, ps.n_poses, device=DEV)
            numpy.testing.assert_allclose(
                sparse.backward(coords, w).cpu().numpy(), dense.backward(coords, w).cpu().numpy(),
                rtol=1e-5, atol=1e-5,
            )
    # a rotamer plan
    ps = synthetic_pose_stack([60, 30], [5, 6], device=DEV)
    rs = synthetic_rotamer_set(ps, max_rots=3, mutate_fraction=0.3, seed=5)
    args = rotamer_score_args(ps, rs, LJLKEnergyTerm(device=DEV))
    dense = _energies(LJLKPlan, args, rs.coords, None, rotamers=True)
    sparse = _energies(LJLKPlan, args, rs.coords, ps, rotamers=True)
    i0, it0 = dense.rotamer_dispatch(rs.coords)
    i1, it1 = sparse.rotamer_dispatch(rs.coords)
    assert torch.equal(i0, i1)
    numpy.testing.assert_allclose(
        sparse.rotamer_forward(rs.coords, it1, i1.shape[1]).cpu().numpy(),
        dense.rotamer_forward(rs.coords, it0, i0.shape[1]).cpu().numpy(),
        rtol=1e-6, atol=1e-6,
    )
