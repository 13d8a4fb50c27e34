"""The LK-ball term's chemistry tables and C oracle against the reference:

- the compiled reference ops (gen_pose_waters, lk_ball_pose_score) run on
  this package's tables reproduce tmol's own stored 1ubq LK-ball energies
  (tmol/tests/data/term_baselines/LKBallEnergyTerm/test_whole_pose_scoring_10.yaml),
  which pins the donor / acceptor / hybridization / bond tables
  (fixture: the reference's outputs, tests/golden/lkball.npz);
- the oracle's waters, four energies and gradient (through the waters)
  against the reference's, float64 to 1e-10, float32 to 1e-5 relative, on
  1ubq and a synthetic pose; live against the compiled op when present;
- the rotamer op (waters on a rotamer set, lk_ball_rotamer_score): dispatch
  indices exact, energies, waters and the gradient of a weighted sum against
  the fixture (tests/golden/lkball_rotamers.npz) and the live op.
"""

import numpy
import pytest
import torch

from oracle import oracle as O
from tests.conftest import load_golden
from tmol_b200.pose.synthetic import synthetic_pose_stack
from tmol_b200.score.lkball_energy_term import LKBallEnergyTerm, score_args, water_gen_args


def cases(ubq_pose_stack):
    g = load_golden("lkball.npz")
    syn = synthetic_pose_stack(list(g["syn_sizes"]), list(g["syn_seeds"]), extra_chi_sd=float(g["syn_chi_sd"]))
    return g, [("ubq", ubq_pose_stack), ("syn", syn)]


def oracle_run(ps, f64, weights=True):
    term = LKBallEnergyTerm()
    dt = torch.float64 if f64 else torch.float32
    wa = water_gen_args(ps, term)
    sa = score_args(ps, term, None)
    coords = ps.coords.flatten(0, 1).to(dt)
    oc = O.OracleCall(coords, sa, f64=f64, term="lkball", lkb_water_args=wa)
    W = oc.lkb_waters()
    E, dx, nbr = oc.lkb_scores(W, weights=numpy.ones((4, ps.n_poses)) if weights else None)
    return W, E, dx, nbr


def test_reference_reproduces_stored_energies(ubq_pose_stack):
    g, _ = cases(ubq_pose_stack)
    numpy.testing.assert_allclose(g["ubq_f32_energies"][:, 0], g["ubq_tmol_test_energies"], rtol=1e-6, atol=1e-5)


@pytest.mark.parametrize("f64", [False, True])
def test_oracle_matches_reference_fixture(ubq_pose_stack, f64):
    g, pss = cases(ubq_pose_stack)
    dn = "f64" if f64 else "f32"
    tol = 1e-10 if f64 else 1e-5
    for tag, ps in pss:
        W, E, dx, _ = oracle_run(ps, f64)
        Wr = g[f"{tag}_{dn}_waters"]
        assert numpy.array_equal(numpy.isnan(W), numpy.isnan(Wr)), tag
        numpy.testing.assert_allclose(W[~numpy.isnan(W)], Wr[~numpy.isnan(Wr)], rtol=0, atol=10 * tol)
        numpy.testing.assert_allclose(E, g[f"{tag}_{dn}_energies"], rtol=tol, atol=tol)
        gr = g[f"{tag}_{dn}_grad"]
        numpy.testing.assert_allclose(dx, gr, rtol=10 * tol, atol=10 * tol * numpy.abs(gr).max())


@pytest.mark.skipif(not O.reference_lkball_available(), reason="compiled reference LK-ball op not built")
def test_oracle_matches_live_reference():
    term = LKBallEnergyTerm()
    for seed in (3, 4):
        ps = synthetic_pose_stack([35], [seed], extra_chi_sd=30.0)
        wa = [a.double() if isinstance(a, torch.Tensor) and a.is_floating_point() else a for a in water_gen_args(ps, term)]
        sa = [a.double() if isinstance(a, torch.Tensor) and a.is_floating_point() else a for a in score_args(ps, term, None)]
        E, Wr, c, nbr = O.reference_lkball(ps.coords.flatten(0, 1).double(), wa, sa)
        E.sum().backward()
        W, Eo, dx, nbro = oracle_run(ps, True)
        numpy.testing.assert_allclose(Eo, E.detach().numpy(), rtol=1e-10, atol=1e-10)
        numpy.testing.assert_allclose(dx, c.grad.numpy(), rtol=1e-9, atol=1e-9 * numpy.abs(dx).max())
        assert numpy.array_equal(nbro, nbr.numpy())


def rotamer_case():
    from tests.test_rotamer_oracle import fixture_case

    _, ps, rs = fixture_case()
    return ps, rs


def oracle_rotamers(ps, rs, f64, weights=None):
    from tmol_b200.score.lkball_energy_term import rotamer_score_args

    lt = LKBallEnergyTerm()
    dt = torch.float64 if f64 else torch.float32
    oc = O.OracleCall(rs.coords.to(dt), rotamer_score_args(ps, rs, lt, None), f64=f64, term="lkball",
                      lkb_water_args=water_gen_args(ps, lt, rs))
    W = oc.lkb_waters()
    E, idx, nbr, dx = oc.lkb_rotamer_scores(W, dTdV=weights)
    return W, E, idx, dx


@pytest.mark.parametrize("f64", [False, True])
def test_rotamer_oracle_matches_reference_fixture(f64):
    """lk_ball_rotamer_score on the rotamer set of rotamers.npz (some blocks
    without rotamers, some rotamers of another residue type)."""
    g = load_golden("lkball_rotamers.npz")
    ps, rs = rotamer_case()
    dn = "f64" if f64 else "f32"
    tol = 1e-10 if f64 else 1e-5
    W, E, idx, dx = oracle_rotamers(ps, rs, f64, weights=g[f"{dn}_weights"])
    assert numpy.array_equal(idx, g["indices"])
    Wr = g[f"{dn}_waters"]
    assert numpy.array_equal(numpy.isnan(W), numpy.isnan(Wr))
    numpy.testing.assert_allclose(W[~numpy.isnan(W)], Wr[~numpy.isnan(Wr)], rtol=0, atol=10 * tol if f64 else 2e-4)
    numpy.testing.assert_allclose(E, g[f"{dn}_energies"], rtol=tol, atol=tol if f64 else 1e-3)
    gr = g[f"{dn}_grad"]
    numpy.testing.assert_allclose(dx, gr, rtol=10 * tol, atol=10 * tol * numpy.abs(gr).max())


@pytest.mark.skipif(not O.reference_lkball_available(), reason="compiled reference LK-ball op not built")
def test_rotamer_oracle_matches_live_reference():
    from tmol_b200.pose.rotamers import synthetic_rotamer_set
    from tmol_b200.score.lkball_energy_term import rotamer_score_args

    lt = LKBallEnergyTerm()
    for seed in (8, 9):
        ps = synthetic_pose_stack([25, 14], [seed, seed + 1], extra_chi_sd=20.0)
        rs = synthetic_rotamer_set(ps, max_rots=3, mutate_fraction=0.3, seed=seed, skip_fraction=0.2)
        wa = [a.double() if isinstance(a, torch.Tensor) and a.is_floating_point() else a
              for a in water_gen_args(ps, lt, rs)]
        sa = [a.double() if isinstance(a, torch.Tensor) and a.is_floating_point() else a
              for a in rotamer_score_args(ps, rs, lt, None)]
        E, idx, _, c = O.reference_lkball_rotamers(rs.coords.double(), wa, sa)
        w = numpy.random.default_rng(seed).normal(size=tuple(E.shape))
        (E * torch.tensor(w)).sum().backward()
        _, Eo, idxo, dx = oracle_rotamers(ps, rs, True, weights=w)
        assert numpy.array_equal(idxo, idx.numpy())
        numpy.testing.assert_allclose(Eo, E.detach().numpy(), rtol=1e-10, atol=1e-10)
        numpy.testing.assert_allclose(dx, c.grad.numpy(), rtol=1e-9, atol=1e-9 * numpy.abs(dx).max())


@pytest.mark.skipif(not O.reference_lkball_available(), reason="compiled reference LK-ball op not built")
def test_oracle_matches_live_reference_on_exotic_blocks():
    """Block types of 40 and 45 atoms (two tiles), three connections and
    ligand fragments."""
    import os
    import sys

    sys.path.insert(0, os.path.dirname(__file__))
    from exotic_blocks import exotic_pose_stack

    term = LKBallEnergyTerm()
    for seed in (4, 5):
        ps = exotic_pose_stack(seed=seed)
        wa = [a.double() if isinstance(a, torch.Tensor) and a.is_floating_point() else a for a in water_gen_args(ps, term)]
        sa = [a.double() if isinstance(a, torch.Tensor) and a.is_floating_point() else a for a in score_args(ps, term, None)]
        E, Wr, c, nbr = O.reference_lkball(ps.coords.flatten(0, 1).double(), wa, sa)
        E.sum().backward()
        W, Eo, dx, nbro = oracle_run(ps, True)
        numpy.testing.assert_allclose(W[~numpy.isnan(W)], Wr.detach().numpy()[~numpy.isnan(W)], rtol=0, atol=1e-10)
        numpy.testing.assert_allclose(Eo, E.detach().numpy(), rtol=1e-10, atol=1e-10)
        # the reference's water adjoint indexes other blocks' base atoms by
        # block instead of rotamer (water.hh:566-575), which is right for the
        # first pose of a stack only; the oracle's gradient is checked against
        # finite differences elsewhere
        if ps.n_poses == 1:
            numpy.testing.assert_allclose(dx, c.grad.numpy(), rtol=1e-9, atol=1e-9 * numpy.abs(dx).max())
        assert numpy.array_equal(nbro, nbr.numpy())
