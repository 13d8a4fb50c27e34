"""The C oracle against the reference's own golden values and against
fixtures produced by the compiled reference op (tests/golden/make_golden.py).

Pins: 1ubq whole-pose energies stored by tmol's test suite
(tmol/tests/data/term_baselines/LJLKEnergyTerm/test_whole_pose_scoring_10.yaml,
compared there with atol 1e-5, rtol 1e-3), and bit-exact agreement with the
reference op's energies, gradients and neighbour matrix.
"""

import os
import sys

import numpy
import pytest
import torch

from oracle import oracle as O
from tmol_b200.score.ljlk_energy_term import pose_score_args


def _oracle(ps, term, f64=False, block_pair=False):
    args = pose_score_args(ps, term, block_pair=block_pair)
    return O.OracleCall(ps.coords.flatten(0, 1), args, f64=f64)


def test_ubq_matches_tmol_test_baseline(ubq_pose_stack, term, ubq_golden):
    E, dV, nbr = _oracle(ubq_pose_stack, term).pose_scores(require_gradient=True)
    numpy.testing.assert_allclose(E[:, 0], ubq_golden["tmol_test_energies"], atol=1e-5, rtol=1e-3)
    # atr and lk reproduce the stored values to the last digit
    assert E[0, 0] == numpy.float32(ubq_golden["tmol_test_energies"][0])
    assert E[2, 0] == numpy.float32(ubq_golden["tmol_test_energies"][2])


def test_ubq_bit_exact_with_reference_op(ubq_pose_stack, term, ubq_golden):
    E, dV, nbr = _oracle(ubq_pose_stack, term).pose_scores(require_gradient=True)
    assert numpy.array_equal(E, ubq_golden["ref_energies"])
    assert numpy.array_equal(dV.sum(0), ubq_golden["ref_grad"])
    assert numpy.array_equal(nbr, ubq_golden["ref_neighbors"])


def test_ubq_block_pair_bit_exact(ubq_pose_stack, term):
    from conftest import load_golden

    ref = load_golden("ubq_blockpair.npz")["ref_block_pair_energies"]
    E, _, _ = _oracle(ubq_pose_stack, term, block_pair=True).pose_scores(block_pair=True)
    assert numpy.array_equal(E, ref)


def test_synthetic_bit_exact_with_reference_op(synthetic_pose_stack_golden, term, synthetic_golden):
    E, dV, nbr = _oracle(synthetic_pose_stack_golden, term).pose_scores(require_gradient=True)
    assert numpy.array_equal(E, synthetic_golden["ref_energies"])
    assert numpy.array_equal(dV.sum(0), synthetic_golden["ref_grad"])
    assert numpy.array_equal(nbr, synthetic_golden["ref_neighbors"])


def test_block_pairs_sum_to_whole_pose(synthetic_pose_stack_golden, term):
    ps = synthetic_pose_stack_golden
    Ew, _, _ = _oracle(ps, term, f64=True).pose_scores()
    Eb, _, _ = _oracle(ps, term, f64=True, block_pair=True).pose_scores(block_pair=True)
    numpy.testing.assert_allclose(Eb.sum(axis=(2, 3)), Ew, rtol=1e-12, atol=1e-9)


def test_whole_pose_gradient_matches_finite_differences(synthetic_pose_stack_golden, term):
    """float64 oracle: analytic gradient vs central differences (h = 1e-6)."""
    ps = synthetic_pose_stack_golden
    coords = ps.coords.flatten(0, 1).double()
    args = pose_score_args(ps, term)
    oc = O.OracleCall(coords, args, f64=True)
    _, dV, _ = oc.pose_scores(require_gradient=True)
    g = dV.sum(0)
    rng = numpy.random.default_rng(0)
    n_real = int((ps.pose_ind_for_atom >= 0).sum())
    atoms = rng.choice(coords.shape[0], 40, replace=False)
    h = 1e-6
    for a in atoms:
        for k in range(3):
            cp = coords.clone()
            cp[a, k] += h
            cm = coords.clone()
            cm[a, k] -= h
            Ep, _, _ = O.OracleCall(cp, args, f64=True).pose_scores()
            Em, _, _ = O.OracleCall(cm, args, f64=True).pose_scores()
            fd = (Ep.sum() - Em.sum()) / (2 * h)
            assert abs(fd - g[a, k]) <= 1e-5 * max(1.0, abs(g[a, k])), (a, k, fd, g[a, k])


def test_weighted_backward_equals_weighted_gradients(synthetic_pose_stack_golden, term):
    ps = synthetic_pose_stack_golden
    oc = _oracle(ps, term, f64=True)
    E, dV, nbr = oc.pose_scores(require_gradient=True)
    rng = numpy.random.default_rng(1)
    w = rng.normal(size=E.shape)
    pose = ps.pose_ind_for_atom.numpy()
    expect = (dV * w[:, pose][:, :, None]).sum(0)
    got = oc.backward(nbr, w, per_pose_weights=True)
    numpy.testing.assert_allclose(got, expect, rtol=1e-10, atol=1e-9)


@pytest.mark.parametrize("f64", [False, True])
def test_lj_known_answers(term, f64):
    """tmol/tests/score/ljlk/potentials/test_compiled_lj_potential.py:45-127."""
    tp = term.type_params.numpy()
    gp = term.global_params.numpy().reshape(-1)
    idx = term.param_db.atom_type_index
    i = tp[idx["CH2"]]
    j = tp[idx["CH3"]]
    sigma = i[0] + j[0]
    eps = numpy.sqrt(i[1] * j[1])
    tol = dict(rtol=1e-5, atol=1e-6)
    # minimum -eps at sigma, split into atr = -eps, rep = 0
    v = O.potential("lj_V_dV", sigma, 6, i, j, gp, f64)
    numpy.testing.assert_allclose(v[0] + v[1], -eps, **tol)
    # zero at and beyond max_dis
    v = O.potential("lj_V_dV", 6.0, 6, i, j, gp, f64)
    numpy.testing.assert_allclose(v[:2], [0, 0], atol=1e-7)
    # connectivity weights: 0.2 at separation 4, 0 at 3 or less
    v5 = O.potential("lj_V_dV", 3.0, 5, i, j, gp, f64)
    v4 = O.potential("lj_V_dV", 3.0, 4, i, j, gp, f64)
    v3 = O.potential("lj_V_dV", 3.0, 3, i, j, gp, f64)
    numpy.testing.assert_allclose(v4, 0.2 * v5, rtol=1e-6)
    assert numpy.all(v3 == 0)
    # linear below 0.6 sigma: equal slope at two points
    d_lin = 0.6 * sigma
    a = O.potential("lj_V_dV", 0.5 * d_lin, 6, i, j, gp, f64)
    b = O.potential("lj_V_dV", 0.8 * d_lin, 6, i, j, gp, f64)
    numpy.testing.assert_allclose(a[3], b[3], rtol=1e-5)
    numpy.testing.assert_allclose((b[1] - a[1]) / (0.3 * d_lin), a[3], rtol=1e-3)


@pytest.mark.parametrize("f64", [False, True])
def test_lk_known_answers(term, f64):
    """tmol/tests/score/ljlk/potentials/test_compiled_lk_isotropic_potential.py:51-110."""
    tp = term.type_params.numpy()
    gp = term.global_params.numpy().reshape(-1)
    idx = term.param_db.atom_type_index
    i = tp[idx["Nbb"]]
    j = tp[idx["OCbb"]]
    # flat close region, zero beyond max_dis, separation weights
    a = O.potential("lk_V_dV", 0.5, 6, i, j, gp, f64)
    b = O.potential("lk_V_dV", 1.0, 6, i, j, gp, f64)
    numpy.testing.assert_allclose(a[0], b[0], rtol=1e-6)
    assert a[1] == 0 and b[1] == 0
    z = O.potential("lk_V_dV", 6.0, 6, i, j, gp, f64)
    numpy.testing.assert_allclose(z, [0, 0], atol=1e-7)
    v4 = O.potential("lk_V_dV", 3.5, 4, i, j, gp, f64)
    v5 = O.potential("lk_V_dV", 3.5, 5, i, j, gp, f64)
    numpy.testing.assert_allclose(v4, 0.2 * v5, rtol=1e-6)
    assert numpy.all(O.potential("lk_V_dV", 3.5, 3, i, j, gp, f64) == 0)
    # C-C pairs are flat up to 4.2 A
    c1 = tp[idx["CH3"]]
    f1 = O.potential("lk_V_dV", 3.0, 6, c1, c1, gp, f64)
    f2 = O.potential("lk_V_dV", 3.8, 6, c1, c1, gp, f64)
    numpy.testing.assert_allclose(f1[0], f2[0], rtol=1e-6)
    # energy-only and energy+derivative evaluators agree
    for d in (1.0, 2.9, 3.3, 4.0, 4.7, 5.5):
        numpy.testing.assert_allclose(
            O.potential("lk_V", d, 6, i, j, gp, f64), O.potential("lk_V_dV", d, 6, i, j, gp, f64)[0], rtol=1e-5
        )


def test_exotic_blocks_oracle_matches_reference(term):
    """Multi-tile blocks, three connections and ligand fragments: the oracle
    against the compiled reference op (skipped where it is not built)."""
    from exotic_blocks import exotic_pose_stack

    if not O.reference_available():
        pytest.skip("reference op not built")
    ps = exotic_pose_stack()
    assert ps.packed_block_types.max_n_conn == 3 and ps.packed_block_types.max_n_atoms > 32
    args = pose_score_args(ps, term)
    E, c, nbr = O.reference_pose_scores(ps.coords.flatten(0, 1), args)
    E.sum().backward()
    Eo, dVo, nbro = O.OracleCall(ps.coords.flatten(0, 1), args).pose_scores(require_gradient=True)
    assert numpy.array_equal(E.detach().numpy(), Eo)
    assert numpy.array_equal(dVo.sum(0), c.grad.numpy())
    assert numpy.array_equal(nbr.numpy(), nbro)


def _degenerate_cases():
    from exotic_blocks import degenerate_pose_stack, with_nan_atom

    ps = degenerate_pose_stack()
    return ps, [("zero-atom block, one-block pose", ps.coords), ("NaN coordinate", with_nan_atom(ps))]


@pytest.mark.skipif(not O.reference_available(), reason="reference op not built")
def test_degenerate_inputs_bit_exact_with_reference(term):
    """A block type without atoms, a one-block pose and a NaN coordinate:
    the oracle defines what the GPU must return, and it is the reference's
    result bit for bit (the NaN block and the empty block are no block's
    neighbours; every energy and gradient stays finite)."""
    ps, cases = _degenerate_cases()
    args = pose_score_args(ps, term)
    for what, coords in cases:
        flat = coords.flatten(0, 1)
        E, dV, nbr = O.OracleCall(flat, args).pose_scores(require_gradient=True)
        Er, c, nbrr = O.reference_pose_scores(flat, args)
        Er.sum().backward()
        assert numpy.array_equal(E, Er.detach().numpy()), what
        assert numpy.array_equal(nbr, nbrr.numpy()), what
        assert numpy.array_equal(dV.sum(0), c.grad.numpy()), what
        assert numpy.isfinite(E).all() and numpy.isfinite(dV).all(), what
    # the NaN block has no neighbours and its atoms no gradient
    E, dV, nbr = O.OracleCall(cases[1][1].flatten(0, 1), args).pose_scores(require_gradient=True)
    assert nbr[2, 3].sum() == 0 and nbr[2, :, 3].sum() == 0
    assert nbr[0, 6].sum() == 0 and nbr[0, :, 6].sum() == 0  # the empty block


@pytest.mark.skipif(not O.reference_available(), reason="reference op not built")
def test_soft_repulsion_bit_exact_with_reference(synthetic_pose_stack_golden):
    """tmol's soft_rep option (lj_dlin_sigma_factor 0.91 instead of 0.6,
    tmol/score/ljlk/ljlk_energy_term.py:44-46,150-156)."""
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm

    ps = synthetic_pose_stack_golden
    soft, hard = LJLKEnergyTerm(), LJLKEnergyTerm()
    soft.set_options({"soft_rep": True})
    assert float(soft.global_params[0, 1]) == pytest.approx(0.91)
    flat = ps.coords.flatten(0, 1)
    args = pose_score_args(ps, soft)
    E, dV, nbr = O.OracleCall(flat, args).pose_scores(require_gradient=True)
    Er, c, nbrr = O.reference_pose_scores(flat, args)
    Er.sum().backward()
    assert numpy.array_equal(E, Er.detach().numpy())
    assert numpy.array_equal(dV.sum(0), c.grad.numpy())
    Eh, _, _ = O.OracleCall(flat, pose_score_args(ps, hard)).pose_scores()
    assert (E[1] < Eh[1]).any()  # a softer wall
