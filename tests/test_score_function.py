"""ScoreFunction (tmol/score/score_function.py): term bookkeeping on the
CPU; on the GPU, the rendered whole-pose and block-pair modules equal the
weighted sum of the terms' own modules, energies and gradients."""

import numpy
import pytest
import torch

from tmol_b200.pose.synthetic import synthetic_pose_stack
from tmol_b200.score.elec_energy_term import ElecEnergyTerm
from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm
from tmol_b200.score.lkball_energy_term import LKBallEnergyTerm
from tmol_b200.score.score_function import ScoreFunction
from tmol_b200.score.score_types import ScoreType

WEIGHTS = {
    "fa_ljatr": 1.0, "fa_ljrep": 0.55, "fa_lk": 1.0, "fa_elec": 1.0,
    "lk_ball_iso": -0.38, "lk_ball": 0.92, "lk_bridge": -0.33, "lk_bridge_uncpl": -0.33,
}


def test_terms_and_weights():
    sfxn = ScoreFunction()
    sfxn.set_weight(ScoreType.lk_ball, 0.92)
    sfxn.set_weight(ScoreType.fa_ljrep, 0.55)
    assert [type(t) for t in sfxn.all_terms()] == [LJLKEnergyTerm, LKBallEnergyTerm]
    assert sfxn.all_score_types()[:3] == [ScoreType.fa_ljatr, ScoreType.fa_ljrep, ScoreType.fa_lk]
    numpy.testing.assert_allclose(sfxn.weights_tensor().numpy(), [0, 0.55, 0, 0, 0.92, 0, 0], rtol=1e-7)
    full = ScoreFunction.from_weights(WEIGHTS)
    assert [type(t) for t in full.all_terms()] == [LJLKEnergyTerm, ElecEnergyTerm, LKBallEnergyTerm]
    assert full.get_weight(ScoreType.lk_bridge) == pytest.approx(-0.33)


@pytest.mark.gpu
def test_rendered_modules_sum_the_terms():
    dev = torch.device("cuda:0")
    ps = synthetic_pose_stack([40, 15], [71, 72], extra_chi_sd=15.0, device=dev)
    sfxn = ScoreFunction.from_weights(WEIGHTS, device=dev)
    whole = sfxn.render_whole_pose_scoring_module(ps)
    coords = ps.coords.clone().requires_grad_(True)
    total = whole(coords)
    total.sum().backward()
    w = sfxn.weights_tensor()
    parts, grad = [], torch.zeros_like(coords)
    for term in sfxn.all_terms():
        c = ps.coords.clone().requires_grad_(True)
        E = term.render_whole_pose_scoring_module(ps)(c)
        parts.append(E.detach())
        k = sum(len(t.score_types()) for t in sfxn.all_terms()[: sfxn.all_terms().index(term)])
        (w[k : k + E.shape[0], None] * E).sum().backward()
        grad += c.grad
    expect = (w[:, None] * torch.cat(parts)).sum(0)
    numpy.testing.assert_allclose(total.detach().cpu().numpy(), expect.cpu().numpy(), rtol=1e-5, atol=1e-3)
    g = coords.grad.cpu().numpy()
    numpy.testing.assert_allclose(g, grad.cpu().numpy(), rtol=1e-4, atol=1e-4 * numpy.abs(g).max())
    assert whole(ps.coords, sum_terms=False).shape == (8, 2)
    pairs = sfxn.render_block_pair_scoring_module(ps)(ps.coords)
    numpy.testing.assert_allclose(pairs.sum(dim=(1, 2)).cpu().numpy(), total.detach().cpu().numpy(), rtol=1e-4,
                                  atol=1e-2)


@pytest.mark.gpu
def test_minimise_the_full_score_function():
    """The ScoreFunction's module drives the batched L-BFGS: the weighted
    LJ/LK + elec + LK-ball energy of every pose falls, and its float64
    gradient (through the LK-ball waters) matches central differences."""
    from tmol_b200.optimization.minimize import minimize_module

    dev = torch.device("cuda:0")
    ps = synthetic_pose_stack([18, 9], [81, 82], extra_chi_sd=25.0, device=dev)
    sfxn = ScoreFunction.from_weights(WEIGHTS, device=dev)
    whole = sfxn.render_whole_pose_scoring_module(ps)
    x0 = ps.coords.double()
    E0 = whole(x0).detach()
    x, E, g, opt = minimize_module(whole, x0, max_iter=40)
    assert (E < E0).all()
    c = x0.clone().requires_grad_(True)
    whole(c).sum().backward()
    gen = numpy.random.default_rng(5)
    real = torch.nonzero(c.grad.abs().sum(-1).flatten() > 0).squeeze(-1).cpu().numpy()
    h = 1e-5
    for flat in gen.choice(real, size=12, replace=False):
        p_, a_ = divmod(int(flat), ps.coords.shape[1])
        k = int(gen.integers(3))
        xp, xm = x0.clone(), x0.clone()
        xp[p_, a_, k] += h
        xm[p_, a_, k] -= h
        fd = (whole(xp).sum() - whole(xm).sum()).item() / (2 * h)
        assert abs(fd - c.grad[p_, a_, k].item()) <= 1e-5 * max(1.0, abs(fd)), (p_, a_, k)
