"""Full-size checks on the GPU.  At these sizes the oracle scores a sample
of poses (poses never interact, so each pose's energy is a property of that
pose alone); the rest are size-independent properties of the path:
linearity of the gradient in the term weights, block-pair energies summing
to whole-pose energies, energy-only forward agreeing with the fused
energy + gradient pass, and translation invariance.  Tolerances as in
test_gpu_parity.py."""

import numpy
import pytest
import torch

from oracle import oracle as O
from tmol_b200.pose.synthetic import log_uniform_sizes, synthetic_pose_stack
from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args
from tmol_b200.score.ljlk_op import LJLKPlan

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _uneven(n=256, seed=2):
    rng = numpy.random.default_rng(seed)
    sizes = log_uniform_sizes(rng, n, 20, 1000)
    seeds = [100000 + k for k in range(n)]
    return sizes, seeds


@pytest.fixture(scope="module")
def uneven_plan():
    term = LJLKEnergyTerm(device=DEV)
    sizes, seeds = _uneven()
    ps = synthetic_pose_stack(sizes, seeds, device=DEV)
    static = pose_score_args(ps, term)[:-1]
    coords = ps.coords.flatten(0, 1).contiguous()
    plan = LJLKPlan(coords, static)
    return plan, coords, sizes, seeds, ps.pose_ind_for_atom


def test_uneven_batch_against_oracle_on_sampled_poses(uneven_plan):
    plan, coords, sizes, seeds, _ = uneven_plan
    E, nbr = plan.forward(coords, want_neighbors=False)
    E = E.cpu().numpy()
    term = LJLKEnergyTerm()
    pick = [int(k) for k in numpy.random.default_rng(11).choice(len(sizes), 8, replace=False)]
    pick.append(int(numpy.argmax(sizes)))
    sub = synthetic_pose_stack([sizes[k] for k in pick], [seeds[k] for k in pick])
    Eo, _, _ = O.OracleCall(sub.coords.flatten(0, 1), pose_score_args(sub, term)).pose_scores()
    numpy.testing.assert_allclose(E[:, pick], Eo, rtol=1e-5, atol=1e-3)


def test_gradient_is_linear_in_the_weights(uneven_plan):
    plan, coords, sizes, _, _ = uneven_plan
    P = len(sizes)
    g = torch.Generator(device=DEV).manual_seed(0)
    w1 = torch.rand((3, P), device=DEV, generator=g)
    w2 = torch.rand((3, P), device=DEV, generator=g)
    E1, g1 = plan.energy_and_gradient(coords, w1)
    E2, g2 = plan.energy_and_gradient(coords, w2)
    E3, g3 = plan.energy_and_gradient(coords, w1 + w2)
    torch.testing.assert_close(E1, E2, rtol=1e-5, atol=1e-3)
    scale = g3.abs().max().item()
    torch.testing.assert_close(g3, g1 + g2, rtol=1e-4, atol=1e-4 * scale)


def test_energy_only_forward_matches_fused_pass(uneven_plan):
    plan, coords, sizes, _, _ = uneven_plan
    E, _ = plan.forward(coords, want_neighbors=False)
    w = torch.ones((3, len(sizes)), device=DEV)
    E2, _ = plan.energy_and_gradient(coords, w)
    torch.testing.assert_close(E, E2, rtol=1e-5, atol=1e-3)


def test_autograd_backward_matches_fused_gradient(uneven_plan):
    plan, coords, sizes, _, _ = uneven_plan
    from tmol_b200.score.ljlk_op import pose_scores_with_plan

    w = torch.rand((3, len(sizes)), device=DEV, generator=torch.Generator(device=DEV).manual_seed(3))
    c = coords.clone().requires_grad_(True)
    E, _ = pose_scores_with_plan(c, plan)
    (w * E).sum().backward()
    _, g = plan.energy_and_gradient(coords, w)
    scale = g.abs().max().item()
    torch.testing.assert_close(c.grad, g, rtol=1e-4, atol=1e-4 * scale)


def test_translation_invariance(uneven_plan):
    plan, coords, sizes, _, pose_of_atom = uneven_plan
    shift = torch.tensor([3.25, -1.5, 0.75], device=DEV)
    moved = coords + shift * (pose_of_atom.to(DEV) % 2 == 0).unsqueeze(1)
    w = torch.ones((3, len(sizes)), device=DEV)
    E1, g1 = plan.energy_and_gradient(coords, w)
    E2, g2 = plan.energy_and_gradient(moved.contiguous(), w)
    torch.testing.assert_close(E2, E1, rtol=1e-5, atol=1e-3)
    scale = g1.abs().max().item()
    torch.testing.assert_close(g2, g1, rtol=1e-4, atol=1e-4 * scale)


def test_block_pair_energies_sum_to_whole_pose():
    term = LJLKEnergyTerm(device=DEV)
    ps = synthetic_pose_stack([150] * 16, list(range(16)), device=DEV)
    static = pose_score_args(ps, term)[:-1]
    coords = ps.coords.flatten(0, 1).contiguous()
    plan = LJLKPlan(coords, static)
    Ew, _ = plan.forward(coords, block_pair=False, want_neighbors=False)
    Eb, nbr = plan.forward(coords, block_pair=True, want_neighbors=True)
    torch.testing.assert_close(Eb.sum(dim=(2, 3)), Ew, rtol=1e-5, atol=1e-3)
    # energies only where the neighbour matrix says so
    assert bool(((Eb != 0).any(dim=0) <= (nbr != 0)).all())
