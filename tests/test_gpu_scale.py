"""Size-independent properties of the path on the uneven 256-pose batch
(every pose of it is checked against the oracle in test_gpu_fullsize.py):
linearity of the gradient in the term weights, block-pair energies summing
to whole-pose energies, energy-only forward agreeing with the fused
energy + gradient pass, the autograd adjoint agreeing with the fused pass,
and translation invariance.  GPU results compared with each other use the
float32-vs-float32 band of tests/tolerances.py, per component.  Translation
is the exception: poses sit up to 6000 A from the origin, where a float32
coordinate is only good to 2.4e-4 A, so moving a pose changes its pair
distances by that much and steep clash gradients by ~1e-4 relative; that
test bounds the change by 1e-4 of the largest component."""

import numpy
import pytest
import torch

from tmol_b200.pose.synthetic import log_uniform_sizes, synthetic_pose_stack
from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args
from tmol_b200.score.ljlk_op import LJLKPlan
from tolerances import E_close, g_close_f32

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


def test_gradient_is_linear_in_the_weights(uneven_plan):
    plan, coords, sizes, _, _ = uneven_plan
    P = len(sizes)
    g = torch.Generator(device=DEV).manual_seed(0)
    w1 = torch.rand((3, P), device=DEV, generator=g)
    w2 = torch.rand((3, P), device=DEV, generator=g)
    E1, g1 = plan.energy_and_gradient(coords, w1)
    E2, g2 = plan.energy_and_gradient(coords, w2)
    E3, g3 = plan.energy_and_gradient(coords, w1 + w2)
    E_close(E1.cpu().numpy(), E2.cpu().numpy())
    g_close_f32(g3.cpu().numpy(), (g1 + g2).cpu().numpy(), what="gradient linearity in the weights")


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
    g_close_f32(c.grad.cpu().numpy(), g.cpu().numpy(), what="autograd adjoint vs fused pass")


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
