"""The drop-in op's speculative gradient: from the second forward + backward
on a plan, the forward's fused pass takes the gradient with the previous
backward's weights and the backward reuses it when its weights match.
Every result must equal the plain path's (the plan's one-call energy and
gradient) within the float32 band, whatever the sequence of calls."""

import numpy
import pytest
import torch

from tmol_b200.pose.synthetic import synthetic_pose_stack
from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args
from tmol_b200.score.ljlk_op import LJLKPlan, clear_plan_cache, ljlk_pose_scores
from tolerances import E_close, g_close_f32

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


@pytest.fixture(scope="module")
def case():
    sizes = [150, 60, 33, 5]
    ps = synthetic_pose_stack(sizes, [400 + k for k in range(len(sizes))], extra_chi_sd=20.0)
    args = [a.to(DEV) if isinstance(a, torch.Tensor) else a for a in pose_score_args(ps, LJLKEnergyTerm())]
    coords = ps.coords.flatten(0, 1).to(DEV)
    moved = coords + 0.05 * torch.randn(coords.shape, device=DEV, generator=torch.Generator(device=DEV).manual_seed(3))
    return ps, args, coords, moved


def dropin(args, coords, w):
    c = coords.clone().requires_grad_(True)
    E, _ = ljlk_pose_scores(c, *args)
    (E * w).sum().backward()
    return E.detach().cpu().numpy(), c.grad.cpu().numpy()


def test_repeated_calls_match_the_plain_path(case):
    ps, args, coords, moved = case
    P = ps.n_poses
    w1 = torch.tensor([1.0, 0.55, 1.0], device=DEV)[:, None].expand(3, P).contiguous()
    w2 = torch.rand((3, P), device=DEV, generator=torch.Generator(device=DEV).manual_seed(5))
    ref = {}
    for name, x in (("start", coords), ("moved", moved)):
        for wn, w in (("w1", w1), ("w2", w2)):
            plan = LJLKPlan(x, args[:-1])
            E, g = plan.energy_and_gradient(x, w)
            ref[name, wn] = (E.cpu().numpy(), g.cpu().numpy())
    clear_plan_cache()
    # the same weights call after call (the speculation's hits), a change of
    # weights (a miss), new coordinates, and back
    for name, wn in [("start", "w1")] * 3 + [("moved", "w1"), ("moved", "w2"), ("start", "w2"), ("start", "w1")]:
        x = coords if name == "start" else moved
        E, g = dropin(args, x, w1 if wn == "w1" else w2)
        E_close(E, ref[name, wn][0], what=f"energies, {name} {wn}")
        g_close_f32(g, ref[name, wn][1], what=f"gradient, {name} {wn}")
    clear_plan_cache()


def test_interleaved_forwards_and_repeated_backward(case):
    """A backward whose forward is not the plan's latest recomputes; a
    second backward of one forward (retain_graph) with other weights too."""
    ps, args, coords, moved = case
    P = ps.n_poses
    w1 = torch.tensor([1.0, 0.55, 1.0], device=DEV)[:, None].expand(3, P).contiguous()
    w2 = torch.rand((3, P), device=DEV, generator=torch.Generator(device=DEV).manual_seed(6))
    ref = {}
    for name, x in (("start", coords), ("moved", moved)):
        for wn, w in (("w1", w1), ("w2", w2)):
            E, g = LJLKPlan(x, args[:-1]).energy_and_gradient(x, w)
            ref[name, wn] = g.cpu().numpy()
    clear_plan_cache()
    for _ in range(2):
        dropin(args, coords, w1)  # the plan now speculates with w1
    a = coords.clone().requires_grad_(True)
    b = moved.clone().requires_grad_(True)
    Ea, _ = ljlk_pose_scores(a, *args)
    Eb, _ = ljlk_pose_scores(b, *args)  # the latest speculative forward
    (Ea * w1).sum().backward()
    g_close_f32(a.grad.cpu().numpy(), ref["start", "w1"], what="earlier forward's gradient")
    (Eb * w2).sum().backward(retain_graph=True)
    g_close_f32(b.grad.cpu().numpy(), ref["moved", "w2"], what="latest forward, other weights")
    b.grad = None
    (Eb * w2).sum().backward()
    g_close_f32(b.grad.cpu().numpy(), ref["moved", "w2"], what="second backward of one forward")
    clear_plan_cache()


def test_backward_takes_the_kept_gradient(case):
    """White-box: after a speculative forward at coordinates A with weights
    w, backward_speculative with w and that forward's id returns A's
    gradient even when handed other coordinates (the scoring launch did no
    work); with a stale id it computes at the coordinates it is given."""
    ps, args, coords, moved = case
    P = ps.n_poses
    w = torch.tensor([1.0, 0.55, 1.0], device=DEV)[:, None].expand(3, P).contiguous()
    plan = LJLKPlan(coords, args[:-1])
    _, gA = plan.energy_and_gradient(coords, w)
    _, gB = plan.energy_and_gradient(moved, w)
    _, _, gen0 = plan.forward_speculative(coords)
    plan.backward_speculative(coords, w, gen0)  # first backward: weights now known
    _, _, gen = plan.forward_speculative(coords)
    kept = plan.backward_speculative(moved, w, gen)
    g_close_f32(kept.cpu().numpy(), gA.cpu().numpy(), what="kept gradient")
    assert not numpy.allclose(gA.cpu().numpy(), gB.cpu().numpy())
    fresh = plan.backward_speculative(moved, w, gen - 1)
    g_close_f32(fresh.cpu().numpy(), gB.cpu().numpy(), what="recomputed gradient")


def test_elec_dropin_speculates_correctly():
    from tmol_b200.score.elec_energy_term import ElecEnergyTerm, elec_pose_score_args
    from tmol_b200.score.elec_op import ElecPlan, elec_pose_scores

    ps = synthetic_pose_stack([120, 40], [21, 22])
    args = [a.to(DEV) if isinstance(a, torch.Tensor) else a for a in elec_pose_score_args(ps, ElecEnergyTerm())]
    coords = ps.coords.flatten(0, 1).to(DEV)
    w = torch.tensor([[0.8, 1.3]], device=DEV)
    E0, g0 = ElecPlan(coords, args[:-1]).energy_and_gradient(coords, w)
    clear_plan_cache()
    for _ in range(3):
        c = coords.clone().requires_grad_(True)
        E, _ = elec_pose_scores(c, *args)
        (E * w).sum().backward()
        E_close(E.detach().cpu().numpy(), E0.cpu().numpy(), what="elec energies")
        g_close_f32(c.grad.cpu().numpy(), g0.cpu().numpy(), what="elec gradient")
    clear_plan_cache()


def test_lkball_dropin_speculates_correctly():
    """gen_pose_waters + lk_ball_pose_score with autograd, call after call:
    the gradient through the waters equals the plan's one-call energy and
    gradient, with repeated weights (the speculation's hits), changed
    weights and moved coordinates."""
    from tmol_b200.score.lkball_energy_term import LKBallEnergyTerm, score_args, water_gen_args
    from tmol_b200.score.lkball_op import LKBallPlan, gen_pose_waters, lk_ball_pose_score

    lt = LKBallEnergyTerm()
    ps = synthetic_pose_stack([70, 30, 45], [61, 62, 63], extra_chi_sd=20.0)

    def dev(args):
        return [a.to(DEV) if isinstance(a, torch.Tensor) else a for a in args]

    wa, sa = dev(water_gen_args(ps, lt)), dev(score_args(ps, lt, None)[:-2])
    coords = ps.coords.flatten(0, 1).to(DEV)
    moved = coords + 0.05 * torch.randn(coords.shape, device=DEV, generator=torch.Generator(device=DEV).manual_seed(9))
    w1 = torch.tensor([1.0, 0.9, 0.8, 0.7], device=DEV)[:, None].expand(4, ps.n_poses).contiguous()
    w2 = torch.rand((4, ps.n_poses), device=DEV, generator=torch.Generator(device=DEV).manual_seed(10))
    ref = {}
    for name, x in (("start", coords), ("moved", moved)):
        for wn, w in (("w1", w1), ("w2", w2)):
            E, g = LKBallPlan(x, water_static=wa, score_static=sa).energy_and_gradient(x, w)
            ref[name, wn] = (E.cpu().numpy(), g.cpu().numpy())
    clear_plan_cache()
    for name, wn in [("start", "w1")] * 3 + [("moved", "w1"), ("moved", "w2"), ("start", "w2"), ("start", "w1")]:
        x = coords if name == "start" else moved
        w = w1 if wn == "w1" else w2
        c = x.clone().requires_grad_(True)
        W = gen_pose_waters(c, *wa)
        E, _ = lk_ball_pose_score(c, *sa, W, False)
        (E * w).sum().backward()
        E_close(E.detach().cpu().numpy(), ref[name, wn][0], what=f"LK-ball energies, {name} {wn}")
        g_close_f32(c.grad.cpu().numpy(), ref[name, wn][1], what=f"LK-ball gradient, {name} {wn}")
    clear_plan_cache()
