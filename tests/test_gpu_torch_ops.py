"""The drop-in ops reached through torch's dispatcher,
``torch.ops.tmol_b200.*`` (and, opt-in, under tmol's own namespaces), give
the Python drop-ins' outputs and gradients: energies and neighbour
matrices, gradients through the autograd functions (for LK-ball through the
waters), the rotamer ops' dispatch."""

import subprocess
import sys

import numpy
import pytest
import torch

import tmol_b200.score.torch_ops  # noqa: F401  (registers the ops)
from tmol_b200.pose.rotamers import synthetic_rotamer_set
from tmol_b200.pose.synthetic import synthetic_pose_stack
from tolerances import E_close, g_close_f32

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")

# Both calls run the same kernels on the same inputs, but a pose's energy is
# a float32 sum whose partial sums arrive by atomics in an order that changes
# from run to run: the two results differ by a few ulps of the largest
# partial sums (up to ~2.5e-6 relative on the elec totals, which cancel).
SAME_SUMS = dict(rtol=2e-5, atol=1e-4)


def _dev(args, dtype=None):
    out = []
    for a in args:
        if isinstance(a, torch.Tensor):
            a = a.to(DEV)
            if dtype is not None and a.is_floating_point():
                a = a.to(dtype)
        out.append(a)
    return out


def _both(op, dropin, coords, args, weights):
    """(energies, neighbours or indices, gradient) through the registered op
    and through the drop-in."""
    res = []
    for fn in (op, dropin):
        c = coords.clone().requires_grad_(True)
        out = fn(c, *args)
        E, other = out[0], out[1]
        (E * weights).sum().backward()
        res.append((E.detach().cpu().numpy(), other.cpu().numpy(), c.grad.cpu().numpy()))
    return res


@pytest.fixture(scope="module")
def poses():
    return synthetic_pose_stack([60, 25, 90], [1, 2, 3], extra_chi_sd=20.0)


def test_ljlk_ops(poses):
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args, rotamer_score_args
    from tmol_b200.score.ljlk_op import ljlk_pose_scores, ljlk_rotamer_scores

    term = LJLKEnergyTerm()
    for dt in (torch.float32, torch.float64):
        args = _dev(pose_score_args(poses, term), dt)
        coords = poses.coords.flatten(0, 1).to(DEV, dt)
        w = torch.rand(3, poses.n_poses, device=DEV, dtype=dt, generator=torch.Generator(device=DEV).manual_seed(1))
        (Ea, na, ga), (Eb, nb, gb) = _both(torch.ops.tmol_b200.ljlk_pose_scores, ljlk_pose_scores, coords, args, w)
        assert numpy.array_equal(na, nb)
        E_close(Ea, Eb, **SAME_SUMS)
        g_close_f32(ga, gb)
    psd = poses.to(DEV)
    rs = synthetic_rotamer_set(psd, max_rots=3, mutate_fraction=0.3, seed=5)
    rargs = _dev(rotamer_score_args(psd, rs, LJLKEnergyTerm(device=DEV)))
    (Ea, ia, ga), (Eb, ib, gb) = _both(
        torch.ops.tmol_b200.ljlk_rotamer_scores, ljlk_rotamer_scores, rs.coords.to(DEV), rargs, 1.0
    )
    assert numpy.array_equal(ia, ib)
    E_close(Ea, Eb, **SAME_SUMS)
    g_close_f32(ga, gb)


def test_elec_ops(poses):
    from tmol_b200.score.elec_energy_term import ElecEnergyTerm, elec_pose_score_args
    from tmol_b200.score.elec_op import elec_pose_scores

    args = _dev(elec_pose_score_args(poses, ElecEnergyTerm()))
    coords = poses.coords.flatten(0, 1).to(DEV)
    (Ea, na, ga), (Eb, nb, gb) = _both(torch.ops.tmol_b200.elec_pose_scores, elec_pose_scores, coords, args, 1.0)
    assert numpy.array_equal(na, nb)
    E_close(Ea, Eb, **SAME_SUMS)
    g_close_f32(ga, gb)


def test_lk_ball_ops(poses):
    from tmol_b200.score.lkball_energy_term import LKBallEnergyTerm, score_args, water_gen_args
    from tmol_b200.score.lkball_op import gen_pose_waters, lk_ball_pose_score

    lt = LKBallEnergyTerm()
    wa = _dev(water_gen_args(poses, lt))
    sa = _dev(score_args(poses, lt, None)[:-2])
    coords = poses.coords.flatten(0, 1).to(DEV)
    res = []
    for waters, score in (
        (torch.ops.tmol_b200.gen_pose_waters, torch.ops.tmol_b200.lk_ball_pose_score),
        (gen_pose_waters, lk_ball_pose_score),
    ):
        c = coords.clone().requires_grad_(True)
        W = waters(c, *wa)
        E, nbr = score(c, *sa, W, False)[:2]
        E.sum().backward()  # through the waters
        res.append((W.detach().cpu().numpy(), E.detach().cpu().numpy(), nbr.cpu().numpy(), c.grad.cpu().numpy()))
    (Wa, Ea, na, ga), (Wb, Eb, nb, gb) = res
    assert numpy.array_equal(numpy.isnan(Wa), numpy.isnan(Wb))
    assert numpy.array_equal(na, nb)
    E_close(Ea, Eb, **SAME_SUMS)
    g_close_f32(ga, gb)


def test_reference_namespace_aliases():
    """In a fresh process (no tmol extension loaded): after
    register_reference_aliases(), torch.ops.tmol_ljlk.ljlk_pose_scores is
    this library's op."""
    code = """
import torch
from tmol_b200.score import torch_ops
from tmol_b200.pose.synthetic import synthetic_pose_stack
from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args
assert torch_ops.register_reference_aliases() == ["tmol_ljlk", "tmol_elec", "tmol_lk_ball"]
ps = synthetic_pose_stack([30, 12], [4, 5])
args = [a.cuda() if isinstance(a, torch.Tensor) else a for a in pose_score_args(ps, LJLKEnergyTerm())]
c = ps.coords.flatten(0, 1).cuda()
E1, n1 = torch.ops.tmol_ljlk.ljlk_pose_scores(c, *args)
E2, n2 = torch.ops.tmol_b200.ljlk_pose_scores(c, *args)
assert torch.equal(n1, n2) and torch.allclose(E1, E2, rtol=1e-6, atol=1e-6)
print("aliases ok")
"""
    import os

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "aliases ok" in r.stdout, r.stderr[-2000:]
