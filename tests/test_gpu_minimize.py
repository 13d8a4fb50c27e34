"""Cartesian L-BFGS minimisation driven by the adjoint, and the adjoint
against central finite differences (h = 1e-3 A, float64, 1000 random atoms)."""

import numpy
import pytest
import torch

from tmol_b200.optimization.minimize import BETA2016_WEIGHTS, finite_difference_check, minimize
from tmol_b200.pose.synthetic import synthetic_pose_stack
from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args
from tmol_b200.score.ljlk_op import LJLKPlan

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def test_lbfgs_lowers_every_pose_energy():
    ps = synthetic_pose_stack([100] * 8, list(range(8)), device=DEV, extra_chi_sd=30.0)
    x, E, g, opt = minimize(ps, max_iter=60)
    hist = torch.stack(opt.history)  # [iters + 1, P]
    assert bool((hist[1:] <= hist[:-1] + 1e-6 * hist[:-1].abs()).all()), "energy rose"
    assert bool((hist[-1] < hist[0]).all())
    # clashes relax: the repulsive term falls by orders of magnitude
    assert float(hist[-1].mean()) < 0.2 * float(hist[0].mean()) or float(hist[-1].mean()) < 0


def test_adjoint_against_finite_differences_float64():
    ps = synthetic_pose_stack([300] * 32, list(range(32)), device=DEV, extra_chi_sd=30.0)
    term = LJLKEnergyTerm(device=DEV)
    static = [a.double() if isinstance(a, torch.Tensor) and a.is_floating_point() else a
              for a in pose_score_args(ps, term)[:-1]]
    coords = ps.coords.flatten(0, 1).double().contiguous()
    plan = LJLKPlan(coords, static)
    fd, g = finite_difference_check(plan, coords, ps.pose_ind_for_atom, BETA2016_WEIGHTS, n_atoms=1000, h=1e-3)
    err = numpy.abs(fd - g)
    # central differences are exact to O(h^2 f''') on smooth regions; a kink
    # of the second derivative at a region boundary costs O(h)
    tol = 1e-3 * numpy.maximum(numpy.abs(g), 1.0)
    assert (err <= tol).mean() > 0.995, (err.max(), numpy.sort(err.ravel())[-5:])
    assert numpy.median(err) < 1e-5
