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
    """Every one of 1000 random atoms x 3 components, none exempt:
    |g - fd| <= 1e-4 |g| + 1e-6 + 2 |fd(h) - fd(h/2)|.  The last term bounds
    the difference quotient's own error, measured per component: a quotient
    converging at order p >= 1 errs by at most |fd(h) - fd(h/2)| / (1 - 2^-p)
    <= 2 |fd(h) - fd(h/2)|.  On a smooth stretch central differences err by
    O(h^2) and the two quotients agree to ~1e-7; near a region boundary of
    the potentials (the LJ linear extension, the spline knots, where the
    second derivative jumps) or on a hard clash (third derivatives of 1e4
    and more) the quotient errs by up to ~0.04 at h = 1e-3 and converges to
    the analytic value as h shrinks."""
    ps = synthetic_pose_stack([300] * 32, list(range(32)), device=DEV, extra_chi_sd=30.0)
    term = LJLKEnergyTerm(device=DEV)
    static = [a.double() if isinstance(a, torch.Tensor) and a.is_floating_point() else a
              for a in pose_score_args(ps, term)[:-1]]
    coords = ps.coords.flatten(0, 1).double().contiguous()
    plan = LJLKPlan(coords, static)
    h = 1e-3
    fd, g = finite_difference_check(plan, coords, ps.pose_ind_for_atom, BETA2016_WEIGHTS, n_atoms=1000, h=h)
    fd2, g2 = finite_difference_check(plan, coords, ps.pose_ind_for_atom, BETA2016_WEIGHTS, n_atoms=1000, h=h / 2)
    # the same atoms (float64 atomics add in a run-dependent order)
    numpy.testing.assert_allclose(g, g2, rtol=1e-12, atol=1e-12)
    fd_err = numpy.abs(fd - fd2)
    err = numpy.abs(fd - g)
    tol = 1e-4 * numpy.abs(g) + 1e-6 + 2 * fd_err
    smooth = fd_err < 1e-5
    print(
        f"[fd] {err.size} components: max |fd - g| {err.max():.3e}; on the {int(smooth.sum())} smooth ones "
        f"max rel {(err[smooth] / numpy.maximum(numpy.abs(g[smooth]), 1e-12)).max():.3e}; "
        f"{int((~smooth).sum())} within h of a region boundary"
    )
    assert (err <= tol).all(), (err[err > tol], g[err > tol], fd_err[err > tol])
    assert numpy.median(err) < 1e-5
