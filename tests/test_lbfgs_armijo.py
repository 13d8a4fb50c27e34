"""tmol_b200.optimization.LBFGS_Armijo against tmol's own minimiser, on the
CPU: step for step against tmol's class (loaded standalone from a tmol
checkout, skipped without one) on segmented test functions, and against the
stored trajectory of tmol's class over the float64 oracle
(tests/golden/lbfgs_armijo.npz, made by tests/golden/make_lbfgs_golden.py):
the same evaluations in the same order, bit for bit."""

import os
import sys

import numpy
import pytest
import torch

from tmol_b200.optimization.lbfgs_armijo import LBFGS_Armijo

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))


def _tmol_optimizer():
    from oracle.build_ref import reference_root

    path = os.path.join(reference_root(), "tmol", "optimization", "lbfgs_armijo.py")
    if not os.path.exists(path):
        pytest.skip("no tmol checkout")
    import make_lbfgs_golden

    return make_lbfgs_golden.load_tmol_optimizer(reference_root())


def _run(cls, x0, seg, **kw):
    x = torch.nn.Parameter(x0.clone())
    trace = []
    opt = cls([x], segment_ids=seg, **kw)

    def closure():
        opt.zero_grad()
        a, b = x[0::2], x[1::2]
        E = (1 - a) ** 2 + 10 * (b - a * a) ** 2 + 0.1 * torch.sin(3 * a) * b
        E.sum().backward()
        trace.append(E.detach().clone())
        return E

    opt.step(closure)
    return x.detach(), torch.stack(trace)


@pytest.mark.parametrize("kw", [dict(max_iter=50), dict(max_iter=200, gradtol=1e-9, history_size=4)])
def test_step_for_step_with_tmols_class(kw):
    ref_cls = _tmol_optimizer()
    gen = torch.Generator().manual_seed(0)
    for _ in range(4):
        n = 2 * int(torch.randint(2, 9, (1,), generator=gen))
        x0 = torch.randn(n, dtype=torch.float64, generator=gen) * 1.5
        seg = torch.arange(n // 2).repeat_interleave(2)
        xa, ta = _run(LBFGS_Armijo, x0, seg, **kw)
        xb, tb = _run(ref_cls, x0, seg, **kw)
        assert torch.equal(ta, tb) and torch.equal(xa, xb)


def test_reproduces_tmols_trajectory_over_the_oracle():
    import make_lbfgs_golden as M

    g = numpy.load(os.path.join(HERE, "golden", "lbfgs_armijo.npz"))
    trace, coords = M.trajectory(LBFGS_Armijo)
    assert trace.shape == g["trace"].shape
    assert numpy.array_equal(trace, g["trace"]) and numpy.array_equal(coords, g["coords"])
    assert (g["trace"][-1] < g["trace"][0]).all()
