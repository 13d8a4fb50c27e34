"""Golden trajectory of tmol's own minimiser over the oracle.

tmol's ``LBFGS_Armijo`` (``tmol/optimization/lbfgs_armijo.py``, which
imports only torch, loaded standalone from the tmol checkout) minimises the
beta2016-weighted LJ/LK energy of a small clashing PoseStack, each pose its
own segment, with the energies and gradients of the float64 oracle
(``oracle/ljlk_oracle.c``, bit-exact with the reference op).  The closure
is tmol's ``run_min`` closure (``tmol/optimization/minimizers.py:108-112``)
over a ``CartesianSfxnNetwork``-shaped parameter (every coordinate of the
[P, max atoms, 3] stack).  Written to ``lbfgs_armijo.npz``: the per-pose
energies of every evaluation, in order, and the final coordinates.

    python tests/golden/make_lbfgs_golden.py [/path/to/tmol/checkout]
"""

import importlib.util
import os
import sys

import numpy
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from tmol_b200.pose.synthetic import synthetic_pose_stack  # noqa: E402
from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args  # noqa: E402

SIZES = [40, 25, 60]
SEEDS = [501, 502, 503]
CHI_SD = 30.0
MAX_ITER = 25
# the score function's weights are a float32 tensor (beta2016: 1, 0.55, 1)
WEIGHTS = torch.tensor([1.0, 0.55, 1.0], dtype=torch.float32).double()


class OracleEnergies(torch.autograd.Function):
    """Per-pose weighted LJ/LK energies of coordinates x [P * A * 3] from
    the float64 oracle; backward scales each pose's gradient."""

    @staticmethod
    def forward(ctx, x, args, pose_of_element):
        oc = O.OracleCall(x.detach().reshape(-1, 3), args, f64=True)
        E, dV, _ = oc.pose_scores(require_gradient=True)
        w = WEIGHTS.numpy()
        ctx.save_for_backward(torch.from_numpy((w[:, None, None] * dV).sum(0)).reshape(-1), pose_of_element)
        return torch.from_numpy((w[:, None] * E).sum(0))

    @staticmethod
    def backward(ctx, gE):
        g, pose = ctx.saved_tensors
        return g * gE[pose], None, None


def stack():
    return synthetic_pose_stack(SIZES, SEEDS, extra_chi_sd=CHI_SD)


def trajectory(optimizer_cls, ps=None):
    """(energies of every evaluation [n_evals, P], final coordinates) of
    ``optimizer_cls`` over the oracle, as ``run_min`` drives it."""
    ps = ps or stack()
    args = pose_score_args(ps, LJLKEnergyTerm())
    x = torch.nn.Parameter(ps.coords.double().reshape(-1).clone())
    pose = torch.arange(ps.n_poses).repeat_interleave(ps.coords.shape[1] * 3)
    opt = optimizer_cls([x], max_iter=MAX_ITER, segment_ids=pose)
    trace = []

    def closure():
        opt.zero_grad()
        E = OracleEnergies.apply(x, args, pose)
        E.sum().backward()
        trace.append(E.detach().numpy().copy())
        return E

    opt.step(closure)
    return numpy.stack(trace), x.detach().reshape(ps.coords.shape).numpy()


def load_tmol_optimizer(root):
    path = os.path.join(root, "tmol", "optimization", "lbfgs_armijo.py")
    spec = importlib.util.spec_from_file_location("tmol_lbfgs_armijo", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.LBFGS_Armijo


def main(root):
    trace, coords = trajectory(load_tmol_optimizer(root))
    numpy.savez_compressed(
        os.path.join(HERE, "lbfgs_armijo.npz"),
        sizes=numpy.array(SIZES), seeds=numpy.array(SEEDS), chi_sd=numpy.float64(CHI_SD),
        max_iter=numpy.int64(MAX_ITER), weights=WEIGHTS.numpy(), trace=trace, coords=coords,
    )
    print(f"{trace.shape[0]} evaluations; energies {trace[0]} -> {trace[-1]}")


if __name__ == "__main__":
    from oracle.build_ref import reference_root

    main(sys.argv[1] if len(sys.argv) > 1 else reference_root())
