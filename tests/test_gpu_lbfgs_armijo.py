"""tmol's minimisation driven through the B200 ops: ``run_min`` over a
``CartesianSfxnNetwork`` of the score function, with ``LBFGS_Armijo``
(tmol's interface and steps; pinned to tmol's own class in
tests/test_lbfgs_armijo.py).

* In float64 the GPU path takes tmol's trajectory: the per-pose energies of
  every evaluation match those tmol's own optimiser saw over the oracle
  (tests/golden/lbfgs_armijo.npz), and so do the final coordinates.
* The minimisation scenario (32 poses x 300 residues, chis + N(0, 30 deg),
  float32, 200 iterations): every pose's energy falls, and the final
  energies and gradient match the float64 oracle at the final coordinates
  (tests/tolerances.py)."""

import os

import numpy
import pytest
import torch

from tmol_b200.optimization.lbfgs_armijo import LBFGS_Armijo
from tmol_b200.optimization.minimizers import run_min
from tmol_b200.optimization.sfxn_modules import CartesianSfxnNetwork
from tmol_b200.pose.synthetic import synthetic_pose_stack
from tmol_b200.score.score_function import ScoreFunction
from tolerances import E_close, g_close

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
BETA2016 = {"fa_ljatr": 1.0, "fa_ljrep": 0.55, "fa_lk": 1.0}
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lbfgs_armijo.npz")


def test_tmol_trajectory_on_the_gpu():
    g = numpy.load(GOLDEN)
    ps = synthetic_pose_stack(list(g["sizes"]), list(g["seeds"]), extra_chi_sd=float(g["chi_sd"]), device=DEV)
    ps.coords = ps.coords.double()
    net = CartesianSfxnNetwork(ScoreFunction.from_weights(BETA2016, device=DEV), ps)
    trace = []
    real_forward = net.forward

    def recorded():
        E = real_forward()
        trace.append(E.detach().cpu().numpy().copy())
        return E

    net.forward = recorded
    out, opt = run_min(net, optimizer_kwargs=dict(max_iter=int(g["max_iter"])))
    trace = numpy.stack(trace)
    assert trace.shape == g["trace"].shape, (trace.shape, g["trace"].shape)
    # the same evaluations in the same order; the energies agree to the
    # float64 rounding of the two paths' sums, carried through 25 steps
    numpy.testing.assert_allclose(trace, g["trace"], rtol=1e-8, atol=1e-9)
    numpy.testing.assert_allclose(out.coords.cpu().numpy(), g["coords"], rtol=0, atol=1e-6)


def test_minimisation_scenario_32x300():
    from oracle_batches import oracle_energies_and_gradient
    from tmol_b200.pose.builder import build_pose_stack
    from tmol_b200.pose.synthetic import synthetic_topologies_and_coords

    topos, coords = synthetic_topologies_and_coords([300] * 32, list(range(32)), 30.0)
    ps = build_pose_stack(topos, coords, device=DEV)
    sfxn = ScoreFunction.from_weights(BETA2016, device=DEV)
    net = CartesianSfxnNetwork(sfxn, ps)
    E0 = net().detach()
    out, opt = run_min(net, optimizer_kwargs=dict(max_iter=200))
    E1 = sfxn.render_whole_pose_scoring_module(out)(out.coords).detach()
    print(f"[lbfgs] {opt.n_evals} evaluations, {len(opt.energy_history) - 1} iterations, "
          f"mean E {float(E0.mean()):.1f} -> {float(E1.mean()):.1f}")
    assert bool((E1 < E0).all()), "a pose's energy did not fall"
    # the final gradient against the oracle at the final coordinates
    c = out.coords.detach().clone().requires_grad_(True)
    sfxn.render_whole_pose_scoring_module(out)(c).sum().backward()
    final = [c.detach()[p, : len(coords[p])].cpu().numpy() for p in range(32)]
    w = numpy.array([BETA2016["fa_ljatr"], BETA2016["fa_ljrep"], BETA2016["fa_lk"]], dtype=numpy.float32)
    Eo, (go,) = oracle_energies_and_gradient(topos, final, [w.astype(numpy.float64)[:, None].repeat(32, 1)])
    E_close(E1.cpu().numpy(), (w.astype(numpy.float64)[:, None] * Eo).sum(0), what="minimised 32x300 energies")
    g_close(c.grad.reshape(-1, 3).cpu().numpy(), go.reshape(-1, 3), what="minimised 32x300 gradient")
