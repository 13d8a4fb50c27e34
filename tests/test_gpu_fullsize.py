"""Every pose of the benchmark batches against the oracle, energies and
gradients, at the per-component tolerances of tests/tolerances.py.

  * the uniform batch (64 poses x 150 residues, seeds 0-63): through the
    plan's fused energy + gradient pass that the benchmark times, through
    the drop-in op and autograd, and in float64;
  * the uneven batch (256 poses, residues log-uniform in [20, 1000]):
    every pose, on coordinates perturbed as one replayed benchmark step
    perturbs them, with the launch re-ordered by measured cost as the
    benchmark runs it;
  * the minimisation batch (32 poses x 300 residues, chis + N(0, 30 deg)):
    the gradient that drives L-BFGS.

The oracle is the float64 restatement of the reference CPU op (bit-exact
with the compiled reference in float32; tests/test_oracle.py), run on the
same float32 coordinates.  tmol's own term tests compare every pose of a
stack the same way (tmol/tests/score/common/test_energy_term.py:243-353).
"""

import numpy
import pytest
import torch

from bench import TERM_WEIGHTS, PERTURB_SD, workload_sizes
from oracle_batches import oracle_energies_and_gradient
from tmol_b200.pose.builder import build_pose_stack
from tmol_b200.pose.synthetic import synthetic_topologies_and_coords
from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args
from tmol_b200.score.ljlk_op import LJLKPlan, clear_plan_cache, ljlk_pose_scores
from tolerances import E_close, g_close

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _batch(sizes, seeds, extra_chi_sd=0.0):
    topos, coords = synthetic_topologies_and_coords(sizes, seeds, extra_chi_sd)
    ps = build_pose_stack(topos, coords, device=DEV)
    return topos, coords, ps


def _per_pose(flat, ps, n_atoms):
    """[P * max atoms, 3] -> the list of each pose's [n_atoms, 3] rows."""
    x = flat.reshape(ps.n_poses, -1, 3).cpu().numpy()
    return [x[p, : n_atoms[p]] for p in range(ps.n_poses)]


def _weights(P, seed):
    rng = numpy.random.default_rng(seed)
    return rng.uniform(0.2, 1.5, size=(3, P))


def test_uniform_bench_batch_every_pose():
    sizes, seeds = workload_sizes("uniform64x150", 0)
    topos, coords, ps = _batch(sizes, seeds)
    P = ps.n_poses
    term = LJLKEnergyTerm(device=DEV)
    args = pose_score_args(ps, term)
    flat = ps.coords.flatten(0, 1).contiguous()
    w_bench = numpy.array(TERM_WEIGHTS)[:, None].repeat(P, 1)
    w_rand = _weights(P, 5)
    Eo, (go_bench, go_rand) = oracle_energies_and_gradient(topos, coords, [w_bench, w_rand])

    # the benchmark's call: the plan's fused energy + gradient pass
    plan = LJLKPlan(flat, args[:-1])
    E, g = plan.energy_and_gradient(flat, torch.tensor(w_bench, device=DEV, dtype=torch.float32))
    E_close(E.cpu().numpy(), Eo, what="uniform 64x150 energies (fused pass)")
    g_close(g.cpu().numpy(), go_bench.reshape(-1, 3), what="uniform 64x150 gradient (fused pass, bench weights)")

    # the drop-in op with autograd, per-pose weights
    c = flat.clone().requires_grad_(True)
    E2, _ = ljlk_pose_scores(c, *args)
    (E2 * torch.tensor(w_rand, device=DEV, dtype=torch.float32)).sum().backward()
    E_close(E2.detach().cpu().numpy(), Eo, what="uniform 64x150 energies (drop-in op)")
    g_close(c.grad.cpu().numpy(), go_rand.reshape(-1, 3), what="uniform 64x150 gradient (drop-in op + autograd)")
    clear_plan_cache()


def test_uniform_bench_batch_float64():
    sizes, seeds = workload_sizes("uniform64x150", 0)
    topos, coords, ps = _batch(sizes, seeds)
    P = ps.n_poses
    term = LJLKEnergyTerm(device=DEV)
    static = [a.double() if isinstance(a, torch.Tensor) and a.is_floating_point() else a
              for a in pose_score_args(ps, term)[:-1]]
    flat = ps.coords.flatten(0, 1).double().contiguous()
    w = _weights(P, 6)
    Eo, (go,) = oracle_energies_and_gradient(topos, coords, [w])
    plan = LJLKPlan(flat, static)
    E, g = plan.energy_and_gradient(flat, torch.tensor(w, device=DEV, dtype=torch.float64))
    E_close(E.cpu().numpy(), Eo, rtol=1e-9, atol=1e-9, what="uniform 64x150 energies (float64)")
    g_close(g.cpu().numpy(), go.reshape(-1, 3), rtol=1e-9, what="uniform 64x150 gradient (float64)")


def test_uneven_bench_batch_every_pose_perturbed():
    sizes, seeds = workload_sizes("uneven256", 0)
    topos, coords, ps = _batch(sizes, seeds)
    P = ps.n_poses
    term = LJLKEnergyTerm(device=DEV)
    static = pose_score_args(ps, term)[:-1]
    base = ps.coords.flatten(0, 1).contiguous()
    plan = LJLKPlan(base, static)
    w = numpy.array(TERM_WEIGHTS)[:, None].repeat(P, 1)
    wt = torch.tensor(w, device=DEV, dtype=torch.float32)
    # the benchmark's replayed step: coordinates + N(0, 0.05 A), after the
    # work items were re-ordered by their measured cost
    plan.balance(lambda: plan.energy_and_gradient(base, wt))
    gen = torch.Generator(device=DEV).manual_seed(17)
    moved = (base + torch.randn(base.shape, device=DEV, generator=gen) * PERTURB_SD).contiguous()
    E, g = plan.energy_and_gradient(moved, wt)
    per_pose = _per_pose(moved, ps, [len(c) for c in coords])
    Eo, (go,) = oracle_energies_and_gradient(topos, per_pose, [w])
    E_close(E.cpu().numpy(), Eo, what="uneven 256 energies (perturbed step)")
    g_close(g.cpu().numpy(), go.reshape(-1, 3), what="uneven 256 gradient (perturbed step)")


def test_minimisation_batch_gradient():
    topos, coords, ps = _batch([300] * 32, list(range(32)), extra_chi_sd=30.0)
    P = ps.n_poses
    term = LJLKEnergyTerm(device=DEV)
    flat = ps.coords.flatten(0, 1).contiguous()
    plan = LJLKPlan(flat, pose_score_args(ps, term)[:-1])
    w = numpy.array(TERM_WEIGHTS)[:, None].repeat(P, 1)
    E, g = plan.energy_and_gradient(flat, torch.tensor(w, device=DEV, dtype=torch.float32))
    Eo, (go,) = oracle_energies_and_gradient(topos, coords, [w])
    E_close(E.cpu().numpy(), Eo, what="minimisation 32x300 energies")
    g_close(g.cpu().numpy(), go.reshape(-1, 3), what="minimisation 32x300 gradient")
