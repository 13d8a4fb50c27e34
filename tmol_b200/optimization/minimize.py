"""Cartesian minimisation of the LJ/LK energy of a PoseStack with the
batched L-BFGS, every energy + gradient evaluation one fused pass of the
B200 kernel.

    python -m tmol_b200.optimization.minimize   # the 32 x 300-residue scenario

prints one JSON line (energies before / after, iterations, evaluations,
milliseconds per evaluation).
"""

import json
import sys
import time

import torch

from ..score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args
from ..score.ljlk_op import LJLKPlan
from .lbfgs import LBFGSArmijo

BETA2016_WEIGHTS = (1.0, 0.55, 1.0)


def make_func(plan, weights, P, max_atoms):
    """x [P, 3 * max_atoms] -> (weighted total energy [P], gradient [P, L])."""
    w = torch.tensor(weights, device=plan.device, dtype=plan.dtype)[:, None].expand(3, P).contiguous()

    def func(x):
        coords = x.reshape(P * max_atoms, 3)
        E, g = plan.energy_and_gradient(coords, w)
        return (w * E).sum(0), g.reshape(P, -1)

    return func


def finite_difference_check(plan, coords, pose_of_atom, weights, n_atoms=1000, h=1e-3, seed=0):
    """Central differences (E(x + h e) - E(x - h e)) / 2h of the weighted
    energy for `n_atoms` random atoms x 3 components, against the adjoint.
    Poses are independent, so every evaluation perturbs one chosen atom in
    each pose at once.  Returns (fd, analytic) as float64 arrays [n, 3]."""
    P = int(pose_of_atom.max()) + 1
    w = torch.tensor(weights, device=coords.device, dtype=coords.dtype)[:, None].expand(3, P).contiguous()
    _, g = plan.energy_and_gradient(coords, w)
    gen = torch.Generator(device="cpu").manual_seed(seed)
    real = torch.nonzero(g.abs().sum(-1).cpu() > 0).squeeze(-1)
    atoms = real[torch.randperm(real.numel(), generator=gen)[:n_atoms]]
    pose = pose_of_atom.cpu()[atoms]
    # rounds: each round takes at most one atom per pose
    rounds = []
    remaining = list(range(atoms.numel()))
    while remaining:
        used, this, rest = set(), [], []
        for i in remaining:
            p_ = int(pose[i])
            (rest if p_ in used else this).append(i)
            used.add(p_)
        rounds.append(this)
        remaining = rest
    fd = torch.zeros((atoms.numel(), 3), dtype=torch.float64)
    for r in rounds:
        idx = atoms[r].to(coords.device)
        pr = pose[r].to(coords.device)
        for k in range(3):
            cp = coords.clone()
            cm = coords.clone()
            cp[idx, k] += h
            cm[idx, k] -= h
            Ep, _ = plan.forward(cp, want_neighbors=False)
            Em, _ = plan.forward(cm, want_neighbors=False)
            dE = ((w * (Ep - Em)).sum(0) / (2 * h)).double()
            fd[r, k] = dE[pr].cpu()
    return fd.numpy(), g[atoms.to(coords.device)].double().cpu().numpy()


def minimize(pose_stack, term=None, max_iter=200, weights=BETA2016_WEIGHTS, **kw):
    term = term or LJLKEnergyTerm(device=pose_stack.device)
    static = pose_score_args(pose_stack, term)[:-1]
    coords = pose_stack.coords.flatten(0, 1).contiguous()
    plan = LJLKPlan(coords, static)
    P, A = pose_stack.n_poses, pose_stack.max_n_pose_atoms
    func = make_func(plan, weights, P, A)
    opt = LBFGSArmijo(func, pose_stack.coords.reshape(P, -1), max_iter=max_iter, **kw)
    x, E, g = opt.run()
    return x.reshape(P, A, 3), E, g, opt


def minimize_module(module, coords, max_iter=200, **kw):
    """Minimise any whole-pose scoring module (a term's, or a
    ScoreFunction's: ``(coords [P, A, 3]) -> [P]`` per-pose energies,
    differentiable) from coords [P, A, 3]; the gradient comes from autograd
    through the terms' adjoint kernels.  Returns (coords, E, g, optimiser)."""
    P, A = coords.shape[0], coords.shape[1]

    def func(x):
        c = x.detach().reshape(P, A, 3).requires_grad_(True)
        E = module(c)
        if E.dim() > 1:
            E = E.sum(0)
        (g,) = torch.autograd.grad(E.sum(), c)
        return E.detach(), g.reshape(P, -1)

    opt = LBFGSArmijo(func, coords.detach().reshape(P, -1), max_iter=max_iter, **kw)
    x, E, g = opt.run()
    return x.reshape(P, A, 3), E, g, opt


def main():
    from ..pose.synthetic import synthetic_pose_stack

    dev = torch.device("cuda:0")
    ps = synthetic_pose_stack([300] * 32, list(range(32)), device=dev, extra_chi_sd=30.0)
    term = LJLKEnergyTerm(device=dev)
    static = pose_score_args(ps, term)[:-1]
    coords = ps.coords.flatten(0, 1).contiguous()
    plan = LJLKPlan(coords, static)
    P, A = ps.n_poses, ps.max_n_pose_atoms
    func = make_func(plan, BETA2016_WEIGHTS, P, A)
    E0, _ = func(ps.coords.reshape(P, -1))
    opt = LBFGSArmijo(func, ps.coords.reshape(P, -1), max_iter=200)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    x, E, g = opt.run()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    print(
        json.dumps(
            {
                "scenario": "32 poses x 300 residues, chis + N(0, 30 deg), beta2016 LJ/LK weights",
                "iterations": len(opt.history) - 1,
                "evaluations": opt.n_evals,
                "wall_s": wall,
                "ms_per_evaluation": 1e3 * wall / opt.n_evals,
                "energy_before_mean": float(E0.mean()),
                "energy_after_mean": float(E.mean()),
                "max_abs_grad_after": float(g.abs().max()),
            }
        )
    )


if __name__ == "__main__":
    sys.exit(main())
