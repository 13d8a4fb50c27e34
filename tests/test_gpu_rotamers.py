"""GPU parity of rotamer scoring (tmol's ljlk_rotamer_scores).

- against the reference op's outputs committed in tests/golden/rotamers.npz:
  dispatch indices bit-exact, energies within 1e-5 relative / 1e-3 kcal/mol,
  the gradient of sum(w * E) per component (tests/tolerances.py, the
  float32-vs-float32 band);
- against the C oracle on larger seeded rotamer sets (mutations, blocks
  without rotamers, up to 6 rotamers per block): dispatch from the float32
  oracle, gradients against the float64 oracle over the same pairs
  (per component, the rotamer band of tests/tolerances.py), float64 runs
  to 1e-9;
- a rotamer set with exactly the native rotamer per block scores like the
  pose op (the rotamer-pair energies add up to the whole-pose energies);
- torch gradcheck in float64 through ``ljlk_rotamer_scores``, and the
  rendered scoring module;
- rotamers of blocks with several tiles, three connections and ligand
  fragments against the oracle.
"""

import numpy
import pytest
import torch

from oracle import oracle as O
from tests.test_rotamer_oracle import fixture_case
from tmol_b200 import native
from tmol_b200.pose.rotamers import synthetic_rotamer_set
from tmol_b200.pose.synthetic import synthetic_pose_stack
from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args, rotamer_score_args
from tmol_b200.score.ljlk_op import LJLKPlan, ljlk_rotamer_scores
from tolerances import E_close, g_close, g_close_f32, g_close_rotamers

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def oracle64_backward(coords, args, nbr, w):
    """The rotamer adjoint in float64 over the float32 oracle's dispatch."""
    oc = O.OracleCall(coords.cpu().double(), [a.cpu() if isinstance(a, torch.Tensor) else a for a in args], f64=True)
    return oc.rotamer_backward(nbr, numpy.asarray(w, dtype=numpy.float64))


def gpu_args(ps, rs):
    term = LJLKEnergyTerm(device=DEV)
    return rotamer_score_args(ps, rs, term)


def test_fixture_parity():
    g, ps, rs = fixture_case(DEV)
    args = gpu_args(ps, rs)
    coords = rs.coords.clone().requires_grad_(True)
    E, idx = ljlk_rotamer_scores(coords, *args)
    assert numpy.array_equal(idx.cpu().numpy(), g["ref_indices"])
    E_close(E.detach().cpu().numpy(), g["ref_energies"])
    (E * torch.tensor(g["weights"], device=DEV)).sum().backward()
    g_close_f32(coords.grad.cpu().numpy(), g["ref_grad"])


@pytest.mark.parametrize("sizes,seed,mut,skip", [([60, 120, 7], 41, 0.4, 0.1), ([200], 42, 0.0, 0.0)])
def test_oracle_parity(sizes, seed, mut, skip):
    ps = synthetic_pose_stack(sizes, [seed + k for k in range(len(sizes))], device=DEV, extra_chi_sd=15.0)
    rs = synthetic_rotamer_set(ps, max_rots=6, mutate_fraction=mut, seed=seed, skip_fraction=skip)
    args = gpu_args(ps, rs)
    plan = LJLKPlan(rs.coords, args[:-1], rotamers=True)
    idx, items = plan.rotamer_dispatch(rs.coords)
    E = plan.rotamer_forward(rs.coords, items, idx.shape[1])
    oc = O.OracleCall(rs.coords.cpu(), [a.cpu() if isinstance(a, torch.Tensor) else a for a in args])
    Eo, idxo, nbr = oc.rotamer_scores()
    assert numpy.array_equal(idx.cpu().numpy(), idxo)
    E_close(E.cpu().numpy(), Eo)
    w = torch.rand(E.shape, device=DEV, generator=torch.Generator(device=DEV).manual_seed(seed))
    dx = plan.rotamer_backward(rs.coords, items, w)
    g_close_rotamers(dx.cpu().numpy(), oracle64_backward(rs.coords, args, nbr, w.cpu().numpy()))


def test_float64_matches_oracle():
    ps = synthetic_pose_stack([50, 31], [51, 52], device=DEV, extra_chi_sd=15.0)
    rs = synthetic_rotamer_set(ps, max_rots=4, mutate_fraction=0.3, seed=51)
    args = gpu_args(ps, rs)
    c64 = rs.coords.double()
    plan = LJLKPlan(c64, args[:-1], rotamers=True)
    idx, items = plan.rotamer_dispatch(c64)
    E = plan.rotamer_forward(c64, items, idx.shape[1])
    oc = O.OracleCall(c64.cpu(), [a.cpu() if isinstance(a, torch.Tensor) else a for a in args], f64=True)
    Eo, idxo, nbr = oc.rotamer_scores()
    assert numpy.array_equal(idx.cpu().numpy(), idxo)
    E_close(E.cpu().numpy(), Eo, rtol=1e-9, atol=1e-9)
    w = torch.rand(E.shape, device=DEV, dtype=torch.float64)
    dx = plan.rotamer_backward(c64, items, w)
    g_close(dx.cpu().numpy(), oc.rotamer_backward(nbr, w.cpu().numpy()), rtol=1e-9)


def test_native_rotamers_reproduce_the_pose_op():
    ps = synthetic_pose_stack([80, 35], [61, 62], device=DEV)
    rs = synthetic_rotamer_set(ps, max_rots=1, seed=61)
    term = LJLKEnergyTerm(device=DEV)
    E_rot, idx = ljlk_rotamer_scores(rs.coords, *rotamer_score_args(ps, rs, term))
    per_pose = torch.zeros((3, ps.n_poses), dtype=torch.float64, device=DEV)
    per_pose.index_add_(1, idx[0].long(), E_rot.double())
    coords = ps.coords.flatten(0, 1).contiguous()
    plan = LJLKPlan(coords, pose_score_args(ps, term)[:-1])
    E_pose, _ = plan.forward(coords, want_neighbors=False)
    E_close(per_pose.cpu().numpy(), E_pose.double().cpu().numpy())


def test_gradcheck_float64():
    ps = synthetic_pose_stack([6, 4], [71, 72], device=DEV)
    rs = synthetic_rotamer_set(ps, max_rots=3, mutate_fraction=0.5, seed=71)
    args = gpu_args(ps, rs)
    c = rs.coords.double().clone().requires_grad_(True)

    def f(x):
        return ljlk_rotamer_scores(x, *args)[0]

    # the adjoint sums float64 forces with atomics, whose order (and the drop-in
    # plan's work order, rebalanced after its first calls) varies between calls
    assert torch.autograd.gradcheck(f, (c,), eps=1e-6, atol=1e-5, rtol=1e-3, nondet_tol=1e-10)


def test_rendered_module_and_plan_kinds():
    g, ps, rs = fixture_case(DEV)
    term = LJLKEnergyTerm(device=DEV)
    mod = term.render_rotamer_scoring_module(ps, rs)
    E, idx = mod(rs.coords)
    assert numpy.array_equal(idx.cpu().numpy(), g["ref_indices"])
    E_close(E.detach().cpu().numpy(), g["ref_energies"])
    sparse = mod.forward_split(rs.coords)
    assert sparse.shape == (3, ps.n_poses, rs.n_rotamers_total, rs.n_rotamers_total)
    # a rotamer plan serves only the rotamer entry points, a pose plan only
    # the pose ones
    rplan = LJLKPlan(rs.coords, rotamer_score_args(ps, rs, term)[:-1], rotamers=True)
    with pytest.raises(native.NativeError):
        rplan.forward(rs.coords)
    coords = ps.coords.flatten(0, 1).contiguous()
    pplan = LJLKPlan(coords, pose_score_args(ps, term)[:-1])
    with pytest.raises(native.NativeError):
        pplan.rotamer_dispatch(coords)


def test_exotic_block_rotamers_against_oracle():
    """Rotamers of blocks with more than 32 atoms, three connections and
    ligand fragments (copies of each native block moved by N(0, 0.4 A))."""
    import sys
    import os

    sys.path.insert(0, os.path.dirname(__file__))
    from exotic_blocks import exotic_pose_stack
    from tmol_b200.pose.rotamers import rotamer_set_from_arrays

    ps = exotic_pose_stack(seed=3)
    rng = numpy.random.default_rng(8)
    X = ps.coords.numpy()
    bti = ps.block_type_ind.numpy()
    offs = ps.block_coord_offset.numpy()
    pbt = ps.packed_block_types
    block_ind, pose_for, bt_for, xyz = [], [], [], []
    for p in range(ps.n_poses):
        for b in range(ps.max_n_blocks):
            if bti[p, b] < 0:
                continue
            n = pbt.active_block_types[bti[p, b]].n_atoms
            native = X[p, offs[p, b]:offs[p, b] + n]
            for k in range(int(rng.integers(1, 4))):
                block_ind.append(b)
                pose_for.append(p)
                bt_for.append(int(bti[p, b]))
                xyz.append(native if k == 0 else native + rng.normal(scale=0.4, size=native.shape))
    rs = rotamer_set_from_arrays(block_ind, pose_for, bt_for, xyz, ps.n_poses, ps.max_n_blocks, "cpu")
    term = LJLKEnergyTerm()
    args = rotamer_score_args(ps, rs, term)
    oc = O.OracleCall(rs.coords, args)
    Eo, idxo, nbr = oc.rotamer_scores()
    gargs = [a.to(DEV) if isinstance(a, torch.Tensor) else a for a in args]
    c = rs.coords.to(DEV).requires_grad_(True)
    E, idx = ljlk_rotamer_scores(c, *gargs)
    assert numpy.array_equal(idx.cpu().numpy(), idxo)
    E_close(E.detach().cpu().numpy(), Eo)
    w = rng.normal(size=Eo.shape).astype(numpy.float32)
    (E * torch.tensor(w, device=DEV)).sum().backward()
    g_close_rotamers(c.grad.cpu().numpy(), oracle64_backward(rs.coords, args, nbr, w))
