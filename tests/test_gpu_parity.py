"""CUDA path vs the oracle and the reference's golden fixtures.

Tolerances (tests/tolerances.py, the parity bar for this path):
  per-pose energies   |dE| <= 1e-3 kcal/mol + 1e-5 * |E|
  gradients           |dg| <= 1e-4 * |g| + 1e-3 kcal/mol/A per component,
                      against the oracle in float64; against the reference
                      op's stored float32 output both terms are doubled
  neighbour matrix    bit-exact
float64 runs are held to 1e-9 relative (+ 1e-9 absolute).
"""

import numpy
import pytest
import torch

from oracle import oracle as O
from tmol_b200.score.ljlk_energy_term import pose_score_args
from tmol_b200.score.ljlk_op import LJLKPlan, ljlk_pose_scores, clear_plan_cache
from tolerances import E_close, g_close, g_close_f32

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def oracle64(ps, args):
    """The oracle in float64 on the stack's (float32) coordinates."""
    return O.OracleCall(ps.coords.flatten(0, 1).double(), args, f64=True)


def gpu_scores(ps, term, dtype=torch.float32, block_pair=False, grad_weights=None):
    args = [a.to(DEV) if isinstance(a, torch.Tensor) else a for a in pose_score_args(ps, term, block_pair)]
    coords = ps.coords.flatten(0, 1).to(DEV, dtype).requires_grad_(True)
    args = [a.to(dtype) if isinstance(a, torch.Tensor) and a.is_floating_point() else a for a in args]
    E, nbr = ljlk_pose_scores(coords, *args)
    g = None
    if grad_weights is not None:
        (E * torch.as_tensor(grad_weights, device=DEV, dtype=dtype)).sum().backward()
        g = coords.grad.detach().cpu().numpy()
    return E.detach().cpu().numpy(), g, nbr.cpu().numpy()


def test_ubq_against_reference_fixture(ubq_pose_stack, term, ubq_golden):
    E, g, nbr = gpu_scores(ubq_pose_stack, term, grad_weights=numpy.ones((3, 1)))
    E_close(E, ubq_golden["ref_energies"])
    numpy.testing.assert_allclose(E[:, 0], ubq_golden["tmol_test_energies"], atol=1e-5, rtol=1e-3)
    g_close_f32(g, ubq_golden["ref_grad"])
    _, dVo, _ = oracle64(ubq_pose_stack, pose_score_args(ubq_pose_stack, term)).pose_scores(require_gradient=True)
    g_close(g, dVo.sum(0))
    assert numpy.array_equal(nbr, ubq_golden["ref_neighbors"])


def test_synthetic_jagged_against_reference_fixture(synthetic_pose_stack_golden, term, synthetic_golden):
    ps = synthetic_pose_stack_golden
    E, g, nbr = gpu_scores(ps, term, grad_weights=numpy.ones((3, 1)))
    E_close(E, synthetic_golden["ref_energies"])
    g_close_f32(g, synthetic_golden["ref_grad"])
    _, dVo, _ = oracle64(ps, pose_score_args(ps, term)).pose_scores(require_gradient=True)
    g_close(g, dVo.sum(0))
    assert numpy.array_equal(nbr, synthetic_golden["ref_neighbors"])


@pytest.mark.parametrize("sizes,seed", [([150] * 8, 100), ([5, 80, 20, 1, 300, 47], 7)])
def test_batches_against_oracle(term, sizes, seed):
    from tmol_b200.pose.synthetic import synthetic_pose_stack

    ps = synthetic_pose_stack(sizes, [seed + k for k in range(len(sizes))])
    rng = numpy.random.default_rng(seed)
    w = rng.uniform(0.2, 1.5, size=(3, len(sizes)))
    E, g, nbr = gpu_scores(ps, term, grad_weights=w)
    Eo, dVo, nbro = oracle64(ps, pose_score_args(ps, term)).pose_scores(require_gradient=True)
    E_close(E, Eo)
    assert numpy.array_equal(nbr, nbro)
    pose = ps.pose_ind_for_atom.numpy()
    g_ref = (dVo * w[:, pose][:, :, None]).sum(0)
    g_close(g, g_ref)


def test_block_pair_mode_and_adjoint(synthetic_pose_stack_golden, term):
    ps = synthetic_pose_stack_golden
    P, B = ps.n_poses, ps.max_n_blocks
    rng = numpy.random.default_rng(3)
    w = rng.normal(size=(3, P, B, B))
    E, g, nbr = gpu_scores(ps, term, block_pair=True, grad_weights=w)
    oc = oracle64(ps, pose_score_args(ps, term, True))
    Eo, _, nbro = oc.pose_scores(block_pair=True)
    E_close(E, Eo)
    assert numpy.array_equal(nbr, nbro)
    go = oc.backward(nbro, w.astype(numpy.float32).astype(numpy.float64), per_pose_weights=False)
    g_close(g, go)


def test_float64_path(synthetic_pose_stack_golden, term):
    ps = synthetic_pose_stack_golden
    E, g, nbr = gpu_scores(ps, term, dtype=torch.float64, grad_weights=numpy.ones((3, 1)))
    oc = O.OracleCall(ps.coords.flatten(0, 1).double(), pose_score_args(ps, term), f64=True)
    Eo, dVo, _ = oc.pose_scores(require_gradient=True)
    E_close(E, Eo, rtol=1e-9, atol=1e-9)
    g_close(g, dVo.sum(0), rtol=1e-9)


def test_gradcheck_float64(term):
    from tmol_b200.pose.synthetic import synthetic_pose_stack

    ps = synthetic_pose_stack([4, 3], [21, 22])
    args = [a.to(DEV) if isinstance(a, torch.Tensor) else a for a in pose_score_args(ps, term)]
    args = [a.double() if isinstance(a, torch.Tensor) and a.is_floating_point() else a for a in args]
    wt = torch.rand(3, 1, device=DEV, dtype=torch.float64)

    def f(c):
        E, _ = ljlk_pose_scores(c, *args)
        return (wt * E).sum()

    c = ps.coords.flatten(0, 1).to(DEV, torch.float64).requires_grad_(True)
    # the adjoint sums float64 forces with atomics, whose order (and the drop-in
    # plan's work order, rebalanced after its first calls) varies between calls
    assert torch.autograd.gradcheck(f, (c,), eps=1e-6, atol=1e-5, rtol=1e-3, nondet_tol=1e-10)


def test_plan_errors_are_raised(ubq_pose_stack, term):
    from tmol_b200.native import NativeError

    args = [a.to(DEV) if isinstance(a, torch.Tensor) else a for a in pose_score_args(ubq_pose_stack, term)]
    bad = list(args)
    at = bad[17].clone()
    at[0, 0] = 10_000  # atom type index past the type table
    bad[17] = at
    coords = ubq_pose_stack.coords.flatten(0, 1).to(DEV)
    with pytest.raises(NativeError, match="index out of range"):
        LJLKPlan(coords, bad[:-1])
    clear_plan_cache()


@pytest.mark.parametrize("block_pair", [False, True])
def test_exotic_blocks_against_oracle(term, block_pair):
    from exotic_blocks import exotic_pose_stack

    ps = exotic_pose_stack()
    P, B = ps.n_poses, ps.max_n_blocks
    rng = numpy.random.default_rng(5)
    w = rng.normal(size=(3, P, B, B) if block_pair else (3, P))
    E, g, nbr = gpu_scores(ps, term, block_pair=block_pair, grad_weights=w)
    oc = oracle64(ps, pose_score_args(ps, term, block_pair))
    Eo, dVo, nbro = oc.pose_scores(block_pair=block_pair, require_gradient=not block_pair)
    E_close(E, Eo)
    assert numpy.array_equal(nbr, nbro)
    if block_pair:
        go = oc.backward(nbro, w.astype(numpy.float32).astype(numpy.float64), per_pose_weights=False)
    else:
        pose = ps.pose_ind_for_atom.numpy()
        go = (dVo * w[:, pose][:, :, None]).sum(0)
    g_close(g, go)


def test_coincident_atoms_and_an_empty_pose(synthetic_pose_stack_golden, term):
    """Two atoms of different blocks on the same point (d = 0: the linear LJ
    and flat LK regions, no force) and a pose whose blocks are all absent
    (no energy, no gradient), against the oracle."""
    ps = synthetic_pose_stack_golden
    args = list(pose_score_args(ps, term))
    coords = ps.coords.clone()
    offs = ps.block_coord_offset
    coords[4, offs[4, 30]] = coords[4, offs[4, 10]]
    coords[4, offs[4, 31] + 2] = coords[4, offs[4, 12] + 3]
    # pose 1: every block absent
    first_bt = args[3].clone()
    first_bt[1] = -1
    bt_for_rot = args[6].clone().view(ps.n_poses, -1)
    bt_for_rot[1] = -1
    args[3] = first_bt
    args[6] = bt_for_rot.reshape(-1)
    flat = coords.flatten(0, 1)
    oc = O.OracleCall(flat.double(), args, f64=True)
    Eo, dVo, nbro = oc.pose_scores(require_gradient=True)
    gpu_args = [a.to(DEV) if isinstance(a, torch.Tensor) else a for a in args]
    c = flat.to(DEV).requires_grad_(True)
    E, nbr = ljlk_pose_scores(c, *gpu_args)
    w = torch.tensor([1.0, 0.55, 1.0], device=DEV)[:, None]
    (E * w).sum().backward()
    E_close(E.detach().cpu().numpy(), Eo)
    assert numpy.array_equal(nbr.cpu().numpy(), nbro)
    assert (E[:, 1] == 0).all() and nbr[1].sum() == 0
    go = (dVo * numpy.array([1.0, 0.55, 1.0])[:, None, None]).sum(0)
    g_close(c.grad.cpu().numpy(), go)
    pose1 = (ps.pose_ind_for_atom == 1).numpy()
    assert (c.grad.cpu().numpy()[pose1] == 0).all()
    clear_plan_cache()


def test_soft_repulsion_against_oracle(synthetic_pose_stack_golden):
    """tmol's soft_rep option: the plan reads lj_dlin_sigma_factor 0.91 from
    the global parameters (tmol/score/ljlk/ljlk_energy_term.py:44-46)."""
    from tmol_b200.pose.synthetic import synthetic_pose_stack
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm

    soft = LJLKEnergyTerm()
    soft.set_options({"soft_rep": True})
    for ps in (synthetic_pose_stack_golden, synthetic_pose_stack([150] * 4, [301, 302, 303, 304], extra_chi_sd=30.0)):
        w = numpy.random.default_rng(9).uniform(0.2, 1.5, size=(3, ps.n_poses))
        E, g, nbr = gpu_scores(ps, soft, grad_weights=w)
        Eo, dVo, nbro = oracle64(ps, pose_score_args(ps, soft)).pose_scores(require_gradient=True)
        E_close(E, Eo, what="soft_rep energies")
        g_close(g, (dVo * w[:, ps.pose_ind_for_atom.numpy()][:, :, None]).sum(0), what="soft_rep gradient")
        assert numpy.array_equal(nbr, nbro)
    clear_plan_cache()


def test_degenerate_inputs_against_oracle(term):
    """A block type without atoms, a one-block pose and a NaN coordinate
    (host-injected): the GPU returns what the reference does (pinned in
    tests/test_oracle.py): the empty block and the block holding the NaN
    are no block's neighbours, score nothing and get no gradient; every
    other energy and gradient is as without them, and all are finite."""
    from exotic_blocks import degenerate_pose_stack, with_nan_atom

    ps = degenerate_pose_stack()
    args = pose_score_args(ps, term)
    gargs = [a.to(DEV) if isinstance(a, torch.Tensor) else a for a in args]
    w = torch.tensor([1.0, 0.55, 1.0], device=DEV)[:, None]
    for what, coords in (("zero-atom block, one-block pose", ps.coords), ("NaN coordinate", with_nan_atom(ps))):
        flat = coords.flatten(0, 1)
        Eo, dVo, _ = O.OracleCall(flat.double(), args, f64=True).pose_scores(require_gradient=True)
        _, _, nbro = O.OracleCall(flat, args).pose_scores()
        c = flat.to(DEV).requires_grad_(True)
        E, nbr = ljlk_pose_scores(c, *gargs)
        (E * w).sum().backward()
        E = E.detach().cpu().numpy()
        assert numpy.isfinite(E).all() and torch.isfinite(c.grad).all(), what
        E_close(E, Eo, what=what)
        assert numpy.array_equal(nbr.cpu().numpy(), nbro), what
        g_close(c.grad.cpu().numpy(), (dVo * numpy.array([1.0, 0.55, 1.0])[:, None, None]).sum(0), what=what)
    # the NaN block's atoms: no gradient
    nan_block = slice(int(ps.block_coord_offset[2, 3]), int(ps.block_coord_offset[2, 4]))
    assert (c.grad.reshape(ps.n_poses, -1, 3)[2, nan_block] == 0).all()
    clear_plan_cache()


def test_work_counters_against_oracle(term):
    """Work counting is off by default (every counter reads zero); the
    counting kernel's block-pair, atom-pair and heavy-pair counts equal the
    oracle's over the same neighbour list, and its results equal those of
    the kernel without counters."""
    from tmol_b200.pose.synthetic import synthetic_pose_stack

    sizes = [150, 150, 37, 5, 80]
    ps = synthetic_pose_stack(sizes, [300 + k for k in range(len(sizes))])
    args = pose_score_args(ps, term)
    gargs = [a.to(DEV) if isinstance(a, torch.Tensor) else a for a in args]
    coords = ps.coords.flatten(0, 1).to(DEV)
    plan = LJLKPlan(coords, gargs[:-1])
    w = torch.tensor([1.0, 0.55, 1.0], device=DEV)[:, None].expand(3, len(sizes)).contiguous()
    E0, g0 = (t.clone() for t in plan.energy_and_gradient(coords, w))
    assert all(v == 0 for v in plan.last_counts().values())
    plan.set_counting(True)
    E1, g1 = (t.clone() for t in plan.energy_and_gradient(coords, w))
    counts = plan.last_counts()
    _, nbr = plan.forward(coords)
    fwd_counts = plan.last_counts()
    plan.set_counting(False)
    nbr = nbr.cpu().numpy()
    ap, hp = oracle64(ps, args).count_pairs(nbr)
    n_block_pairs = int(sum(numpy.triu(nbr[p] != 0).sum() for p in range(len(sizes))))
    for c in (counts, fwd_counts):
        assert (c["block_pairs"], c["atom_pairs"], c["heavy_pairs"]) == (n_block_pairs, ap, hp), c
        assert 0 < c["heavy_pairs_in_range"] <= c["atom_pairs_in_range"] <= c["atom_pairs"], c
    E_close(E1.cpu().numpy(), E0.cpu().numpy(), what="energies, counting kernel")
    g_close_f32(g1.cpu().numpy(), g0.cpu().numpy(), what="gradient, counting kernel")
