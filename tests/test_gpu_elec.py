"""GPU parity of the elec term (tmol's elec_pose_scores and
elec_rotamer_scores) through the C ABI.

- against the reference op's outputs committed in tests/golden/elec.npz
  (1ubq, a jagged synthetic batch, a rotamer set): per-pose and block-pair
  energies within 1e-5 relative / 1e-3 kcal/mol, gradients per component
  (tests/tolerances.py: the float32-vs-float32 band), neighbour matrix and
  rotamer dispatch bit-exact;
- against the C oracle in float64 on larger seeded batches: float32 runs
  per component within 1e-4 relative + 1e-3 kcal/mol/A, float64 runs
  within 1e-9;
- per-pose and block-pair adjoints, energy_and_gradient, float64
  gradcheck;
- blocks with several tiles, three connections and ligand fragments, with
  seeded partial charges;
- plan kinds: elec plans serve the elec entry points only.
"""

import numpy
import pytest
import torch

from oracle import oracle as O
from tests.conftest import load_golden
from tmol_b200 import native
from tmol_b200.pose.rotamers import synthetic_rotamer_set
from tmol_b200.pose.synthetic import synthetic_pose_stack
from tmol_b200.score.elec_energy_term import ElecEnergyTerm, elec_pose_score_args, elec_rotamer_score_args
from tmol_b200.score.elec_op import ElecPlan, elec_pose_scores, elec_rotamer_scores
from tolerances import E_close, g_close, g_close_f32

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
CHARGE_ARG = 15  # index of bt_partial_charge in the static arguments


@pytest.fixture(scope="module")
def eterm():
    return ElecEnergyTerm()


def to_dev(args, dtype=torch.float32):
    out = []
    for a in args:
        if isinstance(a, torch.Tensor):
            a = a.to(DEV)
            if a.is_floating_point():
                a = a.to(dtype)
        out.append(a)
    return out


def gpu_scores(ps, eterm, dtype=torch.float32, block_pair=False, weights=None, args=None):
    args = to_dev(args if args is not None else elec_pose_score_args(ps, eterm, block_pair), dtype)
    coords = ps.coords.flatten(0, 1).to(DEV, dtype).requires_grad_(True)
    E, nbr = elec_pose_scores(coords, *args)
    g = None
    if weights is not None:
        (E * torch.as_tensor(weights, device=DEV, dtype=dtype)).sum().backward()
        g = coords.grad.detach().cpu().numpy()
    return E.detach().cpu().numpy(), g, nbr.cpu().numpy()


def test_fixture_parity(ubq_pose_stack, eterm):
    g = load_golden("elec.npz")
    syn = synthetic_pose_stack(list(g["sizes"]), list(g["seeds"]))
    for tag, ps in (("ubq", ubq_pose_stack), ("syn", syn)):
        E, grad, nbr = gpu_scores(ps, eterm, weights=numpy.ones((1, 1)))
        assert E.shape == (1, ps.n_poses)
        E_close(E, g[f"{tag}_energies"])
        if tag == "ubq":
            # tmol's own stored 1ubq elec energy, at that test's tolerance
            numpy.testing.assert_allclose(E[0, 0], g["ubq_tmol_test_energy"][0], atol=1e-5, rtol=1e-3)
        g_close_f32(grad, g[f"{tag}_grad"])
        assert numpy.array_equal(nbr, g[f"{tag}_neighbors"]), tag
        Eb, _, _ = gpu_scores(ps, eterm, block_pair=True)
        E_close(Eb, g[f"{tag}_block_pair"])


@pytest.mark.parametrize("sizes,seed", [([150] * 6, 200), ([5, 80, 20, 1, 300, 47], 9)])
def test_batches_against_oracle(eterm, sizes, seed):
    ps = synthetic_pose_stack(sizes, [seed + k for k in range(len(sizes))], extra_chi_sd=20.0)
    args = elec_pose_score_args(ps, eterm)
    oc = O.OracleCall(ps.coords.flatten(0, 1).double(), args, f64=True, term="elec")
    Eo, dVo, nbro = oc.pose_scores(require_gradient=True)
    w = numpy.random.default_rng(seed).normal(size=(1, ps.n_poses))
    E, g, nbr = gpu_scores(ps, eterm, weights=w)
    E_close(E, Eo[:1])
    assert numpy.array_equal(nbr, nbro)
    ref = dVo[0] * w[0, ps.pose_ind_for_atom.numpy()][:, None]
    g_close(g, ref)


def test_float64_matches_oracle(eterm):
    ps = synthetic_pose_stack([90, 33, 4], [61, 62, 63], extra_chi_sd=20.0)
    args = elec_pose_score_args(ps, eterm)
    c64 = ps.coords.flatten(0, 1).double()
    oc = O.OracleCall(c64, args, f64=True, term="elec")
    Eo, dVo, nbro = oc.pose_scores(require_gradient=True)
    E, g, nbr = gpu_scores(ps, eterm, dtype=torch.float64, weights=numpy.ones((1, 1)))
    E_close(E, Eo[:1], rtol=1e-9, atol=1e-9)
    g_close(g, dVo[0], rtol=1e-9)
    assert numpy.array_equal(nbr, nbro)
    Ebo, _, _ = oc.pose_scores(block_pair=True)
    Eb, _, _ = gpu_scores(ps, eterm, dtype=torch.float64, block_pair=True)
    E_close(Eb, Ebo[:1], rtol=1e-9, atol=1e-9)


def test_block_pair_backward_and_energy_and_gradient(eterm):
    ps = synthetic_pose_stack([70, 12], [71, 72], extra_chi_sd=20.0)
    args = elec_pose_score_args(ps, eterm)
    oc = O.OracleCall(ps.coords.flatten(0, 1).double(), args, f64=True, term="elec")
    _, _, nbr = oc.pose_scores()
    P, B = ps.n_poses, ps.max_n_blocks
    rng = numpy.random.default_rng(5)
    wb = numpy.zeros((3, P, B, B))
    wb[0] = rng.normal(size=(P, B, B)).astype(numpy.float32)
    ref = oc.backward(nbr, wb, per_pose_weights=False)
    coords = ps.coords.flatten(0, 1).to(DEV)
    plan = ElecPlan(coords, to_dev(args)[:-1])
    dx = plan.backward(coords, torch.tensor(wb[:1], device=DEV), block_pair=True)
    g_close(dx.cpu().numpy(), ref)
    # one-pass energies + per-pose weighted gradient
    wp = torch.tensor(rng.normal(size=(1, P)), device=DEV, dtype=torch.float32)
    E1, dx1 = plan.energy_and_gradient(coords, wp)
    E0, _ = plan.forward(coords, want_neighbors=False)
    dx0 = plan.backward(coords, wp)
    # the same pair terms, summed by atomics in another order
    E_close(E1.cpu().numpy(), E0.cpu().numpy(), rtol=1e-5, atol=1e-5)
    g_close_f32(dx1.cpu().numpy(), dx0.cpu().numpy())


def test_gradcheck_float64(eterm):
    ps = synthetic_pose_stack([7, 4], [81, 82], extra_chi_sd=20.0)
    args = to_dev(elec_pose_score_args(ps, eterm), torch.float64)
    c = ps.coords.flatten(0, 1).to(DEV, torch.float64).clone().requires_grad_(True)

    def f(x):
        return elec_pose_scores(x, *args)[0]

    # gradient atomics add in a run-dependent order: repeated backward
    # passes agree to rounding, not bit for bit
    assert torch.autograd.gradcheck(f, (c,), eps=1e-6, atol=1e-5, rtol=1e-3, nondet_tol=1e-10)


def test_exotic_blocks_against_oracle(eterm):
    """Several tiles, three connections, ligand fragments; the charges are
    seeded (the synthetic block types have none in the database)."""
    import os
    import sys

    sys.path.insert(0, os.path.dirname(__file__))
    from exotic_blocks import exotic_pose_stack

    ps = exotic_pose_stack(seed=3)
    args = elec_pose_score_args(ps, eterm)
    q = args[CHARGE_ARG]
    args[CHARGE_ARG] = torch.tensor(
        numpy.random.default_rng(4).normal(scale=0.4, size=tuple(q.shape)), dtype=torch.float32
    )
    oc = O.OracleCall(ps.coords.flatten(0, 1).double(), args, f64=True, term="elec")
    Eo, dVo, nbro = oc.pose_scores(require_gradient=True)
    assert numpy.abs(Eo[0]).max() > 1.0
    E, g, nbr = gpu_scores(ps, eterm, weights=numpy.ones((1, 1)), args=args)
    E_close(E, Eo[:1])
    g_close(g, dVo[0])
    assert numpy.array_equal(nbr, nbro)


def test_rotamer_fixture_parity(eterm):
    from tests.test_rotamer_oracle import fixture_case

    g = load_golden("elec.npz")
    _, ps, rs = fixture_case(DEV)
    args = elec_rotamer_score_args(ps, rs, eterm)
    coords = rs.coords.clone().requires_grad_(True)
    E, idx = elec_rotamer_scores(coords, *args)
    assert E.shape == (1, g["rot_indices"].shape[1])
    assert numpy.array_equal(idx.cpu().numpy(), g["rot_indices"])
    E_close(E.detach().cpu().numpy(), g["rot_energies"])
    (E * torch.tensor(g["rot_weights"], device=DEV)).sum().backward()
    g_close_f32(coords.grad.cpu().numpy(), g["rot_grad"])


@pytest.mark.parametrize("f64", [False, True])
def test_rotamers_against_oracle(eterm, f64):
    dt = torch.float64 if f64 else torch.float32
    ps = synthetic_pose_stack([60, 120, 7], [91, 92, 93], device=DEV, extra_chi_sd=15.0)
    rs = synthetic_rotamer_set(ps, max_rots=5, mutate_fraction=0.4, seed=91, skip_fraction=0.1)
    args = to_dev(elec_rotamer_score_args(ps, rs, eterm), dt)
    c = rs.coords.to(dt)
    plan = ElecPlan(c, args[:-1], rotamers=True)
    idx, items = plan.rotamer_dispatch(c)
    E = plan.rotamer_forward(c, items, idx.shape[1])
    # the oracle in float64 on the same (float32 or float64) inputs
    oc = O.OracleCall(c.cpu().double(), [a.cpu() if isinstance(a, torch.Tensor) else a for a in args], f64=True,
                      term="elec")
    Eo, idxo, nbr = oc.rotamer_scores()
    assert numpy.array_equal(idx.cpu().numpy(), idxo)
    tol = dict(rtol=1e-9, atol=1e-9) if f64 else {}
    E_close(E.cpu().numpy(), Eo[:1], **tol)
    w = torch.rand(E.shape, device=DEV, dtype=dt, generator=torch.Generator(device=DEV).manual_seed(3))
    dx = plan.rotamer_backward(c, items, w)
    W = numpy.zeros((3, E.shape[1]), dtype=numpy.float64)
    W[0] = w[0].cpu().numpy()
    g_close(dx.cpu().numpy(), oc.rotamer_backward(nbr, W), rtol=1e-9 if f64 else 1e-4)


def test_rendered_modules_and_plan_kinds(ubq_pose_stack, eterm):
    g = load_golden("elec.npz")
    ps = ubq_pose_stack
    dev_ps = ps.to(DEV)
    coords = dev_ps.coords
    E = eterm.render_whole_pose_scoring_module(dev_ps)(coords)
    E_close(E.detach().cpu().numpy(), g["ubq_energies"])
    pair = eterm.render_block_pair_scoring_module(dev_ps)
    E_close(pair(coords).detach().cpu().numpy(), g["ubq_block_pair"])
    # an elec plan serves the elec entry points only, and the reverse
    args = to_dev(elec_pose_score_args(ps, eterm))
    flat = coords.flatten(0, 1).contiguous()
    plan = ElecPlan(flat, args[:-1])
    E = torch.empty((3, 1), device=DEV)
    with pytest.raises(native.NativeError):
        native.call("tmol_b200_ljlk_forward", plan.ptr, flat.data_ptr(), 0, E.data_ptr(), None, None)
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args
    from tmol_b200.score.ljlk_op import LJLKPlan

    lplan = LJLKPlan(flat, to_dev(pose_score_args(ps, LJLKEnergyTerm()))[:-1])
    with pytest.raises(native.NativeError):
        native.call("tmol_b200_elec_forward", lplan.ptr, flat.data_ptr(), 0, E.data_ptr(), None, None)
    with pytest.raises(native.NativeError):
        native.call("tmol_b200_elec_plan_destroy", lplan.ptr)


def test_full_size_batch_properties(eterm):
    """The bench's batch (64 poses x 150 residues): energies and gradient
    against the oracle, block-pair energies summing to the whole-pose ones,
    translation invariance, and linearity of the gradient in the weights."""
    ps = synthetic_pose_stack([150] * 64, list(range(64)))
    args = elec_pose_score_args(ps, eterm)
    coords = ps.coords.flatten(0, 1).to(DEV).contiguous()
    plan = ElecPlan(coords, to_dev(args[:-1]))
    ones = torch.ones(1, 64, device=DEV)
    E, g = plan.energy_and_gradient(coords, ones)
    Eo, dVo, _ = O.OracleCall(ps.coords.flatten(0, 1).double(), args, f64=True, term="elec").pose_scores(
        require_gradient=True
    )
    E_close(E.cpu().numpy(), Eo[:1])
    g_close(g.cpu().numpy(), dVo[0])
    Ebp, _ = plan.forward(coords, block_pair=True)
    E_close(Ebp.sum(dim=(2, 3)).cpu().numpy(), E.cpu().numpy(), rtol=1e-5, atol=1e-3)
    Es, _ = plan.energy_and_gradient(coords + torch.tensor([3.1, -2.2, 5.7], device=DEV), ones)
    E_close(Es.cpu().numpy(), E.cpu().numpy(), rtol=1e-4, atol=1e-3)
    w1 = torch.rand(1, 64, device=DEV, generator=torch.Generator(device=DEV).manual_seed(1))
    w2 = torch.rand(1, 64, device=DEV, generator=torch.Generator(device=DEV).manual_seed(2))
    _, ga = plan.energy_and_gradient(coords, w1)
    _, gb = plan.energy_and_gradient(coords, w2)
    _, gab = plan.energy_and_gradient(coords, w1 + w2)
    g_close_f32(gab.cpu().numpy(), (ga + gb).cpu().numpy())
