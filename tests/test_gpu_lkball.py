"""GPU parity of the LK-ball term (tmol's gen_pose_waters and
lk_ball_pose_score) through the C ABI.

- against the reference ops' outputs committed in tests/golden/lkball.npz
  (1ubq and a synthetic pose, float32 and float64): waters, the four
  energies (1e-5 relative / 1e-3 kcal/mol in float32) and the gradient
  through the waters per component (tests/tolerances.py; float32 against
  the stored float32 output: the doubled band);
- against the C oracle on seeded multi-pose batches: float32 runs against
  the oracle in float64 (per component, 1e-4 relative + 1e-3 kcal/mol/A;
  the neighbour matrix against the float32 oracle, bit-exact), float64 to
  1e-9; and on the bench's full 64 x 150 batch with size-independent
  properties (block-pair sums, translation invariance, linearity in the
  weights);
- block-pair energies (upper triangle, summing to the whole-pose ones) and
  their adjoint, against the reference op (tests/golden/lkball_block_pair.npz);
  float64 gradcheck of both ops;
- plan kinds: a water plan and a score plan serve their own entry points;
  corrupted polar / occluder and hbond tables are rejected with a status;
- the rotamer op (waters on a rotamer set, lk_ball_rotamer_score): dispatch
  exact, energies and the gradient of a weighted sum against the reference
  fixture (tests/golden/lkball_rotamers.npz) and the oracle; gradcheck.
"""

import numpy
import pytest
import torch

from oracle import oracle as O
from tests.conftest import load_golden
from tmol_b200 import native
from tmol_b200.pose.synthetic import synthetic_pose_stack
from tmol_b200.score.lkball_energy_term import LKBallEnergyTerm, score_args, water_gen_args
from tmol_b200.score.lkball_op import LKBallPlan, gen_pose_waters, lk_ball_pose_score
from tolerances import E_close, g_close, g_close_f32

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


@pytest.fixture(scope="module")
def lterm():
    return LKBallEnergyTerm()


def to_dev(args, dtype):
    out = []
    for a in args:
        if isinstance(a, torch.Tensor):
            a = a.to(DEV)
            if a.is_floating_point():
                a = a.to(dtype)
        out.append(a)
    return out


def static_args(ps, lterm, dtype):
    wa = to_dev(water_gen_args(ps, lterm), dtype)
    sa = to_dev(score_args(ps, lterm, None)[:-2], dtype)
    return wa, sa


def gpu_run(ps, lterm, dtype, block_pair=False):
    """(waters, energies, d(sum E)/dcoords through the waters, neighbours)"""
    wa, sa = static_args(ps, lterm, dtype)
    coords = ps.coords.flatten(0, 1).to(DEV, dtype).requires_grad_(True)
    W = gen_pose_waters(coords, *wa)
    E, nbr = lk_ball_pose_score(coords, *sa, W, block_pair)
    E.sum().backward()
    return W.detach(), E.detach(), coords.grad, nbr


def _oracle(ps, lterm, f64, weights=None):
    dt = torch.float64 if f64 else torch.float32
    oc = O.OracleCall(ps.coords.flatten(0, 1).to(dt), score_args(ps, lterm, None), f64=f64, term="lkball",
                      lkb_water_args=water_gen_args(ps, lterm))
    W = oc.lkb_waters()
    E, dx, nbr = oc.lkb_scores(W, weights=numpy.ones((4, ps.n_poses)) if weights is None else weights)
    return W, E, dx, nbr


def oracle_run(ps, lterm, f64, weights=None):
    """The oracle's (waters, energies, gradient, neighbours), the values from
    the oracle in float64.  For a float32 GPU run (f64 False) the neighbour
    matrix comes from the float32 oracle: the rule's float32 rounding
    decides borderline block pairs."""
    W, E, dx, nbr = _oracle(ps, lterm, True, weights)
    if not f64:
        nbr = _oracle(ps, lterm, False, weights)[3]
    return W, E, dx, nbr


def W_close(W, ref, atol):
    assert numpy.array_equal(numpy.isnan(W), numpy.isnan(ref))
    numpy.testing.assert_allclose(W[~numpy.isnan(W)], ref[~numpy.isnan(ref)], rtol=0, atol=atol)


def fixture_cases(ubq_pose_stack):
    g = load_golden("lkball.npz")
    syn = synthetic_pose_stack(list(g["syn_sizes"]), list(g["syn_seeds"]), extra_chi_sd=float(g["syn_chi_sd"]))
    return g, [("ubq", ubq_pose_stack), ("syn", syn)]


@pytest.mark.parametrize("f64", [False, True])
def test_matches_reference_fixture(ubq_pose_stack, lterm, f64):
    g, cases = fixture_cases(ubq_pose_stack)
    dn = "f64" if f64 else "f32"
    for tag, ps in cases:
        W, E, dx, _ = gpu_run(ps, lterm, torch.float64 if f64 else torch.float32)
        W_close(W.cpu().numpy(), g[f"{tag}_{dn}_waters"], 1e-9 if f64 else 1e-4)
        if f64:
            E_close(E.cpu().numpy(), g[f"{tag}_{dn}_energies"], rtol=1e-10, atol=1e-10)
            g_close(dx.cpu().numpy(), g[f"{tag}_{dn}_grad"], rtol=1e-9)
        else:
            E_close(E.cpu().numpy(), g[f"{tag}_{dn}_energies"])
            g_close_f32(dx.cpu().numpy(), g[f"{tag}_{dn}_grad"])


def test_ubq_reproduces_stored_energies(ubq_pose_stack, lterm):
    g = load_golden("lkball.npz")
    _, E, _, _ = gpu_run(ubq_pose_stack, lterm, torch.float32)
    E_close(E[:, 0].cpu().numpy(), g["ubq_tmol_test_energies"])


@pytest.mark.parametrize("f64", [False, True])
def test_batches_match_oracle(lterm, f64):
    dt = torch.float64 if f64 else torch.float32
    for sizes, seeds in (([40, 3, 75, 1, 22], [5, 6, 7, 8, 9]), ([120, 64], [11, 12])):
        ps = synthetic_pose_stack(sizes, seeds, extra_chi_sd=25.0)
        W, E, dx, nbr = gpu_run(ps, lterm, dt)
        Wo, Eo, dxo, nbro = oracle_run(ps, lterm, f64)
        assert numpy.array_equal(nbr.cpu().numpy(), nbro)
        if f64:
            W_close(W.cpu().numpy(), Wo, 1e-9)
            E_close(E.cpu().numpy(), Eo, rtol=1e-9, atol=1e-9)
            g_close(dx.cpu().numpy(), dxo, rtol=1e-9)
        else:
            W_close(W.cpu().numpy(), Wo, 1e-4)
            E_close(E.cpu().numpy(), Eo)
            g_close(dx.cpu().numpy(), dxo)


def test_block_pair_energies_and_adjoint(lterm):
    ps = synthetic_pose_stack([50, 17, 33], [21, 22, 23], extra_chi_sd=20.0)
    dt = torch.float64
    wa, sa = static_args(ps, lterm, dt)
    coords = ps.coords.flatten(0, 1).to(DEV, dt)
    plan = LKBallPlan(coords, water_static=wa, score_static=sa)
    W = plan.waters(coords)
    E, nbr = plan.forward(coords, W)
    Ebp, nbr2 = plan.forward(coords, W, block_pair=True)
    assert torch.equal(nbr, nbr2)
    E_close(Ebp.sum(dim=(2, 3)).cpu().numpy(), E.cpu().numpy(), rtol=1e-12, atol=1e-12)
    B = ps.max_n_blocks
    lower = torch.tril(torch.ones(B, B, dtype=torch.bool, device=DEV), diagonal=-1)
    assert not Ebp[:, :, lower].any()
    # block-pair weights that are constant per pose give the whole-pose adjoint
    w = torch.rand(4, ps.n_poses, device=DEV, dtype=dt)
    dx0, dw0 = plan.backward(coords, W, w)
    dx1, dw1 = plan.backward(coords, W, w[:, :, None, None].expand(4, ps.n_poses, B, B), block_pair=True)
    numpy.testing.assert_allclose(dx1.cpu().numpy(), dx0.cpu().numpy(), rtol=1e-10, atol=1e-10)
    numpy.testing.assert_allclose(dw1.cpu().numpy(), dw0.cpu().numpy(), rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("f64", [False, True])
def test_energy_and_gradient_in_one_call(lterm, f64):
    dt = torch.float64 if f64 else torch.float32
    ps = synthetic_pose_stack([60, 25, 44], [51, 52, 53], extra_chi_sd=20.0)
    wa, sa = static_args(ps, lterm, dt)
    coords = ps.coords.flatten(0, 1).to(DEV, dt)
    plan = LKBallPlan(coords, water_static=wa, score_static=sa)
    w = torch.rand(4, ps.n_poses, dtype=torch.float64, generator=torch.Generator().manual_seed(3))
    plan.set_counting(True)
    for _ in range(2):  # the plan's scratch is reused
        E, dx = plan.energy_and_gradient(coords, w.to(DEV, dt))
    _, Eo, dxo, _ = oracle_run(ps, lterm, f64, weights=w.numpy())
    if f64:
        E_close(E.cpu().numpy(), Eo, rtol=1e-9, atol=1e-9)
        g_close(dx.cpu().numpy(), dxo, rtol=1e-9)
    else:
        E_close(E.cpu().numpy(), Eo)
        g_close(dx.cpu().numpy(), dxo)
    c = plan.last_counts()
    assert 0 < c["bridged_pairs"] <= c["pairs_evaluated"] <= c["polar_occluder_pairs"]
    assert c["block_pairs"] > 0
    # a water-only plan has no one-call path
    with pytest.raises(native.NativeError):
        LKBallPlan(coords, water_static=wa).energy_and_gradient(coords, w.to(DEV, dt))


def test_gradcheck(lterm):
    ps = synthetic_pose_stack([9, 6], [31, 32], extra_chi_sd=30.0)
    wa, sa = static_args(ps, lterm, torch.float64)
    coords = ps.coords.flatten(0, 1).to(DEV, torch.float64).requires_grad_(True)

    def whole(c):
        return lk_ball_pose_score(c, *sa, gen_pose_waters(c, *wa), False)[0]

    def pairs(c):
        return lk_ball_pose_score(c, *sa, gen_pose_waters(c, *wa), True)[0]

    assert torch.autograd.gradcheck(whole, (coords,), eps=1e-6, atol=1e-6, nondet_tol=1e-10)
    assert torch.autograd.gradcheck(pairs, (coords,), eps=1e-6, atol=1e-6, nondet_tol=1e-10)


def test_plan_parts(ubq_pose_stack, lterm):
    wa, sa = static_args(ubq_pose_stack, lterm, torch.float32)
    coords = ubq_pose_stack.coords.flatten(0, 1).to(DEV)
    water_plan = LKBallPlan(coords, water_static=wa)
    score_plan = LKBallPlan(coords, score_static=sa)
    W = water_plan.waters(coords)
    with pytest.raises(native.NativeError):
        water_plan.forward(coords, W)
    with pytest.raises(native.NativeError):
        score_plan.waters(coords)
    E, _ = score_plan.forward(coords, W)
    both = LKBallPlan(coords, water_static=wa, score_static=sa)
    E2, _ = both.forward(coords, both.waters(coords))
    E_close(E2.cpu().numpy(), E.cpu().numpy(), rtol=1e-6, atol=1e-6)
    # an LK-ball plan is not an LJ/LK plan
    with pytest.raises(native.NativeError):
        native.call("tmol_b200_ljlk_forward", both.ptr, coords.data_ptr(), 0, E.data_ptr(), None, None)


def test_short_poses_with_padding(lterm):
    ps = synthetic_pose_stack([1, 4], [41, 42])
    W, E, dx, nbr = gpu_run(ps, lterm, torch.float64)
    Wo, Eo, dxo, nbro = oracle_run(ps, lterm, True)
    W_close(W.cpu().numpy(), Wo, 1e-9)
    E_close(E.cpu().numpy(), Eo, rtol=1e-9, atol=1e-9)
    assert numpy.array_equal(nbr.cpu().numpy(), nbro)


def gpu_rotamers(ps, rs, lterm, dtype, weights=None):
    """(waters, energies [4, n], indices, gradient of sum(weights * E))"""
    from tmol_b200.score.lkball_energy_term import rotamer_score_args
    from tmol_b200.score.lkball_op import lk_ball_rotamer_score

    wa = to_dev(water_gen_args(ps, lterm, rs), dtype)
    sa = to_dev(rotamer_score_args(ps, rs, lterm, None)[:-2], dtype)
    coords = rs.coords.to(DEV, dtype).requires_grad_(True)
    W = gen_pose_waters(coords, *wa)
    E, idx = lk_ball_rotamer_score(coords, *sa, W, True)
    if weights is not None:
        (E * torch.as_tensor(weights, device=DEV, dtype=dtype)).sum().backward()
    return W.detach(), E.detach(), idx, coords.grad


@pytest.mark.parametrize("f64", [False, True])
def test_rotamers_match_reference_fixture(lterm, f64):
    """lk_ball_rotamer_score on the rotamer set of rotamers.npz against the
    reference op's outputs (tests/golden/lkball_rotamers.npz)."""
    from tests.test_rotamer_oracle import fixture_case

    g = load_golden("lkball_rotamers.npz")
    _, ps, rs = fixture_case()
    dn = "f64" if f64 else "f32"
    W, E, idx, dx = gpu_rotamers(ps, rs, lterm, torch.float64 if f64 else torch.float32, g[f"{dn}_weights"])
    assert numpy.array_equal(idx.cpu().numpy(), g["indices"])
    W_close(W.cpu().numpy(), g[f"{dn}_waters"], 1e-9 if f64 else 2e-4)
    if f64:
        E_close(E.cpu().numpy(), g[f"{dn}_energies"], rtol=1e-10, atol=1e-10)
        g_close(dx.cpu().numpy(), g[f"{dn}_grad"], rtol=1e-9)
    else:
        E_close(E.cpu().numpy(), g[f"{dn}_energies"])
        g_close_f32(dx.cpu().numpy(), g[f"{dn}_grad"])


def test_rotamers_match_oracle(lterm):
    from tests.test_lkball_oracle import oracle_rotamers
    from tmol_b200.pose.rotamers import synthetic_rotamer_set

    for seed in (13, 14):
        ps = synthetic_pose_stack([70, 22, 5], [seed, seed + 1, seed + 2], extra_chi_sd=20.0)
        rs = synthetic_rotamer_set(ps, max_rots=5, mutate_fraction=0.3, seed=seed, skip_fraction=0.2)
        _, Eo, idxo, _ = oracle_rotamers(ps, rs, True)
        w = numpy.random.default_rng(seed).normal(size=Eo.shape)
        Wo, Eo, idxo, dxo = oracle_rotamers(ps, rs, True, weights=w)
        W, E, idx, dx = gpu_rotamers(ps, rs, lterm, torch.float64, w)
        assert numpy.array_equal(idx.cpu().numpy(), idxo)
        W_close(W.cpu().numpy(), Wo, 1e-9)
        E_close(E.cpu().numpy(), Eo, rtol=1e-9, atol=1e-9)
        g_close(dx.cpu().numpy(), dxo, rtol=1e-9)


def test_rotamer_gradcheck(lterm):
    from tmol_b200.pose.rotamers import synthetic_rotamer_set
    from tmol_b200.score.lkball_energy_term import rotamer_score_args
    from tmol_b200.score.lkball_op import lk_ball_rotamer_score

    ps = synthetic_pose_stack([7, 4], [33, 34], extra_chi_sd=30.0)
    rs = synthetic_rotamer_set(ps, max_rots=2, mutate_fraction=0.3, seed=3)
    wa = to_dev(water_gen_args(ps, lterm, rs), torch.float64)
    sa = to_dev(rotamer_score_args(ps, rs, lterm, None)[:-2], torch.float64)
    coords = rs.coords.to(DEV, torch.float64).requires_grad_(True)

    def f(c):
        return lk_ball_rotamer_score(c, *sa, gen_pose_waters(c, *wa), True)[0]

    assert torch.autograd.gradcheck(f, (coords,), eps=1e-6, atol=1e-6, nondet_tol=1e-10)


@pytest.mark.parametrize("f64", [False, True])
def test_exotic_blocks_match_oracle(lterm, f64):
    """Block types of 40 and 45 atoms (two tiles), three connections and
    ligand fragments."""
    import os
    import sys

    sys.path.insert(0, os.path.dirname(__file__))
    from exotic_blocks import exotic_pose_stack

    dt = torch.float64 if f64 else torch.float32
    for seed in (4, 5):
        ps = exotic_pose_stack(seed=seed)
        W, E, dx, nbr = gpu_run(ps, lterm, dt)
        Wo, Eo, dxo, nbro = oracle_run(ps, lterm, f64)
        assert numpy.array_equal(nbr.cpu().numpy(), nbro)
        if f64:
            W_close(W.cpu().numpy(), Wo, 1e-9)
            E_close(E.cpu().numpy(), Eo, rtol=1e-9, atol=1e-9)
            g_close(dx.cpu().numpy(), dxo, rtol=1e-9)
        else:
            W_close(W.cpu().numpy(), Wo, 1e-4)
            E_close(E.cpu().numpy(), Eo)
            g_close(dx.cpu().numpy(), dxo)


def test_rendered_scoring_modules(lterm):
    """LKBallEnergyTerm's whole-pose, block-pair and rotamer scoring modules
    (tmol's energy-term surface) score like the ops they wrap."""
    from tmol_b200.pose.rotamers import synthetic_rotamer_set

    ps = synthetic_pose_stack([30, 12], [61, 62], extra_chi_sd=20.0)
    W, E, dx, _ = gpu_run(ps, lterm, torch.float32)
    psd = ps.to(DEV)
    coords = psd.coords.clone().requires_grad_(True)
    whole = lterm.render_whole_pose_scoring_module(psd)
    Em = whole(coords)
    E_close(Em.detach().cpu().numpy(), E.cpu().numpy(), rtol=1e-6, atol=1e-6)
    Em.sum().backward()
    g_close_f32(coords.grad.flatten(0, 1).cpu().numpy(), dx.cpu().numpy())
    pairs = lterm.render_block_pair_scoring_module(psd)
    Eb = pairs(psd.coords)
    E_close(Eb.sum(dim=(2, 3)).cpu().numpy(), E.cpu().numpy(), rtol=1e-5, atol=1e-5)
    rs = synthetic_rotamer_set(ps, max_rots=3, mutate_fraction=0.3, seed=7)
    _, Er, idxr, _ = gpu_rotamers(ps, rs, lterm, torch.float32)
    rot = lterm.render_rotamer_scoring_module(psd, rs.to(DEV))
    Em2, idx2 = rot(rs.coords.to(DEV))
    assert torch.equal(idx2, idxr)
    E_close(Em2.cpu().numpy(), Er.cpu().numpy(), rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("f64", [False, True])
def test_block_pair_matches_reference_fixture(lterm, f64):
    """Block-pair energies [4, P, B, B] (upper triangle, as the reference
    writes them) and the gradient of sum(w * E) through the waters against
    the reference op (tests/golden/lkball_block_pair.npz)."""
    g = load_golden("lkball_block_pair.npz")
    lk = load_golden("lkball.npz")
    ps = synthetic_pose_stack(list(lk["syn_sizes"]), list(lk["syn_seeds"]), extra_chi_sd=float(lk["syn_chi_sd"]))
    dn = "f64" if f64 else "f32"
    dt = torch.float64 if f64 else torch.float32
    wa, sa = static_args(ps, lterm, dt)
    coords = ps.coords.flatten(0, 1).to(DEV, dt).requires_grad_(True)
    E, _ = lk_ball_pose_score(coords, *sa, gen_pose_waters(coords, *wa), True)
    (E * torch.as_tensor(g[f"{dn}_weights"], device=DEV)).sum().backward()
    if f64:
        E_close(E.detach().cpu().numpy(), g[f"{dn}_energies"], rtol=1e-10, atol=1e-10)
        g_close(coords.grad.cpu().numpy(), g[f"{dn}_grad"], rtol=1e-9)
    else:
        E_close(E.detach().cpu().numpy(), g[f"{dn}_energies"])
        g_close_f32(coords.grad.cpu().numpy(), g[f"{dn}_grad"])


def test_bad_tables_are_rejected(lterm):
    """Out-of-range entries in the polar / occluder lists or the hbond
    tables stop plan creation with a status (checked before any use)."""
    ps = synthetic_pose_stack([12, 5], [91, 92])
    wa, sa = static_args(ps, lterm, torch.float32)
    coords = ps.coords.flatten(0, 1).to(DEV)
    # lk_ball_pose_score's tile_pol_occ_inds (argument 12 + 8): an index past the tile
    bad = list(sa)
    t = bad[20].clone()
    nz = torch.nonzero(bad[19] > 0)[0]  # a tile with occluders
    t[nz[0], nz[1], 0] = 40
    bad[20] = t
    with pytest.raises(native.NativeError) as e:
        LKBallPlan(coords, score_static=bad)
    assert e.value.status == 3  # index range
    # gen_pose_waters' tile_donH_hvy_inds (argument 12 + 10): a heavy atom
    # past the block, in a block type the poses use (water sites are resolved
    # for the blocks present)
    bad = list(wa)
    t = bad[22].clone()
    used = [int(b) for b in ps.block_type_ind.flatten() if b >= 0 and bad[19][int(b), 0] > 0]
    t[used[0], 0, 0] = 999
    bad[22] = t
    with pytest.raises(native.NativeError) as e:
        LKBallPlan(coords, water_static=bad)
    assert e.value.status == 3


@pytest.mark.parametrize("f64", [False, True])
def test_large_ragged_batch_matches_oracle(lterm, f64):
    """Poses of 700, 30, 250 and 1 residues in one stack (blocks padded to
    700 per pose)."""
    dt = torch.float64 if f64 else torch.float32
    ps = synthetic_pose_stack([700, 30, 250, 1], [101, 102, 103, 104], extra_chi_sd=15.0)
    W, E, dx, nbr = gpu_run(ps, lterm, dt)
    Wo, Eo, dxo, nbro = oracle_run(ps, lterm, f64)
    assert numpy.array_equal(nbr.cpu().numpy(), nbro)
    if f64:
        W_close(W.cpu().numpy(), Wo, 1e-9)
        E_close(E.cpu().numpy(), Eo, rtol=1e-9, atol=1e-9)
        g_close(dx.cpu().numpy(), dxo, rtol=1e-9)
    else:
        W_close(W.cpu().numpy(), Wo, 1e-4)
        E_close(E.cpu().numpy(), Eo)
        g_close(dx.cpu().numpy(), dxo)


def test_plans_from_connectivity_score_like_dense_plans(lterm, ubq_pose_stack):
    """A plan built from the PoseStack's connectivity (no min_bondsep /
    inter_block_bondsep tensors) scores like one built from them."""
    from tmol_b200.pose.rotamers import synthetic_rotamer_set
    from tmol_b200.score.lkball_energy_term import rotamer_score_args

    for ps in (ubq_pose_stack, synthetic_pose_stack([60, 25], [111, 112], extra_chi_sd=20.0)):
        psd = ps.to(DEV)
        wa, sa = static_args(ps, lterm, torch.float32)
        coords = psd.coords.flatten(0, 1).contiguous()
        dense = LKBallPlan(coords, water_static=wa, score_static=sa)
        sparse_sa = [None if i in (13, 14) else a for i, a in enumerate(sa)]
        sparse = LKBallPlan(coords, water_static=wa, score_static=sparse_sa, connectivity=psd)
        W = dense.waters(coords)
        assert torch.equal(torch.isnan(sparse.waters(coords)), torch.isnan(W))
        for bp in (False, True):
            E0, n0 = dense.forward(coords, W, block_pair=bp)
            E1, n1 = sparse.forward(coords, W, block_pair=bp)
            E_close(E1.cpu().numpy(), E0.cpu().numpy(), rtol=1e-6, atol=1e-6)
            assert torch.equal(n0, n1)
        w = torch.rand(4, ps.n_poses, device=DEV)
        E0, g0 = dense.energy_and_gradient(coords, w)
        E1, g1 = sparse.energy_and_gradient(coords, w)
        g_close_f32(g1.cpu().numpy(), g0.cpu().numpy())
    # a rotamer plan
    ps = synthetic_pose_stack([40, 20], [113, 114])
    rs = synthetic_rotamer_set(ps, max_rots=3, mutate_fraction=0.3, seed=9)
    wa = to_dev(water_gen_args(ps, lterm, rs), torch.float32)
    sa = to_dev(rotamer_score_args(ps, rs, lterm, None)[:-2], torch.float32)
    rc = rs.coords.to(DEV)
    dense = LKBallPlan(rc, water_static=wa, score_static=sa, rotamers=True)
    sparse = LKBallPlan(rc, water_static=wa, score_static=[None if i in (13, 14) else a for i, a in enumerate(sa)],
                        rotamers=True, connectivity=ps.to(DEV))
    W = dense.waters(rc)
    i0, it0 = dense.rotamer_dispatch(rc)
    i1, it1 = sparse.rotamer_dispatch(rc)
    assert torch.equal(i0, i1)
    E_close(sparse.rotamer_forward(rc, it1, i1.shape[1], W).cpu().numpy(),
            dense.rotamer_forward(rc, it0, i0.shape[1], W).cpu().numpy(), rtol=1e-6, atol=1e-6)


def test_full_size_batch_properties(lterm):
    """The bench's batch (64 poses x 150 residues): energies and gradient
    against the oracle, the forward against the one-call energies,
    block-pair energies summing to the whole-pose ones, translation
    invariance, and linearity of the gradient in the weights."""
    ps = synthetic_pose_stack([150] * 64, list(range(64)))
    wa, sa = static_args(ps, lterm, torch.float32)
    coords = ps.coords.flatten(0, 1).to(DEV).contiguous()
    plan = LKBallPlan(coords, water_static=wa, score_static=sa)
    W = plan.waters(coords)
    E, _ = plan.forward(coords, W)
    ones = torch.ones(4, 64, device=DEV)
    E1, g1 = plan.energy_and_gradient(coords, ones)
    E_close(E1.cpu().numpy(), E.cpu().numpy(), rtol=1e-5, atol=1e-4)
    # Poses sit up to 3000 A from the origin, where a float32 coordinate is
    # good to 2.4e-4 A: the absolute float32 waters (the reference API's
    # water tensor) round by up to 1.2e-4 A, and the steep occlusion terms
    # carry that into the gradient (the reference's own float32 ops land up
    # to 0.014 kcal/mol/A from float64 here, 1677 components outside the
    # bar).  So the waters are checked on their own, and the scoring and its
    # adjoint against the oracle in float64 evaluated on this path's float32
    # waters, where the bar holds
    Wo, _, _, _ = oracle_run(ps, lterm, False)
    # a few float32 roundings at the waters' magnitude (2.4e-4 A at 3000 A)
    W_close(W.cpu().numpy(), Wo, 4 * float(numpy.spacing(numpy.float32(numpy.nanmax(numpy.abs(Wo))))))
    oc = O.OracleCall(ps.coords.flatten(0, 1).double(), score_args(ps, lterm, None), f64=True, term="lkball",
                      lkb_water_args=water_gen_args(ps, lterm))
    Eo, dxo, _ = oc.lkb_scores(W.cpu().double().numpy(), weights=numpy.ones((4, ps.n_poses)))
    E_close(E.cpu().numpy(), Eo, what="LK-ball 64x150 energies (oracle on these waters)")
    # the gradient also runs through the waters' adjoint, whose frames come
    # from float32 coordinates at that magnitude: the float32 band (one
    # component of 491 904 lies between the single and the doubled band)
    g_close_f32(g1.cpu().numpy(), dxo, what="LK-ball 64x150 gradient (oracle on these waters)")
    Ebp, _ = plan.forward(coords, W, block_pair=True)
    E_close(Ebp.sum(dim=(2, 3)).cpu().numpy(), E.cpu().numpy(), rtol=1e-5, atol=1e-3)
    shift = torch.tensor([3.1, -2.2, 5.7], device=DEV)
    Es, _ = plan.energy_and_gradient(coords + shift, ones)
    E_close(Es.cpu().numpy(), E1.cpu().numpy(), rtol=1e-4, atol=1e-3)
    w1 = torch.rand(4, 64, device=DEV, generator=torch.Generator(device=DEV).manual_seed(1))
    w2 = torch.rand(4, 64, device=DEV, generator=torch.Generator(device=DEV).manual_seed(2))
    _, ga = plan.energy_and_gradient(coords, w1)
    _, gb = plan.energy_and_gradient(coords, w2)
    _, gab = plan.energy_and_gradient(coords, w1 + w2)
    g_close_f32(gab.cpu().numpy(), (ga + gb).cpu().numpy())
