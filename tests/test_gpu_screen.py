"""GPU checks of the learned block-pair screen.

- the BF16 tensor-core GEMM against an fp32 matmul of the same bf16 values;
- candidate enumeration and features against the NumPy oracle (the
  candidate set bit-exact, features to fp32 rounding of coordinates that lie
  up to ~1e3 A from the origin);
- the skip mask's meaning: scoring with a mask equals the plain block-pair
  energies summed over the pairs left in (the diagonal and count-pair
  partners are never left out), and the gradient equals the C oracle's
  adjoint over the same pairs;
- a training step's gradients against the NumPy oracle (bf16 rounding
  emulated), fused inference against the training forward pass, and a short
  training run that lowers the loss.

Energies: 1e-5 relative / 1e-3 absolute; gradients: 1e-4 relative to the
largest component; network gradients: 2e-2 relative in norm (bf16 rounding
of activations flips with fp32 summation order).
"""

import ctypes

import numpy
import pytest
import torch

from oracle import oracle as O
from oracle import screen_mlp as SM
from tmol_b200.pose.synthetic import synthetic_pose_stack
from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args
from tmol_b200.score.ljlk_op import LJLKPlan
from tmol_b200.screen import BlockPairScreen, ScreenMLP, block_pair_labels

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def bf16(x):
    return x.to(torch.bfloat16)


def gemm(A, a_rs, a_cs, B, b_rs, b_cs, M, N, K, **kw):
    st = ctypes.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)
    ScreenMLP._gemm(st, A, a_rs, a_cs, B, b_rs, b_cs, M, N, K, **kw)


@pytest.mark.parametrize("M,N,K", [(1000, 128, 32), (70, 50, 33), (5, 128, 128), (257, 1, 128)])
def test_gemm_matches_fp32_matmul(M, N, K):
    g = torch.Generator(device=DEV).manual_seed(M + N + K)
    A = bf16(torch.randn(M, K, device=DEV, generator=g))
    W = bf16(torch.randn(N, K, device=DEV, generator=g))
    bias = torch.randn(N, device=DEV, generator=g)
    C = torch.empty(M, N, device=DEV)
    Cb = torch.empty(M, N, device=DEV, dtype=torch.bfloat16)
    gemm(A, K, 1, W, 1, K, M, N, K, C=C, c_rs=N, Cb=Cb, cb_rs=N, bias=bias, relu=True)
    ref = torch.relu(A.float() @ W.float().T + bias)
    torch.testing.assert_close(C, ref, rtol=1e-5, atol=1e-5 * K**0.5)
    # bf16 output: within one bf16 rounding of the fp32 result
    assert ((Cb.float() - ref).abs() <= ref.abs() * 2**-8 + 1e-6).all()


def test_gemm_transposed_operands_and_split_k():
    g = torch.Generator(device=DEV).manual_seed(5)
    n, m, k = 5000, 128, 96
    dZ = bf16(torch.randn(n, m, device=DEV, generator=g))
    H = bf16(torch.randn(n, k, device=DEV, generator=g))
    C = torch.zeros(m, k, device=DEV)
    # C = dZ^T H with A(m, k) = dZ[k, m]
    gemm(dZ, 1, m, H, k, 1, m, k, n, C=C, c_rs=k, accumulate=True, k_split=8)
    ref = dZ.float().T @ H.float()
    torch.testing.assert_close(C, ref, rtol=1e-4, atol=1e-4 * n**0.5)
    # accumulate adds onto what is there
    gemm(dZ, 1, m, H, k, 1, m, k, n, C=C, c_rs=k, accumulate=True, k_split=3)
    torch.testing.assert_close(C, 2 * ref, rtol=1e-4, atol=2e-4 * n**0.5)


def _plan(sizes, seeds, chi_sd=20.0):
    term = LJLKEnergyTerm(device=DEV)
    ps = synthetic_pose_stack(sizes, seeds, device=DEV, extra_chi_sd=chi_sd)
    args = pose_score_args(ps, term)
    coords = ps.coords.flatten(0, 1).contiguous()
    return LJLKPlan(coords, args[:-1]), coords, ps, args


@pytest.fixture(scope="module")
def small():
    return _plan([60, 45, 80], [501, 502, 503])


def test_candidates_match_oracle(small):
    plan, coords, ps, args = small
    cand = plan.screen_candidates(coords, 100000)
    n = int(cand["count"].item())
    oc = O.OracleCall(coords.cpu(), [a.cpu() if isinstance(a, torch.Tensor) else a for a in args])
    _, _, nbr = oc.pose_scores()
    P, B = plan.n_poses, plan.max_n_blocks
    row = cand["row"][:n].cpu().numpy()
    b2 = cand["b2"][:n].cpu().numpy()
    feats = cand["features"][:n].cpu().numpy()
    bt = cand["bt"][:n].cpu().numpy()
    got = {(int(r), int(b)): k for k, (r, b) in enumerate(zip(row, b2))}
    assert len(got) == n
    X = coords.cpu().numpy()
    block_type = args[3].cpu().numpy()
    offsets = args[0].cpu().numpy().reshape(P, B)
    minsep = args[12].cpu().numpy()
    bt_n_atoms = args[14].cpu().numpy()
    n_expected = 0
    for p in range(P):
        pairs, f = SM.candidate_features(X, block_type[p], offsets[p], bt_n_atoms, nbr[p], minsep[p], p)
        n_expected += len(pairs)
        for (b1, bb2), fe in zip(pairs, f):
            k = got[(p * B + int(b1), int(bb2))]
            # poses sit up to ~1e3 A from the origin: fp32 centroids carry
            # ~1e-4 A of rounding, features are distances / 5
            numpy.testing.assert_allclose(feats[k], fe, rtol=1e-4, atol=1e-4)
            assert tuple(bt[k]) == (block_type[p, b1], block_type[p, bb2])
    assert n == n_expected


def _dense_skip(mask, P, B):
    words = mask.shape[1]
    m = mask.cpu().numpy().view(numpy.uint32).reshape(P, B, words)
    bits = (m[..., :, None] >> numpy.arange(32, dtype=numpy.uint32)) & 1
    return bits.reshape(P, B, words * 32)[..., :B].astype(bool)


def test_skip_mask_leaves_out_exactly_the_masked_pairs(small):
    plan, coords, ps, args = small
    P, B = plan.n_poses, plan.max_n_blocks
    plan.set_skip_mask(None)
    Ebp, nbr = plan.forward(coords, block_pair=True)
    E0, _ = plan.forward(coords)
    g = torch.Generator(device=DEV).manual_seed(9)
    mask = torch.randint(-(2**31), 2**31 - 1, (P * B, plan.skip_mask_words()), generator=g, device=DEV,
                         dtype=torch.int32)
    skip = _dense_skip(mask, P, B)
    minsep = args[12].cpu().numpy()
    eye = numpy.eye(B, dtype=bool)[None]
    effective = skip & ~eye & ~(minsep <= 4)
    keep = torch.tensor(~effective, device=DEV)
    Ebp_np = Ebp.cpu().numpy()
    expected = (Ebp_np * (~effective)[None]).sum((2, 3))
    plan.set_skip_mask(mask)
    try:
        E1, _ = plan.forward(coords)
        numpy.testing.assert_allclose(E1.cpu().numpy(), expected, rtol=1e-5, atol=1e-3)
        assert (E1 != E0).any()
        Ebp1, nbr1 = plan.forward(coords, block_pair=True)
        numpy.testing.assert_allclose(Ebp1.cpu().numpy(), Ebp_np * (~effective)[None], rtol=1e-5, atol=1e-5)
        # the neighbour matrix still reports the sphere test
        assert torch.equal(nbr1, nbr)
        w = torch.rand((3, P), device=DEV, generator=g)
        E2, dx = plan.energy_and_gradient(coords, w)
        numpy.testing.assert_allclose(E2.cpu().numpy(), expected, rtol=1e-5, atol=1e-3)
        oc = O.OracleCall(coords.cpu(), [a.cpu() if isinstance(a, torch.Tensor) else a for a in args])
        nbr_kept = (nbr & keep).cpu().numpy()
        ref = oc.backward(nbr_kept, w.cpu().numpy(), per_pose_weights=True)
        scale = numpy.abs(ref).max()
        numpy.testing.assert_allclose(dx.cpu().numpy(), ref, rtol=1e-4, atol=1e-4 * scale)
    finally:
        plan.set_skip_mask(None)
    E3, _ = plan.forward(coords)
    # per-pose sums are accumulated atomically: equal up to summation order
    torch.testing.assert_close(E3, E0, rtol=1e-6, atol=1e-6)


def _random_rows(n, nbt, seed):
    g = torch.Generator(device=DEV).manual_seed(seed)
    feats = torch.randn(n, 12, device=DEV, generator=g)
    bt = torch.randint(0, nbt, (n, 2), device=DEV, generator=g, dtype=torch.int32)
    return feats, bt


def test_training_step_gradients_match_oracle():
    nbt = 23
    mlp = ScreenMLP(nbt, DEV, seed=3)
    with torch.no_grad():
        for k in ("b1", "b2", "b3"):
            mlp.params[k].normal_(0, 0.1)
    feats, bt = _random_rows(700, nbt, 4)
    pred = mlp.forward(feats, bt).clone()
    net = SM.MLP(mlp.state_dict(), bf16=True)
    pred_o = net.forward(feats.cpu().numpy(), bt.cpu().numpy())
    scale = numpy.abs(pred_o).max() + 1
    numpy.testing.assert_allclose(pred.cpu().numpy(), pred_o, atol=2e-3 * scale, rtol=0)
    # targets well away from the predictions: the pinball gradient's sign is
    # then the same on both sides
    rng = numpy.random.default_rng(5)
    y = pred_o + rng.choice([-1.0, 1.0], len(pred_o)) * rng.uniform(0.2, 1.0, len(pred_o))
    tau = 0.9
    loss = mlp.loss_and_backward(torch.tensor(y, dtype=torch.float32, device=DEV), tau)
    loss_o, d = SM.pinball(pred_o, y, tau)
    assert float(loss.item()) == pytest.approx(loss_o, rel=1e-3)
    go = net.backward(d)
    for k, v in go.items():
        gk = mlp.grads[k].cpu().numpy().reshape(v.shape)
        err = numpy.linalg.norm(gk - v) / max(numpy.linalg.norm(v), 1e-12)
        assert err < 2e-2, (k, err)


def test_adam_step_matches_formula():
    mlp = ScreenMLP(5, DEV, seed=1)
    w0 = {k: v.clone() for k, v in mlp.params.items()}
    for k, g in mlp.grads.items():
        g.copy_(torch.linspace(-1, 1, g.numel(), device=DEV).view_as(g))
    mlp.adam(lr=1e-2, weight_decay=0.0)
    for k, w in mlp.params.items():
        gk = mlp.grads[k]
        m = 0.1 * gk
        v = 0.001 * gk * gk
        ref = w0[k] - 1e-2 * (m / 0.1) / ((v / 0.001).sqrt() + 1e-8)
        torch.testing.assert_close(w, ref, rtol=1e-5, atol=1e-6)
    torch.testing.assert_close(mlp.bf16["w2"], mlp.params["w2"].to(torch.bfloat16), rtol=0, atol=0)


def test_fused_inference_matches_training_forward(small):
    plan, coords, ps, args = small
    mlp = ScreenMLP(int(args[14].shape[0]), DEV, seed=7)
    with torch.no_grad():
        for k in ("b1", "b2", "b3"):
            mlp.params[k].normal_(0, 0.1)
    screen = BlockPairScreen(mlp, plan, threshold=0.0)
    screen.update(coords, keep_predictions=True)
    n = screen.n_candidates()
    assert n > 100
    fused = screen.pred[:n].clone()
    ref = mlp.forward(screen.cand["features"][:n], screen.cand["bt"][:n])
    torch.testing.assert_close(fused, ref, rtol=1e-3, atol=1e-3)
    # the mask holds exactly the candidates predicted below the threshold
    P, B = plan.n_poses, plan.max_n_blocks
    skip = _dense_skip(screen.mask, P, B)
    row = screen.cand["row"][:n].cpu().numpy()
    b2 = screen.cand["b2"][:n].cpu().numpy()
    below = (fused < 0.0).cpu().numpy()
    expect = numpy.zeros_like(skip)
    expect.reshape(P * B, B)[row[below], b2[below]] = True
    assert (skip == expect).all()
    assert screen.n_skipped() == int(below.sum())


def test_short_training_run_lowers_the_loss():
    plan, coords, ps, args = _plan([120, 150, 90, 200], [601, 602, 603, 604])
    cand, n, e, label = block_pair_labels(plan, coords, 200000)
    assert n > 1000
    mlp = ScreenMLP(int(args[14].shape[0]), DEV, seed=11)
    feats, bt = cand["features"][:n], cand["bt"][:n]
    g = torch.Generator(device=DEV).manual_seed(0)
    losses = []
    for step in range(300):
        idx = torch.randint(0, n, (1024,), device=DEV, generator=g)
        mlp.forward(feats[idx].contiguous(), bt[idx].contiguous())
        losses.append(float(mlp.loss_and_backward(label[idx].contiguous(), 0.9).item()))
        mlp.adam(lr=2e-3)
    first, last = numpy.mean(losses[:20]), numpy.mean(losses[-20:])
    assert last < 0.6 * first, (first, last)


def test_trained_screen_beats_the_sphere_gap_rule():
    """The shipped network against the geometric rule it refines, on poses
    none of its training, calibration or evaluation sets contain: it skips
    more than twice as many candidate pairs as the sphere-gap rule
    calibrated to the same budget, and the per-pose error it introduces
    (float64 plan, same mask) stays within 0.01 kcal/mol."""
    from tmol_b200.screen.screen import TRAINED_WEIGHTS

    st = numpy.load(TRAINED_WEIGHTS)
    gap_threshold = float(st["gap_threshold"])
    plan, coords, ps, args = _plan([1000] * 6, [40_000_000 + k for k in range(6)])
    names = [bt.name for bt in ps.packed_block_types.active_block_types]
    screen = BlockPairScreen.trained(plan, names)
    screen.update(coords)
    n = screen.n_candidates()
    learned = screen.n_skipped() / n
    gap = screen.cand["features"][:n, 1] * 6.0
    by_gap = float((gap > gap_threshold).float().mean().item())
    assert learned > 2 * by_gap, (learned, by_gap)
    c64 = coords.double()
    plan64 = LJLKPlan(c64, args[:-1])
    E0, _ = plan64.forward(c64, want_neighbors=False)
    E0 = E0.clone()
    plan64.set_skip_mask(screen.mask)
    E1, _ = plan64.forward(c64, want_neighbors=False)
    w = torch.tensor([1.0, 0.55, 1.0], dtype=torch.float64, device=DEV).view(3, 1)
    assert (E1 - E0).abs().max().item() <= 0.01
    assert ((E1 - E0) * w).sum(0).abs().max().item() <= 0.01
