"""Train the block-pair screen on the GPU and measure what it buys.

    python -m tmol_b200.screen.train --out DIR [--train-poses 2000] ...

1. Labels: synthetic proteins (residue counts uniform in [50, 1000], chis
   perturbed by N(0, 20 deg)) are scored in block-pair mode by the plain
   kernel; every screen candidate (a neighbouring, non-count-pair block pair)
   gets label log10(|E_atr| + |E_rep| + |E_lk| + 1e-6).
2. Training: pinball loss at quantile tau, Adam, all on the library's BF16
   kernels.
3. Calibration: on validation poses of the test size (other seeds), the
   largest threshold whose worst per-pose |dE| (each term and the
   beta2016-weighted total, from the pairs' block-pair energies) stays
   within half the error budget.
4. Evaluation on held-out poses (16 x 1000 residues): skipped fraction,
   per-pose |dE| of the screened kernel against the plain one (both run),
   and the time of one energy + gradient evaluation, plain against screened
   (screen update included, and with the mask reused), each replayed from a
   captured CUDA graph with L2 flushed between replays.  The same numbers
   for the sphere-gap rule (skip when the sphere gap exceeds a calibrated
   distance), the exact sub-sphere rule (skip when no pair of sub-spheres is
   within reach) and the exact zero-energy mask (the labels themselves: the
   most any block-pair screen can skip) show what the network adds.

Writes ``screen_weights.npz`` and ``screen_results.json`` into DIR.
"""

import argparse
import concurrent.futures as cf
import json
import math
import multiprocessing
import os
import time

import numpy
import torch

from ..chem.restypes import default_packed_block_types
from ..pose.builder import build_pose_stack
from ..pose.synthetic import synthetic_topologies_and_coords
from ..score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args
from ..score.ljlk_op import LJLKPlan
from .mlp import ScreenMLP
from .screen import BlockPairScreen, block_pair_labels

BETA2016 = (1.0, 0.55, 1.0)


def _host_chunk(job):
    sizes, seeds, chi_sd = job
    return synthetic_topologies_and_coords(sizes, seeds, extra_chi_sd=chi_sd)


def chunk_jobs(sizes, seeds, chi_sd, max_residues=48000, max_poses=64):
    """Poses sorted by size, grouped so that a chunk's padded block count
    stays close to its poses' own."""
    order = numpy.argsort(sizes, kind="stable")
    jobs, cur, tot = [], [], 0
    for k in order:
        if cur and (len(cur) == max_poses or tot + sizes[k] > max_residues):
            jobs.append(cur)
            cur, tot = [], 0
        cur.append(int(k))
        tot += sizes[k]
    if cur:
        jobs.append(cur)
    return [([int(sizes[k]) for k in ks], [int(seeds[k]) for k in ks], chi_sd) for ks in jobs], jobs


def pose_chunks(sizes, seeds, chi_sd, device, workers):
    """Yields (pose indices, PoseStack on device) chunk by chunk; the host
    geometry is built by a spawn-started process pool."""
    jobs, index = chunk_jobs(sizes, seeds, chi_sd)
    pbt = default_packed_block_types(device)
    if workers > 1:
        ctx = multiprocessing.get_context("spawn")
        with cf.ProcessPoolExecutor(max_workers=workers, mp_context=ctx) as pool:
            for ks, (topos, coords) in zip(index, pool.map(_host_chunk, jobs)):
                yield ks, build_pose_stack(topos, coords, pbt=pbt, device=device)
    else:
        for ks, job in zip(index, jobs):
            topos, coords = _host_chunk(job)
            yield ks, build_pose_stack(topos, coords, pbt=pbt, device=device)


def collect(sizes, seeds, chi_sd, term, device, workers, keep_energies=False, log=print):
    """Screen candidates of all poses with labels (and energies): a dict of
    device tensors; ``pose`` is each candidate's index into ``sizes``."""
    out = {k: [] for k in ("features", "bt", "label", "energies", "pose")}
    t0 = time.time()
    n_res = 0
    for ks, ps in pose_chunks(sizes, seeds, chi_sd, device, workers):
        static = pose_score_args(ps, term)[:-1]
        coords = ps.coords.flatten(0, 1).contiguous()
        plan = LJLKPlan(coords, static)
        cap = max(1024, 64 * plan.n_poses * plan.max_n_blocks)
        cand, n, e, label = block_pair_labels(plan, coords, cap)
        out["features"].append(cand["features"][:n].clone())
        out["bt"].append(cand["bt"][:n].clone())
        out["label"].append(label)
        if keep_energies:
            out["energies"].append(e)
        pose_of_row = torch.tensor(ks, dtype=torch.int64, device=device)
        out["pose"].append(pose_of_row[cand["row"][:n].long() // plan.max_n_blocks])
        n_res += sum(sizes[k] for k in ks)
        del plan, ps, cand
    data = {k: torch.cat(out[k]) for k in ("features", "bt", "label", "pose")}
    data["energies"] = torch.cat(out["energies"], dim=1) if keep_energies else None
    log(f"collected {data['label'].shape[0]} candidate pairs from {len(sizes)} poses "
        f"({n_res} residues) in {time.time() - t0:.1f} s")
    return data


def train(mlp, data, epochs, batch, lr, tau, log=print, seed=0):
    N = data["label"].shape[0]
    steps_per_epoch = max(1, N // batch)
    total = epochs * steps_per_epoch
    g = torch.Generator(device=mlp.device).manual_seed(seed)
    step = 0
    hist = []
    t0 = time.time()
    for ep in range(epochs):
        perm = torch.randperm(N, device=mlp.device, generator=g)
        run = torch.zeros((), device=mlp.device)
        for i in range(steps_per_epoch):
            idx = perm[i * batch:(i + 1) * batch]
            mlp.forward(data["features"][idx].contiguous(), data["bt"][idx].contiguous())
            run += mlp.loss_and_backward(data["label"][idx].contiguous(), tau)[0]
            # cosine decay to 5% of the initial rate
            rate = lr * (0.05 + 0.95 * 0.5 * (1 + math.cos(math.pi * step / total)))
            mlp.adam(rate)
            step += 1
        hist.append(float(run.item()) / steps_per_epoch)
        log(f"epoch {ep}: mean pinball loss {hist[-1]:.4f} ({time.time() - t0:.1f} s)")
    return hist


def predictions(mlp, data, chunk=1 << 20):
    n = data["label"].shape[0]
    out = torch.empty(n, device=mlp.device)
    for i in range(0, n, chunk):
        j = min(n, i + chunk)
        out[i:j] = mlp.forward(data["features"][i:j].contiguous(), data["bt"][i:j].contiguous())
    return out


def per_pose_error(score, energies, pose, pose_scale, thresholds):
    """Worst per-pose |dE| (max over the three terms and the weighted total,
    pose p's error multiplied by pose_scale[p]) when the candidates with
    score < t are skipped, for each t."""
    w = torch.tensor(BETA2016, device=energies.device).view(3, 1)
    e4 = torch.cat([energies, (energies * w).sum(0, keepdim=True)]).double()
    scale = torch.as_tensor(pose_scale, dtype=torch.float64, device=energies.device)
    worst, frac = [], []
    for t in thresholds:
        skip = score < t
        dE = torch.zeros((4, scale.shape[0]), dtype=torch.float64, device=energies.device)
        dE.index_add_(1, pose[skip], e4[:, skip])
        worst.append(float((dE.abs() * scale).max().item()))
        frac.append(float(skip.float().mean().item()))
    return numpy.array(worst), numpy.array(frac)


def calibrate(score, energies, pose, n_poses, budget, max_fraction=0.7, n_grid=281):
    """Largest threshold t, among quantiles of `score` up to max_fraction,
    such that every smaller one keeps the worst per-pose |dE| within
    budget.  Returns (t, worst |dE|, skipped fraction)."""
    qs = torch.linspace(0.0, max_fraction, n_grid, device=score.device, dtype=torch.float64)
    ts = torch.quantile(score.double(), qs).cpu().numpy()
    ts[0] = -numpy.inf
    worst, frac = per_pose_error(score, energies, pose, [1.0] * n_poses, ts)
    bad = numpy.nonzero(worst > budget)[0]
    k = (int(bad[0]) - 1) if len(bad) else n_grid - 1
    k = max(k, 0)
    return float(ts[k]), float(worst[k]), float(frac[k])


def pack_mask(skip_dense):
    """Bool [rows, B] -> int32 [rows, ceil(B/32)] skip words."""
    rows, B = skip_dense.shape
    W = (B + 31) // 32
    pad = torch.zeros((rows, W * 32), dtype=torch.int64, device=skip_dense.device)
    pad[:, :B] = skip_dense.long()
    bits = pad.view(rows, W, 32) << torch.arange(32, device=skip_dense.device)
    words = bits.sum(-1)
    words = torch.where(words >= 2**31, words - 2**32, words)
    return words.to(torch.int32).contiguous()


def time_graph(fn, reps, flush, warmup=3):
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(warmup):
            fn()
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    ms = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(warmup):
        g.replay()
    for _ in range(reps):
        flush.zero_()
        e0.record()
        g.replay()
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    del g
    return float(numpy.median(ms))


def evaluate(mlp, threshold, gap_threshold, sizes, seeds, chi_sd, term, device, reps, log=print):
    """Plain against screened scoring on one batch of held-out poses.

    |dE| is measured three ways: in float64 (a float64 plan run with and
    without the mask: the error the screen introduces), as the float64 sum
    of the skipped pairs' block-pair energies (the same quantity, from the
    labels) and in float32 (dominated by the order of the atomic per-pose
    sums at these energies; the plain kernel run twice gives that floor)."""
    (ks, ps), = list(pose_chunks(sizes, seeds, chi_sd, device, 1))
    static = pose_score_args(ps, term)[:-1]
    coords = ps.coords.flatten(0, 1).contiguous()
    plan = LJLKPlan(coords, static)
    coords64 = coords.double()
    plan64 = LJLKPlan(coords64, static)
    P, B = plan.n_poses, plan.max_n_blocks
    weights = torch.tensor(BETA2016, device=device).view(3, 1).repeat(1, P).contiguous()
    w64 = weights.double()
    flush = torch.empty(64 << 20, dtype=torch.float32, device=device)  # 256 MB > L2
    E = torch.empty((3, P), device=device)
    dx = torch.empty_like(coords)

    plan.set_skip_mask(None)
    cand, n, e, label = block_pair_labels(plan, coords, 64 * P * B)
    E0, g0 = (t.clone() for t in plan.energy_and_gradient(coords, weights))
    plan.set_counting(True)
    E0b, _ = plan.energy_and_gradient(coords, weights)
    counts0 = plan.last_counts()
    plan.set_counting(False)
    E64_0, g64_0 = (t.clone() for t in plan64.energy_and_gradient(coords64, w64))
    rows = cand["row"][:n].long()
    b2 = cand["b2"][:n].long()
    pose = rows // B

    def step():
        plan.energy_and_gradient(coords, weights, energies=E, dcoords=dx)

    zero = label <= math.log10(1.5e-6)
    res = {
        "poses": P, "residues": int(sum(sizes)), "candidates": n,
        "neighbour_block_pairs": int(counts0["block_pairs"]),
        "zero_energy_candidates": int(zero.sum().item()),
        "max_abs_E_per_pose": float(E64_0.abs().max().item()),
        "fp32_noise_floor_abs_dE": float((E0 - E0b).abs().max().item()),
    }
    plain_ms = time_graph(step, reps, flush)
    res["plain_ms"] = plain_ms

    def report(name, mask, skipped, update=None):
        plan.set_skip_mask(mask)
        plan64.set_skip_mask(mask)
        if update is not None:
            update()
        plan.set_counting(True)
        E1, g1 = plan.energy_and_gradient(coords, weights)
        counts = plan.last_counts()
        plan.set_counting(False)
        E64_1, g64_1 = plan64.energy_and_gradient(coords64, w64)
        d64 = E64_1 - E64_0
        tot64 = (d64 * w64).sum(0)
        d32 = (E1 - E0).double()
        # the same error from the labels: sum of the skipped pairs' energies
        lab = torch.zeros((3, P), dtype=torch.float64, device=device)
        lab.index_add_(1, pose[skipped], e[:, skipped].double())
        r = {
            "skipped_block_pairs": int(counts0["block_pairs"] - counts["block_pairs"]),
            "skipped_fraction_of_candidates": (counts0["block_pairs"] - counts["block_pairs"]) / max(n, 1),
            "max_abs_dE_f64_per_term": [float(v) for v in d64.abs().max(1).values],
            "max_abs_dE_f64_total": float(tot64.abs().max().item()),
            "max_abs_dE_from_pair_energies": float(lab.abs().max().item()),
            "max_abs_dgrad_f64": float((g64_1 - g64_0).abs().max().item()),
            "max_abs_dE_f32_total": float((d32 * w64).sum(0).abs().max().item()),
            "atom_pairs_in_range_skipped": int(counts0["atom_pairs_in_range"] - counts["atom_pairs_in_range"]),
            "kernel_only_ms": time_graph(step, reps, flush),
        }
        if update is not None:
            def step_with_update():
                update()
                step()

            r["with_update_ms"] = time_graph(step_with_update, reps, flush)
            r["update_ms"] = time_graph(update, reps, flush)
            r["speedup_with_update"] = plain_ms / r["with_update_ms"]
        r["speedup_kernel_only"] = plain_ms / r["kernel_only_ms"]
        plan.set_skip_mask(None)
        plan64.set_skip_mask(None)
        log(f"{name}: {json.dumps(r)}")
        return r

    def dense(skip):
        d = torch.zeros((P * B, B), dtype=torch.bool, device=device)
        d[rows[skip], b2[skip]] = True
        return pack_mask(d)

    screen = BlockPairScreen(mlp, plan, threshold, capacity=64 * P * B)
    pred = mlp.forward(cand["features"][:n].contiguous(), cand["bt"][:n].contiguous()).clone()
    res["learned"] = report("learned", screen.mask, pred < threshold, update=lambda: screen.update(coords))
    res["learned"]["threshold"] = threshold
    gap = cand["features"][:n, 1] * 6.0
    res["sphere_gap_rule"] = report("sphere_gap_rule", dense(gap > gap_threshold), gap > gap_threshold)
    res["sphere_gap_rule"]["gap_threshold_A"] = gap_threshold
    # exact geometric rule: no sub-sphere pair within reach, so no atom pair
    # either (zero error by construction)
    sub_gap = cand["features"][:n, 8:12].min(1).values * 6.0
    far = sub_gap >= 6.0
    res["sub_sphere_rule"] = report("sub_sphere_rule", dense(far), far)
    res["exact_zero_mask"] = report("exact_zero_mask", dense(zero), zero)
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--out", required=True)
    ap.add_argument("--train-poses", type=int, default=2000)
    ap.add_argument("--val-poses", type=int, default=48)
    ap.add_argument("--val-residues", type=int, default=1000)
    ap.add_argument("--test-poses", type=int, default=16)
    ap.add_argument("--test-residues", type=int, default=1000)
    ap.add_argument("--min-res", type=int, default=50)
    ap.add_argument("--max-res", type=int, default=1000)
    ap.add_argument("--chi-sd", type=float, default=20.0)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--tau", type=float, default=0.999)
    ap.add_argument("--budget", type=float, default=0.01, help="per-pose |dE| budget, kcal/mol")
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--workers", type=int, default=min(16, os.cpu_count() or 1))
    ap.add_argument("--weights", default=None, help="skip training, evaluate these weights")
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args(argv)
    os.makedirs(args.out, exist_ok=True)
    device = torch.device("cuda:0")
    torch.cuda.set_device(device)
    term = LJLKEnergyTerm(device=device)
    pbt = default_packed_block_types(device)
    n_bt = len(pbt.active_block_types)
    log_lines = []

    def log(msg):
        print(msg, flush=True)
        log_lines.append(msg)

    rng = numpy.random.default_rng(20240601 + args.seed)
    res = {"config": vars(args)}
    t_start = time.time()
    mlp = ScreenMLP(n_bt, device, seed=args.seed)
    if args.weights:
        st = dict(numpy.load(args.weights, allow_pickle=False))
        mlp.load_state_dict(st)
    else:
        sizes = [int(v) for v in rng.integers(args.min_res, args.max_res + 1, args.train_poses)]
        seeds = [10_000_000 + k for k in range(args.train_poses)]
        data = collect(sizes, seeds, args.chi_sd, term, device, args.workers, log=log)
        res["train_pairs"] = int(data["label"].shape[0])
        res["train_zero_fraction"] = float((data["label"] <= math.log10(1.5e-6)).float().mean().item())
        t0 = time.time()
        res["loss_history"] = train(mlp, data, args.epochs, args.batch, args.lr, args.tau, log=log, seed=args.seed)
        torch.cuda.synchronize()
        res["train_seconds"] = time.time() - t0
        del data
    # calibration on validation poses
    # validation poses of the test poses' size, other seeds; half the budget
    vsizes = [args.val_residues] * args.val_poses
    vseeds = [20_000_000 + k for k in range(args.val_poses)]
    val = collect(vsizes, vseeds, args.chi_sd, term, device, args.workers, keep_energies=True, log=log)
    vpred = predictions(mlp, val)
    half = 0.5 * args.budget
    thr, worst, frac = calibrate(vpred, val["energies"], val["pose"], len(vsizes), half)
    gap = val["features"][:, 1] * 6.0
    gthr_neg, gworst, gfrac = calibrate(-gap, val["energies"], val["pose"], len(vsizes), half)
    gap_thr = -gthr_neg
    res["validation"] = {
        "pairs": int(val["label"].shape[0]),
        "learned": {"threshold": thr, "worst_abs_dE": worst, "skipped_fraction": frac},
        "sphere_gap_rule": {"gap_threshold_A": gap_thr, "worst_abs_dE": gworst, "skipped_fraction": gfrac},
        "zero_fraction": float((val["label"] <= math.log10(1.5e-6)).float().mean().item()),
    }
    log(f"validation: {json.dumps(res['validation'])}")
    del val
    state = mlp.state_dict()
    numpy.savez(
        os.path.join(args.out, "screen_weights.npz"),
        threshold=numpy.float32(thr),
        tau=numpy.float32(args.tau),
        gap_threshold=numpy.float32(gap_thr),
        block_type_names=numpy.array([bt.name for bt in pbt.active_block_types]),
        **state,
    )
    # held-out evaluation
    tsizes = [args.test_residues] * args.test_poses
    tseeds = [30_000_000 + k for k in range(args.test_poses)]
    res["test"] = evaluate(mlp, thr, gap_thr, tsizes, tseeds, args.chi_sd, term, device, args.reps, log=log)
    res["wall_seconds"] = time.time() - t_start
    res["device"] = torch.cuda.get_device_name(device)
    with open(os.path.join(args.out, "screen_results.json"), "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps({"test": res["test"], "validation": res["validation"]}))


if __name__ == "__main__":
    main()
