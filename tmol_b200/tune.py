"""Autotuner for the scoring kernel's launch shape and work order.

The tunables are the fields of ``tmol_b200_ljlk_launch``: work items per
ticket, warps per CTA, CTAs per SM, candidate blocks per work item (how a
row's block pairs are partitioned into work items) and neighbouring blocks
per screening group (how many block pairs share one pass of a warp's 32
lanes: the kernel's "threads per block pair"); and the order of the work
items (longest-first by measured cost, see ``LJLKPlan.rebalance``).  Each
candidate shape is timed with the library's CUDA events around the scoring
kernel; the winner is cached in a JSON file keyed by GPU name and a
signature of the workload (poses, block slots, real blocks per pose and
the histogram of atoms per block), so a later plan for a similar PoseStack
starts from it.

Cache file: ``$TMOL_B200_TUNE_CACHE`` or ``~/.cache/tmol_b200/launch.json``.
"""

import itertools
import json
import os

import torch

DEFAULT_GRID = {
    "rows_per_item": (1, 2),
    # (warps per CTA, CTAs per SM): 16 warps per SM, the register limit at
    # 128 registers a thread (the LK-ball and rotamer kernels take at most
    # 8 warps per CTA)
    "cta_shape": ((4, 4), (8, 2), (16, 1)),
    "candidates_per_item": (32, 64, 128),
    "slots_per_group": (8, 12),
}


def launch_shapes(grid):
    """(items per ticket, warps per CTA, CTAs per SM, candidates per item,
    slots per group) of every grid point."""
    for rows, (warps, ctas), cands, slots in itertools.product(
        grid["rows_per_item"], grid["cta_shape"], grid["candidates_per_item"], grid["slots_per_group"]
    ):
        yield (rows, warps, ctas, cands, slots)

# atoms per block: histogram bin edges of the signature
SIZE_BINS = (8, 16, 24, 32)


def _cache_path():
    return os.environ.get("TMOL_B200_TUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "tmol_b200", "launch.json"
    )


def block_size_summary(plan):
    """(real blocks per pose, mean atoms per block, fraction of blocks per
    SIZE_BINS bin) of the plan's PoseStack, from its block types."""
    block_type, bt_n_atoms = plan.block_sizes
    bt = block_type.reshape(-1).to(torch.int64)
    real = bt >= 0
    n = bt_n_atoms.to(torch.int64)[bt.clamp(min=0)][real].float()
    if n.numel() == 0:
        return 0.0, 0.0, (0.0,) * (len(SIZE_BINS) + 1)
    edges = torch.tensor(SIZE_BINS, dtype=n.dtype, device=n.device)
    bins = torch.bucketize(n, edges, right=False)
    hist = torch.bincount(bins, minlength=len(SIZE_BINS) + 1).float() / n.numel()
    return float(n.numel()) / plan.n_poses, float(n.mean()), tuple(float(h) for h in hist.cpu())


def signature(plan):
    """The cache key: GPU, term, dtype, poses and block slots, and the
    block-size summary (real blocks per pose to the nearest 10, mean atoms
    per block to the nearest atom, the size histogram to the nearest 5 %)."""
    name = torch.cuda.get_device_name(plan.device)
    term = getattr(plan, "NAME", "LJ/LK")
    per_pose, mean_atoms, hist = block_size_summary(plan)
    h = ",".join(f"{round(20 * x) * 5}" for x in hist)
    return (
        f"{name}|{term}|{plan.dtype}|P={plan.n_poses}|B={plan.max_n_blocks}|"
        f"blocks/pose={10 * round(per_pose / 10)}|atoms/block={mean_atoms:.0f}|sizes%={h}"
    )


def _load_cache():
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _store_cache(cache):
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path + ".tmp", "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(path + ".tmp", path)
    except OSError:
        pass


def time_kernel(plan, run, reps=5):
    """Mean scoring-kernel milliseconds of `reps` calls of run()."""
    plan.profile(True)
    for _ in range(reps):
        run()
    ms, n = plan.profile_read()
    plan.profile(False)
    return ms / max(n, 1)


def autotune(plan, run, grid=None, reps=5, use_cache=True, verbose=False):
    """Pick the fastest launch shape for `run` (a closure making one scoring
    call on `plan`), leave it set, rebalance the work order, and return
    (shape, milliseconds)."""
    key = signature(plan)
    cache = _load_cache() if use_cache else {}
    if key in cache:
        shape = tuple(cache[key]["shape"])
        plan.set_launch(*shape)
        plan.balance(run)
        return shape, time_kernel(plan, run, reps)
    grid = grid or DEFAULT_GRID
    results = []
    for shape in launch_shapes(grid):
        plan.set_launch(*shape)
        plan.balance(run)
        run()
        ms = time_kernel(plan, run, reps)
        results.append((ms, shape))
        if verbose:
            print(f"  launch {shape}: {ms * 1e3:.1f} us")
    results.sort()
    ms, shape = results[0]
    plan.set_launch(*shape)
    plan.balance(run)
    if use_cache:
        cache[key] = {"shape": list(shape), "ms": ms}
        _store_cache(cache)
    return shape, ms
