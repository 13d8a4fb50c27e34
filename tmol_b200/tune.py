"""Autotuner for the scoring kernel's launch shape and work order.

The tunables are the fields of ``tmol_b200_ljlk_launch`` (work items per
ticket, warps per CTA, CTAs per SM, candidate blocks per work item) and the
order of the work items (longest-first by measured cost, see
``LJLKPlan.rebalance``).  Each candidate shape is timed with the library's
CUDA events around the scoring kernel; the winner is cached in a JSON file
keyed by GPU name and a signature of the workload (poses, rows, mean block
size), so a later plan for a similar PoseStack starts from it.

Cache file: ``$TMOL_B200_TUNE_CACHE`` or ``~/.cache/tmol_b200/launch.json``.
"""

import itertools
import json
import os

import torch

DEFAULT_GRID = {
    "rows_per_item": (1, 2),
    "warps_per_cta": (4, 8),
    "ctas_per_sm": (2, 3, 4),
    "candidates_per_item": (32, 64, 128),
}


def _cache_path():
    return os.environ.get("TMOL_B200_TUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "tmol_b200", "launch.json"
    )


def signature(plan, mean_block_atoms):
    name = torch.cuda.get_device_name(plan.device)
    term = getattr(plan, "NAME", "LJ/LK")
    return f"{name}|{term}|P={plan.n_poses}|B={plan.max_n_blocks}|atoms/block={mean_block_atoms:.0f}|{plan.dtype}"


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


def autotune(plan, run, grid=None, reps=5, mean_block_atoms=16.0, use_cache=True, verbose=False):
    """Pick the fastest launch shape for `run` (a closure making one scoring
    call on `plan`), leave it set, rebalance the work order, and return
    (shape, milliseconds)."""
    key = signature(plan, mean_block_atoms)
    cache = _load_cache() if use_cache else {}
    if key in cache:
        shape = tuple(cache[key]["shape"])
        plan.set_launch(*shape)
        run()
        plan.rebalance()
        return shape, time_kernel(plan, run, reps)
    grid = grid or DEFAULT_GRID
    results = []
    for shape in itertools.product(*(grid[k] for k in DEFAULT_GRID)):
        plan.set_launch(*shape)
        run()
        plan.rebalance()
        run()
        ms = time_kernel(plan, run, reps)
        results.append((ms, shape))
        if verbose:
            print(f"  launch {shape}: {ms * 1e3:.1f} us")
    results.sort()
    ms, shape = results[0]
    plan.set_launch(*shape)
    run()
    plan.rebalance()
    if use_cache:
        cache[key] = {"shape": list(shape), "ms": ms}
        _store_cache(cache)
    return shape, ms
