"""The oracle over the full benchmark batches, for the full-size parity tests.

Poses never interact (no term couples two poses), so the oracle scores a
large batch as chunks of poses, each chunk its own PoseStack built from the
same per-pose topologies and coordinate arrays as the GPU's stack (identical
float32 values: the placement on the grid happens once, before chunking).
Chunks go to a process pool started with `spawn` (safe after the parent has
used the GPU); sorting poses by size keeps each chunk's dense bond-separation
tensor small.  Test infrastructure only.
"""

import concurrent.futures
import multiprocessing
import os

import numpy


def _score_chunk(payload):
    import torch

    from oracle import oracle as O
    from tmol_b200.pose.builder import build_pose_stack
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args

    topos, coords, weight_sets, f64, soft = payload
    torch.set_num_threads(1)
    ps = build_pose_stack(topos, coords)
    term = LJLKEnergyTerm()
    if soft:
        term.set_options({"soft_rep": True})
    flat = ps.coords.flatten(0, 1)
    oc = O.OracleCall(flat.double() if f64 else flat, pose_score_args(ps, term), f64=f64)
    E, dV, _ = oc.pose_scores(require_gradient=True)
    pose = ps.pose_ind_for_atom.numpy()
    gs = []
    for w in weight_sets:
        w = numpy.asarray(w, dtype=numpy.float64)
        g = (dV.astype(numpy.float64) * w[:, pose][:, :, None]).sum(0)
        gs.append(g.reshape(ps.n_poses, -1, 3))
    return E.astype(numpy.float64), gs


def oracle_energies_and_gradient(topos, coords, weight_sets, f64=True, soft=False, chunk=16, workers=None):
    """Per-pose energies [3, P] and, for each [3, P] array w of
    `weight_sets`, the gradient of sum_t,p w[t, p] E[t, p] as
    [P, max atoms, 3] (float64 arrays), for poses given as topologies and
    [n_atoms, 3] coordinate arrays."""
    P = len(topos)
    n_atoms = [len(c) for c in coords]
    order = numpy.argsort(n_atoms, kind="stable")
    weight_sets = [numpy.asarray(w, dtype=numpy.float64) for w in weight_sets]
    jobs = []
    for c0 in range(0, P, chunk):
        idx = order[c0 : c0 + chunk]
        ws = [w[:, idx] for w in weight_sets]
        jobs.append((idx, ([topos[k] for k in idx], [coords[k] for k in idx], ws, f64, soft)))
    workers = workers or max(1, min(len(jobs), (os.cpu_count() or 2) - 1, 16))
    if workers > 1 and len(jobs) > 1:
        ctx = multiprocessing.get_context("spawn")
        with concurrent.futures.ProcessPoolExecutor(max_workers=workers, mp_context=ctx) as ex:
            results = list(ex.map(_score_chunk, [j[1] for j in jobs]))
    else:
        results = [_score_chunk(j[1]) for j in jobs]
    E = numpy.zeros((3, P))
    gs = [numpy.zeros((P, max(n_atoms), 3)) for _ in weight_sets]
    for (idx, _), (Ec, gcs) in zip(jobs, results):
        E[:, idx] = Ec
        for g, gc in zip(gs, gcs):
            for q, k in enumerate(idx):
                g[k, : gc.shape[1]] = gc[q]
    return E, gs
