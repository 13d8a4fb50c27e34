#!/usr/bin/env python
"""LJ + LK energy + gradient throughput on B200 (tmol's LJLK pose scoring).

Workload (one "step"): the uniform batch of 64 synthetic proteins x 150
residues (seeded; residues uniform over the 20 canonical amino acids, ideal
geometry from tmol's internal coordinates, 60% helix / 40% strand dihedrals,
rotameric chis), float32; per step, the per-pose LJ-attractive, LJ-repulsive
and LK energies and the gradient of their weighted sum with respect to every
coordinate (weights 1.0 / 0.55 / 1.0, tmol's beta2016 weights).

Arms:
  (default)         the B200 path: one fused energy + gradient pass per step
                    (sphere kernel + fused neighbour/atom-pair kernel),
                    replayed as a CUDA graph; inputs resident in HBM.
  --impl reference  tmol's own CPU implementation of the op (compiled from
                    its sources into oracle/_ref), on all host cores: one
                    process per core, each scoring a slice of the poses.

Other workloads (--workload): the uneven 256-pose batch, rotamer-pair
scoring (rotamers16x150), the elec term on the uniform batch (elec64x150:
per-pose fa_elec and the gradient of its sum) and PoseStack bond separation
(bondsep256: inter_block_bondsep and min_bondsep of the uneven batch from its
connectivity).  The default line also carries an "elec" summary measured on
the same batch.

Under torchrun each rank scores its own batch (independent seeds); the
timing is the maximum over ranks (weak scaling, no collective on the data
path).  Prints one JSON line (rank 0).
"""

import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

N_POSES = 64
N_RES = 150
TERM_WEIGHTS = (1.0, 0.55, 1.0)
METRIC = "LJ+LK energy+grad poses/s (64x150-residue batch, 1 B200)"
# the uneven batch: 256 poses, residue counts log-uniform in [20, 1000],
# coordinates perturbed by N(0, 0.05 A) inside every replayed step
UNEVEN_POSES = 256
UNEVEN_SEED = 2
PERTURB_SD = 0.05
UNEVEN_REPLAYS = 100  # graph replays of the uneven batch's sub-record
LAUNCH_FIELDS = ("items_per_ticket", "warps_per_cta", "ctas_per_sm", "candidates_per_item", "slots_per_group")
L2_FLUSH_BYTES = 256 << 20
# the rotamer workload: 16 poses x 150 residues, every block with 1..31
# rotamers (the native one first; chis resampled, a quarter mutated)
ROT_POSES = 16
ROT_RES = 150
ROT_SET = dict(max_rots=31, mutate_fraction=0.25, seed=9)
ROT_METRIC = "LJ+LK rotamer-pair energies/s (16 poses x 150 residues, 1-31 rotamers per block, 1 B200)"
ELEC_METRIC = "elec energy+grad poses/s (64x150-residue batch, 1 B200)"
LKBALL_METRIC = "LK-ball energy+grad poses/s (64x150-residue batch, waters included, 1 B200)"
LKB_ROT_METRIC = (
    "LK-ball rotamer-pair energies/s (16 poses x 150 residues, 1-31 rotamers per block, waters included, 1 B200)"
)
SFXN_METRIC = "score function (LJ/LK + elec + LK-ball) energy+grad poses/s (64x150-residue batch, 1 B200)"
# weights of the eight score types (fa_ljatr, fa_ljrep, fa_lk, fa_elec,
# lk_ball_iso, lk_ball, lk_bridge, lk_bridge_uncpl), as in tmol's beta-2016
# style score functions
SFXN_WEIGHTS = (1.0, 0.55, 1.0, 1.0, -0.38, 0.92, -0.33, -0.33)
BONDSEP_METRIC = "inter-block bond separation poses/s (256-pose uneven batch, dense [P,B,B,C,C] + min, 1 B200)"

# Algorithmic FLOPs per unit (E + dE), counted on the restatement's most
# populated branch (far cubic fade, 4.5-6 A); FMA = 2, div/sqrt/exp/floor = 1.
F_PAIR_TEST = 8  # every atom pair of a neighbouring block pair: distance^2 test
F_LJ = 64  # each pair inside max_dis with non-zero count-pair weight
F_LK = 111  # each heavy-atom pair among those (both LK directions)
# elec: each pair inside max_dis with non-zero count-pair weight, counted on
# the restatement's Coulomb branch (1.85-4.5 A, the most populated):
# distance and unit vector 12, eps 14, deps 10, E 4, dE 8, weights 2,
# energy sum 1, gradient on both atoms 9, charge product 1
F_ELEC = 61
# LK-ball, energy and gradient in one pass (counted on the restatement,
# the isotropic term on its 2-4.5 A branch): each polar / occluder pair in
# reach (bond separation > 3, inside max_dis, polar atom with waters):
# distance 9, sigma 1, isotropic LK and its derivative 38, desolvation
# fraction over 4 waters with its adjoint 139, combination and adjoint onto
# both atoms and the polar waters 64, energy sums 4.
F_LKB_PAIR = 255
# ...and when the occluder is a donor or acceptor, the water-bridge term
# over 4 x 4 water pairs with its adjoint onto both atoms' waters (481) and
# its share of the combination (180)
F_LKB_BRIDGE = 661
# energies alone (the rotamer op's forward): 112 per evaluated pair
# (distance 9, sigma 1, isotropic LK 38, desolvation fraction 57, sums 7)
# and 225 more per bridged pair
F_LKB_PAIR_E = 112
F_LKB_BRIDGE_E = 225


def workload_sizes(name, rank):
    import numpy

    from tmol_b200.pose.synthetic import log_uniform_sizes

    if name in ("uniform64x150", "elec64x150", "lkball64x150", "sfxn64x150"):
        return [N_RES] * N_POSES, [rank * N_POSES + k for k in range(N_POSES)]
    rng = numpy.random.default_rng(UNEVEN_SEED + 1000 * rank)
    sizes = log_uniform_sizes(rng, UNEVEN_POSES, 20, 1000)
    return sizes, [100000 * (rank + 1) + k for k in range(UNEVEN_POSES)]


def workload(rank, name="uniform64x150", device="cpu"):
    from tmol_b200.pose.synthetic import synthetic_pose_stack

    sizes, seeds = workload_sizes(name, rank)
    return synthetic_pose_stack(sizes, seeds, device=device)


def rotamer_workload(rank, device, sizes=None, seeds=None):
    from tmol_b200.pose.rotamers import synthetic_rotamer_set
    from tmol_b200.pose.synthetic import synthetic_pose_stack

    if sizes is None:
        sizes = [ROT_RES] * ROT_POSES
        seeds = [7000 + rank * ROT_POSES + k for k in range(ROT_POSES)]
    ps = synthetic_pose_stack(sizes, seeds, device=device)
    rs = synthetic_rotamer_set(ps, pose_seeds=seeds, **ROT_SET)
    return ps, rs, sizes, seeds


def workload_label(name):
    if name == "elec64x150":
        return f"{N_POSES} poses x {N_RES} residues, fa_elec energy + gradient"
    if name == "sfxn64x150":
        return (
            f"{N_POSES} poses x {N_RES} residues, fa_ljatr + fa_ljrep + fa_lk + fa_elec + the four LK-ball terms, "
            f"weighted sum and its gradient, weights {list(SFXN_WEIGHTS)}"
        )
    if name == "lkball64x150":
        return (
            f"{N_POSES} poses x {N_RES} residues, lk_ball_iso + lk_ball + lk_bridge + lk_bridge_uncpl "
            "energies + gradient through the waters"
        )
    if name == "uniform64x150":
        return f"{N_POSES} poses x {N_RES} residues, energy + gradient, weights {list(TERM_WEIGHTS)}"
    return (
        f"{UNEVEN_POSES} poses, residues log-uniform in [20, 1000], energy + gradient, "
        f"coordinates + N(0, {PERTURB_SD} A) each replayed step, weights {list(TERM_WEIGHTS)}"
    )


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    REASONS = {
        "hw_slowdown": 0x8,
        "hw_thermal_slowdown": 0x40,
        "sw_thermal_slowdown": 0x20,
        "sw_power_cap": 0x4,
        "hw_power_brake_slowdown": 0x80,
    }

    def __init__(self, index):
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for name, bit in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        if self.nv is not None:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self.nv is not None:
            self.t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"]}
        return {
            "sm_mhz": statistics.median(self.samples),
            "sm_max_mhz": self.max_mhz,
            "reasons": sorted(self.reasons),
            "samples": len(self.samples),
        }


def dist_setup():
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def _reduce_device():
    import torch.distributed as dist

    # NCCL reduces device tensors; gloo (the CPU tests of this logic) host ones
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def sum_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.item()


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def cpu_reference_sample(ps, term, reps=3):
    """tmol's CPU op (oracle/_ref, else the bit-exact C restatement) on the
    whole batch, energies + gradient, single thread; best of `reps`."""
    import torch

    from oracle import oracle as O
    from tmol_b200.score.ljlk_energy_term import pose_score_args

    torch.set_num_threads(1)
    args = pose_score_args(ps, term)
    coords = ps.coords.flatten(0, 1)
    if O.reference_available():
        kind = "reference"

        def run():
            E, c, _ = O.reference_pose_scores(coords, args, require_gradient=True)
            (torch.tensor(TERM_WEIGHTS)[:, None] * E).sum().backward()

    else:
        kind = "port"
        oc = O.OracleCall(coords, args)

        def run():
            oc.pose_scores(require_gradient=True)

    run()
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        run()
        best = min(best, time.perf_counter() - t0)
    return kind, best


def _ref_worker(conn, sizes, seeds, term="ljlk"):
    """One single-threaded process of the reference arm: builds its share of
    the poses (same sizes and seeds as the GPU arm) and scores it on demand
    (`term`: "ljlk", "elec", "lkball" or "sfxn": all three, weighted)."""
    import torch

    torch.set_num_threads(1)
    from oracle import oracle as O
    from tmol_b200.pose.synthetic import synthetic_pose_stack

    ps = synthetic_pose_stack(sizes, seeds)
    coords = ps.coords.flatten(0, 1).clone()
    if term == "sfxn":
        import numpy

        from tmol_b200.score.elec_energy_term import ElecEnergyTerm, elec_pose_score_args
        from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args
        from tmol_b200.score.lkball_energy_term import LKBallEnergyTerm, score_args, water_gen_args

        lt = LKBallEnergyTerm()
        la, ea = pose_score_args(ps, LJLKEnergyTerm()), elec_pose_score_args(ps, ElecEnergyTerm())
        wa, sa = water_gen_args(ps, lt), score_args(ps, lt, None)
        avail = O.reference_available() and O.reference_elec_available() and O.reference_lkball_available()
        if avail:
            O.reference_elec_pose_scores(coords, ea)  # loads the op libraries
            ljlk_op, elec_op = O.load_reference(), torch.ops.tmol_elec.elec_pose_scores
        else:
            ocs = (O.OracleCall(coords, la), O.OracleCall(coords, ea, term="elec"),
                   O.OracleCall(coords, sa, term="lkball", lkb_water_args=wa))
        wts = torch.tensor(SFXN_WEIGHTS)
        conn.send("ready")
        while True:
            msg = conn.recv()
            if msg is None:
                break
            t0 = time.perf_counter()
            if avail:
                c = coords.clone().requires_grad_(True)
                E1, _ = ljlk_op(c, *la)
                E2, _ = elec_op(c, *ea)
                El, _, cl, _ = O.reference_lkball(coords, wa, sa)
                ((wts[:3, None] * E1).sum() + (wts[3] * E2).sum()).backward()
                (wts[4:, None] * El).sum().backward()
            else:
                ocs[0].pose_scores(require_gradient=True)
                ocs[1].pose_scores(require_gradient=True)
                ocs[2].lkb_scores(ocs[2].lkb_waters(), weights=numpy.ones((4, ps.n_poses)))
            conn.send(time.perf_counter() - t0)
        return
    if term == "lkball":
        import numpy

        from tmol_b200.score.lkball_energy_term import LKBallEnergyTerm, score_args, water_gen_args

        lt = LKBallEnergyTerm()
        wa, sa = water_gen_args(ps, lt), score_args(ps, lt, None)
        ref = O.reference_lkball_available()
        oc = None if ref else O.OracleCall(coords, sa, term="lkball", lkb_water_args=wa)
        ones = numpy.ones((4, ps.n_poses))
        conn.send("ready")
        while True:
            msg = conn.recv()
            if msg is None:
                break
            t0 = time.perf_counter()
            if ref:
                E, _, c, _ = O.reference_lkball(coords, wa, sa)
                E.sum().backward()
            else:
                oc.lkb_scores(oc.lkb_waters(), weights=ones)
            conn.send(time.perf_counter() - t0)
        return
    if term == "elec":
        from tmol_b200.score.elec_energy_term import ElecEnergyTerm, elec_pose_score_args

        args = elec_pose_score_args(ps, ElecEnergyTerm())
        if O.reference_elec_available():
            O.reference_elec_pose_scores(coords, args)  # loads the op library
            op = torch.ops.tmol_elec.elec_pose_scores
        else:
            op = None
        oc = None if op is not None else O.OracleCall(coords, args, term="elec")
        w = torch.ones((1, 1))
    else:
        from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args

        args = pose_score_args(ps, LJLKEnergyTerm())
        op = O.load_reference() if O.reference_available() else None
        oc = None if op is not None else O.OracleCall(coords, args)
        w = torch.tensor(TERM_WEIGHTS)[:, None]
    conn.send("ready")
    while True:
        msg = conn.recv()
        if msg is None:
            break
        t0 = time.perf_counter()
        if op is not None:
            c = coords.clone().requires_grad_(True)
            E, _ = op(c, *args)
            (w * E).sum().backward()
        else:
            oc.pose_scores(require_gradient=True)
        conn.send(time.perf_counter() - t0)


def _ref_rot_worker(conn, sizes, seeds, term="ljlk"):
    """One single-threaded process of the rotamer reference arm (`term`:
    "ljlk", or "lkball": waters on the rotamers, then the rotamer op)."""
    import torch

    torch.set_num_threads(1)
    from oracle import oracle as O
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, rotamer_score_args

    ps, rs, _, _ = rotamer_workload(0, "cpu", sizes, seeds)
    if term == "lkball":
        from tmol_b200.score.lkball_energy_term import LKBallEnergyTerm, water_gen_args
        from tmol_b200.score.lkball_energy_term import rotamer_score_args as lkb_rotamer_score_args

        lt = LKBallEnergyTerm()
        wa, sa = water_gen_args(ps, lt, rs), lkb_rotamer_score_args(ps, rs, lt, None)
        ref = O.reference_lkball_available()
        oc = None if ref else O.OracleCall(rs.coords, sa, term="lkball", lkb_water_args=wa)
        conn.send("ready")
        while True:
            msg = conn.recv()
            if msg is None:
                break
            t0 = time.perf_counter()
            if ref:
                with torch.no_grad():
                    O.reference_lkball_rotamers(rs.coords, wa, sa)
            else:
                oc.lkb_rotamer_scores(oc.lkb_waters())
            conn.send(time.perf_counter() - t0)
        return
    args = rotamer_score_args(ps, rs, LJLKEnergyTerm())
    conn.send("ready")
    while True:
        msg = conn.recv()
        if msg is None:
            break
        t0 = time.perf_counter()
        if O.reference_available():
            O.reference_rotamer_scores(rs.coords, args, require_gradient=False)
        else:
            O.OracleCall(rs.coords, args).rotamer_scores()
        conn.send(time.perf_counter() - t0)


def run_reference(args, world, rank):
    """tmol's CPU op on all host cores: one process per core, poses dealt
    out longest-first so that every process gets a similar share."""
    import multiprocessing as mp

    from oracle import oracle as O

    if rank != 0:
        return 0
    if args.workload == "rotamers16x150":
        return run_reference_rotamers(args)
    if args.workload == "lkball_rotamers16x150":
        return run_reference_rotamers(args, term="lkball")
    if args.workload == "bondsep256":
        return run_reference_bondsep(args)
    elec = args.workload == "elec64x150"
    lkball = args.workload == "lkball64x150"
    sfxn = args.workload == "sfxn64x150"
    term = "elec" if elec else ("lkball" if lkball else ("sfxn" if sfxn else "ljlk"))
    sizes, seeds = workload_sizes(args.workload, 0)
    n_poses = len(sizes)
    n_proc = min(os.cpu_count() or 1, n_poses)
    shares = [[] for _ in range(n_proc)]
    load = [0] * n_proc
    for k in sorted(range(n_poses), key=lambda k: -sizes[k]):
        q = load.index(min(load))
        shares[q].append(k)
        load[q] += sizes[k] * 16 * 20  # ~ atoms x neighbour atoms
    ctx = mp.get_context("spawn")
    workers = []
    for share in shares:
        parent, child = ctx.Pipe()
        pr = ctx.Process(
            target=_ref_worker,
            args=(child, [sizes[k] for k in share], [seeds[k] for k in share], term),
        )
        pr.start()
        workers.append((pr, parent))
    for _, c in workers:
        c.recv()

    def step():
        t0 = time.perf_counter()
        for _, c in workers:
            c.send(1)
        for _, c in workers:
            c.recv()
        return time.perf_counter() - t0

    for _ in range(max(args.warmup, 1)):
        step()
    times = [step() for _ in range(args.steps)]
    for pr, c in workers:
        c.send(None)
        pr.join()
    t = sum(times)
    value = n_poses * args.steps / t
    if elec:
        kind = "reference" if O.reference_elec_available() else "port"
    elif lkball:
        kind = "reference" if O.reference_lkball_available() else "port"
    elif sfxn:
        both = O.reference_available() and O.reference_elec_available() and O.reference_lkball_available()
        kind = "reference" if both else "port"
    else:
        kind = "reference" if O.reference_available() else "port"
    line = {
        "impl": "reference",
        "metric": ELEC_METRIC if elec else (LKBALL_METRIC if lkball else (SFXN_METRIC if sfxn else METRIC)),
        "value": value,
        "unit": "poses/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded proteins, ideal geometry)",
        "config": {"workload": workload_label(args.workload), "poses": n_poses},
        "cpu_baseline": {
            "value": value,
            "unit": "poses/s",
            "cores": n_proc,
            "kind": kind,
            "sample": f"the full {n_poses}-pose batch per step, dealt to {n_proc} single-threaded processes",
        },
        "e2e": {"value": value, "unit": "poses/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference_rotamers(args, term="ljlk"):
    """tmol's CPU rotamer op, one process per pose (energies of every
    rotamer pair, as the packer asks for them); LK-ball with its waters."""
    import multiprocessing as mp

    from oracle import oracle as O

    sizes = [ROT_RES] * ROT_POSES
    seeds = [7000 + k for k in range(ROT_POSES)]
    n_proc = min(os.cpu_count() or 1, ROT_POSES)
    shares = [list(range(q, ROT_POSES, n_proc)) for q in range(n_proc)]
    ctx = mp.get_context("spawn")
    workers = []
    for share in shares:
        parent, child = ctx.Pipe()
        pr = ctx.Process(
            target=_ref_rot_worker, args=(child, [sizes[k] for k in share], [seeds[k] for k in share], term)
        )
        pr.start()
        workers.append((pr, parent))
    for _, c in workers:
        c.recv()

    def step():
        t0 = time.perf_counter()
        for _, c in workers:
            c.send(1)
        for _, c in workers:
            c.recv()
        return time.perf_counter() - t0

    for _ in range(max(args.warmup, 1)):
        step()
    times = [step() for _ in range(args.steps)]
    for pr, c in workers:
        c.send(None)
        pr.join()
    # the same batch's pair count, for the unit
    import torch

    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, rotamer_score_args

    ps, rs, _, _ = rotamer_workload(0, "cpu", sizes, seeds)
    n_pairs = O.OracleCall(rs.coords, rotamer_score_args(ps, rs, LJLKEnergyTerm())).rotamer_scores()[0].shape[1]
    t = sum(times)
    value = n_pairs * args.steps / t
    if term == "lkball":
        kind = "reference" if O.reference_lkball_available() else "port"
    else:
        kind = "reference" if O.reference_available() else "port"
    line = {
        "impl": "reference",
        "metric": LKB_ROT_METRIC if term == "lkball" else ROT_METRIC,
        "value": value,
        "unit": "rotamer pairs/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded proteins and rotamers, ideal geometry)",
        "config": {
            "workload": (
                "16 poses x 150 residues, 1-31 rotamers per block, waters and the four LK-ball energies of every "
                "rotamer pair"
                if term == "lkball"
                else "16 poses x 150 residues, 1-31 rotamers per block, energies of every rotamer pair"
            ),
            "rotamer_pairs": n_pairs,
        },
        "cpu_baseline": {
            "value": value,
            "unit": "rotamer pairs/s",
            "cores": n_proc,
            "kind": kind,
            "sample": f"the full 16-pose batch per step, one pose per single-threaded process ({n_proc} processes)",
        },
        "e2e": {"value": value, "unit": "rotamer pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    del torch
    return 0


def run_rotamers(args, world, rank, local):
    """Rotamer scoring (tmol's ljlk_rotamer_scores): per step the op's full
    call, dispatch (rotamer and block spheres, neighbour blocks, pair list:
    one host synchronisation to size the output) and the energies of every
    rotamer pair of neighbouring blocks."""
    import torch

    from tmol_b200 import native
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, rotamer_score_args
    from tmol_b200.score.ljlk_op import LJLKPlan

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ps, rs, sizes, seeds = rotamer_workload(rank, dev)
    rargs = rotamer_score_args(ps, rs, LJLKEnergyTerm(device=dev))
    coords = rs.coords.contiguous()
    plan = LJLKPlan(coords, rargs[:-1], rotamers=True, launch=(1, 8, 2, 32))
    flush = torch.empty(L2_FLUSH_BYTES // 4, device=dev, dtype=torch.float32)

    def op():
        idx, items = plan.rotamer_dispatch(coords)
        return plan.rotamer_forward(coords, items, idx.shape[1]), idx, items

    for _ in range(max(args.warmup, 3)):
        E, idx, items = op()
    torch.cuda.synchronize()
    n_pairs = idx.shape[1]
    counts = counted_work(plan, op)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            op()
            ev[k][1].record()
        torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), world)
    value = sum_over_ranks(n_pairs * args.steps, world) / (ms / 1e3)
    # energies alone (a fixed pair list, as a packer reuses it): graph replays
    energies = torch.empty((3, n_pairs), device=dev)

    def energies_only():
        native.call(
            "tmol_b200_ljlk_rotamer_forward", plan.ptr, ctypes_ptr(coords), ctypes_ptr(items), items.shape[0],
            n_pairs, ctypes_ptr(energies), plan._stream(),
        )

    e_ms = time_replays(energies_only, args.steps, flush) / args.steps
    # end to end: host coordinates in, energies and pair indices out (into
    # pinned host buffers sized by the pair count)
    h_coords = coords.cpu().pin_memory()
    d_in = torch.empty_like(coords)
    h_E = torch.empty((3, n_pairs), pin_memory=True)
    h_I = torch.empty((3, n_pairs), dtype=torch.int32, pin_memory=True)
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    d2h = 0
    for k in range(args.steps):
        flush.zero_()
        e2e_ev[k][0].record()
        d_in.copy_(h_coords, non_blocking=True)
        idx2, items2 = plan.rotamer_dispatch(d_in)
        E2 = plan.rotamer_forward(d_in, items2, idx2.shape[1])
        if idx2.shape[1] != h_E.shape[1]:
            h_E = torch.empty(tuple(E2.shape), pin_memory=True)
            h_I = torch.empty(tuple(idx2.shape), dtype=torch.int32, pin_memory=True)
        h_E.copy_(E2, non_blocking=True)
        h_I.copy_(idx2, non_blocking=True)
        d2h = h_E.numel() * 4 + h_I.numel() * 4
        e2e_ev[k][1].record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in e2e_ev), world)
    fp32_peak = native.measure_fp32_peak_tflops(torch.cuda.current_stream().cuda_stream)
    flops = counts["atom_pairs"] * F_PAIR_TEST + counts["atom_pairs_in_range"] * F_LJ + counts["heavy_pairs_in_range"] * F_LK
    achieved = flops / (e_ms * 1e-3) / 1e12
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O

        ps0, rs0, _, _ = rotamer_workload(0, "cpu", sizes[:1], seeds[:1])
        a0 = rotamer_score_args(ps0, rs0, LJLKEnergyTerm())
        torch.set_num_threads(1)
        best = float("inf")
        for _ in range(2):
            t0 = time.perf_counter()
            if O.reference_available():
                E0, _, _ = O.reference_rotamer_scores(rs0.coords, a0, require_gradient=False)
            else:
                E0 = torch.tensor(O.OracleCall(rs0.coords, a0).rotamer_scores()[0])
            best = min(best, time.perf_counter() - t0)
        cpu = {
            "value": E0.shape[1] / best,
            "unit": "rotamer pairs/s",
            "cores": 1,
            "kind": "reference" if O.reference_available() else "port",
            "sample": "pose 0 of the batch (all its rotamer pairs), one thread, best of 2",
        }
    if rank == 0:
        line = {
            "metric": ROT_METRIC,
            "value": value,
            "unit": "rotamer pairs/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded proteins and rotamers, ideal geometry)",
            "config": {
                "workload": "16 poses x 150 residues, 1-31 rotamers per block, energies of every rotamer pair",
                "rotamers": int(rs.n_rotamers_total),
                "rotamer_pairs": n_pairs,
                "l2": "flushed (256 MiB write) before every timed step",
                "parallelism": f"weak, {world} independent batch(es)",
            },
            "atom_pairs_per_s": counts["atom_pairs"] * args.steps * world / (ms / 1e3),
            "energies_only_ms_per_step": e_ms,
            "work_per_step": counts,
            "gpu_launches": 7 * args.steps,
            "clocks": clk.summary(),
            "roofline": {
                "bound": "fp32",
                "achieved": achieved,
                "peak": fp32_peak,
                "unit": "TFLOP/s",
                "frac": achieved / fp32_peak,
                "traffic": None,
                "kernel": "rotamer_kernel<float, energies> (+ rotamer spheres), timed as graph replays",
                "kernel_ms": e_ms,
                "flops_per_launch": flops,
                "peak_source": "measured: FMA-loop probe over all SMs in this run (tmol_b200_measure_fp32_peak)",
            },
            "e2e": {
                "value": sum_over_ranks(n_pairs * args.steps, world) / (e2e_ms / 1e3),
                "unit": "rotamer pairs/s",
                "h2d_bytes_per_step": coords.numel() * 4,
                "d2h_bytes_per_step": d2h,
            },
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def run_lkball_rotamers(args, world, rank, local):
    """LK-ball rotamer scoring (tmol's rotamer scoring of the term): per step
    the waters of every rotamer (gen_pose_waters on the rotamers'
    coordinates), the dispatch (one host synchronisation to size the
    output) and the four energies of every rotamer pair of neighbouring
    blocks (lk_ball_rotamer_score)."""
    import torch

    from tmol_b200 import native
    from tmol_b200.score.lkball_energy_term import LKBallEnergyTerm, rotamer_score_args, water_gen_args
    from tmol_b200.score.lkball_op import LKBallPlan

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ps, rs, sizes, seeds = rotamer_workload(rank, dev)
    lt = LKBallEnergyTerm()
    on = lambda a: [x.to(dev) if isinstance(x, torch.Tensor) else x for x in a]  # noqa: E731
    wa = on(water_gen_args(ps, lt, rs))
    sa = on(rotamer_score_args(ps, rs, lt, None)[:-2])
    coords = rs.coords.contiguous()
    plan = LKBallPlan(coords, water_static=wa, score_static=sa, rotamers=True, launch=(1, 8, 2, 32))
    flush = torch.empty(L2_FLUSH_BYTES // 4, device=dev, dtype=torch.float32)
    W = torch.empty((coords.shape[0], 4, 3), device=dev)

    def op():
        plan.waters(coords, W)
        idx, items = plan.rotamer_dispatch(coords)
        return plan.rotamer_forward(coords, items, idx.shape[1], W), idx, items

    for _ in range(max(args.warmup, 3)):
        E, idx, items = op()
    torch.cuda.synchronize()
    n_pairs = idx.shape[1]
    counts = counted_work(plan, op)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            op()
            ev[k][1].record()
        torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), world)
    value = sum_over_ranks(n_pairs * args.steps, world) / (ms / 1e3)
    # the scoring kernel alone on a fixed pair list (as a packer reuses it)
    energies = torch.empty((4, n_pairs), device=dev)

    def energies_only():
        native.call(
            "tmol_b200_lkball_rotamer_forward", plan.ptr, ctypes_ptr(coords), ctypes_ptr(W), ctypes_ptr(items),
            items.shape[0], n_pairs, ctypes_ptr(energies), plan._stream(),
        )

    e_ms = time_replays(energies_only, args.steps, flush) / args.steps
    h_coords = coords.cpu().pin_memory()
    d_in = torch.empty_like(coords)
    h_E = torch.empty((4, n_pairs), pin_memory=True)
    h_I = torch.empty((3, n_pairs), dtype=torch.int32, pin_memory=True)
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    d2h = 0
    for k in range(args.steps):
        flush.zero_()
        e2e_ev[k][0].record()
        d_in.copy_(h_coords, non_blocking=True)
        plan.waters(d_in, W)
        idx2, items2 = plan.rotamer_dispatch(d_in)
        E2 = plan.rotamer_forward(d_in, items2, idx2.shape[1], W)
        if idx2.shape[1] != h_E.shape[1]:
            h_E = torch.empty(tuple(E2.shape), pin_memory=True)
            h_I = torch.empty(tuple(idx2.shape), dtype=torch.int32, pin_memory=True)
        h_E.copy_(E2, non_blocking=True)
        h_I.copy_(idx2, non_blocking=True)
        d2h = h_E.numel() * 4 + h_I.numel() * 4
        e2e_ev[k][1].record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in e2e_ev), world)
    fp32_peak = native.measure_fp32_peak_tflops(torch.cuda.current_stream().cuda_stream)
    flops = counts["pairs_evaluated"] * F_LKB_PAIR_E + counts["bridged_pairs"] * F_LKB_BRIDGE_E
    achieved = flops / (e_ms * 1e-3) / 1e12
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O

        ps0, rs0, _, _ = rotamer_workload(0, "cpu", sizes[:1], seeds[:1])
        wa0, sa0 = water_gen_args(ps0, lt, rs0), rotamer_score_args(ps0, rs0, lt, None)
        torch.set_num_threads(1)
        best = float("inf")
        for _ in range(2):
            t0 = time.perf_counter()
            if O.reference_lkball_available():
                with torch.no_grad():
                    E0 = O.reference_lkball_rotamers(rs0.coords, wa0, sa0)[0]
            else:
                oc = O.OracleCall(rs0.coords, sa0, term="lkball", lkb_water_args=wa0)
                E0 = torch.tensor(oc.lkb_rotamer_scores(oc.lkb_waters())[0])
            best = min(best, time.perf_counter() - t0)
        cpu = {
            "value": E0.shape[1] / best,
            "unit": "rotamer pairs/s",
            "cores": 1,
            "kind": "reference" if O.reference_lkball_available() else "port",
            "sample": "pose 0 of the batch (its waters and all its rotamer pairs), one thread, best of 2",
        }
    if rank == 0:
        line = {
            "metric": LKB_ROT_METRIC,
            "value": value,
            "unit": "rotamer pairs/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded proteins and rotamers, ideal geometry)",
            "config": {
                "workload": "16 poses x 150 residues, 1-31 rotamers per block, waters and the four LK-ball "
                "energies of every rotamer pair",
                "rotamers": int(rs.n_rotamers_total),
                "rotamer_pairs": n_pairs,
                "l2": "flushed (256 MiB write) before every timed step",
                "parallelism": f"weak, {world} independent batch(es)",
            },
            "scoring_only_ms_per_step": e_ms,
            "work_per_step": counts,
            # waters, 4 dispatch kernels (rotamer and block spheres, row
            # counts, scan), the fill, the rotamer spheres and the scoring
            # kernel
            "gpu_launches": 8 * args.steps,
            "clocks": clk.summary(),
            "roofline": {
                "bound": "fp32",
                "achieved": achieved,
                "peak": fp32_peak,
                "unit": "TFLOP/s",
                "frac": achieved / fp32_peak,
                "traffic": load_traffic("lkb_rotamer"),
                "kernel": "lkb_rotamer_kernel<float, energies>, timed as graph replays",
                "traffic_source": "ncu capture, profiles/lkb_rotamer_traffic.json",
                "kernel_ms": e_ms,
                "flops_per_launch": flops,
                "peak_source": "measured: FMA-loop probe over all SMs in this run (tmol_b200_measure_fp32_peak)",
            },
            "e2e": {
                "value": sum_over_ranks(n_pairs * args.steps, world) / (e2e_ms / 1e3),
                "unit": "rotamer pairs/s",
                "h2d_bytes_per_step": coords.numel() * 4,
                "d2h_bytes_per_step": d2h,
            },
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


E2E_MIN_STEPS = 100


def pipelined_e2e_ms(plan, weights, h_coords, flush, steps, world, P, n_terms=3):
    """Device time (max over ranks) of `steps` energy + gradient steps
    through the plan's C entry point, each with its host->device copy of
    the coordinates, an L2 flush and the device->host copy of energies and
    gradient, double-buffered over a copy-in, a compute and a copy-out
    stream.  The pipeline runs max(steps, E2E_MIN_STEPS) steps, so that
    its fill and drain (one copy-in and one copy-out outside any overlap)
    are not counted 1/steps times over; the time returned is that run's,
    scaled to `steps` steps."""
    import torch

    dev = h_coords.device if h_coords.is_cuda else torch.device("cuda", torch.cuda.current_device())
    s_in, s_run, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    d_in = [torch.empty(h_coords.shape, device=dev) for _ in range(2)]
    E = [torch.empty((n_terms, P), device=dev) for _ in range(2)]
    dx = [torch.empty(h_coords.shape, device=dev) for _ in range(2)]
    h_E = [torch.empty((n_terms, P), pin_memory=True) for _ in range(2)]
    h_g = [torch.empty(h_coords.shape, pin_memory=True) for _ in range(2)]
    ev = lambda: torch.cuda.Event()  # noqa: E731
    copied_in = [ev(), ev()]
    computed = [ev(), ev()]
    copied_out = [ev(), ev()]
    for e in copied_in + computed + copied_out:
        e.record(torch.cuda.current_stream(dev))
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def run(n, timed):
        cur = torch.cuda.current_stream(dev)
        if timed:
            start.record(cur)
        for s_ in (s_in, s_run, s_out):
            s_.wait_stream(cur)
        for k in range(n):
            b = k & 1
            with torch.cuda.stream(s_in):
                s_in.wait_event(computed[b])  # d_in[b] no longer read
                d_in[b].copy_(h_coords, non_blocking=True)
                copied_in[b].record(s_in)
            with torch.cuda.stream(s_run):
                s_run.wait_event(copied_in[b])
                s_run.wait_event(copied_out[b])  # E[b], dx[b] copied out
                flush.zero_()
                plan.energy_and_gradient(d_in[b], weights, E[b], dx[b])
                computed[b].record(s_run)
            with torch.cuda.stream(s_out):
                s_out.wait_event(computed[b])
                h_E[b].copy_(E[b], non_blocking=True)
                h_g[b].copy_(dx[b], non_blocking=True)
                copied_out[b].record(s_out)
        for s_ in (s_in, s_run, s_out):
            cur.wait_stream(s_)
        if timed:
            end.record(cur)

    n = max(steps, E2E_MIN_STEPS)
    run(3, False)
    torch.cuda.synchronize()
    barrier(world)
    run(n, True)
    torch.cuda.synchronize()
    barrier(world)
    return max_over_ranks(start.elapsed_time(end) * steps / n, world)


def counted_work(plan, call):
    """The plan's work counters for one run of `call()` with counting on; the
    timed calls run the kernel instantiation without counters."""
    plan.set_counting(True)
    call()
    counts = plan.last_counts()
    plan.set_counting(False)
    return counts


def ctypes_ptr(t):
    import ctypes

    return ctypes.c_void_p(t.data_ptr())


def flops_per_step(counts):
    return (
        counts["atom_pairs"] * F_PAIR_TEST
        + counts["atom_pairs_in_range"] * F_LJ
        + counts["heavy_pairs_in_range"] * F_LK
    )


def load_traffic(name="ljlk_score"):
    """DRAM bytes per launch of a scoring kernel from its committed ncu
    capture (profiles/<name>_traffic.json), or None."""
    path = os.path.join(ROOT, "profiles", f"{name}_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d.get("dram_bytes_per_launch")
    except Exception:
        return None


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def cpu_baseline_for(name, ps_sizes_seeds, full_atom_pairs):
    """The reference CPU op on one core, on a bounded sample of the workload
    (the whole uniform batch; 16 seeded poses of the uneven batch, scaled to
    the whole batch by atom pairs)."""
    import numpy
    import torch

    from oracle import oracle as O
    from tmol_b200.pose.synthetic import synthetic_pose_stack
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args

    sizes, seeds = ps_sizes_seeds
    term = LJLKEnergyTerm()
    if name == "uniform64x150":
        ps = synthetic_pose_stack(sizes, seeds)
        kind, t = cpu_reference_sample(ps, term)
        return {
            "value": len(sizes) / t,
            "unit": "poses/s",
            "cores": 1,
            "kind": kind,
            "sample": f"the full {len(sizes)}x{N_RES} batch, energies + gradient, best of 3, one thread",
        }
    pick = numpy.random.default_rng(7).choice(len(sizes), 16, replace=False)
    sub = synthetic_pose_stack([sizes[k] for k in pick], [seeds[k] for k in pick])
    kind, t = cpu_reference_sample(sub, term, reps=1)
    args = pose_score_args(sub, term)
    _, _, nbr = O.OracleCall(sub.coords.flatten(0, 1), args).pose_scores()
    ap_sample, _ = O.OracleCall(sub.coords.flatten(0, 1), args).count_pairs(nbr)
    t_full = t * full_atom_pairs / max(ap_sample, 1)
    return {
        "value": len(sizes) / t_full,
        "unit": "poses/s",
        "cores": 1,
        "kind": kind,
        "sample": f"16 seeded poses of the batch ({ap_sample} atom pairs), one thread; "
        f"extrapolated to the batch's {full_atom_pairs} atom pairs",
    }


def time_replays(fn, steps, flush):
    """Milliseconds of `steps` replays of fn captured as a CUDA graph, L2
    flushed before each replay (outside the events)."""
    import torch

    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        fn()
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    for _ in range(3):
        g.replay()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        flush.zero_()
        ev[k][0].record()
        g.replay()
        ev[k][1].record()
    torch.cuda.synchronize()
    del g
    return sum(a.elapsed_time(b) for a, b in ev)


def measure_screen(plan, plan64, coords, weights, step, flush, steps, names, plain_ms):
    """The learned block-pair screen on the same batch: the time of a step
    with the screen rebuilt inside it and with the mask reused, the skipped
    fraction and the per-pose |dE| it introduces (float64 plan, same mask)."""
    import torch

    from tmol_b200.screen import BlockPairScreen

    screen = BlockPairScreen.trained(plan, names)
    screen.update(coords)
    torch.cuda.synchronize()
    n_cand = screen.n_candidates()
    n_skip = screen.n_skipped()
    c64 = coords.double()
    w64 = weights.double()
    plan64.set_skip_mask(None)
    E0, _ = plan64.energy_and_gradient(c64, w64)
    E0 = E0.clone()
    plan64.set_skip_mask(screen.mask)
    E1, _ = plan64.energy_and_gradient(c64, w64)
    plan64.set_skip_mask(None)
    dE = (E1 - E0).abs()
    tot = ((E1 - E0) * w64).sum(0).abs()
    screen.attach()

    def screened_step():
        screen.update(coords)
        step()

    with_update = time_replays(screened_step, steps, flush) / steps
    reused = time_replays(step, steps, flush) / steps
    screen.detach()
    return {
        "threshold": screen.threshold,
        "candidates": n_cand,
        "skipped_block_pairs": n_skip,
        "skipped_fraction": n_skip / max(n_cand, 1),
        "max_abs_dE_per_pose_f64": float(max(dE.max().item(), tot.max().item())),
        "ms_per_step_with_screen_update": with_update,
        "ms_per_step_mask_reused": reused,
        "ms_per_step_plain": plain_ms,
        "speedup_with_update": plain_ms / with_update,
        "speedup_mask_reused": plain_ms / reused,
    }


def elec_plan_for(ps, coords, launch_shape=None):
    """An elec plan of the batch (float32), on the launch shape given."""
    import torch

    from tmol_b200.score.elec_energy_term import ElecEnergyTerm, elec_pose_score_args
    from tmol_b200.score.elec_op import ElecPlan

    dev = coords.device
    static = [a.to(dev) if isinstance(a, torch.Tensor) else a for a in elec_pose_score_args(ps, ElecEnergyTerm())[:-1]]
    plan = ElecPlan(coords, static)
    if launch_shape:
        plan.set_launch(*launch_shape)
    return plan


def measure_elec(plan, coords, flush, steps):
    """elec energy + gradient on the batch: graph-replayed step time (L2
    flushed before each), the scoring kernel's average launch time and its
    FP32 figures."""
    import torch

    P = plan.n_poses
    w = torch.ones((1, P), device=coords.device)
    E = torch.empty((1, P), device=coords.device)
    dx = torch.empty_like(coords)

    def step():
        plan.energy_and_gradient(coords, w, E, dx)

    plan.balance(step)
    for _ in range(3):
        step()
    torch.cuda.synchronize()
    counts = counted_work(plan, step)
    ms = time_replays(step, steps, flush) / steps
    plan.profile(True)
    for _ in range(steps):
        flush.zero_()
        step()
    kern_ms, n_launch = plan.profile_read()
    plan.profile(False)
    kern = kern_ms / max(n_launch, 1)
    flops = counts["atom_pairs"] * F_PAIR_TEST + counts["atom_pairs_in_range"] * F_ELEC
    return {
        "ms_per_step": ms,
        "poses_per_s": P / (ms / 1e3),
        "kernel_ms": kern,
        "flops_per_launch": flops,
        "achieved_tflops": flops / (kern * 1e-3) / 1e12,
        "work_per_step": {k: counts[k] for k in ("block_pairs", "atom_pairs", "atom_pairs_in_range")},
    }, step


def cpu_elec_sample(ps, reps=3):
    """tmol's CPU elec op (oracle/_ref/elec, else the C restatement) on the
    whole batch, energies + gradient, single thread; best of `reps`."""
    import torch

    from oracle import oracle as O
    from tmol_b200.score.elec_energy_term import ElecEnergyTerm, elec_pose_score_args

    torch.set_num_threads(1)
    args = elec_pose_score_args(ps, ElecEnergyTerm())
    coords = ps.coords.flatten(0, 1)
    if O.reference_elec_available():
        kind = "reference"

        def run():
            E, c, _ = O.reference_elec_pose_scores(coords, args, require_gradient=True)
            E.sum().backward()

    else:
        kind = "port"
        oc = O.OracleCall(coords, args, term="elec")

        def run():
            oc.pose_scores(require_gradient=True)

    run()
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        run()
        best = min(best, time.perf_counter() - t0)
    return kind, best


def run_elec(args, world, rank, local):
    """The elec term on the uniform batch: per-pose fa_elec and the gradient
    of its sum, one fused pass per step, replayed as a CUDA graph."""
    import torch

    from tmol_b200 import native

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    sizes, seeds = workload_sizes("uniform64x150", rank)
    ps = workload(rank, "uniform64x150", device=dev)
    coords = ps.coords.flatten(0, 1).to(dev).contiguous()
    plan = elec_plan_for(ps, coords)
    P = ps.n_poses
    del ps
    flush = torch.empty(L2_FLUSH_BYTES // 4, device=dev, dtype=torch.float32)
    # warm-up: W graph replays (and the work order from one call's costs),
    # then the launch shape: given, or autotuned as the LJ/LK arm does
    m, step = measure_elec(plan, coords, flush, max(args.warmup, 3))
    if args.launch:
        launch = tuple(int(v) for v in args.launch.split(","))
        plan.set_launch(*launch)
        plan.balance(step)
    else:
        from tmol_b200.tune import autotune

        launch, _ = autotune(plan, step, use_cache=False)
    m, step = measure_elec(plan, coords, flush, max(args.warmup, 3))
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        step()
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=s):
            step()
    torch.cuda.current_stream().wait_stream(s)
    for _ in range(max(args.warmup, 3)):
        g.replay()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            g.replay()
            ev[k][1].record()
        torch.cuda.synchronize()
    barrier(world)
    ms_max = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), world)
    poses_total = sum_over_ranks(P * args.steps, world)
    value = poses_total / (ms_max / 1e3)
    m, _ = measure_elec(plan, coords, flush, args.steps)

    # end to end with host buffers: pinned coordinates in, energies and
    # gradient out
    w = torch.ones((1, P), device=dev)
    E = torch.empty((1, P), device=dev)
    dx = torch.empty_like(coords)
    h_coords = coords.cpu().pin_memory()
    h_E = torch.empty((1, P), pin_memory=True)
    h_g = torch.empty(coords.shape, pin_memory=True)
    d_in = torch.empty_like(coords)
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    for k in range(args.steps):
        flush.zero_()
        e2e_ev[k][0].record()
        d_in.copy_(h_coords, non_blocking=True)
        plan.energy_and_gradient(d_in, w, E, dx)
        h_E.copy_(E, non_blocking=True)
        h_g.copy_(dx, non_blocking=True)
        e2e_ev[k][1].record()
    torch.cuda.synchronize()
    barrier(world)
    serial_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in e2e_ev), world)
    e2e_ms = pipelined_e2e_ms(plan, w, h_coords, flush, args.steps, world, P, n_terms=1)

    fp32_peak = native.measure_fp32_peak_tflops(torch.cuda.current_stream().cuda_stream)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from tmol_b200.pose.synthetic import synthetic_pose_stack

        kind, t = cpu_elec_sample(synthetic_pose_stack(sizes, seeds))
        cpu = {
            "value": len(sizes) / t,
            "unit": "poses/s",
            "cores": 1,
            "kind": kind,
            "sample": f"the full {len(sizes)}x{N_RES} batch, elec energies + gradient, best of 3, one thread",
        }
    if rank == 0:
        line = {
            "metric": ELEC_METRIC,
            "value": value,
            "unit": "poses/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded proteins, ideal geometry)",
            "config": {
                "workload": f"{N_POSES} poses x {N_RES} residues, fa_elec energy + gradient",
                "poses_per_gpu": P,
                "atoms_per_gpu": int(coords.shape[0]),
                "l2": "flushed (256 MiB write) before every timed step",
                "launch": "CUDA graph replay: 2 kernels per step",
                "launch_shape": dict(
                    zip(LAUNCH_FIELDS, launch)
                ),
                "parallelism": f"weak, {world} independent batch(es)",
            },
            "work_per_step": m["work_per_step"],
            "gpu_launches": 2 * args.steps,
            "clocks": clk.summary(),
            "roofline": {
                "bound": "fp32",
                "achieved": m["achieved_tflops"],
                "peak": fp32_peak,
                "unit": "TFLOP/s",
                "frac": m["achieved_tflops"] / fp32_peak,
                "traffic": load_traffic("elec_score"),
                "kernel": "score_kernel<float, GRAD, elec> (fused neighbour + atom-pair energy and gradient)",
                "traffic_source": "ncu capture, profiles/elec_score_traffic.json",
                "kernel_ms": m["kernel_ms"],
                "flops_per_launch": m["flops_per_launch"],
                "peak_source": "measured: FMA-loop probe over all SMs in this run (tmol_b200_measure_fp32_peak)",
            },
            "e2e": {
                "value": poses_total / (e2e_ms / 1e3),
                "unit": "poses/s",
                "h2d_bytes_per_step": coords.numel() * 4,
                "d2h_bytes_per_step": (P + coords.numel()) * 4,
                "schedule": "double-buffered over copy-in / compute / copy-out streams; L2 flushed before every "
                "step's compute, inside the timed region; timed over max(steps, %d) steps" % E2E_MIN_STEPS,
                "serial_value": poses_total / (serial_ms / 1e3),
            },
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    del g
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def lkball_plan_for(ps, coords):
    """An LK-ball plan of the batch (both parts: waters and scoring)."""
    import torch

    from tmol_b200.score.lkball_energy_term import LKBallEnergyTerm, score_args, water_gen_args
    from tmol_b200.score.lkball_op import LKBallPlan

    dev, dt = coords.device, coords.dtype
    lt = LKBallEnergyTerm()

    def on(args):
        out = []
        for a in args:
            if isinstance(a, torch.Tensor):
                a = a.to(dev)
                if a.is_floating_point():
                    a = a.to(dt)
            out.append(a)
        return out

    return LKBallPlan(coords, water_static=on(water_gen_args(ps, lt)), score_static=on(score_args(ps, lt, None)[:-2]))


def measure_lkball(plan, coords, flush, steps):
    """LK-ball energy + gradient on the batch (waters, one scoring pass, the
    waters' adjoint): graph-replayed step time (L2 flushed before each), the
    scoring kernel's average launch time and its FP32 figures."""
    import torch

    P = plan.n_poses
    w = torch.ones((4, P), device=coords.device, dtype=coords.dtype)
    E = torch.empty((4, P), device=coords.device, dtype=coords.dtype)
    dx = torch.empty_like(coords)

    def step():
        plan.energy_and_gradient(coords, w, E, dx)

    plan.balance(step)
    for _ in range(3):
        step()
    torch.cuda.synchronize()
    counts = counted_work(plan, step)
    ms = time_replays(step, steps, flush) / steps
    plan.profile(True)
    for _ in range(steps):
        flush.zero_()
        step()
    kern_ms, n_launch = plan.profile_read()
    plan.profile(False)
    kern = kern_ms / max(n_launch, 1)
    flops = counts["pairs_evaluated"] * F_LKB_PAIR + counts["bridged_pairs"] * F_LKB_BRIDGE
    return {
        "ms_per_step": ms,
        "poses_per_s": P / (ms / 1e3),
        "kernel_ms": kern,
        "flops_per_launch": flops,
        "achieved_tflops": flops / (kern * 1e-3) / 1e12,
        "work_per_step": {k: counts[k] for k in ("block_pairs", "polar_occluder_pairs", "pairs_evaluated",
                                                 "bridged_pairs")},
    }, step


def cpu_lkball_sample(ps, reps=3):
    """tmol's CPU LK-ball ops (oracle/_ref/lk_ball, else the C restatement)
    on the whole batch: waters, energies, gradient; single thread, best of
    `reps`."""
    import numpy
    import torch

    from oracle import oracle as O
    from tmol_b200.score.lkball_energy_term import LKBallEnergyTerm, score_args, water_gen_args

    torch.set_num_threads(1)
    lt = LKBallEnergyTerm()
    wa, sa = water_gen_args(ps, lt), score_args(ps, lt, None)
    coords = ps.coords.flatten(0, 1)
    if O.reference_lkball_available():
        kind = "reference"

        def run():
            E, _, _, _ = O.reference_lkball(coords, wa, sa)
            E.sum().backward()

    else:
        kind = "port"
        oc = O.OracleCall(coords, sa, term="lkball", lkb_water_args=wa)
        ones = numpy.ones((4, ps.n_poses))

        def run():
            oc.lkb_scores(oc.lkb_waters(), weights=ones)

    run()
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        run()
        best = min(best, time.perf_counter() - t0)
    return kind, best


def run_lkball(args, world, rank, local):
    """The LK-ball term on the uniform batch: waters, the four energies per
    pose and the gradient of their sum through the waters, one call per
    step (4 kernels and the sphere pass), replayed as a CUDA graph."""
    import torch

    from tmol_b200 import native
    from tmol_b200.score.lkball_op import gen_pose_waters, lk_ball_pose_score

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    sizes, seeds = workload_sizes("lkball64x150", rank)
    ps = workload(rank, "lkball64x150", device=dev)
    coords = ps.coords.flatten(0, 1).to(dev).contiguous()
    plan = lkball_plan_for(ps, coords)
    P = ps.n_poses
    flush = torch.empty(L2_FLUSH_BYTES // 4, device=dev, dtype=torch.float32)
    m, step = measure_lkball(plan, coords, flush, max(args.warmup, 3))
    if args.launch:
        launch = tuple(int(v) for v in args.launch.split(","))
        plan.set_launch(*launch)
        plan.balance(step)
    else:
        from tmol_b200.tune import autotune

        launch, _ = autotune(plan, step, use_cache=False)
    m, step = measure_lkball(plan, coords, flush, max(args.warmup, 3))
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        step()
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=s):
            step()
    torch.cuda.current_stream().wait_stream(s)
    for _ in range(max(args.warmup, 3)):
        g.replay()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            g.replay()
            ev[k][1].record()
        torch.cuda.synchronize()
    barrier(world)
    ms_max = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), world)
    poses_total = sum_over_ranks(P * args.steps, world)
    value = poses_total / (ms_max / 1e3)
    m, _ = measure_lkball(plan, coords, flush, args.steps)

    # end to end, pinned coordinates in and energies and gradient out: through
    # the C entry point (e2e), and through the drop-in ops as tmol's LK-ball
    # term calls them (gen_pose_waters, lk_ball_pose_score, backward through
    # both)
    from tmol_b200.score.lkball_energy_term import LKBallEnergyTerm, score_args, water_gen_args

    lt = LKBallEnergyTerm()
    wa = [a.to(dev) if isinstance(a, torch.Tensor) else a for a in water_gen_args(ps, lt)]
    sa = [a.to(dev) if isinstance(a, torch.Tensor) else a for a in score_args(ps, lt, None)[:-2]]
    del ps
    h_coords = coords.cpu().pin_memory()
    h_E = torch.empty((4, P), pin_memory=True)
    h_g = torch.empty(coords.shape, pin_memory=True)

    def e2e_step():
        d_in = h_coords.to(dev, non_blocking=True).requires_grad_(True)
        W = gen_pose_waters(d_in, *wa)
        E, _ = lk_ball_pose_score(d_in, *sa, W, False, return_block_neighbors=False)
        E.sum().backward()
        h_E.copy_(E.detach(), non_blocking=True)
        h_g.copy_(d_in.grad, non_blocking=True)

    def timed(fn):
        for _ in range(max(args.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        barrier(world)
        for k in range(args.steps):
            flush.zero_()
            evs[k][0].record()
            fn()
            evs[k][1].record()
        torch.cuda.synchronize()
        barrier(world)
        return max_over_ranks(sum(a.elapsed_time(b) for a, b in evs), world)

    # the plan's one-call C entry point with host buffers (pinned coordinates
    # in; energies and gradient out), as the LJ/LK arm measures it
    w1 = torch.ones((4, P), device=dev)
    E1 = torch.empty((4, P), device=dev)
    dx1 = torch.empty_like(coords)
    d_in = torch.empty_like(coords)

    def e2e_c_abi():
        d_in.copy_(h_coords, non_blocking=True)
        plan.energy_and_gradient(d_in, w1, E1, dx1)
        h_E.copy_(E1, non_blocking=True)
        h_g.copy_(dx1, non_blocking=True)

    serial_ms = timed(e2e_c_abi)
    e2e_ms = pipelined_e2e_ms(plan, w1, h_coords, flush, args.steps, world, P, n_terms=4)
    dropin_ms = timed(e2e_step)

    fp32_peak = native.measure_fp32_peak_tflops(torch.cuda.current_stream().cuda_stream)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from tmol_b200.pose.synthetic import synthetic_pose_stack

        n_sample = 8
        kind, t = cpu_lkball_sample(synthetic_pose_stack(sizes[:n_sample], seeds[:n_sample]))
        cpu = {
            "value": n_sample / t,
            "unit": "poses/s",
            "cores": 1,
            "kind": kind,
            "sample": f"{n_sample} of the {len(sizes)} {N_RES}-residue poses, waters + energies + gradient, "
            "best of 3, one thread",
        }
    if rank == 0:
        line = {
            "metric": LKBALL_METRIC,
            "value": value,
            "unit": "poses/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded proteins, ideal geometry)",
            "config": {
                "workload": workload_label("lkball64x150"),
                "poses_per_gpu": P,
                "atoms_per_gpu": int(coords.shape[0]),
                "l2": "flushed (256 MiB write) before every timed step",
                "launch": "CUDA graph replay: 4 kernels per step (waters, block spheres, scoring with its "
                "adjoint, waters adjoint) and 5 memsets",
                "launch_shape": dict(
                    zip(LAUNCH_FIELDS, launch)
                ),
                "parallelism": f"weak, {world} independent batch(es)",
            },
            "work_per_step": m["work_per_step"],
            "gpu_launches": 4 * args.steps,
            "clocks": clk.summary(),
            "roofline": {
                "bound": "fp32",
                "achieved": m["achieved_tflops"],
                "peak": fp32_peak,
                "unit": "TFLOP/s",
                "frac": m["achieved_tflops"] / fp32_peak,
                "traffic": load_traffic("lkb_score"),
                "kernel": "lkb_score_kernel<float, GRAD> (neighbour test + polar/occluder energies and adjoint)",
                "traffic_source": "ncu capture, profiles/lkb_score_traffic.json",
                "kernel_ms": m["kernel_ms"],
                "flops_per_launch": m["flops_per_launch"],
                "peak_source": "measured: FMA-loop probe over all SMs in this run (tmol_b200_measure_fp32_peak)",
            },
            "e2e": {
                "value": poses_total / (e2e_ms / 1e3),
                "unit": "poses/s",
                "h2d_bytes_per_step": coords.numel() * 4,
                "d2h_bytes_per_step": (4 * P + coords.numel()) * 4,
                "path": "tmol_b200_lkball_energy_and_gradient (C ABI) with host buffers",
                "schedule": "double-buffered over copy-in / compute / copy-out streams; L2 flushed before every "
                "step's compute, inside the timed region; timed over max(steps, %d) steps" % E2E_MIN_STEPS,
                "serial_value": poses_total / (serial_ms / 1e3),
            },
            "e2e_dropin_ops": {
                "value": poses_total / (dropin_ms / 1e3),
                "unit": "poses/s",
                "path": "gen_pose_waters + lk_ball_pose_score drop-ins, autograd backward, same host copies",
            },
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    del g
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def run_sfxn(args, world, rank, local):
    """The three terms as one score function on the uniform batch: per step
    each plan's one-call energy + gradient (LJ/LK, elec, LK-ball with its
    waters) under the score-type weights, and the summed gradient; replayed
    as a CUDA graph."""
    import torch

    from tmol_b200 import native
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args
    from tmol_b200.score.ljlk_op import LJLKPlan
    from tmol_b200.tune import autotune

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    sizes, seeds = workload_sizes("sfxn64x150", rank)
    ps = workload(rank, "sfxn64x150", device=dev)
    coords = ps.coords.flatten(0, 1).to(dev).contiguous()
    P = ps.n_poses
    plans = [
        LJLKPlan(coords, pose_score_args(ps, LJLKEnergyTerm(device=dev))[:-1]),
        elec_plan_for(ps, coords),
        lkball_plan_for(ps, coords),
    ]
    del ps
    wt = torch.tensor(SFXN_WEIGHTS, device=dev)
    ws = [wt[0:3, None].expand(3, P).contiguous(), wt[3:4, None].expand(1, P).contiguous(),
          wt[4:8, None].expand(4, P).contiguous()]
    Es = [torch.empty((w.shape[0], P), device=dev) for w in ws]
    dxs = [torch.empty_like(coords) for _ in plans]
    dx = torch.empty_like(coords)
    flush = torch.empty(L2_FLUSH_BYTES // 4, device=dev, dtype=torch.float32)

    side = [torch.cuda.Stream(dev) for _ in plans]

    def step(c=coords):
        # the terms are independent: one stream each (parallel branches in
        # the captured graph), joined for the gradient sum
        cur = torch.cuda.current_stream(dev)
        for sd, plan, w, E, g in zip(side, plans, ws, Es, dxs):
            sd.wait_stream(cur)
            with torch.cuda.stream(sd):
                plan.energy_and_gradient(c, w, E, g)
        for sd in side:
            cur.wait_stream(sd)
        torch.add(dxs[0], dxs[1], out=dx)
        dx.add_(dxs[2])

    # each term's launch shape autotuned on its own call, work ordered by cost
    for plan, w, E, g in zip(plans, ws, Es, dxs):
        autotune(plan, lambda plan=plan, w=w, E=E, g=g: plan.energy_and_gradient(coords, w, E, g), use_cache=False)
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    st = torch.cuda.Stream()
    st.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(st):
        step()
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=st):
            step()
    torch.cuda.current_stream().wait_stream(st)
    for _ in range(max(args.warmup, 3)):
        g.replay()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            g.replay()
            ev[k][1].record()
        torch.cuda.synchronize()
    barrier(world)
    ms_max = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), world)
    poses_total = sum_over_ranks(P * args.steps, world)
    value = poses_total / (ms_max / 1e3)
    # the scoring kernels' own times and the FLOP models' work
    kern_ms, flops = 0.0, 0.0
    for i, (plan, w, E, gg) in enumerate(zip(plans, ws, Es, dxs)):
        plan.profile(True)
        for _ in range(args.steps):
            flush.zero_()
            plan.energy_and_gradient(coords, w, E, gg)
        ms, n = plan.profile_read()
        plan.profile(False)
        kern_ms += ms / max(n, 1)
        c = counted_work(plan, lambda: plan.energy_and_gradient(coords, w, E, gg))
        if i == 0:
            flops += c["atom_pairs"] * F_PAIR_TEST + c["atom_pairs_in_range"] * F_LJ + c["heavy_pairs_in_range"] * F_LK
        elif i == 1:
            flops += c["atom_pairs"] * F_PAIR_TEST + c["atom_pairs_in_range"] * F_ELEC
        else:
            flops += c["pairs_evaluated"] * F_LKB_PAIR + c["bridged_pairs"] * F_LKB_BRIDGE
    # end to end: pinned coordinates in, the weighted totals and the summed
    # gradient out, step by step
    h_coords = coords.cpu().pin_memory()
    h_E = torch.empty((P,), pin_memory=True)
    h_g = torch.empty(coords.shape, pin_memory=True)
    d_in = torch.empty_like(coords)
    total = torch.empty((P,), device=dev)
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    for k in range(args.steps + 2):
        flush.zero_()
        if k >= 2:
            e2e_ev[k - 2][0].record()
        d_in.copy_(h_coords, non_blocking=True)
        step(d_in)
        torch.sum(torch.cat([w * E for w, E in zip(ws, Es)]), dim=0, out=total)
        h_E.copy_(total, non_blocking=True)
        h_g.copy_(dx, non_blocking=True)
        if k >= 2:
            e2e_ev[k - 2][1].record()
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in e2e_ev), world)
    fp32_peak = native.measure_fp32_peak_tflops(torch.cuda.current_stream().cuda_stream)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from tmol_b200.pose.synthetic import synthetic_pose_stack

        n_sample = 8
        ps0 = synthetic_pose_stack(sizes[:n_sample], seeds[:n_sample])
        k1, t1 = cpu_reference_sample(ps0, LJLKEnergyTerm(), reps=2)
        k2, t2 = cpu_elec_sample(ps0, reps=2)
        k3, t3 = cpu_lkball_sample(ps0, reps=2)
        cpu = {
            "value": n_sample / (t1 + t2 + t3),
            "unit": "poses/s",
            "cores": 1,
            "kind": "reference" if k1 == k2 == k3 == "reference" else "port",
            "sample": f"{n_sample} of the {len(sizes)} {N_RES}-residue poses, the three reference ops (LK-ball with "
            "its waters), energies + gradient, best of 2 each, one thread",
        }
    if rank == 0:
        achieved = flops / (kern_ms * 1e-3) / 1e12
        line = {
            "metric": SFXN_METRIC,
            "value": value,
            "unit": "poses/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded proteins, ideal geometry)",
            "config": {
                "workload": workload_label("sfxn64x150"),
                "poses_per_gpu": P,
                "atoms_per_gpu": int(coords.shape[0]),
                "l2": "flushed (256 MiB write) before every timed step",
                "launch": "CUDA graph replay: 10 kernels per step (LJ/LK 2, elec 2, LK-ball 4 on three concurrent "
                "streams, gradient sum 2)",
                "parallelism": f"weak, {world} independent batch(es)",
            },
            "gpu_launches": 10 * args.steps,
            "clocks": clk.summary(),
            "roofline": {
                "bound": "fp32",
                "achieved": achieved,
                "peak": fp32_peak,
                "unit": "TFLOP/s",
                "frac": achieved / fp32_peak,
                "traffic": None,
                "kernel": "the three scoring kernels (score_kernel LJ/LK and elec, lkb_score_kernel), FLOPs and "
                "times summed",
                "kernel_ms": kern_ms,
                "flops_per_launch": flops,
                "peak_source": "measured: FMA-loop probe over all SMs in this run (tmol_b200_measure_fp32_peak)",
            },
            "e2e": {
                "value": poses_total / (e2e_ms / 1e3),
                "unit": "poses/s",
                "h2d_bytes_per_step": coords.numel() * 4,
                "d2h_bytes_per_step": (P + coords.numel()) * 4,
                "schedule": "step by step",
            },
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    del g
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def _bondsep_port_worker(conn, sizes, seeds):
    """One single-threaded process of the bond-separation CPU arm: the C
    restatement of the reference route (connection-point matrix, shortest
    paths with cutoff 6, scatter), one pose at a time."""
    from oracle import oracle as O
    from tmol_b200.pose.synthetic import synthetic_topologies_and_coords
    from tmol_b200.pose.builder import build_pose_stack

    stacks = []
    for sz, sd in zip(sizes, seeds):
        topos, _ = synthetic_topologies_and_coords([sz], [sd], with_coords=False)
        stacks.append(build_pose_stack(topos))
    conn.send("ready")
    while True:
        msg = conn.recv()
        if msg is None:
            break
        t0 = time.perf_counter()
        for ps in stacks:
            pbt = ps.packed_block_types
            O.pose_bondsep(ps.block_type_ind, ps.inter_residue_connections, pbt.n_conn, pbt.conn_at_intrablock_bond_sep)
        conn.send(time.perf_counter() - t0)


def bondsep_cpu_sample(sizes, seeds, n=16):
    """The C restatement of the reference route on one core, on n seeded
    poses of the batch (each as its own stack), scaled to the batch by pose
    count; seconds per batch."""
    import numpy

    from oracle import oracle as O
    from tmol_b200.pose.builder import build_pose_stack
    from tmol_b200.pose.synthetic import synthetic_topologies_and_coords

    pick = numpy.random.default_rng(7).choice(len(sizes), n, replace=False)
    stacks = []
    for k in pick:
        topos, _ = synthetic_topologies_and_coords([sizes[k]], [seeds[k]], with_coords=False)
        stacks.append(build_pose_stack(topos))
    best = float("inf")
    for _ in range(3):
        t0 = time.perf_counter()
        for ps in stacks:
            pbt = ps.packed_block_types
            O.pose_bondsep(ps.block_type_ind, ps.inter_residue_connections, pbt.n_conn, pbt.conn_at_intrablock_bond_sep)
        best = min(best, time.perf_counter() - t0)
    return best * len(sizes) / n, [int(sizes[k]) for k in pick]


def run_bondsep(args, world, rank, local):
    """PoseStack bond separation on the GPU: the dense inter_block_bondsep
    [P, B, B, C, C] and min_bondsep [P, B, B] of the uneven batch from its
    connectivity, per step one call of tmol_b200_pose_bondsep (three
    kernels and a status word; its status is read after the timed steps).  Also: scoring-plan creation
    from the connectivity (no dense tensors) against creation from them."""
    import ctypes

    import torch

    from tmol_b200 import native
    from tmol_b200.pose.bondsep import pose_connectivity
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args
    from tmol_b200.score.ljlk_op import LJLKPlan

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    sizes, seeds = workload_sizes("uneven256", rank)
    ps = workload(rank, "uneven256", device=dev)
    P, B, C = ps.n_poses, ps.max_n_blocks, ps.packed_block_types.max_n_conn
    cs, keep = pose_connectivity(ps)
    ibb = torch.empty((P, B, B, C, C), dtype=torch.int32, device=dev)
    mb = torch.empty((P, B, B), dtype=torch.int32, device=dev)
    status = torch.empty(1, dtype=torch.int32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, device=dev, dtype=torch.float32)
    stream = torch.cuda.current_stream(dev)

    def step(dense=True):
        native.call(
            "tmol_b200_pose_bondsep", ctypes.byref(cs), ctypes.c_void_p(ibb.data_ptr() if dense else 0),
            ctypes.c_void_p(mb.data_ptr()), ctypes.c_void_p(status.data_ptr()), ctypes.c_void_p(stream.cuda_stream),
        )

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            step()
            ev[k][1].record()
        torch.cuda.synchronize()
    barrier(world)
    ms_max = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), world)
    value = sum_over_ranks(P * args.steps, world) / (ms_max / 1e3)
    ms_step = ms_max / args.steps
    # min_bondsep alone (the compact output)
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.zero_()
        ev2[k][0].record()
        step(dense=False)
        ev2[k][1].record()
    torch.cuda.synchronize()
    ms_min_only = sum(a.elapsed_time(b) for a, b in ev2) / args.steps
    native.check("tmol_b200_pose_bondsep", int(status.item()))
    step()
    assert torch.equal(ibb, ps.inter_block_bondsep)

    # algorithmic bytes: the dense outputs written once, the connectivity
    # read once (int32)
    n_conn_pts = int(torch.where(ps.block_type_ind >= 0, ps.packed_block_types.n_conn[ps.block_type_ind.clamp(min=0).long()], 0).sum())
    out_bytes = (ibb.numel() + mb.numel()) * 4
    in_bytes = (ps.block_type_ind.numel() + ps.inter_residue_connections.numel()) * 4
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    achieved = (out_bytes + in_bytes) / (ms_step * 1e-3) / 1e9

    # plan creation: from the dense tensors vs from the connectivity
    term = LJLKEnergyTerm(device=dev)
    static = [a.to(dev) if isinstance(a, torch.Tensor) else a for a in pose_score_args(ps, term)[:-1]]
    coords = ps.coords.flatten(0, 1).contiguous()
    sparse_static = [None if i in (12, 13) else a for i, a in enumerate(static)]
    times = {}
    for name, kw, st in (("dense", {}, static), ("connectivity", {"connectivity": ps}, sparse_static)):
        LJLKPlan(coords, st, **kw)  # warm
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(3):
            LJLKPlan(coords, st, **kw)
        torch.cuda.synchronize()
        times[name] = (time.perf_counter() - t0) / 3 * 1e3

    # end to end: connectivity from pinned host memory, min_bondsep back
    h_bt = ps.block_type_ind.cpu().pin_memory()
    h_irc = ps.inter_residue_connections.cpu().pin_memory()
    h_mb = torch.empty(mb.shape, dtype=torch.int32, pin_memory=True)
    d_bt = torch.empty_like(ps.block_type_ind)
    d_irc = torch.empty_like(ps.inter_residue_connections)
    cs2 = native.PoseConnectivity(P, B, cs.n_block_types, C, d_bt.data_ptr(), d_irc.data_ptr(), cs.bt_n_conn,
                                  cs.bt_conn_sep)
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.zero_()
        e2e_ev[k][0].record()
        d_bt.copy_(h_bt, non_blocking=True)
        d_irc.copy_(h_irc, non_blocking=True)
        native.call("tmol_b200_pose_bondsep", ctypes.byref(cs2), ctypes.c_void_p(ibb.data_ptr()),
                    ctypes.c_void_p(mb.data_ptr()), ctypes.c_void_p(status.data_ptr()),
                    ctypes.c_void_p(stream.cuda_stream))
        h_mb.copy_(mb, non_blocking=True)
        e2e_ev[k][1].record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in e2e_ev), world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t_batch, picked = bondsep_cpu_sample(sizes, seeds)
        cpu = {
            "value": len(sizes) / t_batch,
            "unit": "poses/s",
            "cores": 1,
            "kind": "port",
            "sample": f"16 seeded poses of the batch ({sum(picked)} residues), each as its own stack, "
            "C restatement of the reference route (bit-exact with the compiled reference apsp op), "
            "best of 3, one thread; scaled to the batch by pose count",
        }
    if rank == 0:
        line = {
            "metric": BONDSEP_METRIC,
            "value": value,
            "unit": "poses/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "int32",
            "data": "synthetic (seeded single-chain proteins)",
            "config": {
                "workload": f"{P} poses, residues log-uniform in [20, 1000], B = {B}, C = {C}, "
                f"{n_conn_pts} connection points",
                "l2": "flushed (256 MiB write) before every timed step; outputs far larger than L2",
                "parallelism": f"weak, {world} independent batch(es)",
            },
            "gpu_launches": 4 * args.steps,
            "clocks": clk.summary(),
            "roofline": {
                "bound": "hbm",
                "achieved": achieved,
                "peak": hbm,
                "unit": "GB/s",
                "frac": achieved / hbm if hbm else None,
                "traffic": None,
                "kernel": "fill_i32_kernel (x2) + bondsep_sources_kernel + status, one call",
                "bytes_per_step": out_bytes + in_bytes,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (burst copy)",
            },
            "min_bondsep_only_ms": ms_min_only,
            "plan_create_ms": times,
            "dense_tensor_bytes_avoided": int(ps.inter_block_bondsep.numel() * 4 + mb.numel() * 4),
            "e2e": {
                "value": sum_over_ranks(P * args.steps, world) / (e2e_ms / 1e3),
                "unit": "poses/s",
                "h2d_bytes_per_step": in_bytes,
                "d2h_bytes_per_step": mb.numel() * 4,
            },
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    del keep
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def run_reference_bondsep(args):
    """The C restatement of the reference route on all host cores: one
    process per core, poses dealt out longest-first."""
    import multiprocessing as mp

    sizes, seeds = workload_sizes("uneven256", 0)
    n_poses = len(sizes)
    n_proc = min(os.cpu_count() or 1, n_poses)
    shares = [[] for _ in range(n_proc)]
    load = [0] * n_proc
    for k in sorted(range(n_poses), key=lambda k: -sizes[k]):
        q = load.index(min(load))
        shares[q].append(k)
        load[q] += sizes[k] ** 2
    ctx = mp.get_context("spawn")
    workers = []
    for share in shares:
        parent, child = ctx.Pipe()
        pr = ctx.Process(target=_bondsep_port_worker, args=(child, [sizes[k] for k in share], [seeds[k] for k in share]))
        pr.start()
        workers.append((pr, parent))
    for _, c in workers:
        c.recv()

    def step():
        t0 = time.perf_counter()
        for _, c in workers:
            c.send(1)
        for _, c in workers:
            c.recv()
        return time.perf_counter() - t0

    for _ in range(max(args.warmup, 1)):
        step()
    times = [step() for _ in range(args.steps)]
    for pr, c in workers:
        c.send(None)
        pr.join()
    t = sum(times)
    value = n_poses * args.steps / t
    line = {
        "impl": "reference",
        "metric": BONDSEP_METRIC,
        "value": value,
        "unit": "poses/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int32",
        "data": "synthetic (seeded single-chain proteins)",
        "config": {"workload": f"{n_poses} poses, residues log-uniform in [20, 1000]"},
        "cpu_baseline": {
            "value": value,
            "unit": "poses/s",
            "cores": n_proc,
            "kind": "port",
            "sample": f"the full {n_poses}-pose batch per step, each pose as its own stack, dealt to {n_proc} "
            "single-threaded processes (C restatement of the reference route)",
        },
        "e2e": {"value": value, "unit": "poses/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def measure_pose_batch(args, workload_name, world, rank, local, steps, extras=True):
    """One LJ/LK pose workload on this rank's GPU: the timed graph replays,
    the scoring kernel's own time and roofline, the end-to-end figures and
    (rank 0) the CPU baseline.  Returns the JSON line's dict on rank 0."""
    import torch

    from tmol_b200 import native
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args
    from tmol_b200.score.ljlk_op import LJLKPlan, clear_plan_cache, ljlk_pose_scores

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    term = LJLKEnergyTerm()
    sizes_seeds = workload_sizes(workload_name, rank)
    ps = workload(rank, workload_name, device=dev)
    full_args = [a.to(dev) if isinstance(a, torch.Tensor) else a for a in pose_score_args(ps, term)]
    static = full_args[:-1]
    coords = ps.coords.flatten(0, 1).to(dev).contiguous()
    plan = LJLKPlan(coords, static)
    with_screen = extras and not args.no_screen
    with_elec = extras and not args.no_elec
    plan64 = LJLKPlan(coords.double(), static) if with_screen else None
    eplan = elec_plan_for(ps, coords) if with_elec else None
    bt_names = [bt.name for bt in ps.packed_block_types.active_block_types]
    del static
    P = ps.n_poses
    n_residues = int((ps.block_type_ind >= 0).sum())
    del ps
    torch.cuda.empty_cache()
    weights = torch.tensor(TERM_WEIGHTS, device=dev, dtype=torch.float32)[:, None].expand(3, P).contiguous()
    energies = torch.empty((3, P), device=dev)
    dcoords = torch.empty_like(coords)
    flush = torch.empty(L2_FLUSH_BYTES // 4, device=dev, dtype=torch.float32)
    perturb = workload_name == "uneven256"
    base = coords.clone()
    noise = torch.empty_like(coords)

    def step():
        if perturb:
            noise.normal_(0.0, PERTURB_SD)
            torch.add(base, noise, out=coords)
        plan.energy_and_gradient(coords, weights, energies, dcoords)

    # warm-up (also validates the launch), autotuning of the launch shape and
    # work order, then capture of one step as a graph
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    from tmol_b200.tune import autotune

    if args.launch:
        launch_shape = tuple(int(v) for v in args.launch.split(","))
        plan.set_launch(*launch_shape)
        plan.balance(step)
    else:
        launch_shape, _ = autotune(plan, step, use_cache=False)
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    counts = counted_work(plan, step)
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        step()
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=s):
            step()
    torch.cuda.current_stream().wait_stream(s)
    for _ in range(max(args.warmup, 3)):
        g.replay()
    torch.cuda.synchronize()

    # timed region: K graph replays, L2 flushed before each (outside the events)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(steps):
            flush.zero_()
            ev[k][0].record()
            g.replay()
            ev[k][1].record()
        torch.cuda.synchronize()
    barrier(world)
    ms = sum(a.elapsed_time(b) for a, b in ev)
    ms_max = max_over_ranks(ms, world)
    poses_total = sum_over_ranks(P * steps, world)
    value = poses_total / (ms_max / 1e3)

    # kernel-level timing of the scoring kernel (direct launches, events
    # recorded by the library around each launch on the launching stream)
    plan.profile(True)
    for _ in range(steps):
        flush.zero_()
        step()
    kern_ms, n_launch = plan.profile_read()
    plan.profile(False)
    kern_avg_ms = kern_ms / max(n_launch, 1)

    # end to end through the public entry point with host buffers: pinned
    # coordinates in, energies and gradient out, copies inside the timing
    h_coords = coords.cpu().pin_memory()
    h_E = torch.empty((3, P), pin_memory=True)
    h_g = torch.empty(coords.shape, pin_memory=True)
    d_in = torch.empty_like(coords)
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for _ in range(2):
        d_in.copy_(h_coords, non_blocking=True)
        plan.energy_and_gradient(d_in, weights, energies, dcoords)
        h_E.copy_(energies, non_blocking=True)
        h_g.copy_(dcoords, non_blocking=True)
    torch.cuda.synchronize()
    barrier(world)
    for k in range(steps):
        flush.zero_()
        e2e_ev[k][0].record()
        d_in.copy_(h_coords, non_blocking=True)
        plan.energy_and_gradient(d_in, weights, energies, dcoords)
        h_E.copy_(energies, non_blocking=True)
        h_g.copy_(dcoords, non_blocking=True)
        e2e_ev[k][1].record()
    torch.cuda.synchronize()
    barrier(world)
    serial_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in e2e_ev), world)
    # the same steps double-buffered over three streams, as a host pipeline
    # runs them: step k+1's coordinates go in and step k-1's results come out
    # while step k computes; every step still copies its inputs in, flushes
    # L2 and copies its energies and gradient out inside the timed region
    e2e_ms = pipelined_e2e_ms(plan, weights, h_coords, flush, steps, world, P)
    e2e_value = poses_total / (e2e_ms / 1e3)
    h2d = coords.numel() * 4
    d2h = (3 * P + coords.numel()) * 4

    # end to end through tmol's drop-in op, as a tmol caller runs it: the
    # 27-argument ljlk_pose_scores on coordinates copied in from pinned host
    # memory, backward() of the weighted energies through the autograd
    # function, energies and gradient copied back, step by step
    dropin_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    w_col = weights[:, :1].contiguous()

    def dropin_step():
        c = d_in.copy_(h_coords, non_blocking=True).requires_grad_(True)
        E, _ = ljlk_pose_scores(c, *full_args)
        (E * w_col).sum().backward()
        h_E.copy_(E.detach(), non_blocking=True)
        h_g.copy_(c.grad, non_blocking=True)
        c.grad = None
        c.requires_grad_(False)

    for _ in range(3):
        dropin_step()
    torch.cuda.synchronize()
    barrier(world)
    for k in range(steps):
        flush.zero_()
        dropin_ev[k][0].record()
        dropin_step()
        dropin_ev[k][1].record()
    torch.cuda.synchronize()
    barrier(world)
    dropin_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in dropin_ev), world)
    clear_plan_cache()

    screened = None
    if with_screen:
        screened = measure_screen(
            plan, plan64, coords, weights, step, flush, steps, bt_names, ms_max / steps
        )
        del plan64

    fp32_peak = native.measure_fp32_peak_tflops(torch.cuda.current_stream().cuda_stream)
    elec = None
    if eplan is not None:
        # the elec term on the same batch and launch shape (its own workload
        # line: --workload elec64x150)
        eplan.set_launch(*launch_shape)
        elec, _ = measure_elec(eplan, coords, flush, steps)
        elec["roofline_frac"] = elec["achieved_tflops"] / fp32_peak
        elec["metric"] = ELEC_METRIC
        del eplan
    flops = flops_per_step(counts)
    achieved = flops / (kern_avg_ms * 1e-3) / 1e12

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_for(workload_name, sizes_seeds, counts["atom_pairs"])

    line = None
    if rank == 0:
        peaks = measured_peaks()
        traffic = load_traffic()
        line = {
            "metric": METRIC if workload_name == "uniform64x150" else METRIC.replace(
                "64x150-residue batch", "256-pose uneven batch"
            ),
            "value": value,
            "unit": "poses/s",
            "n_gpus": world,
            "steps": steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max / steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded proteins, ideal geometry)",
            "config": {
                "workload": workload_label(workload_name),
                "poses_per_gpu": P,
                "residues_per_gpu": n_residues,
                "atoms_per_gpu": int(coords.shape[0]),
                "l2": "flushed (256 MiB write) before every timed step",
                "launch": "CUDA graph replay: 2 kernels per step" + (" + perturbation" if perturb else ""),
                "launch_shape": dict(
                    zip(LAUNCH_FIELDS, launch_shape)
                ),
                "parallelism": f"weak, {world} independent batch(es)",
            },
            "atom_pairs_per_s": counts["atom_pairs"] * steps * world / (ms_max / 1e3),
            "work_per_step": counts,
            "gpu_launches": 2 * steps,
            "clocks": clk.summary(),
            "roofline": {
                "bound": "fp32",
                "achieved": achieved,
                "peak": fp32_peak,
                "unit": "TFLOP/s",
                "frac": achieved / fp32_peak,
                "traffic": traffic if workload_name == "uniform64x150" else None,
                "kernel": "score_kernel<float, GRAD> (fused neighbour + atom-pair energy and gradient)",
                "kernel_ms": kern_avg_ms,
                "flops_per_launch": flops,
                "peak_source": "measured: FMA-loop probe over all SMs in this run (tmol_b200_measure_fp32_peak)",
                "hbm_peak_gbs": peaks.get("hbm_gbs"),
            },
            "e2e": {
                "value": e2e_value,
                "unit": "poses/s",
                "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "schedule": "double-buffered over copy-in / compute / copy-out streams; L2 flushed before every "
                "step's compute, inside the timed region; timed over max(steps, %d) steps" % E2E_MIN_STEPS,
                "serial_value": poses_total / (serial_ms / 1e3),
                "dropin_value": poses_total / (dropin_ms / 1e3),
                "dropin_schedule": "tmol's drop-in op ljlk_pose_scores (27 arguments) + backward() through its "
                "autograd function (speculative gradient: one fused scoring pass per forward + backward once "
                "the weights repeat), coordinates in from pinned host memory, energies and gradient out, step by "
                "step, L2 flushed before each step inside the timed region",
            },
            "cpu_baseline": cpu,
            "screened": screened,
            "elec": elec,
        }
    del g
    return line


def sub_record(line):
    """The parts of a workload's line that a sub-record keeps."""
    keep = ("metric", "value", "unit", "steps", "ms_per_step", "config", "atom_pairs_per_s", "work_per_step",
            "clocks", "roofline", "e2e", "cpu_baseline")
    return {k: line[k] for k in keep if k in line}


def measure_lbfgs(local, n_poses=32, n_res=300, iters=200):
    """The minimisation scenario: 32 poses x 300 residues with chis + N(0,
    30 deg), 200 iterations of the batched L-BFGS on Cartesian coordinates,
    every energy + gradient one fused pass of the scoring kernel."""
    import torch

    from tmol_b200.optimization.lbfgs import LBFGSArmijo
    from tmol_b200.optimization.minimize import BETA2016_WEIGHTS, make_func
    from tmol_b200.pose.synthetic import synthetic_pose_stack
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args
    from tmol_b200.score.ljlk_op import LJLKPlan

    dev = torch.device("cuda", local)
    ps = synthetic_pose_stack([n_res] * n_poses, list(range(n_poses)), device=dev, extra_chi_sd=30.0)
    term = LJLKEnergyTerm(device=dev)
    coords = ps.coords.flatten(0, 1).contiguous()
    plan = LJLKPlan(coords, pose_score_args(ps, term)[:-1])
    P, A = ps.n_poses, ps.max_n_pose_atoms
    func = make_func(plan, BETA2016_WEIGHTS, P, A)
    x0 = ps.coords.reshape(P, -1)
    plan.balance(lambda: func(x0))
    E0, _ = func(x0)
    LBFGSArmijo(func, x0, max_iter=3).run()  # warm-up
    opt = LBFGSArmijo(func, x0, max_iter=iters)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    wall0 = time.perf_counter()
    t0.record()
    x, E, gr = opt.run()
    t1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    ms = t0.elapsed_time(t1)
    # tmol's route: run_min over a CartesianSfxnNetwork of the score function
    # with LBFGS_Armijo (tmol's interface and steps), every evaluation the
    # drop-in op's forward and its autograd adjoint
    from tmol_b200.optimization.minimizers import run_min
    from tmol_b200.optimization.sfxn_modules import CartesianSfxnNetwork
    from tmol_b200.score.score_function import ScoreFunction

    sfxn = ScoreFunction.from_weights({"fa_ljatr": 1.0, "fa_ljrep": 0.55, "fa_lk": 1.0}, device=dev)
    net = CartesianSfxnNetwork(sfxn, ps)
    run_min(CartesianSfxnNetwork(sfxn, ps), optimizer_kwargs=dict(max_iter=3))  # warm-up
    torch.cuda.synchronize()
    t2, t3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t2.record()
    out, topt = run_min(net, optimizer_kwargs=dict(max_iter=iters))
    t3.record()
    torch.cuda.synchronize()
    tms = t2.elapsed_time(t3)
    E_t = topt.energy_history[-1]
    tmol_route = {
        "what": "tmol's route: run_min over CartesianSfxnNetwork(ScoreFunction beta2016 LJ/LK) with "
        "LBFGS_Armijo (tmol's interface and steps), each evaluation the drop-in op + autograd adjoint",
        "iterations": len(topt.energy_history) - 1,
        "evaluations": topt.n_evals,
        "ms_total": tms,
        "ms_per_evaluation": tms / max(topt.n_evals, 1),
        "energy_after_mean": float(E_t.mean()),
        "poses_whose_energy_fell": int((E_t < topt.energy_history[0]).sum()),
    }
    return {
        "scenario": f"{n_poses} poses x {n_res} residues, chis + N(0, 30 deg), beta2016 LJ/LK weights, "
        f"batched L-BFGS (Armijo) on Cartesian coordinates, {iters} iterations at most",
        "tmol_lbfgs_armijo": tmol_route,
        "iterations": len(opt.history) - 1,
        "evaluations": opt.n_evals,
        "ms_total": ms,
        "wall_s": wall,
        "ms_per_evaluation": ms / max(opt.n_evals, 1),
        "energy_before_mean": float(E0.mean()),
        "energy_after_mean": float(E.mean()),
        "poses_whose_energy_fell": int((E < E0).sum()),
        "max_abs_grad_after": float(gr.abs().max()),
    }


def measure_screen_eval(local, reps=20):
    """The learned block-pair screen on its held-out batch (16 poses x 1000
    residues, chis + N(0, 20 deg)): skipped fraction, per-pose |dE| in
    float64, and the energy + gradient step against the plain kernel, with
    the screen rebuilt every step and with the mask reused; beside it the
    exact zero-energy mask, the most any block-pair screen could skip (its
    speedup is the ceiling of the method on this kernel)."""
    import numpy
    import torch

    from tmol_b200.chem.restypes import default_packed_block_types
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm
    from tmol_b200.screen.mlp import ScreenMLP
    from tmol_b200.screen.screen import TRAINED_WEIGHTS
    from tmol_b200.screen.train import evaluate

    dev = torch.device("cuda", local)
    term = LJLKEnergyTerm(device=dev)
    names = [bt.name for bt in default_packed_block_types(dev).active_block_types]
    mlp, thr = ScreenMLP.load(TRAINED_WEIGHTS, dev, names)
    gap_thr = float(numpy.load(TRAINED_WEIGHTS, allow_pickle=False)["gap_threshold"])
    sizes, seeds = [1000] * 16, [30_000_000 + k for k in range(16)]
    res = evaluate(mlp, thr, gap_thr, sizes, seeds, 20.0, term, dev, reps, log=lambda m: None)
    lr, ceil = res["learned"], res["exact_zero_mask"]
    return {
        "workload": "16 held-out poses x 1000 residues, chis + N(0, 20 deg), energy + gradient, L2 flushed",
        "plain_ms": res["plain_ms"],
        "candidates": res["candidates"],
        "skipped_fraction": lr["skipped_fraction_of_candidates"],
        "max_abs_dE_per_pose_f64": lr["max_abs_dE_f64_total"],
        "budget_kcal_per_mol": 0.01,
        "speedup_with_update": lr.get("speedup_with_update"),
        "speedup_mask_reused": lr["speedup_kernel_only"],
        "update_ms": lr.get("update_ms"),
        "ceiling": {
            "what": "exact zero-energy mask (every candidate whose block-pair energy is zero skipped; no update "
            "cost counted): the most a block-pair screen can save on this kernel",
            "skipped_fraction": ceil["skipped_fraction_of_candidates"],
            "speedup": ceil["speedup_kernel_only"],
        },
        "sphere_gap_rule": {
            "skipped_fraction": res["sphere_gap_rule"]["skipped_fraction_of_candidates"],
            "speedup_mask_reused": res["sphere_gap_rule"]["speedup_kernel_only"],
        },
    }


def run_b200(args, world, rank, local):
    import torch

    line = measure_pose_batch(args, args.workload, world, rank, local, args.steps)
    # the other configurations of the path, as sub-records of the default
    # line (one GPU): the uneven batch through 100 perturbed graph replays,
    # the L-BFGS scenario, and the learned screen against its ceiling
    if args.workload == "uniform64x150" and world == 1 and not args.no_extras:
        torch.cuda.empty_cache()
        uneven = measure_pose_batch(args, "uneven256", world, rank, local, UNEVEN_REPLAYS, extras=False)
        line["uneven256"] = sub_record(uneven)
        torch.cuda.empty_cache()
        line["lbfgs"] = measure_lbfgs(local)
        torch.cuda.empty_cache()
        if not args.no_screen:
            line["screen_eval"] = measure_screen_eval(local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument(
        "--workload",
        default="uniform64x150",
        choices=[
            "uniform64x150", "uneven256", "rotamers16x150", "elec64x150", "lkball64x150", "lkball_rotamers16x150",
            "sfxn64x150", "bondsep256",
        ],
    )
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-screen", action="store_true", help="skip the learned-screen measurement")
    ap.add_argument("--no-elec", action="store_true", help="skip the elec summary of the default line")
    ap.add_argument(
        "--no-extras", action="store_true",
        help="skip the default line's sub-records (uneven batch, L-BFGS, screen evaluation)",
    )
    ap.add_argument(
        "--launch",
        default="",
        help="fixed launch shape items_per_ticket,warps_per_cta,ctas_per_sm,candidates_per_item[,slots_per_group] "
        "(default: autotune)",
    )
    args = ap.parse_args()
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        return run_reference(args, world, rank)
    world, rank, local = dist_setup()
    if args.workload == "rotamers16x150":
        return run_rotamers(args, world, rank, local)
    if args.workload == "elec64x150":
        return run_elec(args, world, rank, local)
    if args.workload == "lkball64x150":
        return run_lkball(args, world, rank, local)
    if args.workload == "lkball_rotamers16x150":
        return run_lkball_rotamers(args, world, rank, local)
    if args.workload == "sfxn64x150":
        return run_sfxn(args, world, rank, local)
    if args.workload == "bondsep256":
        return run_bondsep(args, world, rank, local)
    return run_b200(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
