"""Seeded synthetic proteins for parity tests and benchmarks.

Residue identities are drawn uniformly from the 20 canonical L-amino acids
of tmol's chemical database; geometry is ideal (bond lengths and angles from
the residue types' internal coordinates).  Backbone dihedrals are 60% helical
(phi ~ N(-63, 10), psi ~ N(-41, 10)) and 40% strand (phi ~ N(-120, 15),
psi ~ N(130, 15)); omega = 180; side-chain chis are drawn from
{-60, 60, 180} + N(0, 10), optionally with extra N(0, chi_sd) noise.
Coordinates are float32.
"""

import numpy
import torch

from ..chem.restypes import ResidueTypeSet, default_packed_block_types
from .builder import build_chain_coords, build_pose_stack, topology_from_sequence

CANONICAL_1LC = "ARNDCQEGHILKMFPSTWYV"


def random_sequence(rng, n):
    return "".join(CANONICAL_1LC[i] for i in rng.integers(0, 20, size=n))


def random_dihedrals(rng, n, extra_chi_sd=0.0):
    helix = rng.random(n) < 0.6
    phi = numpy.where(helix, rng.normal(-63.0, 10.0, n), rng.normal(-120.0, 15.0, n))
    psi = numpy.where(helix, rng.normal(-41.0, 10.0, n), rng.normal(130.0, 15.0, n))
    omega = numpy.full(n, 180.0)
    chis = rng.choice([-60.0, 60.0, 180.0], size=(n, 4)) + rng.normal(0.0, 10.0, (n, 4))
    if extra_chi_sd > 0:
        chis = chis + rng.normal(0.0, extra_chi_sd, (n, 4))
    return phi, psi, omega, chis


def synthetic_topologies_and_coords(n_res_per_pose, seeds, extra_chi_sd=0.0, spacing=1000.0, pbt=None,
                                    with_coords=True):
    """The host half of ``synthetic_pose_stack``: per-pose topologies and
    ``[n_pose_atoms, 3]`` coordinates (numpy), already placed on the grid
    (None without ``with_coords``: the sequences only)."""
    rts = ResidueTypeSet.get_default()
    pbt = pbt or default_packed_block_types(torch.device("cpu"))
    topos, phis, psis, omegas, chis = [], [], [], [], []
    for n, seed in zip(n_res_per_pose, seeds):
        rng = numpy.random.default_rng(seed)
        seq = random_sequence(rng, n)
        topos.append(topology_from_sequence(seq, rts))
        ph, ps, om, ch = random_dihedrals(rng, n, extra_chi_sd)
        phis.append(ph)
        psis.append(ps)
        omegas.append(om)
        chis.append(ch)
    if not with_coords:
        return topos, None
    coords = build_chain_coords(pbt, topos, phis, psis, omegas, chis)
    P = len(topos)
    side = max(1, int(numpy.ceil(P ** (1.0 / 3.0))))
    for k in range(P):
        cell = numpy.array([k % side, (k // side) % side, k // (side * side)], dtype=numpy.float64)
        c = coords[k]
        coords[k] = c - c.mean(axis=0) + spacing * cell
    return topos, coords


def synthetic_pose_stack(
    n_res_per_pose,
    seeds,
    device=torch.device("cpu"),
    extra_chi_sd=0.0,
    spacing=1000.0,
    pbt=None,
):
    """One pose per entry of ``n_res_per_pose``; pose k uses
    ``numpy.random.default_rng(seeds[k])``.  Poses are translated onto a cubic
    grid with ``spacing`` angstroms between neighbours so that no two overlap
    (the scoring itself never couples poses)."""
    topos, coords = synthetic_topologies_and_coords(n_res_per_pose, seeds, extra_chi_sd, spacing, pbt)
    # the dense bond-separation tensors are built directly on `device`
    return build_pose_stack(topos, coords, pbt=pbt, device=torch.device(device))


def log_uniform_sizes(rng, n, lo, hi):
    return [int(round(numpy.exp(rng.uniform(numpy.log(lo), numpy.log(hi))))) for _ in range(n)]
