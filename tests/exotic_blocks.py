"""Synthetic block types that exercise the general code paths: blocks with
more than 32 atoms (several tiles), three inter-block connections, and
ligand fragments (the inter-block 3/4 -> 5 count-pair rule).  Chemistry is
arbitrary: the oracle and the kernels must agree on it, nothing more."""

import numpy
import torch

from tmol_b200.chem.restypes import (
    ChemicalDatabase,
    PackedBlockTypes,
    ResidueTypeSet,
)
from tmol_b200.pose.builder import PoseTopology, build_pose_stack

_TYPES = ["CH2", "CH3", "Nbb", "OCbb", "Hapo", "Hpol", "OH", "Caro", "Haro", "NH2O"]


def big_block_type(name, n_atoms, ligand, seed):
    """A branched chain of `n_atoms` atoms with connections down / up / side."""
    from tmol_b200.chem.restypes import ResidueType

    rng = numpy.random.default_rng(seed)
    atoms = [[f"A{k}", _TYPES[rng.integers(len(_TYPES))]] for k in range(n_atoms)]
    bonds = []
    for k in range(1, n_atoms):
        parent = k - 1 if rng.random() < 0.7 else int(rng.integers(0, k))
        bonds.append([f"A{parent}", f"A{k}"])
    conns = [["down", "A0"], ["up", f"A{n_atoms - 1}"], ["side", f"A{n_atoms // 2}"]]
    return ResidueType(
        name=name,
        base_name=name,
        atoms=atoms,
        bonds=bonds,
        connections=conns,
        icoors=[],
        chis=[],
        aliases=[],
        is_polymer=not ligand,
        is_ligand_fragment=ligand,
    )


def exotic_pose_stack(seed=0):
    rts = ResidueTypeSet.get_default()
    db = ChemicalDatabase.get_default()
    bts = list(rts.types.values()) + [
        big_block_type("BIG40", 40, False, 1),
        big_block_type("LIG45", 45, True, 2),
        big_block_type("LIG12", 12, True, 3),
    ]
    pbt = PackedBlockTypes(db, bts)
    rng = numpy.random.default_rng(seed)
    topos, coords = [], []
    for p, names in enumerate(
        [
            ["ALA:nterm", "BIG40", "GLY", "LIG45", "LIG12", "SER:cterm"],
            ["LIG12", "LIG45", "BIG40"],
            ["BIG40"],
        ]
    ):
        bonds = []
        for i in range(len(names) - 1):
            bonds.append((i, "up", i + 1, "down"))
        big = [i for i, n in enumerate(names) if n in ("BIG40", "LIG45", "LIG12")]
        if len(big) >= 2:
            bonds.append((big[0], "side", big[-1], "side"))
        topos.append(PoseTopology(names, bonds))
        n = sum(pbt.active_block_types[pbt.bt_index[x]].n_atoms for x in names)
        # a compact random walk so that many pairs fall inside the cutoff
        steps = rng.normal(size=(n, 3))
        steps = 1.5 * steps / numpy.linalg.norm(steps, axis=1, keepdims=True)
        xyz = numpy.cumsum(steps, axis=0)
        xyz = 0.6 * xyz + rng.normal(scale=0.3, size=xyz.shape)
        coords.append(xyz)
    return build_pose_stack(topos, coords, pbt=pbt)


def degenerate_pose_stack(seed=3):
    """Three poses with the degenerate cases the scoring path must define:
    a block type with no atoms (its sphere's centroid is 0/0 = NaN, so it
    is nobody's neighbour, not even its own) inside pose 0, a pose of a
    single block (pose 1), and an ordinary pose (pose 2)."""
    from tmol_b200.chem.restypes import ResidueType
    from tmol_b200.pose.synthetic import synthetic_topologies_and_coords

    rts = ResidueTypeSet.get_default()
    db = ChemicalDatabase.get_default()
    empty = ResidueType(
        name="EMPTY", base_name="EMPTY", atoms=[], bonds=[], connections=[], icoors=[], chis=[], aliases=[],
        is_polymer=False, is_ligand_fragment=True,
    )
    pbt = PackedBlockTypes(db, list(rts.types.values()) + [empty])
    topos, coords = synthetic_topologies_and_coords([20, 1, 8], [seed, seed + 1, seed + 2], pbt=pbt)
    names = list(topos[0].block_type_names)
    shift = lambda b: b if b < 6 else b + 1  # noqa: E731
    topos[0] = PoseTopology(
        names[:6] + ["EMPTY"] + names[6:], [(shift(a), ca, shift(b), cb) for a, ca, b, cb in topos[0].bonds]
    )
    return build_pose_stack(topos, coords, pbt=pbt)


def with_nan_atom(ps, pose=2, block=3, atom=1, dim=1):
    """The stack's coordinates with one atom coordinate set to NaN: its
    block's sphere is NaN, so the block drops out of neighbour detection and
    scores nothing, while the rest of the pose scores as before."""
    c = ps.coords.clone()
    c[pose, int(ps.block_coord_offset[pose, block]) + atom, dim] = float("nan")
    return c
