"""Minimal PDB reading for single-chain, fully-protonated proteins.

Each residue maps to a canonical block type; the first residue takes the
N-terminus variant and the last the C-terminus variant; a HIS with HD1 and no
HE2 maps to HIS_D.  PDB atom names are resolved through the residue types'
aliases (e.g. ``1HB`` -> ``HB2``, ``1H`` -> ``H1``).  Every block-type atom
must be present; this reader builds no missing atoms.
"""

import numpy

from ..chem.restypes import ResidueTypeSet
from .builder import PoseTopology


def parse_atom_records(text):
    res = []
    key_to_idx = {}
    for line in text.splitlines():
        if not (line.startswith("ATOM") or line.startswith("HETATM")):
            continue
        name = line[12:16].strip()
        resn = line[17:20].strip()
        chain = line[21]
        resi = int(line[22:26])
        icode = line[26]
        xyz = (float(line[30:38]), float(line[38:46]), float(line[46:54]))
        key = (chain, resi, icode)
        if key not in key_to_idx:
            key_to_idx[key] = len(res)
            res.append((resn, {}))
        res[key_to_idx[key]][1][name] = xyz
    return res


def pose_from_pdb_text(text, rts=None):
    """Returns (PoseTopology, coords[n_atoms, 3] float64) for the first chain."""
    rts = rts or ResidueTypeSet.get_default()
    residues = parse_atom_records(text)
    n = len(residues)
    names = []
    coords = []
    for i, (resn, atoms) in enumerate(residues):
        base = resn
        if resn == "HIS":
            base = "HIS_D" if ("HD1" in atoms and "HE2" not in atoms) else "HIS"
        bt_name = rts.variant_name(base, i == 0, i == n - 1)
        bt = rts.types[bt_name]
        lookup = {}
        for pdb_name, xyz in atoms.items():
            lookup[bt.aliases.get(pdb_name, pdb_name)] = xyz
        missing = [a for a in bt.atom_names if a not in lookup]
        if missing:
            raise ValueError(f"residue {i} {bt_name}: missing atoms {missing}")
        coords.extend(lookup[a] for a in bt.atom_names)
        names.append(bt_name)
    bonds = [(i, "up", i + 1, "down") for i in range(n - 1)]
    return PoseTopology(names, bonds), numpy.array(coords, dtype=numpy.float64)
