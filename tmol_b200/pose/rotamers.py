"""Rotamer sets: alternative placements (and identities) of a PoseStack's
blocks, laid out as tmol's ``RotamerSet`` (tmol/pack/rotamer/rotamer_set.py:
9-50), the input of the rotamer-scoring op.

Rotamers are numbered globally, pose by pose and block by block; block b of
pose p owns rotamers ``rot_offset_for_block[p, b] ..
rot_offset_for_block[p, b] + n_rots_for_block[p, b] - 1``, each with its own
block type and coordinates (``coords[coord_offset_for_rot[r] + i]`` is atom
i of rotamer r).

``synthetic_rotamer_set`` builds a seeded set for tests and benchmarks: the
native placement of every block first, then side-chain rebuilds with other
chi angles (rotameric {-60, 60, 180} + N(0, chi_sd)) and, for a fraction of
them, another canonical amino acid with the same termini variant, all on the
native backbone.
"""

from dataclasses import dataclass

import numpy
import torch

from .builder import build_residue_coords
from .synthetic import CANONICAL_1LC


@dataclass
class RotamerSet:
    n_rots_for_pose: torch.Tensor  # [P]
    rot_offset_for_pose: torch.Tensor  # [P]
    n_rots_for_block: torch.Tensor  # [P, B]
    rot_offset_for_block: torch.Tensor  # [P, B] (global rotamer index)
    pose_for_rot: torch.Tensor  # [R]
    block_type_ind_for_rot: torch.Tensor  # [R]
    block_ind_for_rot: torch.Tensor  # [R]
    coord_offset_for_rot: torch.Tensor  # [R]
    coords: torch.Tensor  # [n_rot_atoms, 3]
    first_rot_block_type: torch.Tensor  # [P, B], -1 where a block has no rotamer
    max_n_rots_per_pose: int
    pose_ind_for_atom: torch.Tensor  # [n_rot_atoms]

    @property
    def n_rotamers_total(self):
        return self.block_ind_for_rot.shape[0]

    def to(self, device):
        kw = {k: (v.to(device) if isinstance(v, torch.Tensor) else v) for k, v in self.__dict__.items()}
        return RotamerSet(**kw)


def _variant_suffix(name):
    i = name.find(":")
    return name[i:] if i >= 0 else ""


def rotamer_set_from_arrays(block_ind_for_rot, pose_for_rot, bt_for_rot, rot_coords, P, B, device):
    """A RotamerSet from per-rotamer arrays sorted by (pose, block)."""
    R = len(block_ind_for_rot)
    n_atoms = numpy.array([len(c) for c in rot_coords], dtype=numpy.int64)
    coord_offset = numpy.concatenate([[0], numpy.cumsum(n_atoms)[:-1]]).astype(numpy.int32)
    n_rots_for_block = numpy.zeros((P, B), dtype=numpy.int64)
    rot_offset_for_block = numpy.zeros((P, B), dtype=numpy.int64)
    first_bt = numpy.full((P, B), -1, dtype=numpy.int64)
    for r in range(R - 1, -1, -1):
        p, b = pose_for_rot[r], block_ind_for_rot[r]
        n_rots_for_block[p, b] += 1
        rot_offset_for_block[p, b] = r
        first_bt[p, b] = bt_for_rot[r]
    n_rots_for_pose = n_rots_for_block.sum(1)
    rot_offset_for_pose = numpy.concatenate([[0], numpy.cumsum(n_rots_for_pose)[:-1]])
    coords = numpy.concatenate(rot_coords).astype(numpy.float32)
    pose_ind_for_atom = numpy.repeat(numpy.asarray(pose_for_rot, dtype=numpy.int64), n_atoms)
    t = lambda a, dt: torch.tensor(numpy.asarray(a), dtype=dt, device=device)  # noqa: E731
    return RotamerSet(
        n_rots_for_pose=t(n_rots_for_pose, torch.int64),
        rot_offset_for_pose=t(rot_offset_for_pose, torch.int64),
        n_rots_for_block=t(n_rots_for_block, torch.int64),
        rot_offset_for_block=t(rot_offset_for_block, torch.int64),
        pose_for_rot=t(pose_for_rot, torch.int64),
        block_type_ind_for_rot=t(bt_for_rot, torch.int64),
        block_ind_for_rot=t(block_ind_for_rot, torch.int32),
        coord_offset_for_rot=t(coord_offset, torch.int32),
        coords=t(coords, torch.float32),
        first_rot_block_type=t(first_bt, torch.int64),
        max_n_rots_per_pose=int(n_rots_for_pose.max()) if P else 0,
        pose_ind_for_atom=t(pose_ind_for_atom, torch.int64),
    )


def synthetic_rotamer_set(pose_stack, max_rots=4, mutate_fraction=0.25, seed=0, chi_sd=10.0,
                          skip_fraction=0.0, pose_seeds=None):
    """Seeded rotamers for every block of ``pose_stack`` (a single-chain
    PoseStack from ``tmol_b200.pose``): 1..max_rots per block, the native
    placement first.  With ``skip_fraction``, that fraction of blocks gets
    no rotamers at all (a block absent from the packing problem).  One
    random stream serves the whole stack, or, with ``pose_seeds``, pose p
    has its own (seeded by ``(seed, pose_seeds[p])``), so that any subset of
    poses gets the same rotamers as the whole batch."""
    rng = numpy.random.default_rng(seed)
    pbt = pose_stack.packed_block_types
    bts = pbt.active_block_types
    X = pose_stack.coords.detach().cpu().numpy().astype(numpy.float64)
    bti = pose_stack.block_type_ind.detach().cpu().numpy()
    offs = pose_stack.block_coord_offset.detach().cpu().numpy()
    P, B = bti.shape
    block_ind, pose_for, bt_for, rot_xyz = [], [], [], []
    builds = {}  # block-type name -> [(rotamer index, frame, chis)]; built per type at once
    for p in range(P):
        if pose_seeds is not None:
            rng = numpy.random.default_rng([seed, int(pose_seeds[p])])
        for b in range(B):
            if bti[p, b] < 0 or rng.random() < skip_fraction:
                continue
            bt = bts[bti[p, b]]
            native = X[p, offs[p, b]:offs[p, b] + bt.n_atoms]
            n = int(rng.integers(1, max_rots + 1))
            block_ind.append(b)
            pose_for.append(p)
            bt_for.append(int(bti[p, b]))
            rot_xyz.append(native)
            ia = bt.atom_index
            n_pos, ca_pos, c_pos = (native[ia[a]] for a in ("N", "CA", "C"))
            down, up = n_pos, c_pos
            if b > 0 and bti[p, b - 1] >= 0:
                prev = bts[bti[p, b - 1]]
                down = X[p, offs[p, b - 1] + prev.atom_index["C"]]
            if b + 1 < B and bti[p, b + 1] >= 0:
                nxt = bts[bti[p, b + 1]]
                up = X[p, offs[p, b + 1] + nxt.atom_index["N"]]
            for _ in range(n - 1):
                rbt = bt
                if rng.random() < mutate_fraction:
                    name = CANONICAL_1LC[int(rng.integers(0, 20))]
                    base = [t for t in bts if t.one_letter_code == name and not t.is_ligand_fragment]
                    cand = [t for t in base if _variant_suffix(t.name) == _variant_suffix(bt.name)]
                    if cand:
                        rbt = cand[0]
                chis = rng.choice([-60.0, 60.0, 180.0], size=4) + rng.normal(0.0, chi_sd, 4)
                builds.setdefault(rbt.name, []).append((len(rot_xyz), (n_pos, ca_pos, c_pos, down, up), chis))
                block_ind.append(b)
                pose_for.append(p)
                bt_for.append(pbt.bt_index[rbt.name])
                rot_xyz.append(None)
    for name, specs in builds.items():
        frames = [numpy.stack([f[k] for _, f, _ in specs]) for k in range(5)]
        chis = numpy.stack([c for _, _, c in specs])
        xyz = build_residue_coords(bts[pbt.bt_index[name]], *frames, chis)
        for (r, _, _), x in zip(specs, xyz):
            rot_xyz[r] = x
    return rotamer_set_from_arrays(block_ind, pose_for, bt_for, rot_xyz, P, B, pose_stack.device)
