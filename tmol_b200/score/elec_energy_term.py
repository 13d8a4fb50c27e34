"""The elec term: tmol's ``ElecEnergyTerm`` (tmol/score/elec/elec_energy_term.py:
13-186) and its parameter resolver (tmol/score/elec/params.py:27-175), over
this package's chemistry tables.

Per block type it provides the partial charge of every atom (looked up by
residue name, the block's variants in order, then the unpatched entry) and
the count-pair *representative* path distances: ``inter[a, b]`` is the number
of bonds between atom a and the representative of atom b, and ``intra[a, b]``
the number between the representatives of a and b, with 3 and 4 read as 5
in non-polymer blocks (full weight for 1-4 pairs in ligands).  Its ops,
``elec_pose_scores`` and ``elec_rotamer_scores`` (``tmol_b200.score.elec_op``),
take the same leading PoseStack (or rotamer-set) arguments as the LJ/LK ops
and return one energy per pose, block pair or rotamer pair.
"""

import json
import os

import numpy
import torch

from .score_types import ScoreType

DATA = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "chem", "data",
                    "elec_chemistry.json")


class ElecParams:
    """Partial charges and count-pair representatives, keyed as tmol keys
    them: ``[res][atom][variant]`` (variant "" = unpatched)."""

    def __init__(self, path=DATA):
        with open(path) as f:
            d = json.load(f)
        g = d["global_params"]
        self.D = g["elec_sigmoidal_die_D"]
        self.D0 = g["elec_sigmoidal_die_D0"]
        self.S = g["elec_sigmoidal_die_S"]
        self.min_dis = g["elec_min_dis"]
        self.max_dis = g["elec_max_dis"]
        self.partial_charges = {}
        for res, var, atom, q in d["partial_charges"]:
            self.partial_charges.setdefault(res, {}).setdefault(atom, {})[var] = q
        # later lines override earlier ones (params.py:149-163)
        self.cp_reps = {}
        for res, var, outer, inner in d["cp_reps"]:
            self.cp_reps.setdefault(res, {}).setdefault(outer, {})[var] = inner

    @staticmethod
    def _res_vars(block_type):
        res, *variants = block_type.name.split(":")
        return res, variants + [""]

    def partial_charges_for_block(self, block_type):
        res, variants = self._res_vars(block_type)
        table = self.partial_charges.get(res)
        out = numpy.zeros(block_type.n_atoms, dtype=numpy.float32)
        if table is None:
            return out
        for i, atom in enumerate(block_type.atom_names):
            if atom not in table:
                raise KeyError(f"elec charge for atom {block_type.name},{atom} not found")
            for v in variants:
                if v in table[atom]:
                    out[i] = table[atom][v]
                    break
        return out

    def representative_mapping(self, block_type):
        mapping = numpy.arange(block_type.n_atoms, dtype=numpy.int32)
        res, variants = self._res_vars(block_type)
        reps = self.cp_reps.get(res)
        if reps is None:
            return mapping
        for outer in block_type.atom_names:
            if outer not in reps:
                continue
            inner = next((reps[outer][v] for v in variants if v in reps[outer]), None)
            if inner is None:
                continue
            if inner not in block_type.atom_index:
                raise KeyError(f"invalid elec count-pair mapping: {res} {outer} -> {inner}")
            mapping[block_type.atom_index[inner]] = block_type.atom_index[outer]
        return mapping


class ElecEnergyTerm:
    def __init__(self, device=torch.device("cpu"), params=None):
        self.device = torch.device(device)
        self.params = params or ElecParams()
        self._bt_cache = {}

    @classmethod
    def class_name(cls):
        return "Elec"

    @classmethod
    def score_types(cls):
        return [ScoreType.fa_elec]

    def n_bodies(self):
        return 2

    def block_type_tables(self, block_type):
        hit = self._bt_cache.get(block_type.name)
        if hit is not None:
            return hit
        charge = self.params.partial_charges_for_block(block_type)
        rep = self.params.representative_mapping(block_type)
        pd = numpy.asarray(block_type.path_distance, dtype=numpy.int32)
        inter = pd[:, rep]
        intra = inter[rep, :].copy()
        if not block_type.is_polymer:
            intra[(intra == 3) | (intra == 4)] = 5
        hit = (charge, inter, intra)
        self._bt_cache[block_type.name] = hit
        return hit

    def setup_packed_block_types(self, pbt):
        if getattr(pbt, "_elec_tables", None) is not None:
            return pbt._elec_tables
        nbt, A = pbt.n_types, pbt.max_n_atoms
        q = numpy.zeros((nbt, A), dtype=numpy.float32)
        inter = numpy.zeros((nbt, A, A), dtype=numpy.int32)
        intra = numpy.zeros((nbt, A, A), dtype=numpy.int32)
        lig = numpy.zeros(nbt, dtype=numpy.int32)
        for i, bt in enumerate(pbt.active_block_types):
            c, e, a = self.block_type_tables(bt)
            n = bt.n_atoms
            q[i, :n] = c
            inter[i, :n, :n] = e
            intra[i, :n, :n] = a
            lig[i] = int(bt.is_ligand_fragment)
        dev = pbt.device
        pbt._elec_tables = dict(
            elec_partial_charge=torch.tensor(q, device=dev),
            elec_inter_repr_path_distance=torch.tensor(inter, device=dev),
            elec_intra_repr_path_distance=torch.tensor(intra, device=dev),
            elec_is_ligand_fragment=torch.tensor(lig, device=dev),
        )
        return pbt._elec_tables

    def setup_poses(self, pose_stack):
        if not hasattr(pose_stack, "min_block_bondsep"):
            mbs, _ = torch.min(pose_stack.inter_block_bondsep, dim=4)
            mbs, _ = torch.min(mbs, dim=3)
            pose_stack.min_block_bondsep = mbs.contiguous()

    def global_params_tensor(self, device):
        p = self.params
        return torch.tensor([[p.D, p.D0, p.S, p.min_dis, p.max_dis]], dtype=torch.float32, device=device)

    def get_score_term_attributes(self, pose_stack):
        """The 11 term arguments of the elec op, in tmol's order
        (elec_energy_term.py:153-186)."""
        self.setup_poses(pose_stack)
        pbt = pose_stack.packed_block_types
        t = self.setup_packed_block_types(pbt)
        return [
            pose_stack.min_block_bondsep,
            pose_stack.inter_block_bondsep,
            pbt.n_atoms,
            t["elec_partial_charge"],
            pbt.n_conn,
            pbt.conn_atom,
            t["elec_inter_repr_path_distance"],
            t["elec_intra_repr_path_distance"],
            t["elec_is_ligand_fragment"],
            self.global_params_tensor(pose_stack.device),
            float(self.params.max_dis),
        ]

    def get_pose_score_term_function(self):
        from .elec_op import elec_pose_scores

        return elec_pose_scores

    def render_whole_pose_scoring_module(self, pose_stack):
        from .scoring_module import TermWholePoseScoringModule

        return TermWholePoseScoringModule(
            self.class_name(), pose_stack, self.get_score_term_attributes(pose_stack),
            self.get_pose_score_term_function(),
        )

    def render_block_pair_scoring_module(self, pose_stack):
        from .scoring_module import TermBlockPairScoringModule

        return TermBlockPairScoringModule(
            self.class_name(), pose_stack, self.get_score_term_attributes(pose_stack),
            self.get_pose_score_term_function(),
        )

    def get_rotamer_score_term_function(self):
        from .elec_op import elec_rotamer_scores

        return elec_rotamer_scores

    def render_rotamer_scoring_module(self, pose_stack, rotamer_set):
        """tmol ``energy_term.py:132-147``: the rotamer-pair scoring module
        over ``rotamer_set``."""
        from .scoring_module import TermRotamerScoringModule

        return TermRotamerScoringModule(
            self.class_name(), rotamer_set, self.get_score_term_attributes(pose_stack),
            self.get_rotamer_score_term_function(),
        )


def elec_pose_score_args(pose_stack, term, block_pair=False):
    """The elec op's argument list minus the coordinates (tmol
    ``elec/potentials/compiled.ops.cpp:28-59`` order)."""
    common = [
        pose_stack.rot_coord_offset,
        pose_stack.pose_ind_for_atom,
        pose_stack.first_rot_for_block,
        pose_stack.block_type_ind,
        pose_stack.block_ind_for_rot,
        pose_stack.pose_ind_for_rot,
        pose_stack.block_type_ind_for_rot,
        pose_stack.n_rots_for_pose,
        pose_stack.rot_offset_for_pose,
        pose_stack.n_rots_for_block,
        pose_stack.rot_offset_for_block,
        pose_stack.max_n_rots_per_pose,
    ]
    return common + term.get_score_term_attributes(pose_stack) + [block_pair]


def elec_rotamer_score_args(pose_stack, rotamer_set, term):
    """The elec rotamer op's argument list minus the coordinates: the rotamer
    set's indexing (as ``TermRotamerScoringModule`` passes it,
    tmol/score/common/scoring_module.py:133-170), the pose's term
    attributes and ``output_block_pair_energies=True``."""
    from .ljlk_energy_term import rotamer_score_args

    return rotamer_score_args(pose_stack, rotamer_set, term)
