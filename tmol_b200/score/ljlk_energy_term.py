"""LJLKEnergyTerm: the Lennard-Jones + Lazaridis-Karplus term, with tmol's
``EnergyTerm`` plugin surface (``tmol/score/energy_term.py:35-123``,
``tmol/score/ljlk/ljlk_energy_term.py:16-178``).

The setup hooks annotate block types, packed block types and pose stacks
with the tables the op reads; ``get_score_term_attributes`` returns the
13-item static argument tail in tmol's order; the rendered modules call the
B200 op ``tmol_b200.score.ljlk_op.ljlk_pose_scores`` in place of
``torch.ops.tmol_ljlk.ljlk_pose_scores``.
"""

import torch

from ..chem.restypes import ChemicalDatabase
from .ljlk_params import global_params_tensor, type_params_tensor
from .score_types import ScoreType
from .scoring_module import TermBlockPairScoringModule, TermRotamerScoringModule, TermWholePoseScoringModule


class LJLKEnergyTerm:
    tile_size = 32

    def __init__(self, param_db=None, device=torch.device("cpu")):
        self.param_db = param_db or ChemicalDatabase.get_default()
        self.device = torch.device(device)
        self.type_params = type_params_tensor(self.param_db, self.device)
        self.soft_repulsive = False

    @classmethod
    def class_name(cls):
        return "LJLK"

    @classmethod
    def score_types(cls):
        return [ScoreType.fa_ljatr, ScoreType.fa_ljrep, ScoreType.fa_lk]

    def n_bodies(self):
        return 2

    def set_options(self, options):
        if "soft_rep" in options:
            self.soft_repulsive = bool(options["soft_rep"])

    @property
    def global_params(self):
        return global_params_tensor(self.param_db, self.soft_repulsive, self.device)

    # The packed tables are built eagerly by PackedBlockTypes, so the setup
    # hooks only check that they are present.
    def setup_block_type(self, block_type):
        assert hasattr(block_type, "path_distance")

    def setup_packed_block_types(self, packed_block_types):
        for attr in (
            "ljlk_heavy_atoms_in_tile",
            "ljlk_n_heavy_atoms_in_tile",
            "ljlk_bond_separation",
            "ljlk_is_ligand_fragment",
            "atom_types",
        ):
            assert hasattr(packed_block_types, attr)

    def setup_poses(self, pose_stack):
        if not hasattr(pose_stack, "min_block_bondsep"):
            mbs, _ = torch.min(pose_stack.inter_block_bondsep, dim=4)
            mbs, _ = torch.min(mbs, dim=3)
            pose_stack.min_block_bondsep = mbs.contiguous()

    def get_pose_score_term_function(self):
        from .ljlk_op import ljlk_pose_scores

        return ljlk_pose_scores

    def get_rotamer_score_term_function(self):
        from .ljlk_op import ljlk_rotamer_scores

        return ljlk_rotamer_scores

    def render_rotamer_scoring_module(self, pose_stack, rotamer_set):
        """tmol ``energy_term.py:132-147``: the rotamer-pair scoring module
        over ``rotamer_set`` (see ``tmol_b200.pose.rotamers``)."""
        return TermRotamerScoringModule(
            self.class_name(),
            rotamer_set,
            self.get_score_term_attributes(pose_stack),
            self.get_rotamer_score_term_function(),
        )

    def get_score_term_attributes(self, pose_stack):
        self.setup_poses(pose_stack)
        pbt = pose_stack.packed_block_types
        return [
            pose_stack.min_block_bondsep,
            pose_stack.inter_block_bondsep,
            pbt.n_atoms,
            pbt.ljlk_n_heavy_atoms_in_tile,
            pbt.ljlk_heavy_atoms_in_tile,
            pbt.atom_types,
            pbt.n_conn,
            pbt.conn_atom,
            pbt.ljlk_bond_separation,
            pbt.ljlk_is_ligand_fragment,
            self.type_params,
            self.global_params,
            float(self.param_db.ljlk_global_params["max_dis"]),
        ]

    def render_whole_pose_scoring_module(self, pose_stack):
        return TermWholePoseScoringModule(
            self.class_name(),
            pose_stack,
            self.get_score_term_attributes(pose_stack),
            self.get_pose_score_term_function(),
        )

    def render_block_pair_scoring_module(self, pose_stack):
        return TermBlockPairScoringModule(
            self.class_name(),
            pose_stack,
            self.get_score_term_attributes(pose_stack),
            self.get_pose_score_term_function(),
        )


def pose_score_args(pose_stack, term, block_pair=False):
    """The op's full 27-argument list for ``pose_stack`` minus the coordinates
    (tmol ``compiled.ops.cpp:533-597`` order)."""
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


def rotamer_score_args(pose_stack, rotamer_set, term):
    """The rotamer-score op's argument list minus the coordinates, in the
    order tmol's ``TermRotamerScoringModule`` passes it
    (tmol/score/common/scoring_module.py:133-170; op at
    ``compiled.ops.cpp:599-662``): the rotamer set's indexing, the pose's
    term attributes, and ``output_block_pair_energies=True``."""

    def i32(t):
        return t if isinstance(t, int) else t.to(torch.int32)

    rs = rotamer_set
    common = [
        i32(rs.coord_offset_for_rot),
        i32(rs.pose_ind_for_atom),
        i32(rs.rot_offset_for_block),
        i32(rs.first_rot_block_type),
        i32(rs.block_ind_for_rot),
        i32(rs.pose_for_rot),
        i32(rs.block_type_ind_for_rot),
        i32(rs.n_rots_for_pose),
        i32(rs.rot_offset_for_pose),
        i32(rs.n_rots_for_block),
        i32(rs.rot_offset_for_block),
        int(rs.max_n_rots_per_pose),
    ]
    return common + term.get_score_term_attributes(pose_stack) + [True]
