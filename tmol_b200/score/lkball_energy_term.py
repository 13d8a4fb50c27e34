"""LKBallEnergyTerm: the LK-ball solvation term (lk_ball_iso, lk_ball,
lk_bridge, lk_bridge_uncpl), with tmol's argument lists
(``tmol/score/lk_ball/lk_ball_energy_term.py:17-369``).

Scoring is two ops: water generation (``gen_pose_waters``: up to four
waters per polar atom, built from the polar atom and its bonded
neighbours) and the pose score over polar-atom / heavy-atom pairs of
neighbouring blocks, reading the waters (``lk_ball_pose_score``).  This
module assembles their arguments from a PoseStack; the block-type tables
come from ``tmol_b200.chem.lkball_tables``, the global parameters from the
LJ/LK ones (``max_dis``, the hbond distances) and the LK-ball water
geometry in tmol's ``ljlk.yaml``.
"""

import torch

from ..chem.lkball_tables import packed_lkball_tables
from .score_types import ScoreType


class LKBallEnergyTerm:
    def __init__(self, device=torch.device("cpu")):
        self.device = torch.device(device)

    @classmethod
    def class_name(cls):
        return "LKBall"

    @classmethod
    def score_types(cls):
        return [ScoreType.lk_ball_iso, ScoreType.lk_ball, ScoreType.lk_bridge, ScoreType.lk_bridge_uncpl]

    def n_bodies(self):
        return 2

    def setup_poses(self, pose_stack):
        if not hasattr(pose_stack, "min_block_bondsep"):
            mbs, _ = torch.min(pose_stack.inter_block_bondsep, dim=4)
            mbs, _ = torch.min(mbs, dim=3)
            pose_stack.min_block_bondsep = mbs.contiguous()

    @staticmethod
    def _gp(pbt):
        return pbt.db.ljlk_global_params, pbt.db.lkball_global_params

    # -- the scoring-module surface (tmol energy_term.py:35-147) -----------

    N_WATER_TABLES = 20  # gen_pose_waters' arguments after the 12 indexing ones
    N_SCORE_TABLES = 13  # lk_ball_pose_score's, before the waters and the output flag

    def get_score_term_attributes(self, pose_stack):
        """The pose's LK-ball arguments of both ops, built once: the 20
        water-generation tables, then the 13 scoring ones (tmol passes the
        PoseStack itself and rebuilds these lists per call,
        lk_ball_energy_term.py:236-369)."""
        return water_gen_args(pose_stack, self)[12:] + score_args(pose_stack, self, None)[12:-2]

    @classmethod
    def _split(cls, args):
        common = args[:12]
        wt = args[12 : 12 + cls.N_WATER_TABLES]
        st = args[12 + cls.N_WATER_TABLES : 12 + cls.N_WATER_TABLES + cls.N_SCORE_TABLES]
        return common, wt, st, args[12 + cls.N_WATER_TABLES + cls.N_SCORE_TABLES]

    @classmethod
    def pose_score_lk_ball(cls, coords, *args):
        """tmol ``LKBallEnergyTerm.pose_score_lk_ball``: the waters, then the
        pose scores on them; ``(scores, block_neighbors)``."""
        from .lkball_op import gen_pose_waters, lk_ball_pose_score

        common, wt, st, block_pair = cls._split(args)
        W = gen_pose_waters(coords, *common, *wt)
        return lk_ball_pose_score(coords, *common, *st, W, block_pair)

    @classmethod
    def rotamer_score_lk_ball(cls, coords, *args):
        """tmol ``LKBallEnergyTerm.rotamer_score_lk_ball``: the waters of every
        rotamer, then the rotamer-pair scores; ``(scores, indices)``."""
        from .lkball_op import gen_pose_waters, lk_ball_rotamer_score

        common, wt, st, block_pair = cls._split(args)
        W = gen_pose_waters(coords, *common, *wt)
        return lk_ball_rotamer_score(coords, *common, *st, W, block_pair)

    def get_pose_score_term_function(self):
        return self.pose_score_lk_ball

    def get_rotamer_score_term_function(self):
        return self.rotamer_score_lk_ball

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

    def render_rotamer_scoring_module(self, pose_stack, rotamer_set):
        """tmol ``energy_term.py:132-147``: the rotamer-pair scoring module
        over ``rotamer_set``."""
        from .scoring_module import TermRotamerScoringModule

        return TermRotamerScoringModule(
            self.class_name(), rotamer_set, self.get_score_term_attributes(pose_stack),
            self.get_rotamer_score_term_function(),
        )

    def water_gen_global_params(self, pbt, device):
        """[1, 4] (water distance, sp2 / sp3 / ring angles) and the three
        torsion lists, float32 as tmol's resolver holds them."""
        _, lkb = self._gp(pbt)
        gp = torch.tensor(
            [[lkb["lkb_water_dist"], lkb["lkb_water_angle_sp2"], lkb["lkb_water_angle_sp3"],
              lkb["lkb_water_angle_ring"]]],
            dtype=torch.float32,
            device=device,
        )
        tors = [
            torch.tensor(lkb[k], dtype=torch.float32, device=device)
            for k in ("lkb_water_tors_sp2", "lkb_water_tors_sp3", "lkb_water_tors_ring")
        ]
        return gp, tors

    def score_global_params(self, pbt, device):
        """[1, 5]: hbond distance, OH-donor distance, H distance, water
        distance, max_dis (tmol lk_ball_energy_term.py:32-47)."""
        lj, lkb = self._gp(pbt)
        return torch.tensor(
            [[lj["lj_hbond_dis"], lj["lj_hbond_OH_donor_dis"], lj["lj_hbond_hdis"], lkb["lkb_water_dist"],
              lj["max_dis"]]],
            dtype=torch.float32,
            device=device,
        )


def _common(pose_stack):
    return [
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


def _rotamer_common(rotamer_set):
    """A rotamer set's indexing, as tmol's TermRotamerScoringModule passes
    it (tmol/score/common/scoring_module.py:133-170)."""

    def i32(t):
        return t if isinstance(t, int) else t.to(torch.int32)

    rs = rotamer_set
    return [
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


def water_gen_args(pose_stack, term, rotamer_set=None):
    """gen_pose_waters' argument list minus the coordinates
    (tmol lk_ball_energy_term.py:245-270, compiled.ops.cpp:28-64); with a
    rotamer set, its indexing in front, as tmol's rotamer scoring calls the
    op on the rotamers' coordinates (lk_ball_energy_term.py:300-336)."""
    pbt = pose_stack.packed_block_types
    t = packed_lkball_tables(pbt)
    gp, tors = term.water_gen_global_params(pbt, pose_stack.device)
    common = _common(pose_stack) if rotamer_set is None else _rotamer_common(rotamer_set)
    return common + [
        pose_stack.inter_residue_connections,
        pbt.n_atoms,
        pbt.n_conn,
        pbt.conn_atom,
        t["n_all_bonds"],
        t["all_bonds"],
        t["atom_all_bond_ranges"],
        t["tile_n_donH"],
        t["tile_n_acc"],
        t["tile_donH_inds"],
        t["tile_donH_hvy_inds"],
        t["tile_which_donH_of_donH_hvy"],
        t["tile_acc_inds"],
        t["tile_acceptor_hybridization"],
        t["tile_acceptor_n_attached_H"],
        t["is_hydrogen"],
        gp,
        *tors,
    ]


def rotamer_score_args(pose_stack, rotamer_set, term, water_coords):
    """lk_ball_rotamer_score's argument list minus the coordinates
    (lk_ball_energy_term.py:338-358, compiled.ops.cpp:909-976): the rotamer
    set's indexing, the pose's LK-ball tables, the rotamers' waters and
    ``output_block_pair_energies=True``."""
    return _rotamer_common(rotamer_set) + score_args(pose_stack, term, water_coords, True)[12:]


def score_args(pose_stack, term, water_coords, block_pair=False):
    """lk_ball_pose_score's argument list minus the coordinates
    (tmol lk_ball_energy_term.py:275-300)."""
    term.setup_poses(pose_stack)
    pbt = pose_stack.packed_block_types
    t = packed_lkball_tables(pbt)
    return _common(pose_stack) + [
        pose_stack.inter_residue_connections,
        pose_stack.min_block_bondsep,
        pose_stack.inter_block_bondsep,
        pbt.n_atoms,
        pbt.n_conn,
        pbt.conn_atom,
        t["tile_n_polar_atoms"],
        t["tile_n_occluder_atoms"],
        t["tile_pol_occ_inds"],
        t["tile_lk_ball_params"],
        t["bond_separation"],
        term.score_global_params(pbt, pose_stack.device),
        float(torch.tensor(pbt.db.ljlk_global_params["max_dis"], dtype=torch.float32).item()),
        water_coords,
        block_pair,
    ]
