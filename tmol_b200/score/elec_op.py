"""The elec ops on B200, with tmol's argument lists and outputs.

``elec_pose_scores(coords, <23 static arguments>, output_block_pair_energies)``
takes exactly the arguments of ``torch.ops.tmol_elec.elec_pose_scores``
(``tmol/score/elec/potentials/compiled.ops.cpp:526-585``) and returns
``(scores, block_neighbors)``: scores ``[1, P]`` (whole pose) or
``[1, P, B, B]`` (block pairs), neighbours ``[P, B, B]`` int32.
``elec_rotamer_scores`` is ``torch.ops.tmol_elec.elec_rotamer_scores``
(``compiled.ops.cpp:588-647``): ``(scores [1, n], indices [3, n])``.
Gradients flow to ``coords`` only, through the recompute adjoint kernels.

The plan (count-pair tables, partial charges, the potential's constants) is
built once per set of static tensors and cached as the LJ/LK op's is.  All
tensors must be on one CUDA device; there is no CPU path.
"""

import torch

from .. import native
from .ljlk_op import LJLKPlan, _RotamerScoreFn, get_plan, pose_scores_with_plan

N_STATIC = 24  # arguments after coords, including the output-mode flag


class ElecPlan(LJLKPlan):
    """Owns one ``tmol_b200_elec_plan`` (include/tmol_b200_elec.h): of the
    pose op or, with ``rotamers=True``, of the rotamer op."""

    N_TERMS = 1  # fa_elec
    ABI = "tmol_b200_elec"
    NAME = "elec"

    def __init__(self, coords_like, static_args, launch=None, rotamers=False, connectivity=None):
        (
            rot_coord_offset,
            pose_ind_for_atom,
            first_rot_for_block,
            first_rot_block_type,
            block_ind_for_rot,
            pose_ind_for_rot,
            block_type_ind_for_rot,
            n_rots_for_pose,
            rot_offset_for_pose,
            n_rots_for_block,
            rot_offset_for_block,
            max_n_rots_per_pose,
            min_bondsep,
            inter_block_bondsep,
            bt_n_atoms,
            bt_partial_charge,
            bt_n_conn,
            bt_conn_atom,
            bt_inter_repr_path_distance,
            bt_intra_repr_path_distance,
            bt_is_ligand,
            global_params,
            max_dis,
        ) = static_args
        device = self._set_device(coords_like)
        self.block_sizes = (first_rot_block_type, bt_n_atoms)  # for the autotuner's signature
        ints = dict(
            rot_coord_offset=rot_coord_offset,
            pose_ind_for_atom=pose_ind_for_atom,
            first_rot_for_block=first_rot_for_block,
            first_rot_block_type=first_rot_block_type,
            block_ind_for_rot=block_ind_for_rot,
            pose_ind_for_rot=pose_ind_for_rot,
            block_type_ind_for_rot=block_type_ind_for_rot,
            n_rots_for_pose=n_rots_for_pose,
            rot_offset_for_pose=rot_offset_for_pose,
            n_rots_for_block=n_rots_for_block,
            rot_offset_for_block=rot_offset_for_block,
            min_bondsep=min_bondsep,
            inter_block_bondsep=inter_block_bondsep,
            bt_n_atoms=bt_n_atoms,
            bt_n_conn=bt_n_conn,
            bt_conn_atom=bt_conn_atom,
            bt_inter_repr_path_distance=bt_inter_repr_path_distance,
            bt_intra_repr_path_distance=bt_intra_repr_path_distance,
            bt_is_ligand_fragment=bt_is_ligand,
        )
        keep = []
        if connectivity is not None:
            # count-pair tables from the connectivity: the dense bond
            # separation tensors are not needed
            for name in ("min_bondsep", "inter_block_bondsep"):
                if ints[name] is None:
                    del ints[name]
        s = native.ElecInputs()
        for name, t in ints.items():
            if not isinstance(t, torch.Tensor):
                raise TypeError(f"{name} must be a tensor")
            if t.device != device:
                raise RuntimeError(f"{name} is on {t.device}, coordinates on {device}")
            t = t.to(torch.int32).contiguous()
            keep.append(t)
            setattr(s, name, t.data_ptr())
        for name, t in (("bt_partial_charge", bt_partial_charge), ("global_params", global_params)):
            if t.device != device:
                raise RuntimeError(f"{name} is on {t.device}, coordinates on {device}")
            t = t.to(self.dtype).contiguous()
            keep.append(t)
            setattr(s, name, t.data_ptr())
        P, B = first_rot_for_block.shape
        C = bt_conn_atom.shape[1]
        nbt, A = bt_partial_charge.shape
        if inter_block_bondsep is not None and tuple(inter_block_bondsep.shape) != (P, B, B, C, C):
            raise ValueError(
                f"inter_block_bondsep has shape {tuple(inter_block_bondsep.shape)}, expected {(P, B, B, C, C)}"
            )
        if min_bondsep is not None and tuple(min_bondsep.shape) != (P, B, B):
            raise ValueError(f"min_bondsep has shape {tuple(min_bondsep.shape)}, expected {(P, B, B)}")
        for name, t in (("inter", bt_inter_repr_path_distance), ("intra", bt_intra_repr_path_distance)):
            if tuple(t.shape) != (nbt, A, A):
                raise ValueError(f"{name} representative path distances must be [{nbt}, {A}, {A}]")
        if global_params.numel() != 5:
            raise ValueError("global_params must hold 5 values (D, D0, S, min_dis, max_dis)")
        s.n_poses = P
        s.max_n_blocks = B
        s.n_rots = rot_coord_offset.shape[0]
        s.n_block_types = nbt
        s.max_n_block_atoms = A
        s.max_n_conn = C
        s.max_n_rots_per_pose = int(max_n_rots_per_pose)
        s.max_dis = float(max_dis)
        self.n_poses, self.max_n_blocks = P, B
        self.n_atoms = pose_ind_for_atom.shape[0]
        s.n_atoms = self.n_atoms
        self._create(s, launch, rotamers, connectivity)
        del keep

    def set_skip_mask(self, mask):
        raise NotImplementedError("the learned block-pair screen serves LJ/LK plans")

    def screen_candidates(self, coords, capacity, out=None):
        raise NotImplementedError("the learned block-pair screen serves LJ/LK plans")


def elec_pose_scores(coords, *args, return_block_neighbors=True):
    """Drop-in for ``torch.ops.tmol_elec.elec_pose_scores``."""
    if len(args) != N_STATIC:
        raise TypeError(f"elec_pose_scores takes coords + {N_STATIC} arguments, got {1 + len(args)}")
    static = args[:-1]
    block_pair = bool(args[-1])
    plan = get_plan(coords, static, plan_class=ElecPlan)
    return pose_scores_with_plan(coords, plan, block_pair, return_block_neighbors)


def elec_rotamer_scores(coords, *args):
    """Drop-in for ``torch.ops.tmol_elec.elec_rotamer_scores``: the rotamer
    set's coordinates and the op's 24 further arguments (the last,
    ``output_block_pair_energies``, must be True).  Returns
    ``(scores [1, n], indices [3, n])`` for every rotamer pair of
    neighbouring blocks and every rotamer with itself."""
    if len(args) != N_STATIC:
        raise TypeError(f"elec_rotamer_scores takes coords and {N_STATIC} further arguments")
    static, block_pair = args[:-1], args[-1]
    if not block_pair:
        raise ValueError("rotamer scoring reports rotamer-pair energies (output_block_pair_energies=True)")
    flat = coords.reshape(-1, 3)
    plan = get_plan(flat, static, rotamers=True, plan_class=ElecPlan)
    return _RotamerScoreFn.apply(flat, plan)
