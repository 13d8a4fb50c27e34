"""Per-term scoring modules (tmol ``tmol/score/common/scoring_module.py:7-130``).

A module caches the pose stack's rotamer views and the term's static
arguments as non-trainable parameters; ``forward(coords)`` flattens the
coordinates to ``[n_poses * max_pose_atoms, 3]`` and calls the term's op.
The whole-pose module returns ``[n_terms, n_poses]``; the block-pair module
``[n_terms, n_poses, max_n_blocks, max_n_blocks]``.
"""

import torch


def _p(t):
    return torch.nn.Parameter(t, requires_grad=False) if isinstance(t, torch.Tensor) else t


class TermPoseScoringModule(torch.nn.Module):
    def __init__(self, classname, pose_stack, term_parameters, term_score_poses, block_pair):
        super().__init__()
        self.classname = classname
        self.common_parameters = [
            _p(t)
            for t in [
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
        ]
        self.term_parameters = [_p(t) for t in term_parameters]
        self.term_score_poses = term_score_poses
        self.n_poses = pose_stack.n_poses
        self.max_n_blocks = pose_stack.max_n_blocks
        self._tail = tuple(self.common_parameters) + tuple(self.term_parameters) + (block_pair,)
        for i, t in enumerate(self.common_parameters + self.term_parameters):
            if isinstance(t, torch.nn.Parameter):
                self.register_parameter(f"static_{i}", t)

    def forward(self, coords):
        flat = coords.flatten(start_dim=0, end_dim=-2)
        scores, _ = self.term_score_poses(flat, *self._tail)
        return scores


class TermWholePoseScoringModule(TermPoseScoringModule):
    def __init__(self, classname, pose_stack, term_parameters, term_score_poses):
        super().__init__(classname, pose_stack, term_parameters, term_score_poses, False)


class TermBlockPairScoringModule(TermPoseScoringModule):
    def __init__(self, classname, pose_stack, term_parameters, term_score_poses):
        super().__init__(classname, pose_stack, term_parameters, term_score_poses, True)


class TermRotamerScoringModule(torch.nn.Module):
    """Rotamer scoring (tmol ``scoring_module.py:133-201``): ``forward(coords)``
    with the rotamer set's coordinates ``[n_rot_atoms, 3]`` returns
    ``(scores [n_terms, n], indices [3, n])`` (pose, rot1, rot2 in global
    rotamer numbering) without building a sparse tensor."""

    def __init__(self, classname, rotamer_set, term_parameters, term_score_rotamers):
        super().__init__()
        self.classname = classname

        def i32(t):
            return t if isinstance(t, int) else t.to(torch.int32)

        rs = rotamer_set
        self.common_parameters = [
            _p(i32(t))
            for t in [
                rs.coord_offset_for_rot,
                rs.pose_ind_for_atom,
                rs.rot_offset_for_block,
                rs.first_rot_block_type,
                rs.block_ind_for_rot,
                rs.pose_for_rot,
                rs.block_type_ind_for_rot,
                rs.n_rots_for_pose,
                rs.rot_offset_for_pose,
                rs.n_rots_for_block,
                rs.rot_offset_for_block,
                int(rs.max_n_rots_per_pose),
            ]
        ]
        self.term_parameters = [_p(t) for t in term_parameters]
        self.term_score_rotamers = term_score_rotamers
        self.n_poses = rs.n_rots_for_pose.shape[0]
        self.n_rots = rs.coord_offset_for_rot.shape[0]
        self._tail = tuple(self.common_parameters) + tuple(self.term_parameters) + (True,)
        for i, t in enumerate(self.common_parameters + self.term_parameters):
            if isinstance(t, torch.nn.Parameter):
                self.register_parameter(f"static_{i}", t)

    def forward(self, coords):
        flat = coords.flatten(start_dim=0, end_dim=-2)
        return self.term_score_rotamers(flat, *self._tail)

    def forward_split(self, coords):
        """Per-term sparse [n_poses, n_rots, n_rots] tensors, stacked."""
        scores, indices = self.forward(coords)
        return torch.stack(
            [
                torch.sparse_coo_tensor(
                    indices, scores[t], size=(self.n_poses, self.n_rots, self.n_rots), check_invariants=True
                )
                for t in range(scores.shape[0])
            ]
        )
