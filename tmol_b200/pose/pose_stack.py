"""PoseStack: a batch of molecular systems with per-block chemistry.

The fields and the derived per-"rotamer" views follow tmol's ``PoseStack``
(``tmol/pose/pose_stack.py:86-168``): in whole-pose scoring every block has
exactly one rotamer, so the rotamer index of (pose p, block b) is
``p * max_n_blocks + b`` and the rotamer's first atom is the block's coordinate
offset plus the pose's offset into the flattened coordinate array.
"""

import torch


class PoseStack:
    def __init__(
        self,
        packed_block_types,
        coords,
        block_coord_offset,
        inter_residue_connections,
        inter_block_bondsep,
        block_type_ind,
        device,
    ):
        self.packed_block_types = packed_block_types
        self.coords = coords
        self.block_coord_offset = block_coord_offset
        self.block_coord_offset64 = block_coord_offset.to(torch.int64)
        self.inter_residue_connections = inter_residue_connections
        self.inter_residue_connections64 = inter_residue_connections.to(torch.int64)
        self.inter_block_bondsep = inter_block_bondsep
        self.block_type_ind = block_type_ind
        self.block_type_ind64 = block_type_ind.to(torch.int64)
        self.device = torch.device(device)
        self._derive_rotamer_views()

    def _derive_rotamer_views(self):
        n_poses, n_blocks = self.block_coord_offset.shape
        dev = self.device
        self.block_ind_for_rot = (
            torch.arange(n_blocks, dtype=torch.int32, device=dev).repeat(n_poses)
        )
        self.pose_ind_for_rot = (
            torch.arange(n_poses, dtype=torch.int32, device=dev)
            .unsqueeze(1)
            .expand(n_poses, n_blocks)
            .flatten()
            .contiguous()
        )
        self.block_type_ind_for_rot = self.block_type_ind.flatten().contiguous()
        self.rot_offset_for_block = torch.arange(
            n_poses * n_blocks, dtype=torch.int32, device=dev
        ).view(n_poses, n_blocks)
        self.first_rot_for_block = self.rot_offset_for_block
        self.first_rot_block_type = self.block_type_ind
        self.n_rots_for_pose = torch.full((n_poses,), n_blocks, dtype=torch.int32, device=dev)
        self.rot_offset_for_pose = self.n_rots_for_pose * torch.arange(
            n_poses, dtype=torch.int32, device=dev
        )
        self.n_rots_for_block = torch.ones_like(self.block_coord_offset)
        coord_offset_for_pose = self.coords.size(1) * torch.arange(
            n_poses, dtype=torch.int32, device=dev
        )
        self.rot_coord_offset = (
            self.block_coord_offset.flatten()
            + torch.repeat_interleave(coord_offset_for_pose, n_blocks)
        ).to(torch.int32)
        self.max_n_rots_per_pose = n_blocks
        atom_to_pose = torch.zeros(
            self.coords.size(0) * self.coords.size(1), dtype=torch.int32, device=dev
        )
        pose_atom_offsets = self.rot_coord_offset.index_select(
            0, self.rot_offset_for_pose.to(torch.int64)
        ).to(torch.int64)
        atom_to_pose[pose_atom_offsets] = 1
        atom_to_pose[0] = 0
        self.pose_ind_for_atom = atom_to_pose.cumsum(0, dtype=torch.int32)

    @property
    def n_poses(self):
        return self.block_coord_offset.shape[0]

    @property
    def max_n_blocks(self):
        return self.block_coord_offset.shape[1]

    @property
    def max_n_pose_atoms(self):
        return self.coords.shape[1]

    def n_blocks_per_pose(self):
        return (self.block_type_ind >= 0).sum(dim=1)

    def slice_poses(self, p0, p1):
        """A PoseStack of poses [p0, p1) (same block and atom padding)."""
        return PoseStack(
            self.packed_block_types,
            self.coords[p0:p1],
            self.block_coord_offset[p0:p1],
            self.inter_residue_connections[p0:p1],
            self.inter_block_bondsep[p0:p1],
            self.block_type_ind[p0:p1],
            self.device,
        )

    def to(self, device):
        device = torch.device(device)
        ps = PoseStack(
            self.packed_block_types.to(device),
            self.coords.to(device),
            self.block_coord_offset.to(device),
            self.inter_residue_connections.to(device),
            self.inter_block_bondsep.to(device),
            self.block_type_ind.to(device),
            device,
        )
        return ps
