"""``CartesianSfxnNetwork``: a score function over a PoseStack as a torch
module whose parameters are the (unmasked) Cartesian coordinates, tmol's
``tmol/optimization/sfxn_modules.py:12-69``.  ``forward()`` returns the
per-pose weighted total energies [P]; ``segment_ids`` gives each parameter
element its pose, so that ``LBFGS_Armijo`` minimises poses independently;
``pose_stack_from_dofs()`` returns the PoseStack at the current
coordinates.  The scoring module is the B200 ScoreFunction's, so every
energy and gradient comes from the scoring kernels and their adjoints."""

import copy

import torch


class CartesianSfxnNetwork(torch.nn.Module):
    def __init__(self, score_function, pose_stack, coord_mask=None):
        super().__init__()
        self.whole_pose_scoring_module = score_function.render_whole_pose_scoring_module(pose_stack)
        self.pose_stack = pose_stack
        self.full_coords = pose_stack.coords.clone().detach()
        if coord_mask is None:
            coord_mask = torch.ones(self.full_coords.shape[:-1], dtype=torch.bool, device=self.full_coords.device)
        self.coord_mask = coord_mask
        self._flat = coord_mask.reshape(-1).nonzero(as_tuple=False).squeeze(-1)
        self.masked_coords = torch.nn.Parameter(self.full_coords.view(-1, 3)[self._flat].clone())
        pose = torch.arange(self.full_coords.shape[0], device=self.full_coords.device).unsqueeze(1)
        pose = pose.expand(coord_mask.shape).reshape(-1)
        self.segment_ids = pose[self._flat].repeat_interleave(3)
        self.count = 0

    def forward(self):
        self.count += 1
        full = self.full_coords.detach().clone()
        full.view(-1, 3)[self._flat] = self.masked_coords
        self.full_coords = full
        return self.whole_pose_scoring_module(full)

    def pose_stack_from_dofs(self):
        full = self.full_coords.detach().clone()
        full.view(-1, 3)[self._flat] = self.masked_coords.detach()
        ps = copy.copy(self.pose_stack)
        ps.coords = full
        return ps
