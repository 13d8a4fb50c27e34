"""Candidate enumeration, labels and the skip-mask driver of the screen."""

import os

import torch

from .mlp import ScreenMLP

# the network trained by ``python -m tmol_b200.screen.train`` (2000 synthetic
# poses, 14.1M labelled block pairs), with its calibrated threshold
TRAINED_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "screen_weights.npz")

# label: log10 of the pair's summed energy magnitude, floored at 1e-6
LABEL_FLOOR = 1e-6


def block_pair_labels(plan, coords, capacity):
    """Candidates of ``plan`` at ``coords`` with the energies the plain
    kernel gives them in block-pair mode.  Returns (cand, n, energies [3, n],
    label [n]); ``cand`` is ``LJLKPlan.screen_candidates``'s dict."""
    plan.set_skip_mask(None)
    cand = plan.screen_candidates(coords, capacity)
    E, _ = plan.forward(coords, block_pair=True, want_neighbors=False)
    total = int(cand["count"].item())
    if total > capacity:
        raise RuntimeError(f"{total} screen candidates exceed the capacity {capacity}")
    n = total
    row = cand["row"][:n].long()
    b2 = cand["b2"][:n].long()
    e = E.view(3, -1, plan.max_n_blocks)[:, row, b2]
    del E
    label = torch.log10(e.abs().sum(0) + LABEL_FLOOR)
    return cand, n, e, label


class BlockPairScreen:
    """Screens one plan's block pairs with a trained network.

    ``update(coords)`` enumerates the candidates at ``coords`` and rebuilds
    the skip mask from the network's predictions (all on the device, no host
    synchronisation, so it can sit in a captured CUDA graph next to the
    scoring call); ``attach()`` makes the plan's scoring calls honour the
    mask, ``detach()`` restores plain scoring.  Candidates beyond
    ``capacity`` are never skipped."""

    @classmethod
    def trained(cls, plan, block_type_names=None, capacity=None, path=TRAINED_WEIGHTS):
        """The screen with the trained network shipped in the package."""
        mlp, threshold = ScreenMLP.load(path, plan.device, block_type_names)
        return cls(mlp, plan, threshold, capacity)

    def __init__(self, mlp: ScreenMLP, plan, threshold, capacity=None):
        self.mlp = mlp
        self.plan = plan
        self.threshold = float(threshold)
        rows = plan.n_poses * plan.max_n_blocks
        if capacity is None:
            capacity = max(1024, 48 * rows)
        self.capacity = int(capacity)
        dev = plan.device
        self.mask = torch.zeros((rows, plan.skip_mask_words()), dtype=torch.int32, device=dev)
        self.cand = dict(
            row=torch.empty(self.capacity, dtype=torch.int32, device=dev),
            b2=torch.empty(self.capacity, dtype=torch.int32, device=dev),
            bt=torch.empty((self.capacity, 2), dtype=torch.int32, device=dev),
            features=torch.empty((self.capacity, 12), dtype=torch.float32, device=dev),
            count=torch.zeros(1, dtype=torch.int32, device=dev),
        )
        self.pred = None

    def update(self, coords, keep_predictions=False):
        self.plan.screen_candidates(coords, self.capacity, out=self.cand)
        if keep_predictions and self.pred is None:
            self.pred = torch.empty(self.capacity, dtype=torch.float32, device=self.plan.device)
        self.mlp.infer(self.cand, self.threshold, mask=self.mask, pred=self.pred if keep_predictions else None)

    def attach(self):
        self.plan.set_skip_mask(self.mask)

    def detach(self):
        self.plan.set_skip_mask(None)

    def n_candidates(self):
        return int(self.cand["count"].item())

    def n_skipped(self):
        """Set bits of the mask (pairs the scoring kernel leaves out)."""
        m = self.mask.view(torch.uint8)
        table = torch.tensor([bin(i).count("1") for i in range(256)], dtype=torch.int64, device=m.device)
        return int(table[m.long()].sum().item())
