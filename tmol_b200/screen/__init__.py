"""Learned block-pair screen for LJ/LK scoring.

A small MLP, trained on block-pair energies that the plain scoring kernel
produces, predicts an upper quantile of each candidate block pair's energy
magnitude; pairs predicted negligible are left out of scoring through the
plan's skip mask.  Training and inference run on hand-written BF16 tensor-core
kernels (``tmol_b200/csrc/screen.cu``).
"""

from .mlp import ScreenMLP  # noqa: F401
from .screen import BlockPairScreen, block_pair_labels  # noqa: F401
