"""ScoreFunction: weighted sums of the terms this package provides (LJ/LK,
elec, LK-ball), with tmol's interface (``tmol/score/score_function.py``).

``set_weight(score_type, w)`` pulls in the term that owns the score type;
``render_whole_pose_scoring_module(pose_stack)`` returns a callable whose
``(coords)`` gives the weighted per-pose total ``[n_poses]`` (or, with
``sum_terms=False``, the weighted per-score-type rows), differentiable with
respect to the coordinates through every term's adjoint kernels;
``render_block_pair_scoring_module`` gives ``[n_poses, B, B]``.  Terms are
ordered by their first score type and their outputs concatenated in that
order, as tmol does (``ScoreFunction.get_sorted_terms``).
"""

import torch

from .elec_energy_term import ElecEnergyTerm
from .ljlk_energy_term import LJLKEnergyTerm
from .lkball_energy_term import LKBallEnergyTerm
from .score_types import ScoreType

N_SCORE_TYPES = len(ScoreType)

# the term class providing each score type (tmol's ScoreTermFactory)
TERM_FOR_SCORE_TYPE = {
    ScoreType.fa_ljatr: LJLKEnergyTerm,
    ScoreType.fa_ljrep: LJLKEnergyTerm,
    ScoreType.fa_lk: LJLKEnergyTerm,
    ScoreType.fa_elec: ElecEnergyTerm,
    ScoreType.lk_ball_iso: LKBallEnergyTerm,
    ScoreType.lk_ball: LKBallEnergyTerm,
    ScoreType.lk_bridge: LKBallEnergyTerm,
    ScoreType.lk_bridge_uncpl: LKBallEnergyTerm,
}


class ScoreFunction:
    def __init__(self, device=torch.device("cpu")):
        self._device = torch.device(device)
        self._weights = torch.zeros(N_SCORE_TYPES)
        self._terms = {}  # term class -> instance

    @classmethod
    def from_weights(cls, weights, device=torch.device("cpu")):
        """A score function from {ScoreType or its name: weight} (the
        ``weights`` block of tmol's .sfxn files)."""
        sfxn = cls(device)
        for st, w in weights.items():
            sfxn.set_weight(ScoreType[st] if isinstance(st, str) else st, w)
        return sfxn

    def set_weight(self, st, weight):
        cls = TERM_FOR_SCORE_TYPE[ScoreType(st)]
        if cls not in self._terms:
            self._terms[cls] = cls(device=self._device)
        self._weights[int(st)] = float(weight)

    def get_weight(self, st):
        return float(self._weights[int(st)])

    def all_terms(self):
        """The terms in score-type order."""
        return sorted(self._terms.values(), key=lambda t: min(int(s) for s in t.score_types()))

    def all_score_types(self):
        return [st for t in self.all_terms() for st in t.score_types()]

    def weights_tensor(self):
        """The weights of all_score_types(), in that order."""
        return torch.tensor([float(self._weights[int(st)]) for st in self.all_score_types()], dtype=torch.float32,
                            device=self._device)

    def pre_work_initialization(self, pose_stack):
        for term in self.all_terms():
            if hasattr(term, "setup_poses"):
                term.setup_poses(pose_stack)

    def render_whole_pose_scoring_module(self, pose_stack):
        self.pre_work_initialization(pose_stack)
        return WholePoseScoringModule(
            self.weights_tensor(), [t.render_whole_pose_scoring_module(pose_stack) for t in self.all_terms()]
        )

    def render_block_pair_scoring_module(self, pose_stack):
        self.pre_work_initialization(pose_stack)
        return BlockPairScoringModule(
            self.weights_tensor(), [t.render_block_pair_scoring_module(pose_stack) for t in self.all_terms()]
        )


class WholePoseScoringModule:
    """``(coords) -> [n_poses]`` weighted totals (tmol score_function.py
    WholePoseScoringModule)."""

    def __init__(self, weights, term_modules):
        self.weights = weights.unsqueeze(1)
        self.term_modules = term_modules

    def unweighted_scores(self, coords):
        return torch.cat([m(coords) for m in self.term_modules], dim=0)

    def __call__(self, coords, sum_terms=True, apply_weights=True):
        scores = self.unweighted_scores(coords)
        if apply_weights:
            scores = self.weights.to(scores.dtype) * scores
        return scores.sum(dim=0) if sum_terms else scores


class BlockPairScoringModule(WholePoseScoringModule):
    """``(coords) -> [n_poses, B, B]`` weighted block-pair totals."""

    def __init__(self, weights, term_modules):
        super().__init__(weights, term_modules)
        self.weights = weights.view(-1, 1, 1, 1)
