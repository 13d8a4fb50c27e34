"""Score types of the LJ/LK and elec terms (tmol ``tmol/score/score_types.py``)."""

import enum


class ScoreType(enum.IntEnum):
    fa_ljatr = 0
    fa_ljrep = 1
    fa_lk = 2
    fa_elec = 3
