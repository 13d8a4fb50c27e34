"""Score types of the LJ/LK, elec and LK-ball terms (tmol ``tmol/score/score_types.py``)."""

import enum


class ScoreType(enum.IntEnum):
    fa_ljatr = 0
    fa_ljrep = 1
    fa_lk = 2
    fa_elec = 3
    lk_ball_iso = 4
    lk_ball = 5
    lk_bridge = 6
    lk_bridge_uncpl = 7
