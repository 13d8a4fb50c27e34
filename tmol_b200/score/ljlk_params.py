"""LJ/LK parameters packed as the op expects them.

``type_params[T, 10]`` columns (``tmol/score/ljlk/ljlk_energy_term.py:130-146``):
lj_radius, lj_wdepth, lk_dgfree, lk_lambda, lk_volume, is_donor,
is_hydroxyl, is_polarh, is_acceptor, is_carbon_lk.  ``is_carbon_lk`` marks
CH1/CH2/CH3/Caro, the carbon types whose C-C LK is flattened
(``tmol/score/ljlk/params.py:132-136``).

``global_params[1, 5]`` (``ljlk_energy_term.py:147-162``): max_dis,
lj_dlin_sigma_factor (the soft value when ``soft_rep`` is set), lj_hbond_dis,
lj_hbond_OH_donor_dis, lj_hbond_hdis.
"""

import math

import torch

CARBON_LK_TYPES = ("CH1", "CH2", "CH3", "Caro")
TYPE_PARAM_COLUMNS = (
    "lj_radius",
    "lj_wdepth",
    "lk_dgfree",
    "lk_lambda",
    "lk_volume",
    "is_donor",
    "is_hydroxyl",
    "is_polarh",
    "is_acceptor",
    "is_carbon_lk",
)


def type_params_tensor(db, device=torch.device("cpu")):
    rows = []
    for at in db.atom_types:
        row = []
        for col in TYPE_PARAM_COLUMNS:
            if col == "is_carbon_lk":
                row.append(1.0 if at["name"] in CARBON_LK_TYPES else 0.0)
            else:
                v = at[col]
                row.append(float(v) if v is not None else math.nan)
        rows.append(row)
    return torch.tensor(rows, dtype=torch.float32, device=device)


def global_params_tensor(db, soft_rep=False, device=torch.device("cpu")):
    g = db.ljlk_global_params
    return torch.tensor(
        [
            [
                g["max_dis"],
                g["lj_dlin_sigma_factor_soft"] if soft_rep else g["lj_dlin_sigma_factor"],
                g["lj_hbond_dis"],
                g["lj_hbond_OH_donor_dis"],
                g["lj_hbond_hdis"],
            ]
        ],
        dtype=torch.float32,
        device=device,
    )
