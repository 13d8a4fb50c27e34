"""The C oracle's rotamer scoring (ljlk_rotamer_scores) against the
reference: bit for bit against the committed fixture (rotamer-pair energies,
dispatch indices, gradient of a weighted sum) and, where the compiled
reference op is present, against it on further seeded rotamer sets."""

import numpy
import pytest
import torch

from oracle import oracle as O
from tests.conftest import load_golden
from tmol_b200.pose.rotamers import RotamerSet, synthetic_rotamer_set
from tmol_b200.pose.synthetic import synthetic_pose_stack
from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, rotamer_score_args

FIELDS = (
    "n_rots_for_pose", "rot_offset_for_pose", "n_rots_for_block", "rot_offset_for_block", "pose_for_rot",
    "block_type_ind_for_rot", "block_ind_for_rot", "coord_offset_for_rot", "coords", "first_rot_block_type",
    "pose_ind_for_atom",
)


def fixture_case(device="cpu"):
    g = load_golden("rotamers.npz")
    ps = synthetic_pose_stack(list(g["sizes"]), list(g["seeds"]), device=device)
    rs = RotamerSet(
        max_n_rots_per_pose=int(g["max_n_rots_per_pose"]),
        **{f: torch.tensor(g[f], device=device) for f in FIELDS},
    )
    return g, ps, rs


def test_rotamer_set_is_reproducible():
    g, ps, rs = fixture_case()
    again = synthetic_rotamer_set(ps, max_rots=4, mutate_fraction=0.25, seed=5, skip_fraction=0.1)
    for f in FIELDS:
        a, b = getattr(again, f).numpy(), g[f]
        if f == "coords":
            numpy.testing.assert_allclose(a, b, atol=1e-4)
        else:
            assert numpy.array_equal(a, b), f
    # some blocks have no rotamers, some rotamers change the residue type
    assert (g["n_rots_for_block"] == 0).sum() > 0
    bt_first = g["block_type_ind_for_rot"][g["rot_offset_for_block"]]
    assert (g["block_type_ind_for_rot"] != numpy.repeat(bt_first.reshape(-1), g["n_rots_for_block"].reshape(-1))).any()


def test_oracle_matches_reference_fixture():
    g, ps, rs = fixture_case()
    args = rotamer_score_args(ps, rs, LJLKEnergyTerm())
    oc = O.OracleCall(rs.coords, args)
    E, idx, nbr = oc.rotamer_scores()
    assert numpy.array_equal(idx, g["ref_indices"])
    assert numpy.array_equal(E, g["ref_energies"])
    dx = oc.rotamer_backward(nbr, g["weights"])
    assert numpy.array_equal(dx, g["ref_grad"])


@pytest.mark.skipif(not O.reference_available(), reason="compiled reference op not built")
@pytest.mark.parametrize("seed,mut,skip", [(31, 0.0, 0.0), (32, 0.5, 0.2)])
def test_oracle_matches_reference_op(seed, mut, skip):
    ps = synthetic_pose_stack([40, 17], [seed, seed + 1], extra_chi_sd=15.0)
    rs = synthetic_rotamer_set(ps, max_rots=5, mutate_fraction=mut, seed=seed, skip_fraction=skip)
    args = rotamer_score_args(ps, rs, LJLKEnergyTerm())
    E_ref, c, idx_ref = O.reference_rotamer_scores(rs.coords, args)
    oc = O.OracleCall(rs.coords, args)
    E, idx, nbr = oc.rotamer_scores()
    assert numpy.array_equal(idx, idx_ref.numpy())
    assert numpy.array_equal(E, E_ref.detach().numpy())
    w = torch.tensor(numpy.random.default_rng(seed).normal(size=tuple(E_ref.shape)), dtype=E_ref.dtype)
    (E_ref * w).sum().backward()
    assert numpy.array_equal(oc.rotamer_backward(nbr, w.numpy()), c.grad.numpy())
