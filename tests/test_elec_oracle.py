"""The C oracle's elec term against the reference elec op: bit for bit
against the committed fixture (1ubq and a jagged synthetic batch: per-pose
energies, gradient, neighbour matrix, block-pair energies), against the
live compiled op where it is present, and the partial-charge and count-pair
representative tables against tmol's rules."""

import numpy
import pytest
import torch

from oracle import oracle as O
from tests.conftest import load_golden
from tmol_b200.pose.synthetic import synthetic_pose_stack
from tmol_b200.score.elec_energy_term import ElecEnergyTerm, ElecParams, elec_pose_score_args


@pytest.fixture(scope="module")
def eterm():
    return ElecEnergyTerm()


def cases(ubq_pose_stack):
    g = load_golden("elec.npz")
    return g, [("ubq", ubq_pose_stack), ("syn", synthetic_pose_stack(list(g["sizes"]), list(g["seeds"])))]


def test_oracle_matches_reference_fixture(ubq_pose_stack, eterm):
    g, pss = cases(ubq_pose_stack)
    for tag, ps in pss:
        coords = ps.coords.flatten(0, 1)
        oc = O.OracleCall(coords, elec_pose_score_args(ps, eterm), term="elec")
        E, dV, nbr = oc.pose_scores(require_gradient=True)
        assert numpy.array_equal(E[:1], g[f"{tag}_energies"]), tag
        assert numpy.array_equal(dV[0], g[f"{tag}_grad"]), tag
        assert numpy.array_equal(nbr, g[f"{tag}_neighbors"]), tag
        Eb, _, _ = oc.pose_scores(block_pair=True)
        assert numpy.array_equal(Eb[:1], g[f"{tag}_block_pair"]), tag


@pytest.mark.skipif(not O.reference_elec_available(), reason="compiled reference elec op not built")
@pytest.mark.parametrize("f64", [False, True])
def test_oracle_matches_reference_op(eterm, f64):
    ps = synthetic_pose_stack([60, 25], [41, 42], extra_chi_sd=20.0)
    args = elec_pose_score_args(ps, eterm)
    dt = torch.float64 if f64 else torch.float32
    coords = ps.coords.flatten(0, 1).to(dt)
    args64 = [a.to(dt) if isinstance(a, torch.Tensor) and a.is_floating_point() else a for a in args]
    E_ref, c, nbr_ref = O.reference_elec_pose_scores(coords, args64)
    E_ref.sum().backward()
    oc = O.OracleCall(coords, args, f64=f64, term="elec")
    E, dV, nbr = oc.pose_scores(require_gradient=True)
    assert numpy.array_equal(nbr, nbr_ref.numpy())
    if not f64:
        assert numpy.array_equal(E[:1], E_ref.detach().numpy())
        assert numpy.array_equal(dV[0], c.grad.numpy())
    else:
        # float64: the same operations, the last bit of some pair energies
        # differs (the reference compiler's evaluation of the dielectric)
        numpy.testing.assert_allclose(E[:1], E_ref.detach().numpy(), rtol=1e-13, atol=0)
        g_ref = c.grad.numpy()
        numpy.testing.assert_allclose(dV[0], g_ref, rtol=1e-12, atol=1e-12 * numpy.abs(g_ref).max())
    w = numpy.random.default_rng(3).normal(size=(3,) + E.shape[1:])
    w[1:] = 0
    dx = oc.backward(nbr, w, per_pose_weights=True)
    ref = dV[0] * w[0, ps.pose_ind_for_atom.numpy()][:, None]
    # the same terms summed in another order
    numpy.testing.assert_allclose(dx, ref, rtol=1e-5, atol=1e-5 * numpy.abs(ref).max())


def test_charge_and_representative_tables(eterm):
    from tmol_b200.chem.restypes import ResidueTypeSet

    rts = ResidueTypeSet.get_default()
    p = ElecParams()
    # variants take their own charges, falling back to the unpatched entry
    ala_n = rts.types["ALA:nterm"]
    q = dict(zip(ala_n.atom_names, p.partial_charges_for_block(ala_n)))
    assert q["N"] == pytest.approx(-0.10440) and q["CB"] == pytest.approx(-0.36465)
    # a hydrogen's representative is its heavy atom: the pair distances use
    # the heavy atom's path distances
    ala = rts.types["ALA"]
    rep = p.representative_mapping(ala)
    assert rep[ala.atom_index["N"]] == ala.atom_index["H"]
    charge, inter, intra = eterm.block_type_tables(ala)
    pd = numpy.asarray(ala.path_distance)
    assert (inter == pd[:, rep]).all() and (intra == pd[rep][:, rep]).all()
    assert abs(charge.sum()) < 1e-4  # neutral residue


def test_oracle_rotamer_scores_match_reference_fixture(eterm):
    """Elec rotamer scoring (elec_rotamer_scores) on the rotamer set of
    rotamers.npz: dispatch, energies and the gradient of sum(w * E)."""
    from tests.test_rotamer_oracle import fixture_case
    from tmol_b200.score.elec_energy_term import elec_rotamer_score_args

    g = load_golden("elec.npz")
    _, ps, rs = fixture_case()
    oc = O.OracleCall(rs.coords, elec_rotamer_score_args(ps, rs, eterm), term="elec")
    E, idx, nbr = oc.rotamer_scores()
    assert numpy.array_equal(idx, g["rot_indices"])
    assert numpy.array_equal(E[:1], g["rot_energies"])
    w = numpy.zeros((3, E.shape[1]), dtype=numpy.float32)
    w[0] = g["rot_weights"][0]
    assert numpy.array_equal(oc.rotamer_backward(nbr, w), g["rot_grad"])


def test_oracle_reproduces_the_reference_suites_stored_energy(ubq_pose_stack, eterm):
    """1ubq elec energy stored by tmol's own test suite
    (tmol/tests/data/term_baselines/ElecEnergyTerm/test_whole_pose_scoring_10.yaml;
    that test's tolerance is atol 1e-5, rtol 1e-3): pins this package's charge
    and count-pair representative tables."""
    g = load_golden("elec.npz")
    oc = O.OracleCall(ubq_pose_stack.coords.flatten(0, 1), elec_pose_score_args(ubq_pose_stack, eterm), term="elec")
    E, _, _ = oc.pose_scores()
    numpy.testing.assert_allclose(E[0, 0], g["ubq_tmol_test_energy"][0], rtol=1e-6, atol=1e-5)
