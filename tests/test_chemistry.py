"""Host-side chemistry and PoseStack construction (tmol semantics)."""

import numpy
import torch

from tmol_b200.chem.restypes import (
    MAX_SIG_BOND_SEPARATION,
    ResidueTypeSet,
    default_packed_block_types,
    tile_subset_indices,
)
from tmol_b200.pose.builder import build_pose_stack, topology_from_sequence
from tmol_b200.pose.synthetic import synthetic_pose_stack


def test_tile_subset_indices_matches_reference_docstring_example():
    # tmol/score/common/stack_condense.py:316-327
    tiles, counts = tile_subset_indices([0, 3, 4, 7, 10, 12, 14], 8)
    assert tiles.tolist() == [0, 3, 4, 7, -1, -1, -1, -1, 2, 4, 6, -1, -1, -1, -1, -1]
    assert counts.tolist() == [4, 3]


def test_path_distance_and_variants():
    rts = ResidueTypeSet.get_default()
    ala = rts.types["ALA"]
    i = ala.atom_index
    assert ala.path_distance[i["N"], i["CA"]] == 1
    assert ala.path_distance[i["N"], i["C"]] == 2
    assert ala.path_distance[i["H"], i["HB1"]] == 4
    assert ala.path_distance[i["O"], i["HB1"]] == 4
    nt = rts.types["ALA:nterm"]
    assert "H" not in nt.atom_index and {"H1", "H2", "H3"} <= set(nt.atom_names)
    assert nt.atom_type_names[nt.atom_index["N"]] == "Nlys"
    assert nt.connection_names == ["up"]
    ct = rts.types["ALA:cterm"]
    assert "OXT" in ct.atom_index and ct.connection_names == ["down"]
    assert ct.atom_type_names[ct.atom_index["O"]] == "OOC"
    pro = rts.types["PRO:nterm"]
    assert {"H2", "H3"} <= set(pro.atom_names) and "H1" not in pro.atom_index
    # path distances are capped at MAX_SIG_BOND_SEPARATION
    arg = rts.types["ARG"]
    assert arg.path_distance.max() == MAX_SIG_BOND_SEPARATION


def test_packed_block_types_tables():
    pbt = default_packed_block_types()
    assert pbt.max_n_conn == 2
    n = pbt.n_atoms.numpy()
    at = pbt.atom_types.numpy()
    for k, bt in enumerate(pbt.active_block_types):
        assert n[k] == bt.n_atoms
        assert (at[k, : n[k]] >= 0).all() and (at[k, n[k] :] == -1).all()
    # heavy atoms in tile: canonical residues fit one tile
    nh = pbt.ljlk_n_heavy_atoms_in_tile.numpy()
    assert nh.shape[1] == 1
    trp = pbt.bt_index["TRP"]
    assert nh[trp, 0] == 14


def test_inter_block_bondsep_linear_chain():
    ps = build_pose_stack([topology_from_sequence("AGSA")])
    ibb = ps.inter_block_bondsep[0].numpy()
    # residue 0 (nterm) has only "up" (conn 0); residue 1 has down(0), up(1)
    assert ibb[0, 1, 0, 0] == 1  # C(0) - N(1)
    assert ibb[0, 2, 0, 0] == 4  # C(0) - N(1)-CA-C(1) - N(2)
    assert ibb[1, 2, 1, 0] == 1
    assert ibb[0, 3].min() == MAX_SIG_BOND_SEPARATION
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm

    LJLKEnergyTerm().setup_poses(ps)
    mbs = ps.min_block_bondsep[0].numpy()
    assert mbs[0, 1] == 1 and mbs[0, 2] == 4 and mbs[1, 3] == 4 and mbs[0, 3] == 6


def test_rotamer_views():
    ps = synthetic_pose_stack([3, 5], [0, 1])
    P, B = 2, 5
    assert ps.rot_coord_offset.shape == (P * B,)
    assert ps.pose_ind_for_atom.shape == (P * ps.max_n_pose_atoms,)
    assert ps.pose_ind_for_atom[ps.max_n_pose_atoms].item() == 1
    assert ps.block_type_ind[0, 3].item() == -1
    assert ps.rot_coord_offset[B].item() == ps.max_n_pose_atoms


def test_synthetic_geometry_is_ideal():
    ps = synthetic_pose_stack([12], [3])
    pbt = ps.packed_block_types
    c = ps.coords[0].numpy()
    for b in range(12):
        bt = pbt.active_block_types[ps.block_type_ind[0, b]]
        off = ps.block_coord_offset[0, b].item()
        for x, y in bt.bonds:
            d = numpy.linalg.norm(c[off + bt.atom_index[x]] - c[off + bt.atom_index[y]])
            assert 0.9 < d < 1.9, (bt.name, x, y, d)
