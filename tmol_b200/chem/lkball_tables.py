"""Block-type tables of the LK-ball term, from this package's chemistry.

The LK-ball term builds waters on polar atoms and scores them against the
heavy atoms around; it reads, per block type (tmol's ``HBondDependentTerm``,
``BondDependentTerm`` and ``LKBallEnergyTerm`` setup,
``tmol/score/hbond/hbond_dependent_term.py:20-358``,
``tmol/score/bond_dependent_term.py:19-90``,
``tmol/score/lk_ball/lk_ball_energy_term.py:67-228``):

* hydrogen flags and the hbond donors / acceptors, tiled by 32 atoms: donor
  hydrogens with their heavy atom and their rank among its hydrogens,
  acceptors with their hybridization (none / sp2 / sp3 / ring = 0..3) and
  attached-hydrogen count;
* "all bonds": each atom's intra-block bonds (both directions, in sorted
  order) followed by its inter-block connections (``tmol/chemical/
  all_bonds.py:8-80``), with per-atom ranges — the water builder walks them
  to find acceptor base atoms, across connections when needed;
* per tile, the polar atoms (those that carry waters: donor heavy atoms and
  acceptors) followed by the other heavy atoms ("occluders"), as tile-local
  indices, with nine per-atom parameters (LJ radius, LK dgfree / lambda /
  volume, donor, hydroxyl, polar-H, acceptor and carbon-LK flags).

Donor and acceptor atom types come from tmol's ``hbond.yaml``; the
hybridization from ``chemical.yaml``; both are in the committed chemistry
extract.
"""

import numpy
import torch

from .restypes import MAX_SIG_BOND_SEPARATION, TILE_SIZE

HYBRIDIZATION = {None: 0, "sp2": 1, "sp3": 2, "ring": 3}
N_LKB_PARAMS = 9


def _tile_args(indices, tile_size, n_atoms):
    """Positions in `indices` grouped by tile (index // tile_size), left
    justified, -1 padded; and the per-tile counts.  ceil(n_atoms / tile)
    tiles (tmol ``stack_condense.arg_tile_subset_indices``)."""
    n_tiles = max(n_atoms - 1, 0) // tile_size + 1
    out = numpy.full(n_tiles * tile_size, -1, dtype=numpy.int32)
    counts = numpy.zeros(n_tiles, dtype=numpy.int32)
    for k, ind in enumerate(indices):
        t = int(ind) // tile_size
        out[t * tile_size + counts[t]] = k
        counts[t] += 1
    return out.reshape(n_tiles, tile_size), counts


def sorted_bond_pairs(bt):
    """Intra-block bonds in both directions, sorted (tmol's bond_indices)."""
    pairs = set()
    for a, b in bt.bonds:
        i, j = bt.atom_index[a], bt.atom_index[b]
        pairs.add((i, j))
        pairs.add((j, i))
    return sorted(pairs)


def all_bonds(bt):
    """(all_bonds [n, 3] = (atom, other atom or -1, connection or -1),
    atom_all_bond_ranges [n_atoms, 2])."""
    n = bt.n_atoms
    intra = sorted_bond_pairs(bt)
    conn_atoms = [bt.atom_index[a] for _, a in bt.connections]
    count = numpy.zeros(n, dtype=numpy.int64)
    for i, _ in intra:
        count[i] += 1
    for a in conn_atoms:
        count[a] += 1
    # the reference's rule: atom 0 starts at 0 (or stays (-1, -1) without
    # bonds), every later atom starts where the previous one ended
    ranges = numpy.full((n, 2), -1, dtype=numpy.int32)
    for i in range(n):
        if i == 0:
            if count[0] > 0:
                ranges[0] = (0, count[0])
        else:
            ranges[i] = (ranges[i - 1, 1], ranges[i - 1, 1] + count[i])
    bonds = numpy.zeros((len(intra) + len(conn_atoms), 3), dtype=numpy.int32)
    fill = numpy.zeros(n, dtype=numpy.int64)
    for i, j in intra:
        k = ranges[i, 0] + fill[i]
        fill[i] += 1
        bonds[k] = (i, j, -1)
    for c, a in enumerate(conn_atoms):
        k = ranges[a, 0] + fill[a]
        fill[a] += 1
        bonds[k] = (a, -1, c)
    return bonds, ranges


def hbond_block_params(bt, db):
    """Donors, acceptors and their tiles for one block type (a dict of the
    fields of tmol's HBondBlockTypeParams that LK-ball reads)."""
    n = bt.n_atoms
    types = [db.atom_types[db.atom_type_index[t]] for t in bt.atom_type_names]
    is_h = numpy.array([t["is_hydrogen"] for t in types], dtype=numpy.int32)
    hyb = numpy.array([HYBRIDIZATION[t.get("acceptor_hybridization")] for t in types], dtype=numpy.int32)
    acc_types = set(db.hbond_acceptor_atom_types)
    don_types = set(db.hbond_donor_atom_types)
    A_idx = numpy.array([i for i, t in enumerate(bt.atom_type_names) if t in acc_types], dtype=numpy.int32)
    D_idx = numpy.array([i for i, t in enumerate(bt.atom_type_names) if t in don_types], dtype=numpy.int32)

    # hydrogens bonded to each donor, in bond order; then sorted by H index
    nbrs = [[] for _ in range(n)]
    for i, j in sorted_bond_pairs(bt):
        nbrs[i].append(j)
    H, D_for_H, which, n_H_for_D = [], [], [], []
    for d in D_idx:
        k = 0
        for j in nbrs[d]:
            if is_h[j]:
                H.append(j)
                D_for_H.append(int(d))
                which.append(k)
                k += 1
        n_H_for_D.append(k)
    order = numpy.argsort(numpy.array(H, dtype=numpy.int64), kind="stable")
    H = numpy.array(H, dtype=numpy.int32)[order]
    D_for_H = numpy.array(D_for_H, dtype=numpy.int32)[order]
    which = numpy.array(which, dtype=numpy.int32)[order]
    n_H_for_at = numpy.zeros(n, dtype=numpy.int32)
    n_H_for_at[D_idx] = numpy.array(n_H_for_D, dtype=numpy.int32)

    acc_args, tile_n_acc = _tile_args(A_idx, TILE_SIZE, n)
    n_tiles = tile_n_acc.shape[0]
    tile_acc_inds = numpy.full((n_tiles, TILE_SIZE), -1, dtype=numpy.int32)
    tile_acc_hyb = numpy.full((n_tiles, TILE_SIZE), -1, dtype=numpy.int32)
    tile_acc_nH = numpy.full((n_tiles, TILE_SIZE), -1, dtype=numpy.int32)
    m = acc_args >= 0
    tile_acc_inds[m] = A_idx[acc_args[m]] % TILE_SIZE
    tile_acc_hyb[m] = hyb[A_idx[acc_args[m]]]
    tile_acc_nH[m] = n_H_for_at[A_idx[acc_args[m]]]

    h_args, tile_n_donH = _tile_args(H, TILE_SIZE, n)
    tile_donH_inds = numpy.full((n_tiles, TILE_SIZE), -1, dtype=numpy.int32)
    tile_donH_hvy = numpy.full((n_tiles, TILE_SIZE), -1, dtype=numpy.int32)
    tile_which = numpy.full((n_tiles, TILE_SIZE), -1, dtype=numpy.int32)
    m = h_args >= 0
    tile_donH_inds[m] = H[h_args[m]] % TILE_SIZE
    tile_donH_hvy[m] = D_for_H[h_args[m]]
    tile_which[m] = which[h_args[m]]
    return dict(
        is_hydrogen=is_h,
        don_hvy_inds=D_idx,
        acc_inds=A_idx,
        tile_n_donH=tile_n_donH,
        tile_n_acc=tile_n_acc,
        tile_donH_inds=tile_donH_inds,
        tile_donH_hvy_inds=tile_donH_hvy,
        tile_which_donH_of_donH_hvy=tile_which,
        tile_acc_inds=tile_acc_inds,
        tile_acceptor_hybridization=tile_acc_hyb,
        tile_acceptor_n_attached_H=tile_acc_nH,
    )


def lkball_block_params(bt, db, hb):
    """Polar-then-occluder tiles and their nine parameters for one block
    type (tmol's LKBallBlockTypeParams)."""
    n = bt.n_atoms
    is_polar = numpy.zeros(n, dtype=bool)
    is_polar[hb["don_hvy_inds"]] = True
    is_polar[hb["acc_inds"]] = True
    polar = numpy.nonzero(is_polar)[0].astype(numpy.int32)
    pol_args, tile_n_polar = _tile_args(polar, TILE_SIZE, n)
    n_tiles = tile_n_polar.shape[0]
    heavy_apolar = numpy.nonzero((hb["is_hydrogen"] == 0) & ~is_polar)[0].astype(numpy.int32)
    apo_args, tile_n_apolar = _tile_args(heavy_apolar, TILE_SIZE, n)
    pol_occ = numpy.full((n_tiles, TILE_SIZE), -1, dtype=numpy.int32)
    tile_n_occ = numpy.zeros(n_tiles, dtype=numpy.int32)
    for t in range(n_tiles):
        k = 0
        for s in range(TILE_SIZE):
            if pol_args[t, s] >= 0:
                pol_occ[t, k] = polar[pol_args[t, s]]
                k += 1
        for s in range(TILE_SIZE):
            if apo_args[t, s] >= 0:
                pol_occ[t, k] = heavy_apolar[apo_args[t, s]]
                k += 1
        tile_n_occ[t] = k
    params = numpy.zeros((n_tiles, TILE_SIZE, N_LKB_PARAMS), dtype=numpy.float32)
    for t in range(n_tiles):
        for s in range(tile_n_occ[t]):
            at = db.atom_types[db.atom_type_index[bt.atom_type_names[pol_occ[t, s]]]]
            params[t, s] = [
                at["lj_radius"],
                at["lk_dgfree"],
                at["lk_lambda"],
                at["lk_volume"],
                float(at["is_donor"]),
                float(at["is_hydroxyl"]),
                float(at["is_polarh"]),
                float(at["is_acceptor"]),
                float(_is_carbon_lk(at["name"])),
            ]
    tile_pol_occ_inds = numpy.where(pol_occ >= 0, pol_occ % TILE_SIZE, -1).astype(numpy.int32)
    return dict(
        tile_n_polar_atoms=tile_n_polar,
        tile_n_occluder_atoms=tile_n_occ,
        tile_pol_occ_inds=tile_pol_occ_inds,
        tile_lk_ball_params=params,
    )


def _is_carbon_lk(type_name):
    # tmol/score/ljlk/params.py:132-136: CH1, CH2, CH3 and aromatic carbons
    return type_name in ("CH1", "CH2", "CH3", "Caro")


def packed_lkball_tables(pbt):
    """The packed tensors of every LK-ball table for `pbt`, cached on it."""
    cached = getattr(pbt, "_lkball_tables", None)
    if cached is not None:
        return cached
    db = pbt.db
    nt, A = pbt.n_types, pbt.max_n_atoms
    n_tiles = (A - 1) // TILE_SIZE + 1
    hbs = [hbond_block_params(bt, db) for bt in pbt.active_block_types]
    lkbs = [lkball_block_params(bt, db, hb) for bt, hb in zip(pbt.active_block_types, hbs)]
    abs_ = [all_bonds(bt) for bt in pbt.active_block_types]

    def tiles(key, fill, src, dtype=numpy.int32, extra=()):
        out = numpy.full((nt, n_tiles) + tuple(extra), fill, dtype=dtype)
        for i, d in enumerate(src):
            v = d[key]
            out[i, : v.shape[0]] = v
        return out

    keys3 = (
        "tile_donH_inds",
        "tile_donH_hvy_inds",
        "tile_which_donH_of_donH_hvy",
        "tile_acc_inds",
        "tile_acceptor_hybridization",
        "tile_acceptor_n_attached_H",
    )
    t = {k: tiles(k, -1, hbs, extra=(TILE_SIZE,)) for k in keys3}
    t["tile_n_donH"] = tiles("tile_n_donH", 0, hbs)
    t["tile_n_acc"] = tiles("tile_n_acc", 0, hbs)
    is_h = numpy.zeros((nt, A), dtype=numpy.int32)
    for i, hb in enumerate(hbs):
        is_h[i, : hb["is_hydrogen"].shape[0]] = hb["is_hydrogen"]
    t["is_hydrogen"] = is_h
    t["tile_n_polar_atoms"] = tiles("tile_n_polar_atoms", 0, lkbs)
    t["tile_n_occluder_atoms"] = tiles("tile_n_occluder_atoms", 0, lkbs)
    t["tile_pol_occ_inds"] = tiles("tile_pol_occ_inds", -1, lkbs, extra=(TILE_SIZE,))
    t["tile_lk_ball_params"] = tiles(
        "tile_lk_ball_params", 0, lkbs, dtype=numpy.float32, extra=(TILE_SIZE, N_LKB_PARAMS)
    )
    max_nb = max(b.shape[0] for b, _ in abs_)
    n_all = numpy.full(nt, -1, dtype=numpy.int32)
    allb = numpy.full((nt, max_nb, 3), -1, dtype=numpy.int32)
    ranges = numpy.full((nt, A, 2), -1, dtype=numpy.int32)
    for i, (b, r) in enumerate(abs_):
        n_all[i] = b.shape[0]
        allb[i, : b.shape[0]] = b
        ranges[i, : r.shape[0]] = r
    t["n_all_bonds"], t["all_bonds"], t["atom_all_bond_ranges"] = n_all, allb, ranges
    bs = numpy.full((nt, A, A), MAX_SIG_BOND_SEPARATION, dtype=numpy.int32)
    for i, bt in enumerate(pbt.active_block_types):
        bs[i, : bt.n_atoms, : bt.n_atoms] = bt.path_distance
    t["bond_separation"] = bs
    out = {
        k: torch.tensor(v, device=pbt.device) for k, v in t.items()
    }
    pbt._lkball_tables = out
    return out
