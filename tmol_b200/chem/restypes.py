"""Residue ("block") types and their packed tensor form.

A residue type is a small molecule graph: named atoms with atom types, bonds,
inter-residue connection points ("down" = N, "up" = C for amino acids) and
internal coordinates used to build ideal geometry.  The LJ/LK path needs, per
block type:

* ``path_distance[A, A]``: bonds separating two atoms of the type, capped at
  ``MAX_SIG_BOND_SEPARATION`` (tmol ``chemical/restypes.py:406-418``, which
  runs an unweighted, limited Dijkstra; a capped breadth-first search gives
  the same integers);
* heavy atoms, tiled in groups of 32 (``score/common/stack_condense.py:303``);
* connection atoms and their mutual separations
  (``pose/pose_stack_builder.py:874-921``).

Termini variants follow tmol's ``CarboxyTerminus`` / ``AminoTerminus`` /
``AminoTerminusPro`` patches in ``chemical.yaml`` (the ``variants`` section):
the C terminus drops the ``up`` connection and the carbonyl O and adds O and
OXT (type OOC) bonded to C; the N terminus drops ``down`` and H, retypes N to
Nlys and adds H1, H2, H3 (type Hpol); proline's N terminus keeps N's type and
adds H2, H3.
"""

from collections import deque
import json
import os

import numpy
import torch

MAX_SIG_BOND_SEPARATION = 6
TILE_SIZE = 32

_DATA = os.path.join(os.path.dirname(__file__), "data", "ljlk_chemistry.json")


class ChemicalDatabase:
    """Atom types, residue types and LJ/LK parameters, as read from tmol's
    database files (via the committed extract)."""

    _default = None

    def __init__(self, data):
        self.atom_types = data["atom_types"]
        self.atom_type_index = {a["name"]: i for i, a in enumerate(self.atom_types)}
        self.residues = {r["name"]: r for r in data["residues"]}
        self.ljlk_global_params = data["ljlk_global_params"]
        self.lkball_global_params = data.get("lkball_global_params", {})
        self.hbond_donor_atom_types = data.get("hbond_donor_atom_types", [])
        self.hbond_acceptor_atom_types = data.get("hbond_acceptor_atom_types", [])

    @classmethod
    def get_default(cls):
        if cls._default is None:
            with open(_DATA) as f:
                cls._default = cls(json.load(f))
        return cls._default

    def is_hydrogen_type(self, type_name):
        return self.atom_types[self.atom_type_index[type_name]]["is_hydrogen"]


class ResidueType:
    """One block type.  Attributes mirror the fields of tmol's
    ``RefinedResidueType`` that the LJ/LK term reads."""

    def __init__(
        self,
        name,
        base_name,
        atoms,
        bonds,
        connections,
        icoors,
        chis,
        aliases,
        is_polymer=True,
        is_ligand_fragment=False,
        one_letter_code=None,
    ):
        self.name = name
        self.base_name = base_name
        self.atom_names = [a[0] for a in atoms]
        self.atom_type_names = [a[1] for a in atoms]
        self.atom_index = {n: i for i, n in enumerate(self.atom_names)}
        self.bonds = [tuple(b) for b in bonds]
        self.connections = [tuple(c) for c in connections]
        self.icoors = [list(ic) for ic in icoors]
        self.chis = chis
        self.aliases = dict(aliases)
        self.is_polymer = is_polymer
        self.is_ligand_fragment = is_ligand_fragment
        self.one_letter_code = one_letter_code
        self._derive()

    @property
    def n_atoms(self):
        return len(self.atom_names)

    def _derive(self):
        n = self.n_atoms
        bond_indices = numpy.array(
            [[self.atom_index[a], self.atom_index[b]] for a, b in self.bonds],
            dtype=numpy.int64,
        ).reshape(-1, 2)
        self.bond_indices = bond_indices
        self.path_distance = _capped_path_distance(n, bond_indices, MAX_SIG_BOND_SEPARATION)
        self.connection_atoms = numpy.array(
            [self.atom_index[a] for _, a in self.connections], dtype=numpy.int32
        )
        self.connection_names = [c for c, _ in self.connections]
        ca = self.connection_atoms
        self.conn_at_intrablock_bond_sep = self.path_distance[ca[:, None], ca[None, :]].astype(
            numpy.int32
        ) if len(ca) else numpy.zeros((0, 0), dtype=numpy.int32)

    def conn_index(self, name):
        for i, c in enumerate(self.connection_names):
            if c == name:
                return i
        return -1


def _capped_path_distance(n, bond_indices, cap):
    """Bond count between every atom pair, ``cap`` where unreachable or >= cap."""
    adj = [[] for _ in range(n)]
    for a, b in bond_indices:
        adj[a].append(b)
        adj[b].append(a)
    pd = numpy.full((n, n), cap, dtype=numpy.int32)
    for s in range(n):
        pd[s, s] = 0
        q = deque([s])
        while q:
            u = q.popleft()
            du = pd[s, u]
            if du + 1 >= cap:
                continue
            for v in adj[u]:
                if pd[s, v] > du + 1:
                    pd[s, v] = du + 1
                    q.append(v)
    return pd


def residue_type_from_db(db, name):
    r = db.residues[name]
    return ResidueType(
        name=r["name"],
        base_name=r["base_name"],
        atoms=r["atoms"],
        bonds=r["bonds"],
        connections=r["connections"],
        icoors=r["icoors"],
        chis=r["chis"],
        aliases=[(alt, nm) for nm, alt in r["atom_aliases"]],
        is_polymer=r["is_polymer"],
        one_letter_code=r["one_letter_code"],
    )


def _neighbors(rt, atom):
    out = []
    for a, b in rt.bonds:
        if a == atom:
            out.append(b)
        elif b == atom:
            out.append(a)
    return out


def _mainchain_neighbor(rt, atom, exclude):
    """The heavy-atom neighbour of ``atom`` used as the dihedral reference in
    the termini patches' internal coordinates."""
    db = ChemicalDatabase.get_default()
    nbrs = [
        x
        for x in _neighbors(rt, atom)
        if x not in exclude and not db.is_hydrogen_type(rt.atom_type_names[rt.atom_index[x]])
    ]
    for pref in ("CA", "C", "N"):
        if pref in nbrs:
            return pref
    return nbrs[0]


def cterm_variant(rt):
    """tmol ``CarboxyTerminus``: remove ``up`` and the carbonyl O, add O and OXT."""
    c_atom = dict(rt.connections)["up"]
    o_atom = [
        x
        for x in _neighbors(rt, c_atom)
        if rt.atom_type_names[rt.atom_index[x]] == "OCbb"
    ][0]
    ca = _mainchain_neighbor(rt, c_atom, {o_atom})
    n_ = _mainchain_neighbor(rt, ca, {c_atom})
    atoms = [
        [n, t] for n, t in zip(rt.atom_names, rt.atom_type_names) if n != o_atom
    ] + [["O", "OOC"], ["OXT", "OOC"]]
    bonds = [b for b in rt.bonds if o_atom not in b] + [[c_atom, "OXT"], [c_atom, "O"]]
    conns = [c for c in rt.connections if c[0] != "up"]
    icoors = [ic for ic in rt.icoors if ic[0] not in ("up", o_atom)]
    icoors += [
        ["O", 80.0, 60.0, 1.2, c_atom, ca, n_],
        ["OXT", -180.0, 60.0, 1.2, c_atom, ca, "O"],
    ]
    return ResidueType(
        name=rt.name + ":cterm" if ":" not in rt.name else rt.name + ":cterm",
        base_name=rt.base_name,
        atoms=atoms,
        bonds=bonds,
        connections=conns,
        icoors=icoors,
        chis=rt.chis,
        aliases=list(rt.aliases.items()),
        is_polymer=rt.is_polymer,
        one_letter_code=rt.one_letter_code,
    )


def nterm_variant(rt):
    """tmol ``AminoTerminus`` (``AminoTerminusPro`` for an N bonded to two
    carbons): remove ``down`` and the amide H, add H1..H3 (H2, H3 for Pro)."""
    n_atom = dict(rt.connections)["down"]
    heavy_nbrs = [
        x
        for x in _neighbors(rt, n_atom)
        if not ChemicalDatabase.get_default().is_hydrogen_type(rt.atom_type_names[rt.atom_index[x]])
    ]
    is_pro = len(heavy_nbrs) >= 2
    ca = "CA" if "CA" in heavy_nbrs else heavy_nbrs[0]
    c_ = _mainchain_neighbor(rt, ca, {n_atom})
    conns = [c for c in rt.connections if c[0] != "down"]
    if is_pro:
        atoms = [[n, t] for n, t in zip(rt.atom_names, rt.atom_type_names)] + [
            ["H2", "Hpol"],
            ["H3", "Hpol"],
        ]
        bonds = list(rt.bonds) + [[n_atom, "H2"], [n_atom, "H3"]]
        icoors = [ic for ic in rt.icoors if ic[0] != "down"]
        icoors += [
            ["H2", 120.0, 70.5, 1.0, n_atom, ca, c_],
            ["H3", -120.0, 70.5, 1.0, n_atom, ca, c_],
        ]
        aliases = list(rt.aliases.items()) + [("1H", "H2"), ("2H", "H3")]
    else:
        h_atom = [
            x
            for x in _neighbors(rt, n_atom)
            if ChemicalDatabase.get_default().is_hydrogen_type(rt.atom_type_names[rt.atom_index[x]])
        ][0]
        atoms = [
            [n, ("Nlys" if n == n_atom else t)]
            for n, t in zip(rt.atom_names, rt.atom_type_names)
            if n != h_atom
        ] + [["H1", "Hpol"], ["H2", "Hpol"], ["H3", "Hpol"]]
        bonds = [b for b in rt.bonds if h_atom not in b] + [
            [n_atom, "H1"],
            [n_atom, "H2"],
            [n_atom, "H3"],
        ]
        icoors = [ic for ic in rt.icoors if ic[0] not in ("down", h_atom)]
        icoors += [
            ["H1", 180.0, 70.5, 1.0, n_atom, ca, c_],
            ["H2", 120.0, 70.5, 1.0, n_atom, ca, "H1"],
            ["H3", 120.0, 70.5, 1.0, n_atom, ca, "H2"],
        ]
        aliases = list(rt.aliases.items()) + [("1H", "H1"), ("2H", "H2"), ("3H", "H3")]
    return ResidueType(
        name=rt.name + ":nterm",
        base_name=rt.base_name,
        atoms=atoms,
        bonds=bonds,
        connections=conns,
        icoors=icoors,
        chis=rt.chis,
        aliases=aliases,
        is_polymer=rt.is_polymer,
        one_letter_code=rt.one_letter_code,
    )


class ResidueTypeSet:
    """Residue types with termini variants, keyed by name
    (``ALA``, ``ALA:nterm``, ``ALA:cterm``, ``ALA:nterm:cterm``)."""

    _default = None

    def __init__(self, db, base_names):
        self.db = db
        self.types = {}
        for name in base_names:
            base = residue_type_from_db(db, name)
            nt = nterm_variant(base)
            self.types[base.name] = base
            self.types[nt.name] = nt
            self.types[base.name + ":cterm"] = cterm_variant(base)
            self.types[nt.name + ":cterm"] = cterm_variant(nt)
        self.by_one_letter = {}
        for name in base_names:
            r = db.residues[name]
            if r["one_letter_code"] and r["one_letter_code"] not in self.by_one_letter and ":" not in name and name != "HIS_D":
                self.by_one_letter[r["one_letter_code"]] = name

    @classmethod
    def get_default(cls):
        if cls._default is None:
            db = ChemicalDatabase.get_default()
            cls._default = cls(db, list(db.residues.keys()))
        return cls._default

    def variant_name(self, base, nterm, cterm):
        return base + (":nterm" if nterm else "") + (":cterm" if cterm else "")


class PackedBlockTypes:
    """Block-type tables packed into padded int32 tensors, as tmol's
    ``PackedBlockTypes`` annotated by ``AtomTypeDependentTerm``,
    ``BondDependentTerm`` and ``LJLKEnergyTerm``
    (``score/atom_type_dependent_term.py:84-181``,
    ``score/bond_dependent_term.py:31-89``,
    ``score/ljlk/ljlk_energy_term.py:59-111``)."""

    def __init__(self, db, block_types, device=torch.device("cpu")):
        self.db = db
        self.active_block_types = list(block_types)
        self.device = torch.device(device)
        self.bt_index = {bt.name: i for i, bt in enumerate(self.active_block_types)}
        self.n_types = len(self.active_block_types)
        self.max_n_atoms = max(bt.n_atoms for bt in self.active_block_types)
        self.max_n_conn = max(1, max(len(bt.connections) for bt in self.active_block_types))
        self._pack()

    def _pack(self):
        nt, A, C = self.n_types, self.max_n_atoms, self.max_n_conn
        T = TILE_SIZE
        max_n_tiles = (A - 1) // T + 1
        n_atoms = numpy.zeros(nt, dtype=numpy.int32)
        atom_types = numpy.full((nt, A), -1, dtype=numpy.int32)
        bond_sep = numpy.full((nt, A, A), MAX_SIG_BOND_SEPARATION, dtype=numpy.int32)
        n_conn = numpy.zeros(nt, dtype=numpy.int32)
        conn_atom = numpy.full((nt, C), -1, dtype=numpy.int32)
        conn_sep = numpy.full((nt, C, C), -1, dtype=numpy.int32)
        heavy_in_tile = numpy.full((nt, max_n_tiles * T), -1, dtype=numpy.int32)
        n_heavy_in_tile = numpy.zeros((nt, max_n_tiles), dtype=numpy.int32)
        is_ligand = numpy.zeros(nt, dtype=numpy.int32)
        down_conn = numpy.full(nt, -1, dtype=numpy.int32)
        up_conn = numpy.full(nt, -1, dtype=numpy.int32)
        ljlk_bond_sep = numpy.full((nt, A, A), MAX_SIG_BOND_SEPARATION, dtype=numpy.int32)
        for i, bt in enumerate(self.active_block_types):
            n = bt.n_atoms
            n_atoms[i] = n
            atom_types[i, :n] = [self.db.atom_type_index[t] for t in bt.atom_type_names]
            bond_sep[i, :n, :n] = bt.path_distance
            ljlk_bond_sep[i, :n, :n] = bt.path_distance
            if not bt.is_polymer:
                slab = ljlk_bond_sep[i, :n, :n]
                slab[(slab == 3) | (slab == 4)] = 5
            k = len(bt.connections)
            n_conn[i] = k
            conn_atom[i, :k] = bt.connection_atoms
            conn_sep[i, :k, :k] = bt.conn_at_intrablock_bond_sep
            heavy = [
                j for j, t in enumerate(bt.atom_type_names) if not self.db.is_hydrogen_type(t)
            ]
            tiles, counts = tile_subset_indices(heavy, T)
            heavy_in_tile[i, : len(tiles)] = tiles
            n_heavy_in_tile[i, : len(counts)] = counts
            is_ligand[i] = int(bt.is_ligand_fragment)
            down_conn[i] = bt.conn_index("down")
            up_conn[i] = bt.conn_index("up")

        def _t(x):
            return torch.tensor(x, dtype=torch.int32, device=self.device)

        self.n_atoms = _t(n_atoms)
        self.atom_types = _t(atom_types)
        self.bond_separation = _t(bond_sep)
        self.n_conn = _t(n_conn)
        self.conn_atom = _t(conn_atom)
        self.conn_at_intrablock_bond_sep = _t(conn_sep)
        self.ljlk_heavy_atoms_in_tile = _t(heavy_in_tile)
        self.ljlk_n_heavy_atoms_in_tile = _t(n_heavy_in_tile)
        self.ljlk_bond_separation = _t(ljlk_bond_sep)
        self.ljlk_is_ligand_fragment = _t(is_ligand)
        self.down_conn_inds = _t(down_conn)
        self.up_conn_inds = _t(up_conn)

    def to(self, device):
        return PackedBlockTypes(self.db, self.active_block_types, device)


def tile_subset_indices(indices, tile_size):
    """Group sorted subset indices by ``index // tile_size`` and left-justify
    them inside each tile, as tile-local indices; returns the tiled array
    (``-1`` padded) and the per-tile counts
    (tmol ``score/common/stack_condense.py:303-347``)."""
    indices = numpy.asarray(indices, dtype=numpy.int64)
    if indices.size == 0:
        return numpy.full(tile_size, -1, dtype=numpy.int32), numpy.zeros(1, dtype=numpy.int32)
    n_tiles = int(indices.max()) // tile_size + 1
    out = numpy.full(n_tiles * tile_size, -1, dtype=numpy.int32)
    counts = numpy.zeros(n_tiles, dtype=numpy.int32)
    for ind in indices:
        t = int(ind) // tile_size
        out[t * tile_size + counts[t]] = int(ind) - t * tile_size
        counts[t] += 1
    return out, counts


def default_packed_block_types(device=torch.device("cpu")):
    rts = ResidueTypeSet.get_default()
    return PackedBlockTypes(rts.db, list(rts.types.values()), device)
