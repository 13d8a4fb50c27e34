"""Build PoseStacks: block types from sequences, inter-block bond separation
from the connection graph, and coordinates from internal coordinates.

The connectivity rules follow tmol's ``PoseStackBuilder.from_block_type_names``
(``tmol/pose/pose_stack_builder.py:199-330``):

1. residue i's ``up`` connection bonds to residue i+1's ``down`` within a
   chain; chain termini get the N-/C-terminus variants;
2. the nodes of a per-pose graph are the connection points of all blocks;
   two connection points of one block are joined by an edge weighted with the
   bond count between their atoms, and chemically bonded connection points
   of different blocks by an edge of weight 1 (``:436-599``, ``:1230-1254``);
3. shortest paths over that graph, capped at ``MAX_SIG_BOND_SEPARATION``,
   give ``inter_block_bondsep[p, b1, b2, c1, c2]`` (``:1271-1343``), 6 where
   a connection slot does not exist.

The shortest paths come from a bounded search per connection point rather
than tmol's all-pairs pass over a dense matrix; the integers are the same.
On a CUDA device the search runs on the GPU (``tmol_b200.pose.bondsep``,
one thread per connection point); on the host, a capped Dijkstra in Python.
"""

import heapq
import math

import numpy
import torch

from ..chem.restypes import MAX_SIG_BOND_SEPARATION, ResidueTypeSet, default_packed_block_types
from .pose_stack import PoseStack


class PoseTopology:
    """Host-side description of one pose: block type names per residue and
    inter-block chemical bonds as (block1, conn1, block2, conn2)."""

    def __init__(self, block_type_names, bonds):
        self.block_type_names = list(block_type_names)
        self.bonds = list(bonds)


def topology_from_sequence(seq, rts=None, termini=True):
    """One chain of one-letter codes (or three-letter names, as a list)."""
    rts = rts or ResidueTypeSet.get_default()
    names = []
    n = len(seq)
    for i, code in enumerate(seq):
        base = rts.by_one_letter[code] if len(code) == 1 else code
        names.append(rts.variant_name(base, termini and i == 0, termini and i == n - 1))
    bonds = []
    for i in range(n - 1):
        bonds.append((i, "up", i + 1, "down"))
    return PoseTopology(names, bonds)


def _capped_sssp(adj, src, cap):
    dist = {src: 0}
    heap = [(0, src)]
    while heap:
        d, u = heapq.heappop(heap)
        if d > dist.get(u, cap):
            continue
        for v, w in adj[u]:
            nd = d + w
            if nd < cap and nd < dist.get(v, cap):
                dist[v] = nd
                heapq.heappush(heap, (nd, v))
    return dist


def interblock_bondsep_entries(topo, pbt):
    """Sparse entries (b1, c1, b2, c2, sep) with sep < MAX_SIG_BOND_SEPARATION."""
    cap = MAX_SIG_BOND_SEPARATION
    bts = [pbt.active_block_types[pbt.bt_index[n]] for n in topo.block_type_names]
    node_of = {}
    nodes = []
    for b, bt in enumerate(bts):
        for c in range(len(bt.connections)):
            node_of[(b, c)] = len(nodes)
            nodes.append((b, c))
    adj = [[] for _ in nodes]
    for b, bt in enumerate(bts):
        k = len(bt.connections)
        for c1 in range(k):
            for c2 in range(k):
                if c1 != c2:
                    w = int(bt.conn_at_intrablock_bond_sep[c1, c2])
                    adj[node_of[(b, c1)]].append((node_of[(b, c2)], w))
    for b1, cn1, b2, cn2 in topo.bonds:
        c1 = bts[b1].conn_index(cn1) if isinstance(cn1, str) else cn1
        c2 = bts[b2].conn_index(cn2) if isinstance(cn2, str) else cn2
        if c1 < 0 or c2 < 0:
            continue
        u, v = node_of[(b1, c1)], node_of[(b2, c2)]
        adj[u].append((v, 1))
        adj[v].append((u, 1))
    entries = []
    for u, (b1, c1) in enumerate(nodes):
        for v, d in _capped_sssp(adj, u, cap).items():
            b2, c2 = nodes[v]
            entries.append((b1, c1, b2, c2, d))
    return entries


def build_pose_stack(topologies, coords_list=None, pbt=None, device=torch.device("cpu")):
    """PoseStack from per-pose topologies and (optionally) per-pose
    ``[n_pose_atoms, 3]`` coordinate arrays (zeros otherwise)."""
    pbt = pbt or default_packed_block_types(device)
    if pbt.device != torch.device(device):
        pbt = pbt.to(device)
    P = len(topologies)
    B = max(len(t.block_type_names) for t in topologies)
    C = pbt.max_n_conn
    bt_ind = numpy.full((P, B), -1, dtype=numpy.int32)
    n_atoms_bt = pbt.n_atoms.cpu().numpy()
    offsets = numpy.zeros((P, B), dtype=numpy.int32)
    pose_n_atoms = numpy.zeros(P, dtype=numpy.int64)
    irc = numpy.full((P, B, C, 2), -1, dtype=numpy.int32)
    for p, topo in enumerate(topologies):
        idx = [pbt.bt_index[n] for n in topo.block_type_names]
        nb = len(idx)
        bt_ind[p, :nb] = idx
        na = n_atoms_bt[idx]
        offsets[p, :nb] = numpy.concatenate([[0], numpy.cumsum(na)[:-1]]).astype(numpy.int32)
        pose_n_atoms[p] = int(na.sum())
        for b1, cn1, b2, cn2 in topo.bonds:
            bt1 = pbt.active_block_types[idx[b1]]
            bt2 = pbt.active_block_types[idx[b2]]
            c1 = bt1.conn_index(cn1) if isinstance(cn1, str) else cn1
            c2 = bt2.conn_index(cn2) if isinstance(cn2, str) else cn2
            if c1 < 0 or c2 < 0:
                continue
            irc[p, b1, c1] = (b2, c2)
            irc[p, b2, c2] = (b1, c1)
    # padding blocks after a pose's last block get the pose's atom count as
    # their offset, as tmol's exclusive cumulative sum does
    for p in range(P):
        nb = len(topologies[p].block_type_names)
        offsets[p, nb:] = pose_n_atoms[p]
    max_atoms = int(pose_n_atoms.max())

    if torch.device(device).type == "cuda":
        from .bondsep import bondsep_from_connectivity

        ibb, _ = bondsep_from_connectivity(
            torch.tensor(bt_ind, device=device),
            torch.tensor(irc, device=device),
            pbt.n_conn,
            pbt.conn_at_intrablock_bond_sep,
        )
    else:
        ibb = torch.full((P, B, B, C, C), MAX_SIG_BOND_SEPARATION, dtype=torch.int32, device=device)
        for p, topo in enumerate(topologies):
            ent = interblock_bondsep_entries(topo, pbt)
            if ent:
                e = torch.tensor(ent, dtype=torch.int64, device=device)
                ibb[p, e[:, 0], e[:, 2], e[:, 1], e[:, 3]] = e[:, 4].to(torch.int32)

    coords = torch.zeros((P, max_atoms, 3), dtype=torch.float32)
    if coords_list is not None:
        for p, c in enumerate(coords_list):
            c = torch.as_tensor(c, dtype=torch.float32)
            coords[p, : c.shape[0]] = c
    return PoseStack(
        packed_block_types=pbt,
        coords=coords.to(device),
        block_coord_offset=torch.tensor(offsets, device=device),
        inter_residue_connections=torch.tensor(irc, device=device),
        inter_block_bondsep=ibb,
        block_type_ind=torch.tensor(bt_ind, device=device),
        device=device,
    )


# ---------------------------------------------------------------------------
# Geometry from internal coordinates (natural extension reference frame).
# An internal coordinate (phi, theta, d, parent, grand_parent,
# great_grand_parent) places an atom at distance d from its parent, with bond
# angle (180 - theta) at the parent and dihedral phi about the
# grand_parent -> parent axis, measured from the great_grand_parent.


def _place(a, b, c, d, theta_deg, phi_deg):
    """Vectorised NeRF: positions D with |CD| = d, angle(B, C, D) = 180 - theta,
    dihedral(A, B, C, D) = phi.  a, b, c: [..., 3]; d, theta, phi: scalars or
    arrays broadcastable to a.shape[:-1]."""
    shape = a.shape[:-1]
    d = numpy.broadcast_to(numpy.asarray(d, dtype=numpy.float64), shape)
    theta = numpy.radians(numpy.broadcast_to(numpy.asarray(theta_deg, dtype=numpy.float64), shape))
    phi = numpy.radians(numpy.broadcast_to(numpy.asarray(phi_deg, dtype=numpy.float64), shape))
    bc = c - b
    bc = bc / numpy.linalg.norm(bc, axis=-1, keepdims=True)
    ab = b - a
    n = numpy.cross(ab, bc)
    n = n / numpy.linalg.norm(n, axis=-1, keepdims=True)
    m = numpy.cross(n, bc)
    x = (d * numpy.cos(theta))[..., None]
    y = (d * numpy.sin(theta) * numpy.cos(phi))[..., None]
    z = (d * numpy.sin(theta) * numpy.sin(phi))[..., None]
    return c + x * bc + y * m + z * n


def _icoor_map(bt):
    return {ic[0]: ic for ic in bt.icoors}


def build_residue_coords(bt, n_pos, ca_pos, c_pos, down_pos, up_pos, chis):
    """Place all atoms of ``len(n_pos)`` residues of one block type given the
    backbone N, CA, C positions, the neighbouring C(i-1) ("down") and N(i+1)
    ("up") positions, and per-residue chi angles ``chis[k, n_chi]``.

    Atoms are placed in dependency order from their internal coordinates; a
    chi's fourth atom takes the sampled chi as its dihedral."""
    icm = _icoor_map(bt)
    pos = {"N": n_pos, "CA": ca_pos, "C": c_pos}
    nm = dict(bt.connections)
    if "down" in nm:
        pos["down"] = down_pos
    if "up" in nm:
        pos["up"] = up_pos
    chi_phi = {}
    # proline's chis close its ring, so its ideal ring geometry is kept
    ring_closing = bt.base_name == "PRO"
    for k, chi in enumerate([] if ring_closing else bt.chis):
        a, b, c, d = chi["atoms"]
        ic = icm.get(d)
        if ic is None or d in ("N", "CA", "C"):
            continue
        if (ic[4], ic[5], ic[6]) == (c, b, a) and k < chis.shape[1]:
            chi_phi[d] = chis[:, k]
    pending = [ic for ic in bt.icoors if ic[0] not in pos and (ic[0] in bt.atom_index)]
    guard = 0
    while pending:
        guard += 1
        if guard > 200:
            raise RuntimeError(f"unresolvable internal coordinates for {bt.name}")
        rest = []
        for ic in pending:
            name, phi, theta, d, par, gp, ggp = ic
            if par in pos and gp in pos and ggp in pos:
                ph = chi_phi.get(name, numpy.full(n_pos.shape[0], phi))
                pos[name] = _place(pos[ggp], pos[gp], pos[par], d, theta, ph)
            else:
                rest.append(ic)
        if len(rest) == len(pending):
            raise RuntimeError(f"unresolvable internal coordinates for {bt.name}: {rest}")
        pending = rest
    return numpy.stack([pos[a] for a in bt.atom_names], axis=1)


def backbone_geometry(bt):
    """Bond lengths and (180 - angle) values from a block type's icoors:
    (d_N_CA, d_CA_C, d_C_Nnext, theta_CA_C, theta_C_up, theta_N_down)."""
    icm = _icoor_map(bt)
    return (
        icm["CA"][3],
        icm["C"][3],
        icm["up"][3] if "up" in icm else 1.3287,
        icm["C"][2],
        icm["up"][2] if "up" in icm else 63.8,
        icm["down"][2] if "down" in icm else 58.3,
    )


def build_chain_coords(pbt, topologies, phis, psis, omegas, chis):
    """Coordinates for single-chain poses.  ``phis[p][i]`` etc. are degrees;
    ``chis[p][i]`` a length-4 array.  Poses are built in parallel along the
    residue index; side chains are built in parallel per block type."""
    P = len(topologies)
    nres = [len(t.block_type_names) for t in topologies]
    Bmax = max(nres)
    bts = [[pbt.active_block_types[pbt.bt_index[n]] for n in t.block_type_names] for t in topologies]
    N = numpy.zeros((P, Bmax + 1, 3))
    CA = numpy.zeros((P, Bmax + 1, 3))
    C = numpy.zeros((P, Bmax + 1, 3))
    geo = {}

    def g(bt):
        if bt.name not in geo:
            geo[bt.name] = backbone_geometry(bt)
        return geo[bt.name]

    def arr(vals, i):
        return numpy.array([vals[p][i] if i < nres[p] else 180.0 for p in range(P)])

    def geo_arr(i, k):
        return numpy.array([g(bts[p][min(i, nres[p] - 1)])[k] for p in range(P)])

    # first residue: N at origin, CA along x, C in the xy plane
    d_nca, d_cac = geo_arr(0, 0), geo_arr(0, 1)
    th_c = geo_arr(0, 3)
    N[:, 0] = 0.0
    CA[:, 0, 0] = d_nca
    ang = numpy.radians(180.0 - th_c)
    C[:, 0, 0] = d_nca - d_cac * numpy.cos(ang)
    C[:, 0, 1] = d_cac * numpy.sin(ang)
    for i in range(1, Bmax + 1):
        d_cn = geo_arr(i - 1, 2)
        th_up = geo_arr(i - 1, 4)
        N[:, i] = _place(N[:, i - 1], CA[:, i - 1], C[:, i - 1], d_cn, th_up, arr(psis, i - 1))
        d_nca, th_down = geo_arr(i, 0), geo_arr(i, 5)
        CA[:, i] = _place(CA[:, i - 1], C[:, i - 1], N[:, i], d_nca, th_down, arr(omegas, i - 1))
        d_cac, th_c = geo_arr(i, 1), geo_arr(i, 3)
        C[:, i] = _place(C[:, i - 1], N[:, i], CA[:, i], d_cac, th_c, arr(phis, i))
    # "down" of residue 0: a virtual C(-1) placed with the residue's phi
    down0 = _place(C[:, 0], CA[:, 0], N[:, 0], 1.3287, 58.3, 180.0)

    out = [numpy.zeros((sum(b.n_atoms for b in bts[p]), 3)) for p in range(P)]
    groups = {}
    for p in range(P):
        off = 0
        for i, bt in enumerate(bts[p]):
            groups.setdefault(bt.name, []).append((p, i, off))
            off += bt.n_atoms
    for name, items in groups.items():
        bt = pbt.active_block_types[pbt.bt_index[name]]
        ps = numpy.array([it[0] for it in items])
        is_ = numpy.array([it[1] for it in items])
        n_pos = N[ps, is_]
        ca_pos = CA[ps, is_]
        c_pos = C[ps, is_]
        down = numpy.where((is_ > 0)[:, None], C[ps, numpy.maximum(is_ - 1, 0)], down0[ps])
        up = N[ps, is_ + 1]
        ch = numpy.array([numpy.asarray(chis[p][i], dtype=numpy.float64) for p, i in zip(ps, is_)])
        xyz = build_residue_coords(bt, n_pos, ca_pos, c_pos, down, up, ch.reshape(len(items), -1))
        for k, (p, i, off) in enumerate(items):
            out[p][off : off + bt.n_atoms] = xyz[k]
    return out
