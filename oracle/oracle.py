"""ctypes front end of the C oracle (``oracle/ljlk_oracle.c``) and of the
compiled reference op (``oracle/_ref``).

Test infrastructure only: tests, ``__graft_entry__.smoke()`` and the
benchmark's CPU-baseline leg import this module, as the checker.  The
product never does.

Arguments follow the reference op's order (``tmol/score/ljlk/potentials/
compiled.ops.cpp:533-597``): ``coords`` then the 26-item tail that
``tmol_b200.score.ljlk_energy_term.pose_score_args`` returns.
"""

import ctypes
import os
import subprocess

import numpy
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _lib(f64):
    key = "f64" if f64 else "f32"
    if key not in _LIBS:
        path = os.path.join(HERE, f"liboracle_ljlk_{key}.so")
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        lib.oracle_ljlk_rotamer_count.restype = ctypes.c_int64
        _LIBS[key] = lib
    return _LIBS[key]


def _inputs_struct(real_t):
    P = ctypes.POINTER
    i32p = P(ctypes.c_int32)
    rp = P(real_t)

    class Inputs(ctypes.Structure):
        _fields_ = [
            ("coords", rp),
            ("rot_coord_offset", i32p),
            ("first_rot_block_type", i32p),
            ("block_ind_for_rot", i32p),
            ("pose_ind_for_rot", i32p),
            ("block_type_ind_for_rot", i32p),
            ("rot_offset_for_block", i32p),
            ("min_bondsep", i32p),
            ("inter_block_bondsep", i32p),
            ("bt_n_atoms", i32p),
            ("bt_n_heavy_in_tile", i32p),
            ("bt_heavy_in_tile", i32p),
            ("bt_atom_types", i32p),
            ("bt_n_conn", i32p),
            ("bt_conn_atom", i32p),
            ("bt_path_distance", i32p),
            ("bt_is_ligand", i32p),
            ("type_params", rp),
            ("global_params", rp),
            ("max_dis", real_t),
            ("n_atoms", ctypes.c_int),
            ("n_rots", ctypes.c_int),
            ("P", ctypes.c_int),
            ("B", ctypes.c_int),
            ("nbt", ctypes.c_int),
            ("A", ctypes.c_int),
            ("C", ctypes.c_int),
            ("ntiles", ctypes.c_int),
            ("T", ctypes.c_int),
            ("n_rots_for_block", i32p),
            ("term", ctypes.c_int),
            ("bt_charge", rp),
            ("bt_pd_inter", i32p),
            ("elec_D", ctypes.c_float),
            ("elec_D0", ctypes.c_float),
            ("elec_S", ctypes.c_float),
            ("elec_min_dis", ctypes.c_float),
            ("elec_max_dis", ctypes.c_float),
        ]

    return Inputs


class OracleCall:
    """Holds contiguous numpy copies of one op call's inputs and the ctypes
    struct pointing at them.  ``term="elec"`` takes the elec op's argument
    list (``tmol/score/elec/potentials/compiled.ops.cpp:28-59``) instead of
    the LJ/LK op's; energies then come back as [1, ...]."""

    def __init__(self, coords, args, f64=False, term="ljlk", lkb_water_args=None):
        self.f64 = f64
        self.term = term
        if term == "lkball":
            # LK-ball: the score op's arguments (tmol_b200.score.lkball_energy_term.score_args)
            # for the shared tables; the water-generation ones for the rest
            (irc, min_bondsep, ibb, bt_n_atoms, bt_n_conn, bt_conn_atom, t_npol, t_nocc, t_polocc, t_params,
             bond_sep, lkb_global, max_dis) = args[12:25]
            nbt = bt_n_atoms.shape[0]
            lkb_tables = (irc, t_npol, t_nocc, t_polocc, t_params, lkb_global)
            args = list(args[:12]) + [
                min_bondsep, ibb, bt_n_atoms, None, None, None, bt_n_conn, bt_conn_atom, bond_sep,
                torch.zeros(nbt, dtype=torch.int32), None, None, max_dis,
            ]
            lkb_A = bond_sep.shape[1]
        if term == "elec":
            (min_bondsep, ibb, bt_n_atoms, bt_charge, bt_n_conn, bt_conn_atom, inter_rpd, intra_rpd,
             bt_is_ligand, elec_global, max_dis) = args[12:23]
            args = list(args[:12]) + [
                min_bondsep, ibb, bt_n_atoms, None, None, None, bt_n_conn, bt_conn_atom, intra_rpd,
                bt_is_ligand, None, None, max_dis,
            ]
        self.np_real = numpy.float64 if f64 else numpy.float32
        real_t = ctypes.c_double if f64 else ctypes.c_float
        self.real_t = real_t
        (
            rot_coord_offset,
            _pose_ind_for_atom,
            _first_rot_for_block,
            first_rot_block_type,
            block_ind_for_rot,
            pose_ind_for_rot,
            block_type_ind_for_rot,
            _n_rots_for_pose,
            _rot_offset_for_pose,
            n_rots_for_block,
            rot_offset_for_block,
            _max_n_rots_per_pose,
            min_bondsep,
            inter_block_bondsep,
            bt_n_atoms,
            bt_n_heavy_in_tile,
            bt_heavy_in_tile,
            bt_atom_types,
            bt_n_conn,
            bt_conn_atom,
            bt_path_distance,
            bt_is_ligand,
            type_params,
            global_params,
            max_dis,
        ) = args[:25]
        self.keep = []

        def i32(t):
            if t is None:
                return None
            a = numpy.ascontiguousarray(t.detach().cpu().numpy().astype(numpy.int32))
            self.keep.append(a)
            return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))

        def rl(t):
            if t is None:
                return None
            a = numpy.ascontiguousarray(t.detach().cpu().numpy().astype(self.np_real))
            self.keep.append(a)
            return a.ctypes.data_as(ctypes.POINTER(real_t))

        Inputs = _inputs_struct(real_t)
        s = Inputs()
        s.coords = rl(coords.reshape(-1, 3))
        s.rot_coord_offset = i32(rot_coord_offset)
        s.first_rot_block_type = i32(first_rot_block_type)
        s.block_ind_for_rot = i32(block_ind_for_rot)
        s.pose_ind_for_rot = i32(pose_ind_for_rot)
        s.block_type_ind_for_rot = i32(block_type_ind_for_rot)
        s.rot_offset_for_block = i32(rot_offset_for_block)
        s.min_bondsep = i32(min_bondsep)
        s.inter_block_bondsep = i32(inter_block_bondsep)
        s.bt_n_atoms = i32(bt_n_atoms)
        s.bt_n_heavy_in_tile = i32(bt_n_heavy_in_tile)
        s.bt_heavy_in_tile = i32(bt_heavy_in_tile)
        s.bt_atom_types = i32(bt_atom_types)
        s.bt_n_conn = i32(bt_n_conn)
        s.bt_conn_atom = i32(bt_conn_atom)
        s.bt_path_distance = i32(bt_path_distance)
        s.bt_is_ligand = i32(bt_is_ligand)
        s.n_rots_for_block = i32(n_rots_for_block)
        s.type_params = rl(type_params)
        s.global_params = rl(global_params.reshape(-1) if global_params is not None else None)
        s.max_dis = float(max_dis)
        if term == "elec":
            g = elec_global.detach().cpu().reshape(-1).to(torch.float32).numpy()
            s.term = 1
            s.bt_charge = rl(bt_charge)
            s.bt_pd_inter = i32(inter_rpd)
            s.elec_D, s.elec_D0, s.elec_S, s.elec_min_dis, s.elec_max_dis = (float(v) for v in g)
        s.n_atoms = coords.reshape(-1, 3).shape[0]
        s.n_rots = rot_coord_offset.shape[0]
        s.P = first_rot_block_type.shape[0]
        s.B = first_rot_block_type.shape[1]
        s.nbt = bt_n_atoms.shape[0]
        if term == "lkball":
            s.A = lkb_A
        else:
            s.A = (bt_charge if term == "elec" else bt_atom_types).shape[1]
        s.C = bt_conn_atom.shape[1]
        s.ntiles = 0 if term in ("elec", "lkball") else bt_n_heavy_in_tile.shape[1]
        s.T = 0 if term in ("elec", "lkball") else type_params.shape[0]
        self.s = s
        self.P, self.B, self.N = s.P, s.B, s.n_atoms
        if term == "lkball":
            self.k = self._lkb_struct(lkb_tables, lkb_water_args, i32, rl, real_t)

    def _lkb_struct(self, tables, wg, i32, rl, real_t):
        irc, t_npol, t_nocc, t_polocc, t_params, lkb_global = tables
        (_irc, _nat, _nconn, _catom, _n_all, all_bonds, ranges, t_ndonH, t_nacc, t_donH, t_donH_hvy, t_which,
         t_acc, t_hyb, t_nH, is_h, wg_gp, tors_sp2, tors_sp3, tors_ring) = wg[12:32]
        P = ctypes.POINTER
        i32p = P(ctypes.c_int32)
        rp = P(real_t)

        class LKB(ctypes.Structure):
            _fields_ = (
                [("irc", i32p), ("all_bonds", i32p), ("bond_ranges", i32p), ("NB", ctypes.c_int), ("NT", ctypes.c_int)]
                + [(n, i32p) for n in ("tile_n_donH", "tile_n_acc", "tile_donH_inds", "tile_donH_hvy",
                                       "tile_which_donH", "tile_acc_inds", "tile_acc_hyb", "tile_acc_nH",
                                       "is_hydrogen", "tile_n_polar", "tile_n_occ", "tile_pol_occ")]
                + [("tile_params", rp)]
                + [(n, real_t) for n in ("water_dist", "ang_sp2", "ang_sp3", "ang_ring")]
                + [("tors_sp2", rp), ("tors_sp3", rp), ("tors_ring", rp)]
                + [(n, ctypes.c_int) for n in ("n_sp2", "n_sp3", "n_ring")]
                + [(n, real_t) for n in ("hbond_dis", "hbond_OH_donor_dis", "hbond_hdis", "max_dis")]
            )

        k = LKB()
        k.irc = i32(irc)
        k.all_bonds = i32(all_bonds)
        k.bond_ranges = i32(ranges)
        k.NB = all_bonds.shape[1]
        k.NT = t_npol.shape[1]
        for name, t in (("tile_n_donH", t_ndonH), ("tile_n_acc", t_nacc), ("tile_donH_inds", t_donH),
                        ("tile_donH_hvy", t_donH_hvy), ("tile_which_donH", t_which), ("tile_acc_inds", t_acc),
                        ("tile_acc_hyb", t_hyb), ("tile_acc_nH", t_nH), ("is_hydrogen", is_h),
                        ("tile_n_polar", t_npol), ("tile_n_occ", t_nocc), ("tile_pol_occ", t_polocc)):
            setattr(k, name, i32(t))
        k.tile_params = rl(t_params)
        g = wg_gp.detach().cpu().reshape(-1).to(torch.float64).numpy()
        k.water_dist, k.ang_sp2, k.ang_sp3, k.ang_ring = (float(v) for v in g[:4])
        k.tors_sp2, k.tors_sp3, k.tors_ring = rl(tors_sp2), rl(tors_sp3), rl(tors_ring)
        k.n_sp2, k.n_sp3, k.n_ring = tors_sp2.numel(), tors_sp3.numel(), tors_ring.numel()
        sg = lkb_global.detach().cpu().reshape(-1).to(torch.float64).numpy()
        k.hbond_dis, k.hbond_OH_donor_dis, k.hbond_hdis, k.max_dis = float(sg[0]), float(sg[1]), float(sg[2]), float(sg[4])
        return k

    def lkb_waters(self):
        """gen_pose_waters: [N, 4, 3] (NaN where no water)."""
        W = numpy.empty((self.N, 4, 3), dtype=self.np_real)
        rc = _lib(self.f64).oracle_lkb_waters(ctypes.byref(self.s), ctypes.byref(self.k), self._ptr(W))
        assert rc == 0
        return W

    def lkb_scores(self, W, weights=None):
        """(E [4, P], d(sum weights * E)/dcoords [N, 3] or None, neighbours)."""
        E = numpy.zeros((4, self.P), dtype=self.np_real)
        nbr = numpy.zeros((self.P, self.B, self.B), dtype=numpy.int32)
        W = numpy.ascontiguousarray(W, dtype=self.np_real)
        dx = None
        wp = ctypes.c_void_p(0)
        if weights is not None:
            w = numpy.ascontiguousarray(numpy.asarray(weights, dtype=self.np_real).reshape(4, self.P))
            self.keep.append(w)
            wp = self._ptr(w)
            dx = numpy.zeros((self.N, 3), dtype=self.np_real)
        rc = _lib(self.f64).oracle_lkb_pose_scores(
            ctypes.byref(self.s), ctypes.byref(self.k), self._ptr(W), self._ptr(E), wp,
            self._ptr(dx) if dx is not None else ctypes.c_void_p(0), self._ptr(nbr),
        )
        assert rc == 0
        return E, dx, nbr

    def lkb_rotamer_scores(self, W, dTdV=None):
        """lk_ball_rotamer_score on a rotamer set: (E [4, n], indices [3, n]
        (pose, rot1, rot2), block neighbours [P, B, B], and with dTdV
        [4, n] the gradient of sum dTdV * E through the waters [N, 3])."""
        lib = _lib(self.f64)
        nbr = numpy.zeros((self.P, self.B, self.B), dtype=numpy.int32)
        n = lib.oracle_ljlk_rotamer_count(ctypes.byref(self.s), self._ptr(nbr))
        assert n >= 0
        E = numpy.zeros((4, n), dtype=self.np_real)
        idx = numpy.zeros((3, n), dtype=numpy.int32)
        W = numpy.ascontiguousarray(W, dtype=self.np_real)
        dx = None
        wp = ctypes.c_void_p(0)
        if dTdV is not None:
            w = numpy.ascontiguousarray(numpy.asarray(dTdV, dtype=self.np_real).reshape(4, n))
            self.keep.append(w)
            wp = self._ptr(w)
            dx = numpy.zeros((self.N, 3), dtype=self.np_real)
        rc = lib.oracle_lkb_rotamer_scores(
            ctypes.byref(self.s), ctypes.byref(self.k), self._ptr(W), self._ptr(nbr), ctypes.c_int64(n),
            self._ptr(E), self._ptr(idx), wp, self._ptr(dx) if dx is not None else ctypes.c_void_p(0),
        )
        assert rc == 0
        return E, idx, nbr, dx

    def _ptr(self, a):
        return a.ctypes.data_as(ctypes.c_void_p)

    def pose_scores(self, block_pair=False, require_gradient=False):
        """Returns (E [3, P] or [3, P, B, B], dV [3, N, 3] or None, nbr [P, B, B])."""
        lib = _lib(self.f64)
        P, B, N = self.P, self.B, self.N
        E = numpy.zeros((3, P, B, B) if block_pair else (3, P), dtype=self.np_real)
        nbr = numpy.zeros((P, B, B), dtype=numpy.int32)
        dV = numpy.zeros((3, N, 3), dtype=self.np_real) if (require_gradient and not block_pair) else None
        rc = lib.oracle_ljlk_pose_scores(
            ctypes.byref(self.s),
            ctypes.c_int(int(block_pair)),
            self._ptr(E),
            self._ptr(dV) if dV is not None else ctypes.c_void_p(0),
            self._ptr(nbr),
        )
        assert rc == 0
        return E, dV, nbr

    def backward(self, nbr, dTdV, per_pose_weights):
        lib = _lib(self.f64)
        w = numpy.ascontiguousarray(numpy.asarray(dTdV, dtype=self.np_real))
        nb = numpy.ascontiguousarray(nbr.astype(numpy.int32))
        out = numpy.zeros((self.N, 3), dtype=self.np_real)
        rc = lib.oracle_ljlk_backward(
            ctypes.byref(self.s), self._ptr(nb), self._ptr(w), ctypes.c_int(int(per_pose_weights)), self._ptr(out)
        )
        assert rc == 0
        return out

    def rotamer_scores(self):
        """The rotamer-score op: (E [3, n], indices [3, n] (pose, rot1, rot2),
        block neighbours [P, B, B])."""
        lib = _lib(self.f64)
        nbr = numpy.zeros((self.P, self.B, self.B), dtype=numpy.int32)
        n = lib.oracle_ljlk_rotamer_count(ctypes.byref(self.s), self._ptr(nbr))
        assert n >= 0
        E = numpy.zeros((3, n), dtype=self.np_real)
        idx = numpy.zeros((3, n), dtype=numpy.int32)
        rc = lib.oracle_ljlk_rotamer_scores(ctypes.byref(self.s), self._ptr(nbr), ctypes.c_int64(n),
                                            self._ptr(E), self._ptr(idx))
        assert rc == 0
        return E, idx, nbr

    def rotamer_backward(self, nbr, dTdV):
        lib = _lib(self.f64)
        w = numpy.ascontiguousarray(numpy.asarray(dTdV, dtype=self.np_real))
        nb = numpy.ascontiguousarray(nbr.astype(numpy.int32))
        out = numpy.zeros((self.N, 3), dtype=self.np_real)
        rc = lib.oracle_ljlk_rotamer_backward(ctypes.byref(self.s), self._ptr(nb), ctypes.c_int64(w.shape[1]),
                                              self._ptr(w), self._ptr(out))
        assert rc == 0
        return out

    def count_pairs(self, nbr):
        lib = _lib(self.f64)
        nb = numpy.ascontiguousarray(nbr.astype(numpy.int32))
        ap = ctypes.c_int64()
        hp = ctypes.c_int64()
        lib.oracle_count_pairs(ctypes.byref(self.s), self._ptr(nb), ctypes.byref(ap), ctypes.byref(hp))
        return ap.value, hp.value


def potential(name, dist, sep, tp_i, tp_j, gp, f64=True):
    """Scalar potentials: name in {lj_V, lj_V_dV, lk_V, lk_V_dV}."""
    lib = _lib(f64)
    npr = numpy.float64 if f64 else numpy.float32
    real_t = ctypes.c_double if f64 else ctypes.c_float
    ti = numpy.ascontiguousarray(numpy.asarray(tp_i, dtype=npr))
    tj = numpy.ascontiguousarray(numpy.asarray(tp_j, dtype=npr))
    g = numpy.ascontiguousarray(numpy.asarray(gp, dtype=npr).reshape(-1))
    vp = ctypes.c_void_p
    if name == "lk_V":
        f = lib.oracle_lk_score_V
        f.restype = real_t
        return float(
            f(real_t(dist), real_t(sep), vp(ti.ctypes.data), vp(tj.ctypes.data), vp(g.ctypes.data))
        )
    n_out = {"lj_V": 2, "lj_V_dV": 4, "lk_V_dV": 2}[name]
    out = numpy.zeros(n_out, dtype=npr)
    f = {
        "lj_V": lib.oracle_lj_score_V,
        "lj_V_dV": lib.oracle_lj_score_V_dV,
        "lk_V_dV": lib.oracle_lk_score_V_dV,
    }[name]
    f(real_t(dist), real_t(sep), vp(ti.ctypes.data), vp(tj.ctypes.data), vp(g.ctypes.data), vp(out.ctypes.data))
    return out


# ---------------------------------------------------------------------------
# The compiled reference op (built by oracle/build_ref.py into oracle/_ref).

REF_LIB = os.path.join(HERE, "_ref", "tmol_ljlk_ref.so")
_ref_loaded = False


def reference_available():
    return os.path.exists(REF_LIB)


def load_reference():
    global _ref_loaded
    if not _ref_loaded:
        torch.ops.load_library(REF_LIB)
        _ref_loaded = True
    return torch.ops.tmol_ljlk.ljlk_pose_scores


def reference_rotamer_scores(coords, args, require_gradient=True):
    """Runs the reference CPU rotamer op: returns (scores [3, n], coords
    tensor (with grad if requested), indices [3, n])."""
    load_reference()
    op = torch.ops.tmol_ljlk.ljlk_rotamer_scores
    cpu_args = [a.cpu() if isinstance(a, torch.Tensor) else a for a in args]
    c = coords.detach().cpu().reshape(-1, 3).clone()
    if require_gradient:
        c.requires_grad_(True)
    E, idx = op(c, *cpu_args)
    return E, c, idx


ELEC_REF_LIB = os.path.join(HERE, "_ref", "elec", "tmol_elec_ref.so")
_elec_loaded = False


def reference_elec_available():
    return os.path.exists(ELEC_REF_LIB)


def reference_elec_pose_scores(coords, args, require_gradient=True):
    """Runs the reference CPU elec op: returns (E [1, P] or [1, P, B, B],
    coords tensor (with grad if requested), block neighbours)."""
    global _elec_loaded
    if not _elec_loaded:
        torch.ops.load_library(ELEC_REF_LIB)
        _elec_loaded = True
    op = torch.ops.tmol_elec.elec_pose_scores
    cpu_args = [a.cpu() if isinstance(a, torch.Tensor) else a for a in args]
    c = coords.detach().cpu().reshape(-1, 3).clone()
    if require_gradient:
        c.requires_grad_(True)
    E, nbr = op(c, *cpu_args)
    return E, c, nbr


def reference_elec_rotamer_scores(coords, args, require_gradient=True):
    """Runs the reference CPU elec rotamer op: returns (scores [1, n], coords
    tensor (with grad if requested), indices [3, n])."""
    global _elec_loaded
    if not _elec_loaded:
        torch.ops.load_library(ELEC_REF_LIB)
        _elec_loaded = True
    op = torch.ops.tmol_elec.elec_rotamer_scores
    cpu_args = [a.cpu() if isinstance(a, torch.Tensor) else a for a in args]
    c = coords.detach().cpu().reshape(-1, 3).clone()
    if require_gradient:
        c.requires_grad_(True)
    E, idx = op(c, *cpu_args)
    return E, c, idx


LKBALL_REF_LIB = os.path.join(HERE, "_ref", "lk_ball", "tmol_lk_ball_ref.so")


def reference_lkball_available():
    return os.path.exists(LKBALL_REF_LIB)


def reference_lkball(coords, water_args, score_args, require_gradient=True):
    """The reference CPU LK-ball ops: waters from gen_pose_waters, then
    lk_ball_pose_score on them; returns (E [4, P], waters, coords tensor with
    grad of sum(E) when requested, block neighbours)."""
    if "lkball_ref" not in _LIBS:
        torch.ops.load_library(LKBALL_REF_LIB)
        _LIBS["lkball_ref"] = True
    ops = torch.ops.tmol_lk_ball
    c = coords.detach().cpu().reshape(-1, 3).clone()
    if require_gradient:
        c.requires_grad_(True)
    wa = [a.cpu() if isinstance(a, torch.Tensor) else a for a in water_args]
    sa = [a.cpu() if isinstance(a, torch.Tensor) else a for a in score_args]
    W = ops.gen_pose_waters(c, *wa)
    sa[-2] = W
    E, nbr = ops.lk_ball_pose_score(c, *sa)
    return E, W, c, nbr


def reference_lkball_rotamers(coords, water_args, score_args):
    """The reference CPU LK-ball rotamer op on a rotamer set: waters from
    gen_pose_waters on the rotamers' coordinates, then lk_ball_rotamer_score;
    returns (E [4, n], dispatch indices [3, n], waters, coords tensor that
    requires grad)."""
    if "lkball_ref" not in _LIBS:
        torch.ops.load_library(LKBALL_REF_LIB)
        _LIBS["lkball_ref"] = True
    ops = torch.ops.tmol_lk_ball
    c = coords.detach().cpu().reshape(-1, 3).clone().requires_grad_(True)
    wa = [a.cpu() if isinstance(a, torch.Tensor) else a for a in water_args]
    sa = [a.cpu() if isinstance(a, torch.Tensor) else a for a in score_args]
    W = ops.gen_pose_waters(c, *wa)
    sa[-2] = W
    E, idx = ops.lk_ball_rotamer_score(c, *sa)
    return E, idx, W, c


def reference_pose_scores(coords, args, require_gradient=True):
    """Runs the reference CPU op: returns (E, dE/dx or None, nbr)."""
    op = load_reference()
    cpu_args = [a.cpu() if isinstance(a, torch.Tensor) else a for a in args]
    c = coords.detach().cpu().reshape(-1, 3).clone()
    if require_gradient:
        c.requires_grad_(True)
    E, nbr = op(c, *cpu_args)
    return E, c, nbr


# ---------------------------------------------------------------------------
# PoseStack bond separation (oracle/apsp_oracle.c) and the reference's
# stacked all-pairs-shortest-paths op (oracle/_ref/apsp)


def _apsp_lib():
    if "apsp" not in _LIBS:
        path = os.path.join(HERE, "liboracle_apsp.so")
        if not os.path.exists(path):
            build()
        _LIBS["apsp"] = ctypes.CDLL(path)
    return _LIBS["apsp"]


def _np_i32(a):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    return numpy.ascontiguousarray(numpy.asarray(a, dtype=numpy.int32))


def apsp_stacked(weights, cutoff=-1):
    """tmol's stacked_apsp on a copy of int32 weights [G, N, N] (-1 = no
    edge): cutoff -1 = Floyd-Warshall, else distances capped at the cutoff."""
    w = _np_i32(weights).copy()
    G, N = w.shape[0], w.shape[1]
    rc = _apsp_lib().oracle_apsp_stacked(
        w.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(G), ctypes.c_int(N), ctypes.c_int(int(cutoff))
    )
    assert rc == 0
    return w


def pose_bondsep(block_type_ind, inter_residue_connections, bt_n_conn, bt_conn_sep):
    """inter_block_bondsep [P, B, B, C, C] and min_bondsep [P, B, B] of a
    PoseStack from its connectivity, as tmol's builder computes them."""
    bti = _np_i32(block_type_ind)
    irc = _np_i32(inter_residue_connections)
    nc = _np_i32(bt_n_conn)
    cs = _np_i32(bt_conn_sep)
    P, B = bti.shape
    C = cs.shape[1]
    ibb = numpy.empty((P, B, B, C, C), dtype=numpy.int32)
    mb = numpy.empty((P, B, B), dtype=numpy.int32)
    rc = _apsp_lib().oracle_pose_bondsep(
        ctypes.c_int(P), ctypes.c_int(B), ctypes.c_int(C), ctypes.c_int(nc.shape[0]),
        bti.ctypes.data_as(ctypes.c_void_p), irc.ctypes.data_as(ctypes.c_void_p),
        nc.ctypes.data_as(ctypes.c_void_p), cs.ctypes.data_as(ctypes.c_void_p),
        ibb.ctypes.data_as(ctypes.c_void_p), mb.ctypes.data_as(ctypes.c_void_p),
    )
    assert rc == 0, rc
    return ibb, mb


APSP_REF_LIB = os.path.join(HERE, "_ref", "apsp", "tmol_apsp_ref.so")


def reference_apsp_available():
    return os.path.exists(APSP_REF_LIB)


def reference_apsp(weights, cutoff=-1):
    """The reference's CPU stacked_apsp op on a copy of weights."""
    if "apsp_ref" not in _LIBS:
        torch.ops.load_library(APSP_REF_LIB)
        _LIBS["apsp_ref"] = True
    w = torch.as_tensor(_np_i32(weights)).clone()
    torch.ops.tmol_apsp.apsp_op(w, int(cutoff))
    return w.numpy()
