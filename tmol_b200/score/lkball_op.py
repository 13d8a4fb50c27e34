"""The LK-ball ops on B200, with tmol's argument lists and outputs.

``gen_pose_waters(coords, <32 static arguments>)`` takes exactly the
arguments of ``torch.ops.tmol_lk_ball.gen_pose_waters``
(``tmol/score/lk_ball/potentials/compiled.ops.cpp:25-360``) and returns the
waters ``[n_atoms, 4, 3]`` (NaN in unused slots); gradients flow back to
``coords`` through the water-building adjoint.

``lk_ball_rotamer_score(coords, <25 static arguments>, water_coords, True)``
is ``torch.ops.tmol_lk_ball.lk_ball_rotamer_score`` (``compiled.ops.cpp:604-842,
909-976``) on a rotamer set, whose waters come from ``gen_pose_waters`` on the
rotamers' coordinates: ``(scores [4, n], indices [3, n])``.

``lk_ball_pose_score(coords, <25 static arguments>, water_coords,
output_block_pair_energies)`` is ``torch.ops.tmol_lk_ball.lk_ball_pose_score``
(``compiled.ops.cpp:361-603, 843-907``): ``(scores, block_neighbors)``,
scores ``[4, P]`` (lk_ball_iso, lk_ball, lk_bridge, lk_bridge_uncpl) or
``[4, P, B, B]``; gradients flow to ``coords`` and ``water_coords``.

Each op builds its plan (include/tmol_b200_lkball.h) once per set of static
tensors and caches it as the LJ/LK op's is.  All tensors must be on one CUDA
device; there is no CPU path.
"""

import ctypes

import torch

from .. import native
from .ljlk_op import LJLKPlan, get_plan

N_WATER_STATIC = 32  # gen_pose_waters' arguments after coords
N_SCORE_STATIC = 27  # lk_ball_pose_score's after coords (water_coords and the output-mode flag included)
MAX_N_WATER = 4


class LKBallPlan(LJLKPlan):
    """Owns one ``tmol_b200_lkball_plan``.  ``water_static`` (gen_pose_waters'
    32 arguments after coords) enables water generation, ``score_static``
    (lk_ball_pose_score's first 25 arguments after coords) scoring; either
    may be None."""

    N_TERMS = 4  # lk_ball_iso, lk_ball, lk_bridge, lk_bridge_uncpl
    ABI = "tmol_b200_lkball"
    # the score op's own autograd function uses the speculative pair below
    # (LJLKPlan's _ScoreFn is not used for LK-ball)
    SPECULATIVE = False
    NAME = "LK-ball"

    def __init__(self, coords_like, water_static=None, score_static=None, launch=None, rotamers=False,
                 connectivity=None):
        """With ``connectivity`` (a PoseStack, or the tuple (block_type_ind,
        inter_residue_connections, bt_n_conn, bt_conn_sep)) the count-pair
        tables come from it and the scoring arguments' min_bondsep /
        inter_block_bondsep may be None."""
        if water_static is None and score_static is None:
            raise ValueError("an LK-ball plan needs the water-generation or the scoring arguments")
        device = self._set_device(coords_like)
        s = native.LKBallInputs()
        keep = []

        def put(name, t, real=False):
            if not isinstance(t, torch.Tensor):
                raise TypeError(f"{name} must be a tensor")
            if t.device != device:
                raise RuntimeError(f"{name} is on {t.device}, coordinates on {device}")
            t = t.to(self.dtype if real else torch.int32).contiguous()
            keep.append(t)
            setattr(s, name, t.data_ptr())
            return t

        common = water_static[:12] if water_static is not None else score_static[:12]
        names = ("rot_coord_offset", "pose_ind_for_atom", "first_rot_for_block", "first_rot_block_type",
                 "block_ind_for_rot", "pose_ind_for_rot", "block_type_ind_for_rot", "n_rots_for_pose",
                 "rot_offset_for_pose", "n_rots_for_block", "rot_offset_for_block")
        for name, t in zip(names, common[:11]):
            put(name, t)
        s.max_n_rots_per_pose = int(common[11])
        P, B = common[2].shape
        bt_sizes = (water_static if water_static is not None else score_static)[13 if water_static is not None else 15]
        self.block_sizes = (common[3], bt_sizes)  # for the autotuner's signature
        if water_static is not None:
            if len(water_static) != N_WATER_STATIC:
                raise TypeError(f"gen_pose_waters takes coords + {N_WATER_STATIC} arguments")
            (irc, bt_n_atoms, bt_n_conn, bt_conn_atom, bt_n_all_bonds, all_bonds, ranges, t_ndonH, t_nacc,
             t_donH, t_donH_hvy, t_which, t_acc, t_hyb, t_nH, is_h, wg_gp, tors_sp2, tors_sp3,
             tors_ring) = water_static[12:]
            for name, t in (("inter_residue_connections", irc), ("bt_n_all_bonds", bt_n_all_bonds),
                            ("bt_all_bonds", all_bonds), ("bt_atom_all_bond_ranges", ranges),
                            ("bt_tile_n_donH", t_ndonH), ("bt_tile_n_acc", t_nacc), ("bt_tile_donH_inds", t_donH),
                            ("bt_tile_donH_hvy_inds", t_donH_hvy), ("bt_tile_which_donH_for_hvy", t_which),
                            ("bt_tile_acc_inds", t_acc), ("bt_tile_hybridization", t_hyb),
                            ("bt_tile_acc_n_attached_H", t_nH), ("bt_atom_is_hydrogen", is_h)):
                put(name, t)
            if wg_gp.numel() != 4:
                raise ValueError("the water-generation global parameters must hold 4 values")
            put("water_gen_global_params", wg_gp, real=True)
            for name, t in (("sp2", tors_sp2), ("sp3", tors_sp3), ("ring", tors_ring)):
                if t.numel():
                    put(f"{name}_water_tors", t.reshape(-1), real=True)
                setattr(s, f"n_{name}_tors", t.numel())
            s.max_n_all_bonds = all_bonds.shape[1]
            s.max_n_tiles = t_ndonH.shape[1]
            A = is_h.shape[1]
        if score_static is not None:
            if len(score_static) != N_SCORE_STATIC - 2:
                raise TypeError(f"lk_ball_pose_score takes coords + {N_SCORE_STATIC} arguments")
            (irc, min_bondsep, ibb, bt_n_atoms, bt_n_conn, bt_conn_atom, t_npol, t_nocc, t_polocc, t_params,
             path_distance, gp, max_dis) = score_static[12:]
            for name, t in (("inter_residue_connections", irc), ("min_bondsep", min_bondsep),
                            ("inter_block_bondsep", ibb), ("bt_tile_n_polar_atoms", t_npol),
                            ("bt_tile_n_occluder_atoms", t_nocc), ("bt_tile_pol_occ_inds", t_polocc),
                            ("bt_path_distance", path_distance)):
                if t is None and connectivity is not None and name in ("min_bondsep", "inter_block_bondsep"):
                    continue
                put(name, t)
            C = bt_conn_atom.shape[1]
            if (ibb is not None and tuple(ibb.shape) != (P, B, B, C, C)) or (
                min_bondsep is not None and tuple(min_bondsep.shape) != (P, B, B)
            ):
                raise ValueError("bond separation tensors do not match the PoseStack's shape")
            if t_params.shape[-1] != 9:
                raise ValueError("LK-ball atom parameters must be [n_block_types, n_tiles, 32, 9]")
            if gp.numel() != 5:
                raise ValueError("the scoring global parameters must hold 5 values")
            put("bt_tile_lk_ball_params", t_params, real=True)
            put("global_params", gp, real=True)
            s.max_dis = float(max_dis)
            s.max_n_tiles = t_npol.shape[1]
            A = path_distance.shape[1]
        put("bt_n_atoms", bt_n_atoms)
        put("bt_n_conn", bt_n_conn)
        put("bt_conn_atom", bt_conn_atom)
        s.n_poses = P
        s.max_n_blocks = B
        s.n_rots = common[0].shape[0]
        s.n_block_types = bt_n_atoms.shape[0]
        s.max_n_block_atoms = A
        s.max_n_conn = bt_conn_atom.shape[1]
        self.n_poses, self.max_n_blocks = P, B
        self.n_atoms = common[1].shape[0]
        s.n_atoms = self.n_atoms
        self.launch = native.Launch(*(launch or (0, 0, 0, 0)))
        self.rotamers = bool(rotamers)
        ptr = ctypes.c_void_p()
        real_bytes = 4 if self.dtype == torch.float32 else 8
        with torch.cuda.device(self.device):
            if connectivity is None:
                native.call(
                    "tmol_b200_lkball_rotamer_plan_create" if rotamers else "tmol_b200_lkball_plan_create",
                    ctypes.byref(s), real_bytes, ctypes.byref(self.launch), self._stream(), ctypes.byref(ptr),
                )
            else:
                from ..pose.bondsep import connectivity as conn_struct, pose_connectivity

                cs, conn_keep = (
                    conn_struct(*connectivity) if isinstance(connectivity, tuple) else pose_connectivity(connectivity)
                )
                native.call(
                    "tmol_b200_lkball_plan_create_from_connectivity", ctypes.byref(s), ctypes.byref(cs), real_bytes,
                    ctypes.byref(self.launch), self._stream(), int(bool(rotamers)), ctypes.byref(ptr),
                )
                del conn_keep
        self.ptr = ptr
        del keep

    def waters(self, coords, out=None):
        """Waters [n_atoms, 4, 3] at ``coords``."""
        self._check_coords(coords)
        coords = coords.contiguous()
        if out is None:
            out = torch.empty((self.n_atoms, MAX_N_WATER, 3), dtype=self.dtype, device=self.device)
        native.call("tmol_b200_lkball_waters", self.ptr, ctypes.c_void_p(coords.data_ptr()),
                    ctypes.c_void_p(out.data_ptr()), self._stream())
        return out

    def waters_backward(self, coords, dwaters, dcoords=None):
        """dcoords (+)= the adjoint of dL/dwaters (zeros first when
        ``dcoords`` is None)."""
        self._check_coords(coords)
        coords = coords.contiguous()
        dwaters = dwaters.to(self.dtype).contiguous()
        if dcoords is None:
            dcoords = torch.zeros_like(coords)
        native.call("tmol_b200_lkball_waters_backward", self.ptr, ctypes.c_void_p(coords.data_ptr()),
                    ctypes.c_void_p(dwaters.data_ptr()), ctypes.c_void_p(dcoords.data_ptr()), self._stream())
        return dcoords

    def _check_waters(self, waters):
        if waters.device != self.device or waters.dtype != self.dtype:
            raise RuntimeError("waters do not match the plan's device and dtype")
        if tuple(waters.shape) != (self.n_atoms, MAX_N_WATER, 3):
            raise ValueError(f"waters must be [{self.n_atoms}, {MAX_N_WATER}, 3], got {tuple(waters.shape)}")

    def forward(self, coords, waters, block_pair=False, want_neighbors=True, energies=None):
        self._check_coords(coords)
        self._check_waters(waters)
        coords, waters = coords.contiguous(), waters.contiguous()
        P, B = self.n_poses, self.max_n_blocks
        shape = (self.N_TERMS, P, B, B) if block_pair else (self.N_TERMS, P)
        if energies is None:
            energies = torch.empty(shape, dtype=self.dtype, device=self.device)
        nbr = torch.empty((P, B, B), dtype=torch.int32, device=self.device) if want_neighbors else None
        native.call(
            "tmol_b200_lkball_forward", self.ptr, ctypes.c_void_p(coords.data_ptr()),
            ctypes.c_void_p(waters.data_ptr()), int(block_pair), ctypes.c_void_p(energies.data_ptr()),
            ctypes.c_void_p(nbr.data_ptr() if nbr is not None else 0), self._stream(),
        )
        self._after_call()
        return energies, nbr

    def backward(self, coords, waters, dTdV, block_pair=False, dcoords=None, dwaters=None):
        """(dL/dcoords directly, dL/dwaters) from dL/dE."""
        self._check_coords(coords)
        self._check_waters(waters)
        coords, waters = coords.contiguous(), waters.contiguous()
        dTdV = dTdV.to(self.dtype).contiguous()
        if dcoords is None:
            dcoords = torch.empty_like(coords)
        if dwaters is None:
            dwaters = torch.empty_like(waters)
        native.call(
            "tmol_b200_lkball_backward", self.ptr, ctypes.c_void_p(coords.data_ptr()),
            ctypes.c_void_p(waters.data_ptr()), int(block_pair), ctypes.c_void_p(dTdV.data_ptr()),
            ctypes.c_void_p(dcoords.data_ptr()), ctypes.c_void_p(dwaters.data_ptr()), self._stream(),
        )
        self._after_call()
        return dcoords, dwaters

    def forward_speculative(self, coords, waters, want_neighbors=True):
        """Whole-pose energies (and neighbour matrix) for an autograd forward
        whose backward will follow: once the plan has seen a
        backward_speculative call, the same pass also takes the gradients
        (coordinates directly, and waters) with that call's weights and keeps
        them.  Returns (energies, nbr, gen)."""
        self._check_coords(coords)
        self._check_waters(waters)
        coords, waters = coords.contiguous(), waters.contiguous()
        P, B = self.n_poses, self.max_n_blocks
        energies = torch.empty((self.N_TERMS, P), dtype=self.dtype, device=self.device)
        nbr = torch.empty((P, B, B), dtype=torch.int32, device=self.device) if want_neighbors else None
        native.call(
            "tmol_b200_lkball_forward_speculative", self.ptr, ctypes.c_void_p(coords.data_ptr()),
            ctypes.c_void_p(waters.data_ptr()), ctypes.c_void_p(energies.data_ptr()),
            ctypes.c_void_p(nbr.data_ptr() if nbr is not None else 0), self._stream(),
        )
        self.spec_gen += 1
        self._after_call()
        return energies, nbr, self.spec_gen

    def backward_speculative(self, coords, waters, dTdV, gen):
        """(dL/dcoords directly, dL/dwaters) for the forward `gen` returned:
        that forward's kept gradients when it is still the plan's latest and
        its weights equal dTdV (decided on the device), else recomputed."""
        self._check_coords(coords)
        self._check_waters(waters)
        coords, waters = coords.contiguous(), waters.contiguous()
        dTdV = dTdV.to(self.dtype).contiguous()
        dcoords = torch.empty_like(coords)
        dwaters = torch.empty_like(waters)
        native.call(
            "tmol_b200_lkball_backward_speculative", self.ptr, ctypes.c_void_p(coords.data_ptr()),
            ctypes.c_void_p(waters.data_ptr()), ctypes.c_void_p(dTdV.data_ptr()),
            ctypes.c_void_p(dcoords.data_ptr()), ctypes.c_void_p(dwaters.data_ptr()),
            int(gen is not None and gen == self.spec_gen), self._stream(),
        )
        self._after_call()
        return dcoords, dwaters

    COUNT_NAMES = ("block_pairs", "polar_occluder_pairs", "bridged_pairs", "pairs_evaluated", "unused")

    def set_skip_mask(self, mask):
        raise NotImplementedError("the learned block-pair screen serves LJ/LK plans")

    def screen_candidates(self, coords, capacity, out=None):
        raise NotImplementedError("the learned block-pair screen serves LJ/LK plans")

    # rotamer_dispatch (count + fill) is the LJ/LK plan's, on this ABI

    def rotamer_forward(self, coords, items, n_pairs, waters=None):
        """Energies [4, n_pairs] of the dispatched rotamer pairs."""
        self._check_coords(coords)
        self._check_waters(waters)
        coords, waters = coords.contiguous(), waters.contiguous()
        energies = torch.empty((self.N_TERMS, n_pairs), dtype=self.dtype, device=self.device)
        native.call(
            "tmol_b200_lkball_rotamer_forward", self.ptr, ctypes.c_void_p(coords.data_ptr()),
            ctypes.c_void_p(waters.data_ptr()), ctypes.c_void_p(items.data_ptr() if items.numel() else 0),
            items.shape[0], n_pairs, ctypes.c_void_p(energies.data_ptr()), self._stream(),
        )
        return energies

    def rotamer_backward(self, coords, items, dTdV, waters=None):
        """(dL/dcoords directly, dL/dwaters) from dL/dE [4, n_pairs]."""
        self._check_coords(coords)
        self._check_waters(waters)
        coords, waters = coords.contiguous(), waters.contiguous()
        dTdV = dTdV.to(self.dtype).contiguous()
        dcoords = torch.empty_like(coords)
        dwaters = torch.empty_like(waters)
        native.call(
            "tmol_b200_lkball_rotamer_backward", self.ptr, ctypes.c_void_p(coords.data_ptr()),
            ctypes.c_void_p(waters.data_ptr()), ctypes.c_void_p(items.data_ptr() if items.numel() else 0),
            items.shape[0], dTdV.shape[1], ctypes.c_void_p(dTdV.data_ptr()), ctypes.c_void_p(dcoords.data_ptr()),
            ctypes.c_void_p(dwaters.data_ptr()), self._stream(),
        )
        return dcoords, dwaters


class LKBallWaterPlan(LKBallPlan):
    """Water generation; over a rotamer set (more or fewer rotamers than
    blocks) the plan is a rotamer plan."""

    def __init__(self, coords_like, static_args, launch=None, rotamers=False):
        P, B = static_args[2].shape
        rotamers = rotamers or static_args[0].shape[0] != P * B
        super().__init__(coords_like, water_static=static_args, launch=launch, rotamers=rotamers)


class LKBallScorePlan(LKBallPlan):
    def __init__(self, coords_like, static_args, launch=None, rotamers=False):
        super().__init__(coords_like, score_static=static_args, launch=launch, rotamers=rotamers)


class _WaterFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, plan):
        ctx.plan = plan
        ctx.save_for_backward(coords)
        return plan.waters(coords)

    @staticmethod
    def backward(ctx, dW):
        (coords,) = ctx.saved_tensors
        if dW is None:
            return None, None
        return ctx.plan.waters_backward(coords, dW), None


class _LKBallScoreFn(torch.autograd.Function):
    """Whole-pose calls that need a gradient go through the speculative pair
    (one scoring pass per forward + backward from the second call on, as
    the LJ/LK op)."""

    @staticmethod
    def forward(ctx, coords, waters, plan, block_pair, want_neighbors):
        ctx.spec_gen = None
        ctx.speculate = (
            not block_pair and (ctx.needs_input_grad[0] or ctx.needs_input_grad[1])
            and coords.is_cuda and not torch.cuda.is_current_stream_capturing()
        )
        if ctx.speculate:
            E, nbr, ctx.spec_gen = plan.forward_speculative(coords, waters, want_neighbors)
        else:
            E, nbr = plan.forward(coords, waters, block_pair, want_neighbors)
        ctx.plan = plan
        ctx.block_pair = block_pair
        ctx.save_for_backward(coords, waters)
        if nbr is None:
            nbr = torch.empty((0,), dtype=torch.int32, device=coords.device)
        ctx.mark_non_differentiable(nbr)
        return E, nbr

    @staticmethod
    def backward(ctx, dE, _dnbr):
        coords, waters = ctx.saved_tensors
        if dE is None:
            return None, None, None, None, None
        if not ctx.speculate or torch.cuda.is_current_stream_capturing():
            dx, dw = ctx.plan.backward(coords, waters, dE, ctx.block_pair)
        else:
            dx, dw = ctx.plan.backward_speculative(coords, waters, dE, ctx.spec_gen)
        return dx, dw, None, None, None


class _LKBallRotamerScoreFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, waters, plan):
        indices, items = plan.rotamer_dispatch(coords)
        energies = plan.rotamer_forward(coords, items, indices.shape[1], waters)
        ctx.plan = plan
        ctx.save_for_backward(coords, waters, items)
        ctx.mark_non_differentiable(indices)
        return energies, indices

    @staticmethod
    def backward(ctx, dE, _dindices):
        coords, waters, items = ctx.saved_tensors
        if dE is None:
            return None, None, None
        dx, dw = ctx.plan.rotamer_backward(coords, items, dE, waters)
        return dx, dw, None


def gen_pose_waters(coords, *args):
    """Drop-in for ``torch.ops.tmol_lk_ball.gen_pose_waters``."""
    if len(args) != N_WATER_STATIC:
        raise TypeError(f"gen_pose_waters takes coords + {N_WATER_STATIC} arguments, got {1 + len(args)}")
    flat = coords.reshape(-1, 3)
    plan = get_plan(flat, args, plan_class=LKBallWaterPlan)
    return _WaterFn.apply(flat, plan)


def lk_ball_pose_score(coords, *args, return_block_neighbors=True):
    """Drop-in for ``torch.ops.tmol_lk_ball.lk_ball_pose_score``."""
    if len(args) != N_SCORE_STATIC:
        raise TypeError(f"lk_ball_pose_score takes coords + {N_SCORE_STATIC} arguments, got {1 + len(args)}")
    static, waters, block_pair = args[:-2], args[-2], bool(args[-1])
    flat = coords.reshape(-1, 3)
    plan = get_plan(flat, static, plan_class=LKBallScorePlan)
    E, nbr = _LKBallScoreFn.apply(flat, waters, plan, block_pair, return_block_neighbors)
    return E, (nbr if return_block_neighbors else None)


def lk_ball_rotamer_score(coords, *args):
    """Drop-in for ``torch.ops.tmol_lk_ball.lk_ball_rotamer_score``: a rotamer
    set's coordinates, its indexing and the pose's LK-ball tables (25
    arguments), its waters and ``output_block_pair_energies`` (True, as tmol's
    rotamer scoring passes it).  Returns ``(scores [4, n], indices [3, n])``
    for every rotamer pair of neighbouring blocks and every rotamer with
    itself; gradients flow to ``coords`` and the waters."""
    if len(args) != N_SCORE_STATIC:
        raise TypeError(f"lk_ball_rotamer_score takes coords + {N_SCORE_STATIC} arguments, got {1 + len(args)}")
    static, waters, block_pair = args[:-2], args[-2], args[-1]
    if not block_pair:
        raise ValueError("rotamer scoring reports rotamer-pair energies (output_block_pair_energies=True)")
    flat = coords.reshape(-1, 3)
    plan = get_plan(flat, static, rotamers=True, plan_class=LKBallScorePlan)
    return _LKBallRotamerScoreFn.apply(flat, waters, plan)
