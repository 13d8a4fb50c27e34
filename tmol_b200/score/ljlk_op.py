"""The LJ/LK pose-score op on B200, with tmol's argument list and outputs.

``ljlk_pose_scores(coords, <26 static arguments>, output_block_pair_energies)``
takes exactly the arguments of ``torch.ops.tmol_ljlk.ljlk_pose_scores``
(``tmol/score/ljlk/potentials/compiled.ops.cpp:533-597``) and returns
``(scores, block_neighbors)``: scores ``[3, P]`` (whole pose) or
``[3, P, B, B]`` (block pairs), neighbours ``[P, B, B]`` int32.  Gradients
flow to ``coords`` only, through a recompute adjoint kernel.

The static arguments are turned into a device plan (compact count-pair and
parameter tables) once and cached, keyed by the identity, shape and version
of each static tensor.  All tensors must be on one CUDA device; there is no
CPU path.
"""

import collections
import ctypes

import torch

from .. import native

N_STATIC = 26  # arguments after coords, before the output-mode flag


class LJLKPlan:
    """Owns one ``tmol_b200_ljlk_plan``: of the pose op (one rotamer per
    block) or, with ``rotamers=True``, of the rotamer op (any number of
    rotamers per block)."""

    N_TERMS = 3  # fa_ljatr, fa_ljrep, fa_lk
    ABI = "tmol_b200_ljlk"  # prefix of the scoring entry points
    NAME = "LJ/LK"
    # scoring calls after which the work items are reordered by their
    # measured cost (rebalance); the drop-in ops' plans set 2
    auto_balance = 0
    # whole-pose autograd through forward_speculative / backward_speculative
    SPECULATIVE = True
    spec_gen = 0  # count of speculative forwards on this plan

    def __init__(self, coords_like, static_args, launch=None, rotamers=False, connectivity=None):
        (
            rot_coord_offset,
            pose_ind_for_atom,
            first_rot_for_block,
            first_rot_block_type,
            block_ind_for_rot,
            pose_ind_for_rot,
            block_type_ind_for_rot,
            n_rots_for_pose,
            rot_offset_for_pose,
            n_rots_for_block,
            rot_offset_for_block,
            max_n_rots_per_pose,
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
        ) = static_args
        device = self._set_device(coords_like)
        self.block_sizes = (first_rot_block_type, bt_n_atoms)  # for the autotuner's signature
        ints = dict(
            rot_coord_offset=rot_coord_offset,
            pose_ind_for_atom=pose_ind_for_atom,
            first_rot_for_block=first_rot_for_block,
            first_rot_block_type=first_rot_block_type,
            block_ind_for_rot=block_ind_for_rot,
            pose_ind_for_rot=pose_ind_for_rot,
            block_type_ind_for_rot=block_type_ind_for_rot,
            n_rots_for_pose=n_rots_for_pose,
            rot_offset_for_pose=rot_offset_for_pose,
            n_rots_for_block=n_rots_for_block,
            rot_offset_for_block=rot_offset_for_block,
            min_bondsep=min_bondsep,
            inter_block_bondsep=inter_block_bondsep,
            bt_n_atoms=bt_n_atoms,
            bt_n_heavy_atoms_in_tile=bt_n_heavy_in_tile,
            bt_heavy_atoms_in_tile=bt_heavy_in_tile,
            bt_atom_types=bt_atom_types,
            bt_n_conn=bt_n_conn,
            bt_conn_atom=bt_conn_atom,
            bt_path_distance=bt_path_distance,
            bt_is_ligand_fragment=bt_is_ligand,
        )
        keep = []
        if connectivity is not None:
            # count-pair tables from the connectivity: the dense bond
            # separation tensors are not needed
            for name in ("min_bondsep", "inter_block_bondsep"):
                if ints[name] is None:
                    del ints[name]
        s = native.Inputs()
        for name, t in ints.items():
            if not isinstance(t, torch.Tensor):
                raise TypeError(f"{name} must be a tensor")
            if t.device != device:
                raise RuntimeError(f"{name} is on {t.device}, coordinates on {device}")
            t = t.to(torch.int32).contiguous()
            keep.append(t)
            setattr(s, name, t.data_ptr())
        reals = {}
        for name, t in (("type_params", type_params), ("global_params", global_params)):
            if t.device != device:
                raise RuntimeError(f"{name} is on {t.device}, coordinates on {device}")
            t = t.to(self.dtype).contiguous()
            keep.append(t)
            reals[name] = t
            setattr(s, name, t.data_ptr())
        P, B = first_rot_for_block.shape
        C = bt_conn_atom.shape[1]
        if inter_block_bondsep is not None and tuple(inter_block_bondsep.shape) != (P, B, B, C, C):
            raise ValueError(
                f"inter_block_bondsep has shape {tuple(inter_block_bondsep.shape)}, expected {(P, B, B, C, C)}"
            )
        if min_bondsep is not None and tuple(min_bondsep.shape) != (P, B, B):
            raise ValueError(f"min_bondsep has shape {tuple(min_bondsep.shape)}, expected {(P, B, B)}")
        if reals["type_params"].dim() != 2 or reals["type_params"].shape[1] != 10:
            raise ValueError("type_params must be [n_types, 10]")
        if reals["global_params"].numel() != 5:
            raise ValueError("global_params must hold 5 values")
        s.n_poses = P
        s.max_n_blocks = B
        s.n_rots = rot_coord_offset.shape[0]
        s.n_block_types = bt_n_atoms.shape[0]
        s.max_n_block_atoms = bt_atom_types.shape[1]
        s.max_n_conn = C
        s.max_n_tiles = bt_n_heavy_in_tile.shape[1]
        s.n_atom_types = type_params.shape[0]
        s.max_n_rots_per_pose = int(max_n_rots_per_pose)
        s.max_dis = float(max_dis)
        self.n_poses, self.max_n_blocks = P, B
        self.n_atoms = pose_ind_for_atom.shape[0]
        s.n_atoms = self.n_atoms
        self._create(s, launch, rotamers, connectivity)
        del keep

    def _set_device(self, coords_like):
        device = coords_like.device
        if device.type != "cuda":
            raise RuntimeError(f"tmol_b200 {self.NAME} scoring runs on CUDA tensors only")
        self.device = device
        self.dtype = coords_like.dtype
        if self.dtype not in (torch.float32, torch.float64):
            raise TypeError(f"coordinates must be float32 or float64, got {self.dtype}")
        return device

    def _create(self, inputs, launch, rotamers, connectivity=None):
        """Calls the plan-create entry point on the filled inputs struct;
        with ``connectivity`` (a PoseStack, or the tuple (block_type_ind,
        inter_residue_connections, bt_n_conn, bt_conn_sep)) the count-pair
        tables are built from it (include/tmol_b200_pose.h)."""
        self.launch = native.Launch(*(launch or (0, 0, 0, 0)))
        self.rotamers = bool(rotamers)
        ptr = ctypes.c_void_p()
        real_bytes = 4 if self.dtype == torch.float32 else 8
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            if connectivity is None:
                native.call(
                    f"{self.ABI}_rotamer_plan_create" if rotamers else f"{self.ABI}_plan_create",
                    ctypes.byref(inputs),
                    real_bytes,
                    ctypes.byref(self.launch),
                    ctypes.c_void_p(stream),
                    ctypes.byref(ptr),
                )
            else:
                from ..pose.bondsep import connectivity as conn_struct, pose_connectivity

                if isinstance(connectivity, tuple):
                    cs, conn_keep = conn_struct(*connectivity)
                else:
                    cs, conn_keep = pose_connectivity(connectivity)
                native.call(
                    f"{self.ABI}_plan_create_from_connectivity",
                    ctypes.byref(inputs),
                    ctypes.byref(cs),
                    real_bytes,
                    ctypes.byref(self.launch),
                    ctypes.c_void_p(stream),
                    int(bool(rotamers)),
                    ctypes.byref(ptr),
                )
                del conn_keep
        self.ptr = ptr

    def __del__(self):
        ptr = getattr(self, "ptr", None)
        if ptr is not None and ptr.value:
            try:
                native.load().tmol_b200_ljlk_plan_destroy(ptr)
            except Exception:
                pass
            self.ptr = None

    def set_launch(self, rows_per_item=0, warps_per_cta=0, ctas_per_sm=0, candidates_per_item=0,
                   slots_per_group=0):
        """Launch shape (0 = default); see tmol_b200_ljlk_launch."""
        self.launch = native.Launch(rows_per_item, warps_per_cta, ctas_per_sm, candidates_per_item,
                                    slots_per_group)
        native.call("tmol_b200_ljlk_plan_set_launch", self.ptr, ctypes.byref(self.launch))

    def launch_tuple(self):
        l = self.launch
        return (l.rows_per_item, l.warps_per_cta, l.ctas_per_sm, l.candidates_per_item, l.slots_per_group)

    def rebalance(self):
        """Order the work items longest-first by their cost in the last call
        made with counting on (the counting kernels time each item)."""
        native.call("tmol_b200_ljlk_plan_rebalance", self.ptr, self._stream())

    def _after_call(self):
        # the reorder synchronises the stream: never inside a graph capture
        if self.auto_balance > 0 and not torch.cuda.is_current_stream_capturing():
            self.auto_balance -= 1
            self.rebalance()
            if self.auto_balance == 0:
                self.set_counting(False)

    def balance(self, run, passes=2):
        """Runs `run()` (one scoring call on this plan) and orders the work
        items longest-first by their measured costs, `passes` times.  An item
        that ran in the tail of a call, with its SM nearly to itself, measures
        several times cheaper than it runs beside other heavy items; measured
        again in longest-first order, every heavy item runs as it will in the
        calls that follow."""
        self.set_counting(True)  # the counting kernels time each item
        for _ in range(passes):
            run()
            self.rebalance()
        self.set_counting(False)

    def device_bytes(self):
        return native.load().tmol_b200_ljlk_plan_device_bytes(self.ptr)

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _check_coords(self, coords):
        if coords.device != self.device or coords.dtype != self.dtype:
            raise RuntimeError(
                f"coordinates ({coords.device}, {coords.dtype}) do not match the plan "
                f"({self.device}, {self.dtype})"
            )
        if coords.dim() != 2 or coords.shape[1] != 3 or coords.shape[0] != self.n_atoms:
            raise ValueError(f"coordinates must be [{self.n_atoms}, 3], got {tuple(coords.shape)}")

    def forward(self, coords, block_pair=False, want_neighbors=True, energies=None):
        self._check_coords(coords)
        coords = coords.contiguous()
        P, B = self.n_poses, self.max_n_blocks
        shape = (self.N_TERMS, P, B, B) if block_pair else (self.N_TERMS, P)
        if energies is None:
            energies = torch.empty(shape, dtype=self.dtype, device=self.device)
        nbr = torch.empty((P, B, B), dtype=torch.int32, device=self.device) if want_neighbors else None
        native.call(
            f"{self.ABI}_forward",
            self.ptr,
            ctypes.c_void_p(coords.data_ptr()),
            int(block_pair),
            ctypes.c_void_p(energies.data_ptr()),
            ctypes.c_void_p(nbr.data_ptr() if nbr is not None else 0),
            self._stream(),
        )
        self._after_call()
        return energies, nbr

    def backward(self, coords, dTdV, block_pair=False, dcoords=None):
        self._check_coords(coords)
        coords = coords.contiguous()
        dTdV = dTdV.to(self.dtype).contiguous()
        if dcoords is None:
            dcoords = torch.empty_like(coords)
        native.call(
            f"{self.ABI}_backward",
            self.ptr,
            ctypes.c_void_p(coords.data_ptr()),
            int(block_pair),
            ctypes.c_void_p(dTdV.data_ptr()),
            ctypes.c_void_p(dcoords.data_ptr()),
            self._stream(),
        )
        self._after_call()
        return dcoords

    def forward_speculative(self, coords, want_neighbors=True):
        """Whole-pose energies (and neighbour matrix) for an autograd forward
        whose backward will follow: once the plan has seen a
        backward_speculative call, the same pass also takes the gradient with
        that call's weights and keeps it.  Returns (energies, nbr, gen), gen
        identifying this forward for backward_speculative."""
        self._check_coords(coords)
        coords = coords.contiguous()
        P, B = self.n_poses, self.max_n_blocks
        energies = torch.empty((self.N_TERMS, P), dtype=self.dtype, device=self.device)
        nbr = torch.empty((P, B, B), dtype=torch.int32, device=self.device) if want_neighbors else None
        native.call(
            f"{self.ABI}_forward_speculative",
            self.ptr,
            ctypes.c_void_p(coords.data_ptr()),
            ctypes.c_void_p(energies.data_ptr()),
            ctypes.c_void_p(nbr.data_ptr() if nbr is not None else 0),
            self._stream(),
        )
        self.spec_gen += 1
        self._after_call()
        return energies, nbr, self.spec_gen

    def backward_speculative(self, coords, dTdV, gen):
        """sum_t dTdV_t * dE_t/dcoords for the forward `gen` returned: the
        gradient that forward kept when it is still the plan's latest and
        its weights equal dTdV (decided on the device), else a recomputed
        one."""
        self._check_coords(coords)
        coords = coords.contiguous()
        dTdV = dTdV.to(self.dtype).contiguous()
        dcoords = torch.empty_like(coords)
        native.call(
            f"{self.ABI}_backward_speculative",
            self.ptr,
            ctypes.c_void_p(coords.data_ptr()),
            ctypes.c_void_p(dTdV.data_ptr()),
            ctypes.c_void_p(dcoords.data_ptr()),
            int(gen is not None and gen == self.spec_gen),
            self._stream(),
        )
        self._after_call()
        return dcoords

    def energy_and_gradient(self, coords, weights, energies=None, dcoords=None):
        """Energies [n_terms, P] and sum_t weights[t, pose] * dE_t/dcoords in
        one pass."""
        self._check_coords(coords)
        coords = coords.contiguous()
        weights = weights.to(self.dtype).contiguous()
        if tuple(weights.shape) != (self.N_TERMS, self.n_poses):
            raise ValueError(f"weights must be [{self.N_TERMS}, {self.n_poses}]")
        if energies is None:
            energies = torch.empty((self.N_TERMS, self.n_poses), dtype=self.dtype, device=self.device)
        if dcoords is None:
            dcoords = torch.empty_like(coords)
        native.call(
            f"{self.ABI}_energy_and_gradient",
            self.ptr,
            ctypes.c_void_p(coords.data_ptr()),
            ctypes.c_void_p(weights.data_ptr()),
            ctypes.c_void_p(energies.data_ptr()),
            ctypes.c_void_p(dcoords.data_ptr()),
            self._stream(),
        )
        self._after_call()
        return energies, dcoords

    COUNT_NAMES = ("block_pairs", "atom_pairs", "heavy_pairs", "atom_pairs_in_range", "heavy_pairs_in_range")

    def set_counting(self, enable=True):
        """Work counting for the following calls (off by default: the counting
        kernel is slower)."""
        native.call("tmol_b200_ljlk_plan_set_counting", self.ptr, int(bool(enable)))

    def last_counts(self):
        """Work counters of the last forward / energy_and_gradient call (all
        zero when it ran with counting off)."""
        arr = (ctypes.c_int64 * 5)()
        native.call("tmol_b200_ljlk_last_counts", self.ptr, self._stream(), arr)
        return dict(zip(self.COUNT_NAMES, list(arr)))

    # -- rotamer plans ----------------------------------------------------

    def rotamer_dispatch(self, coords):
        """The rotamer pairs the op scores at ``coords``: (indices [3, n]
        int32 (pose, rot1, rot2), work items [n_items, 4] int32).
        Synchronises the current stream once (the counts size the output)."""
        self._check_coords(coords)
        coords = coords.contiguous()
        n_pairs, n_items = ctypes.c_int64(), ctypes.c_int64()
        native.call(
            f"{self.ABI}_rotamer_count", self.ptr, ctypes.c_void_p(coords.data_ptr()),
            ctypes.byref(n_pairs), ctypes.byref(n_items), self._stream(),
        )
        indices = torch.empty((3, n_pairs.value), dtype=torch.int32, device=self.device)
        items = torch.empty((n_items.value, 4), dtype=torch.int32, device=self.device)
        native.call(
            f"{self.ABI}_rotamer_fill", self.ptr, ctypes.c_void_p(indices.data_ptr() if n_pairs.value else 0),
            ctypes.c_void_p(items.data_ptr() if n_items.value else 0), self._stream(),
        )
        return indices, items

    def rotamer_forward(self, coords, items, n_pairs):
        """Energies [n_terms, n_pairs] of the dispatched rotamer pairs."""
        self._check_coords(coords)
        coords = coords.contiguous()
        energies = torch.empty((self.N_TERMS, n_pairs), dtype=self.dtype, device=self.device)
        native.call(
            f"{self.ABI}_rotamer_forward", self.ptr, ctypes.c_void_p(coords.data_ptr()),
            ctypes.c_void_p(items.data_ptr() if items.numel() else 0), items.shape[0], n_pairs,
            ctypes.c_void_p(energies.data_ptr()), self._stream(),
        )
        return energies

    def rotamer_backward(self, coords, items, dTdV):
        """dL/dcoords from dL/dE [n_terms, n_pairs]."""
        self._check_coords(coords)
        coords = coords.contiguous()
        dTdV = dTdV.to(self.dtype).contiguous()
        dcoords = torch.empty_like(coords)
        native.call(
            f"{self.ABI}_rotamer_backward", self.ptr, ctypes.c_void_p(coords.data_ptr()),
            ctypes.c_void_p(items.data_ptr() if items.numel() else 0), items.shape[0], dTdV.shape[1],
            ctypes.c_void_p(dTdV.data_ptr()), ctypes.c_void_p(dcoords.data_ptr()), self._stream(),
        )
        return dcoords

    def skip_mask_words(self):
        """32-bit words per (pose, block) row of a skip mask."""
        return (self.max_n_blocks + 31) // 32

    def set_skip_mask(self, mask):
        """Install a block-pair skip mask (int32 [P * B, words], caller-owned,
        kept alive by the plan) or remove it (None).  Bit b2 of row
        (p, b1) set = later scoring calls leave block pair (b1, b2) out; the
        diagonal and count-pair partners are always scored."""
        if mask is None:
            self._skip_mask = None
            native.call("tmol_b200_ljlk_plan_set_skip_mask", self.ptr, None, 0)
            return
        if mask.device != self.device or mask.dtype != torch.int32 or not mask.is_contiguous():
            raise ValueError("skip mask must be a contiguous int32 tensor on the plan's device")
        if mask.dim() != 2 or mask.shape[0] != self.n_poses * self.max_n_blocks:
            raise ValueError(f"skip mask must be [{self.n_poses * self.max_n_blocks}, words]")
        self._skip_mask = mask
        native.call(
            "tmol_b200_ljlk_plan_set_skip_mask", self.ptr, ctypes.c_void_p(mask.data_ptr()), int(mask.shape[1])
        )

    def screen_candidates(self, coords, capacity, out=None):
        """Block pairs b1 < b2 that pass the sphere test and are not
        count-pair partners, with their screen features.  Returns a dict of
        device tensors: row [cap] (p * B + b1), b2 [cap], bt [cap, 2],
        features [cap, 12] and count [1] (total candidates, may exceed cap)."""
        self._check_coords(coords)
        if self.dtype != torch.float32:
            raise TypeError("screen candidates need a float32 plan")
        coords = coords.contiguous()
        if out is None:
            dev = self.device
            out = dict(
                row=torch.empty(capacity, dtype=torch.int32, device=dev),
                b2=torch.empty(capacity, dtype=torch.int32, device=dev),
                bt=torch.empty((capacity, 2), dtype=torch.int32, device=dev),
                features=torch.empty((capacity, 12), dtype=torch.float32, device=dev),
                count=torch.empty(1, dtype=torch.int32, device=dev),
            )
        capacity = out["row"].shape[0]
        native.call(
            "tmol_b200_ljlk_screen_candidates",
            self.ptr,
            ctypes.c_void_p(coords.data_ptr()),
            int(capacity),
            ctypes.c_void_p(out["row"].data_ptr()),
            ctypes.c_void_p(out["b2"].data_ptr()),
            ctypes.c_void_p(out["bt"].data_ptr()),
            ctypes.c_void_p(out["features"].data_ptr()),
            ctypes.c_void_p(out["count"].data_ptr()),
            self._stream(),
        )
        return out

    def profile(self, enable=True):
        native.call("tmol_b200_ljlk_profile", self.ptr, int(enable))

    def profile_read(self):
        """(total milliseconds, launches) of the scoring kernel since profile()."""
        ms = ctypes.c_double()
        n = ctypes.c_int32()
        native.call("tmol_b200_ljlk_profile_read", self.ptr, ctypes.byref(ms), ctypes.byref(n))
        return ms.value, n.value


class _ScoreFn(torch.autograd.Function):
    """Whole-pose calls whose coordinates need a gradient go through the
    speculative pair: from the second call on, the forward's fused pass also
    takes the gradient with the previous backward's weights, and a backward
    with the same weights reuses it (one scoring pass per forward + backward
    instead of two)."""

    @staticmethod
    def forward(ctx, coords, plan, block_pair, want_neighbors):
        ctx.spec_gen = None
        # not inside a graph capture: the choice between a kept and a fresh
        # gradient uses host-side state of the plan at call time
        ctx.speculate = (
            not block_pair and plan.SPECULATIVE and ctx.needs_input_grad[0]
            and coords.is_cuda and not torch.cuda.is_current_stream_capturing()
        )
        if ctx.speculate:
            E, nbr, ctx.spec_gen = plan.forward_speculative(coords, want_neighbors)
        else:
            E, nbr = plan.forward(coords, block_pair, want_neighbors)
        ctx.plan = plan
        ctx.block_pair = block_pair
        ctx.save_for_backward(coords)
        if nbr is None:
            nbr = torch.empty((0,), dtype=torch.int32, device=coords.device)
        ctx.mark_non_differentiable(nbr)
        return E, nbr

    @staticmethod
    def backward(ctx, dE, _dnbr):
        (coords,) = ctx.saved_tensors
        if dE is None:
            return None, None, None, None
        if not ctx.speculate or torch.cuda.is_current_stream_capturing():
            dx = ctx.plan.backward(coords, dE, ctx.block_pair)
        else:
            dx = ctx.plan.backward_speculative(coords, dE, ctx.spec_gen)
        return dx, None, None, None


_PLAN_CACHE = collections.OrderedDict()
_PLAN_CACHE_SIZE = 8


def _plan_key(coords, static):
    parts = [coords.device, coords.dtype]
    for t in static:
        if isinstance(t, torch.Tensor):
            parts.append((t.data_ptr(), tuple(t.shape), t.dtype, t._version))
        else:
            parts.append(t)
    return tuple(parts)


def get_plan(coords, static, rotamers=False, plan_class=None):
    plan_class = plan_class or LJLKPlan
    key = (plan_class, rotamers) + _plan_key(coords, static)
    entry = _PLAN_CACHE.get(key)
    if entry is not None:
        _PLAN_CACHE.move_to_end(key)
        return entry[0]
    plan = plan_class(coords, static, rotamers=rotamers)
    # the drop-in ops run without a tuning step: their plans order the work
    # items by measured cost after each of their first two calls (made with
    # the counting kernels, which time each item)
    if not rotamers:
        plan.auto_balance = 2
        plan.set_counting(True)
    # the static tensors are held so that their addresses cannot be reused
    # by other tensors while the key is cached
    _PLAN_CACHE[key] = (plan, [t for t in static if isinstance(t, torch.Tensor)])
    while len(_PLAN_CACHE) > _PLAN_CACHE_SIZE:
        _PLAN_CACHE.popitem(last=False)
    return plan


def clear_plan_cache():
    _PLAN_CACHE.clear()


def ljlk_pose_scores(coords, *args, return_block_neighbors=True):
    """Drop-in for ``torch.ops.tmol_ljlk.ljlk_pose_scores``."""
    if len(args) != N_STATIC:
        raise TypeError(f"ljlk_pose_scores takes coords + {N_STATIC} arguments, got {1 + len(args)}")
    static = args[:-1]
    block_pair = bool(args[-1])
    plan = get_plan(coords, static)
    return pose_scores_with_plan(coords, plan, block_pair, return_block_neighbors)


def pose_scores_with_plan(coords, plan, block_pair=False, return_block_neighbors=False):
    scores, nbr = _ScoreFn.apply(coords, plan, block_pair, return_block_neighbors)
    return scores, (nbr if return_block_neighbors else None)


class _RotamerScoreFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, plan):
        indices, items = plan.rotamer_dispatch(coords)
        energies = plan.rotamer_forward(coords, items, indices.shape[1])
        ctx.plan = plan
        ctx.save_for_backward(coords, items)
        ctx.mark_non_differentiable(indices)
        return energies, indices

    @staticmethod
    def backward(ctx, dE, _dindices):
        coords, items = ctx.saved_tensors
        if dE is None:
            return None, None
        return ctx.plan.rotamer_backward(coords, items, dE), None


def ljlk_rotamer_scores(coords, *args):
    """Drop-in for ``torch.ops.tmol_ljlk.ljlk_rotamer_scores``
    (``tmol/score/ljlk/potentials/compiled.ops.cpp:599-662``): the rotamer
    set's coordinates and the op's 26 further arguments (the last,
    ``output_block_pair_energies``, must be True as tmol's rotamer scoring
    module passes it).  Returns ``(scores [3, n], indices [3, n])``: the
    energies of every rotamer pair of neighbouring blocks and of every
    rotamer with itself, and their (pose, rot1, rot2); gradients flow to
    ``coords``."""
    if len(args) != N_STATIC:
        raise TypeError(f"ljlk_rotamer_scores takes coords and {N_STATIC} further arguments")
    static, block_pair = args[:-1], args[-1]
    if not block_pair:
        raise ValueError("rotamer scoring reports rotamer-pair energies (output_block_pair_energies=True)")
    plan = get_plan(coords.reshape(-1, 3), static, rotamers=True)
    return _RotamerScoreFn.apply(coords.reshape(-1, 3), plan)
