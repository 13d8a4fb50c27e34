"""ctypes binding of the C ABI in ``include/tmol_b200_ljlk.h``,
``include/tmol_b200_elec.h``, ``include/tmol_b200_lkball.h``,
``include/tmol_b200_pose.h`` and ``include/tmol_b200_screen.h``.

The shared library is built in-tree (``tmol_b200/lib``) by
``tmol_b200.build``.  There is no fallback: importing this module without the
library raises, and every entry point's status code is turned into an
exception.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("TMOL_B200_LIB") or os.path.join(HERE, "lib", "libtmol_b200_ljlk.so")

_i32p = ctypes.POINTER(ctypes.c_int32)


class Inputs(ctypes.Structure):
    """``tmol_b200_ljlk_inputs``."""

    _fields_ = [
        ("n_atoms", ctypes.c_int64),
        ("n_poses", ctypes.c_int32),
        ("max_n_blocks", ctypes.c_int32),
        ("n_rots", ctypes.c_int32),
        ("n_block_types", ctypes.c_int32),
        ("max_n_block_atoms", ctypes.c_int32),
        ("max_n_conn", ctypes.c_int32),
        ("max_n_tiles", ctypes.c_int32),
        ("n_atom_types", ctypes.c_int32),
        ("rot_coord_offset", ctypes.c_void_p),
        ("pose_ind_for_atom", ctypes.c_void_p),
        ("first_rot_for_block", ctypes.c_void_p),
        ("first_rot_block_type", ctypes.c_void_p),
        ("block_ind_for_rot", ctypes.c_void_p),
        ("pose_ind_for_rot", ctypes.c_void_p),
        ("block_type_ind_for_rot", ctypes.c_void_p),
        ("n_rots_for_pose", ctypes.c_void_p),
        ("rot_offset_for_pose", ctypes.c_void_p),
        ("n_rots_for_block", ctypes.c_void_p),
        ("rot_offset_for_block", ctypes.c_void_p),
        ("max_n_rots_per_pose", ctypes.c_int32),
        ("min_bondsep", ctypes.c_void_p),
        ("inter_block_bondsep", ctypes.c_void_p),
        ("bt_n_atoms", ctypes.c_void_p),
        ("bt_n_heavy_atoms_in_tile", ctypes.c_void_p),
        ("bt_heavy_atoms_in_tile", ctypes.c_void_p),
        ("bt_atom_types", ctypes.c_void_p),
        ("bt_n_conn", ctypes.c_void_p),
        ("bt_conn_atom", ctypes.c_void_p),
        ("bt_path_distance", ctypes.c_void_p),
        ("bt_is_ligand_fragment", ctypes.c_void_p),
        ("type_params", ctypes.c_void_p),
        ("global_params", ctypes.c_void_p),
        ("max_dis", ctypes.c_double),
    ]


class ElecInputs(ctypes.Structure):
    """``tmol_b200_elec_inputs``."""

    _fields_ = [
        ("n_atoms", ctypes.c_int64),
        ("n_poses", ctypes.c_int32),
        ("max_n_blocks", ctypes.c_int32),
        ("n_rots", ctypes.c_int32),
        ("n_block_types", ctypes.c_int32),
        ("max_n_block_atoms", ctypes.c_int32),
        ("max_n_conn", ctypes.c_int32),
        ("rot_coord_offset", ctypes.c_void_p),
        ("pose_ind_for_atom", ctypes.c_void_p),
        ("first_rot_for_block", ctypes.c_void_p),
        ("first_rot_block_type", ctypes.c_void_p),
        ("block_ind_for_rot", ctypes.c_void_p),
        ("pose_ind_for_rot", ctypes.c_void_p),
        ("block_type_ind_for_rot", ctypes.c_void_p),
        ("n_rots_for_pose", ctypes.c_void_p),
        ("rot_offset_for_pose", ctypes.c_void_p),
        ("n_rots_for_block", ctypes.c_void_p),
        ("rot_offset_for_block", ctypes.c_void_p),
        ("max_n_rots_per_pose", ctypes.c_int32),
        ("min_bondsep", ctypes.c_void_p),
        ("inter_block_bondsep", ctypes.c_void_p),
        ("bt_n_atoms", ctypes.c_void_p),
        ("bt_partial_charge", ctypes.c_void_p),
        ("bt_n_conn", ctypes.c_void_p),
        ("bt_conn_atom", ctypes.c_void_p),
        ("bt_inter_repr_path_distance", ctypes.c_void_p),
        ("bt_intra_repr_path_distance", ctypes.c_void_p),
        ("bt_is_ligand_fragment", ctypes.c_void_p),
        ("global_params", ctypes.c_void_p),
        ("max_dis", ctypes.c_double),
    ]


class LKBallInputs(ctypes.Structure):
    """``tmol_b200_lkball_inputs``."""

    _fields_ = (
        [("n_atoms", ctypes.c_int64)]
        + [(n, ctypes.c_int32) for n in ("n_poses", "max_n_blocks", "n_rots", "n_block_types", "max_n_block_atoms",
                                         "max_n_conn", "max_n_tiles", "max_n_all_bonds")]
        + [(n, ctypes.c_void_p) for n in (
            "rot_coord_offset", "pose_ind_for_atom", "first_rot_for_block", "first_rot_block_type",
            "block_ind_for_rot", "pose_ind_for_rot", "block_type_ind_for_rot", "n_rots_for_pose",
            "rot_offset_for_pose", "n_rots_for_block", "rot_offset_for_block")]
        + [("max_n_rots_per_pose", ctypes.c_int32)]
        + [(n, ctypes.c_void_p) for n in (
            "inter_residue_connections", "min_bondsep", "inter_block_bondsep", "bt_n_atoms", "bt_n_conn",
            "bt_conn_atom", "bt_n_all_bonds", "bt_all_bonds", "bt_atom_all_bond_ranges", "bt_tile_n_donH",
            "bt_tile_n_acc", "bt_tile_donH_inds", "bt_tile_donH_hvy_inds", "bt_tile_which_donH_for_hvy",
            "bt_tile_acc_inds", "bt_tile_hybridization", "bt_tile_acc_n_attached_H", "bt_atom_is_hydrogen",
            "water_gen_global_params", "sp2_water_tors", "sp3_water_tors", "ring_water_tors")]
        + [(n, ctypes.c_int32) for n in ("n_sp2_tors", "n_sp3_tors", "n_ring_tors")]
        + [(n, ctypes.c_void_p) for n in (
            "bt_tile_n_polar_atoms", "bt_tile_n_occluder_atoms", "bt_tile_pol_occ_inds", "bt_tile_lk_ball_params",
            "bt_path_distance", "global_params")]
        + [("max_dis", ctypes.c_double)]
    )


class PoseConnectivity(ctypes.Structure):
    """``tmol_b200_pose_connectivity``."""

    _fields_ = [
        ("n_poses", ctypes.c_int32),
        ("max_n_blocks", ctypes.c_int32),
        ("n_block_types", ctypes.c_int32),
        ("max_n_conn", ctypes.c_int32),
        ("block_type_ind", ctypes.c_void_p),
        ("inter_residue_connections", ctypes.c_void_p),
        ("bt_n_conn", ctypes.c_void_p),
        ("bt_conn_sep", ctypes.c_void_p),
    ]


class Launch(ctypes.Structure):
    """``tmol_b200_ljlk_launch``."""

    _fields_ = [
        ("rows_per_item", ctypes.c_int32),
        ("warps_per_cta", ctypes.c_int32),
        ("ctas_per_sm", ctypes.c_int32),
        ("candidates_per_item", ctypes.c_int32),
        ("slots_per_group", ctypes.c_int32),
    ]


# Every symbol the header declares, with its ctypes signature.
_V, _I32, _I64, _F = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float


class ScreenWeights(ctypes.Structure):
    """tmol_b200_screen_weights: device pointers of the screen MLP."""

    _fields_ = [(n, ctypes.c_void_p) for n in ("w1", "w2", "w3", "w4", "b1", "b2", "b3", "b4", "emb")]


SIGNATURES = {
    "tmol_b200_ljlk_plan_create": (
        ctypes.c_int,
        [ctypes.POINTER(Inputs), ctypes.c_int, ctypes.POINTER(Launch), ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)],
    ),
    "tmol_b200_ljlk_plan_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "tmol_b200_ljlk_plan_set_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Launch)]),
    "tmol_b200_ljlk_plan_rebalance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "tmol_b200_ljlk_forward": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "tmol_b200_ljlk_backward": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "tmol_b200_ljlk_forward_speculative": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "tmol_b200_ljlk_backward_speculative": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p],
    ),
    "tmol_b200_ljlk_energy_and_gradient": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "tmol_b200_ljlk_plan_set_counting": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "tmol_b200_ljlk_last_counts": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)],
    ),
    "tmol_b200_ljlk_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "tmol_b200_ljlk_profile_read": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32)],
    ),
    "tmol_b200_ljlk_plan_device_bytes": (ctypes.c_int64, [ctypes.c_void_p]),
    "tmol_b200_measure_fp32_peak": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    "tmol_b200_ljlk_block_neighbors_noalloc": (
        ctypes.c_int,
        [
            ctypes.c_void_p,
            ctypes.c_int64,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_int32,
            ctypes.c_int32,
            ctypes.c_int32,
            ctypes.c_double,
            ctypes.c_void_p,
            ctypes.c_void_p,
        ],
    ),
    "tmol_b200_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    # rotamer scoring
    "tmol_b200_ljlk_rotamer_plan_create": (
        ctypes.c_int,
        [ctypes.POINTER(Inputs), ctypes.c_int, ctypes.POINTER(Launch), ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)],
    ),
    "tmol_b200_ljlk_rotamer_count": (
        ctypes.c_int, [_V, _V, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64), _V]
    ),
    "tmol_b200_ljlk_rotamer_fill": (ctypes.c_int, [_V, _V, _V, _V]),
    "tmol_b200_ljlk_rotamer_forward": (ctypes.c_int, [_V, _V, _V, _I64, _I64, _V, _V]),
    "tmol_b200_ljlk_rotamer_backward": (ctypes.c_int, [_V, _V, _V, _I64, _I64, _V, _V, _V]),
    # elec (include/tmol_b200_elec.h)
    "tmol_b200_elec_plan_create": (
        ctypes.c_int,
        [ctypes.POINTER(ElecInputs), ctypes.c_int, ctypes.POINTER(Launch), _V, ctypes.POINTER(ctypes.c_void_p)],
    ),
    "tmol_b200_elec_rotamer_plan_create": (
        ctypes.c_int,
        [ctypes.POINTER(ElecInputs), ctypes.c_int, ctypes.POINTER(Launch), _V, ctypes.POINTER(ctypes.c_void_p)],
    ),
    "tmol_b200_elec_plan_destroy": (ctypes.c_int, [_V]),
    "tmol_b200_elec_forward": (ctypes.c_int, [_V, _V, ctypes.c_int, _V, _V, _V]),
    "tmol_b200_elec_backward": (ctypes.c_int, [_V, _V, ctypes.c_int, _V, _V, _V]),
    "tmol_b200_elec_energy_and_gradient": (ctypes.c_int, [_V, _V, _V, _V, _V, _V]),
    "tmol_b200_elec_forward_speculative": (ctypes.c_int, [_V, _V, _V, _V, _V]),
    "tmol_b200_elec_backward_speculative": (ctypes.c_int, [_V, _V, _V, _V, ctypes.c_int, _V]),
    "tmol_b200_elec_rotamer_count": (
        ctypes.c_int, [_V, _V, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64), _V]
    ),
    "tmol_b200_elec_rotamer_fill": (ctypes.c_int, [_V, _V, _V, _V]),
    "tmol_b200_elec_rotamer_forward": (ctypes.c_int, [_V, _V, _V, _I64, _I64, _V, _V]),
    "tmol_b200_elec_rotamer_backward": (ctypes.c_int, [_V, _V, _V, _I64, _I64, _V, _V, _V]),
    # LK-ball (include/tmol_b200_lkball.h)
    "tmol_b200_lkball_plan_create": (
        ctypes.c_int,
        [ctypes.POINTER(LKBallInputs), ctypes.c_int, ctypes.POINTER(Launch), _V, ctypes.POINTER(ctypes.c_void_p)],
    ),
    "tmol_b200_lkball_plan_destroy": (ctypes.c_int, [_V]),
    "tmol_b200_lkball_waters": (ctypes.c_int, [_V, _V, _V, _V]),
    "tmol_b200_lkball_waters_backward": (ctypes.c_int, [_V, _V, _V, _V, _V]),
    "tmol_b200_lkball_forward": (ctypes.c_int, [_V, _V, _V, ctypes.c_int, _V, _V, _V]),
    "tmol_b200_lkball_backward": (ctypes.c_int, [_V, _V, _V, ctypes.c_int, _V, _V, _V, _V]),
    "tmol_b200_lkball_forward_speculative": (ctypes.c_int, [_V, _V, _V, _V, _V, _V]),
    "tmol_b200_lkball_backward_speculative": (ctypes.c_int, [_V, _V, _V, _V, _V, _V, ctypes.c_int, _V]),
    "tmol_b200_lkball_energy_and_gradient": (ctypes.c_int, [_V, _V, _V, _V, _V, _V]),
    "tmol_b200_lkball_plan_create_from_connectivity": (
        ctypes.c_int,
        [
            ctypes.POINTER(LKBallInputs), ctypes.POINTER(PoseConnectivity), ctypes.c_int, ctypes.POINTER(Launch), _V,
            ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
        ],
    ),
    "tmol_b200_lkball_rotamer_plan_create": (
        ctypes.c_int,
        [ctypes.POINTER(LKBallInputs), ctypes.c_int, ctypes.POINTER(Launch), _V, ctypes.POINTER(ctypes.c_void_p)],
    ),
    "tmol_b200_lkball_rotamer_count": (
        ctypes.c_int, [_V, _V, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64), _V]
    ),
    "tmol_b200_lkball_rotamer_fill": (ctypes.c_int, [_V, _V, _V, _V]),
    "tmol_b200_lkball_rotamer_forward": (ctypes.c_int, [_V, _V, _V, _V, _I64, _I64, _V, _V]),
    "tmol_b200_lkball_rotamer_backward": (ctypes.c_int, [_V, _V, _V, _V, _I64, _I64, _V, _V, _V, _V]),
    # PoseStack construction (include/tmol_b200_pose.h)
    "tmol_b200_pose_bondsep": (ctypes.c_int, [ctypes.POINTER(PoseConnectivity), _V, _V, _V, _V]),
    "tmol_b200_apsp_stacked": (ctypes.c_int, [_V, _I32, _I32, _I32, _V]),
    "tmol_b200_ljlk_plan_create_from_connectivity": (
        ctypes.c_int,
        [
            ctypes.POINTER(Inputs), ctypes.POINTER(PoseConnectivity), ctypes.c_int, ctypes.POINTER(Launch), _V,
            ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
        ],
    ),
    "tmol_b200_elec_plan_create_from_connectivity": (
        ctypes.c_int,
        [
            ctypes.POINTER(ElecInputs), ctypes.POINTER(PoseConnectivity), ctypes.c_int, ctypes.POINTER(Launch), _V,
            ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
        ],
    ),
    # learned block-pair screen (include/tmol_b200_screen.h)
    "tmol_b200_ljlk_plan_set_skip_mask": (ctypes.c_int, [_V, _V, _I32]),
    "tmol_b200_ljlk_screen_candidates": (ctypes.c_int, [_V, _V, _I32, _V, _V, _V, _V, _V, _V]),
    "tmol_b200_screen_infer": (
        ctypes.c_int,
        [ctypes.POINTER(ScreenWeights), _V, _V, _V, _V, _V, _I32, _F, _V, _I32, _I64, _V, _V],
    ),
    "tmol_b200_screen_gemm": (
        ctypes.c_int,
        [_V, _I64, _I64, _V, _I64, _I64, _V, _I64, _V, _I64, _V, _I32, _I32, _I32, _I32, _I32, _I32, _V],
    ),
    "tmol_b200_screen_relu_backward": (ctypes.c_int, [_V, _V, _V, _V, _I64, _V]),
    "tmol_b200_screen_col_sum": (ctypes.c_int, [_V, _I64, _I32, _V, _V]),
    "tmol_b200_screen_pinball": (ctypes.c_int, [_V, _V, _I64, _F, _V, _V, _V, _V]),
    "tmol_b200_screen_adam": (ctypes.c_int, [_V, _V, _V, _V, _V, _I64, _F, _F, _F, _F, _I32, _F, _V]),
    "tmol_b200_screen_assemble_features": (ctypes.c_int, [_V, _V, _V, _I64, _V, _V]),
    "tmol_b200_screen_embedding_backward": (ctypes.c_int, [_V, _V, _I64, _V, _V]),
}

_lib = None


class NativeError(RuntimeError):
    def __init__(self, func, status, text):
        super().__init__(f"{func} failed with status {status}: {text}")
        self.status = status


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"the tmol_b200 CUDA library is not built ({LIB_PATH} is missing); "
                "run `python -m tmol_b200.build`"
            )
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def check(func, status):
    if status != 0:
        text = load().tmol_b200_status_string(status).decode()
        raise NativeError(func, status, text)


def call(name, *args):
    lib = load()
    check(name, getattr(lib, name)(*args))


def measure_fp32_peak_tflops(stream_handle=0):
    """Device FP32 FMA throughput in TFLOP/s (see the C declaration)."""
    v = ctypes.c_double()
    call("tmol_b200_measure_fp32_peak", ctypes.c_void_p(stream_handle), ctypes.byref(v))
    return v.value
