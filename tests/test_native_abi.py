"""The C-ABI library loads and exports every function include/ declares.

No GPU work is done here: only host-side entry points are called."""

import ctypes
import os
import re

import pytest

from tmol_b200 import native

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_functions():
    names = []
    inc = os.path.join(ROOT, "include")
    for fn in sorted(os.listdir(inc)):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(inc, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(tmol_b200_\w+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "tmol_b200_ljlk_forward" in names and "tmol_b200_ljlk_backward" in names


def test_library_exports_every_declared_symbol():
    lib = native.load()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_binding_covers_header():
    assert set(declared_functions()) <= set(native.SIGNATURES)


def test_status_strings_and_argument_checks():
    lib = native.load()
    assert lib.tmol_b200_status_string(0) == b"ok"
    assert b"index" in lib.tmol_b200_status_string(3)
    out = ctypes.c_void_p()
    # null inputs are rejected before any device work
    assert lib.tmol_b200_ljlk_plan_create(None, 4, None, None, ctypes.byref(out)) == 1
    s = native.Inputs()
    assert lib.tmol_b200_ljlk_plan_create(ctypes.byref(s), 3, None, None, ctypes.byref(out)) == 6
    s.max_n_conn = 5
    assert lib.tmol_b200_ljlk_plan_create(ctypes.byref(s), 4, None, None, ctypes.byref(out)) == 2
    assert lib.tmol_b200_ljlk_plan_destroy(None) == 1
    assert lib.tmol_b200_ljlk_forward(None, None, 0, None, None, None) == 1
    assert lib.tmol_b200_ljlk_plan_device_bytes(None) == -1
    assert lib.tmol_b200_ljlk_plan_set_counting(None, 1) == 1
    # the elec entry points check their arguments the same way
    assert lib.tmol_b200_elec_plan_create(None, 4, None, None, ctypes.byref(out)) == 1
    e = native.ElecInputs()
    assert lib.tmol_b200_elec_plan_create(ctypes.byref(e), 3, None, None, ctypes.byref(out)) == 6
    e.max_n_conn = 5
    assert lib.tmol_b200_elec_plan_create(ctypes.byref(e), 4, None, None, ctypes.byref(out)) == 2
    assert lib.tmol_b200_elec_plan_destroy(None) == 1
    assert lib.tmol_b200_elec_forward(None, None, 0, None, None, None) == 1
    assert lib.tmol_b200_elec_rotamer_fill(None, None, None, None) == 1
    # and the LK-ball ones: a plan needs the water or the scoring tables
    assert lib.tmol_b200_lkball_plan_create(None, 4, None, None, ctypes.byref(out)) == 1
    k = native.LKBallInputs()
    assert lib.tmol_b200_lkball_plan_create(ctypes.byref(k), 4, None, None, ctypes.byref(out)) == 1
    assert lib.tmol_b200_lkball_rotamer_plan_create(ctypes.byref(k), 4, None, None, ctypes.byref(out)) == 1
    assert lib.tmol_b200_lkball_plan_destroy(None) == 1
    assert lib.tmol_b200_lkball_waters(None, None, None, None) == 1
    assert lib.tmol_b200_lkball_forward(None, None, None, 0, None, None, None) == 1
    assert lib.tmol_b200_lkball_energy_and_gradient(None, None, None, None, None, None) == 1
    assert lib.tmol_b200_lkball_rotamer_fill(None, None, None, None) == 1


def test_op_refuses_cpu_tensors(ubq_pose_stack, term):
    import torch
    from tmol_b200.score.ljlk_energy_term import pose_score_args
    from tmol_b200.score.ljlk_op import ljlk_pose_scores

    args = pose_score_args(ubq_pose_stack, term)
    with pytest.raises(RuntimeError, match="CUDA"):
        ljlk_pose_scores(ubq_pose_stack.coords.flatten(0, 1), *args)


def test_autotuner_block_size_summary():
    """The autotuner's cache key summarises the PoseStack's blocks: real
    blocks per pose, mean atoms per block, the share of blocks per size bin."""
    import types

    import torch

    from tmol_b200.tune import SIZE_BINS, block_size_summary

    bt = torch.tensor([[0, 1, 2, -1], [2, 2, -1, -1]])
    n_atoms = torch.tensor([7, 20, 40])
    per_pose, mean, hist = block_size_summary(types.SimpleNamespace(block_sizes=(bt, n_atoms), n_poses=2))
    assert per_pose == 2.5 and abs(mean - (7 + 20 + 40 + 40 + 40) / 5) < 1e-5
    assert len(hist) == len(SIZE_BINS) + 1 and abs(sum(hist) - 1) < 1e-6
    assert abs(hist[0] - 0.2) < 1e-6 and abs(hist[2] - 0.2) < 1e-6 and abs(hist[-1] - 0.6) < 1e-6
