"""The drop-in ops registered with torch's dispatcher (tmol_b200.score.
torch_ops), on the CPU: their schemas against the reference's own
registrations (compiled into oracle/_ref; the reference registers them by
function pointer, so its schemas carry types and positions but no names),
the opt-in alias's refusal when tmol's own extension is loaded, and the
error on CPU tensors (the ops run on CUDA only)."""

import pytest
import torch

from oracle import oracle as O
from tmol_b200.score import torch_ops


def _types(schema):
    return [str(a.type) for a in schema.arguments], [str(r.type) for r in schema.returns]


def _reference_libraries():
    loaded = []
    if O.reference_available():
        O.load_reference()
        loaded.append("tmol_ljlk")
    if O.reference_elec_available():
        torch.ops.load_library(O.ELEC_REF_LIB)
        loaded.append("tmol_elec")
    if O.reference_lkball_available():
        torch.ops.load_library(O.LKBALL_REF_LIB)
        loaded.append("tmol_lk_ball")
    return loaded


def test_schemas_match_the_reference_registrations():
    loaded = _reference_libraries()
    if not loaded:
        pytest.skip("reference ops not built")
    for ns in loaded:
        for name, *_ in torch_ops.OPS[ns]:
            ref = getattr(getattr(torch.ops, ns), name).default._schema
            ours = getattr(torch.ops.tmol_b200, name).default._schema
            assert _types(ours) == _types(ref), name


def test_reference_aliases_refuse_a_loaded_extension():
    if "tmol_ljlk" not in _reference_libraries():
        pytest.skip("reference op not built")
    with pytest.raises(RuntimeError, match="tmol's own extension is loaded"):
        torch_ops.register_reference_aliases()


def test_cpu_tensors_are_refused():
    from tmol_b200.pose.synthetic import synthetic_pose_stack
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm, pose_score_args

    ps = synthetic_pose_stack([5, 3], [1, 2])
    with pytest.raises(RuntimeError, match="CUDA tensors only"):
        torch.ops.tmol_b200.ljlk_pose_scores(ps.coords.flatten(0, 1), *pose_score_args(ps, LJLKEnergyTerm()))
