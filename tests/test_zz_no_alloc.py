"""The block-neighbour entry point that allocates no device memory.

Some callers of this library may not allocate GPU memory while they run
(code inside a memory pool it does not own, or a loop that must never enter
the allocator).  tmol_b200_ljlk_block_neighbors_noalloc serves them: its
only scratch is a fixed array inside the library.  These tests call it
through the C ABI and compare it with the neighbour matrix of the scoring
path (tmol_b200_ljlk_forward), which must agree bit for bit.  The file name
makes pytest collect it last.
"""

import ctypes

import numpy
import pytest
import torch

from tmol_b200 import native
from tmol_b200.pose.synthetic import synthetic_pose_stack
from tmol_b200.score.ljlk_energy_term import pose_score_args
from tmol_b200.score.ljlk_op import LJLKPlan

MAX_BLOCKS = 1 << 18


def _noalloc(coords, block_type, block_coord_offset, bt_n_atoms, P, B, max_dis, out, stream):
    lib = native.load()
    return lib.tmol_b200_ljlk_block_neighbors_noalloc(
        ctypes.c_void_p(coords.data_ptr() if coords is not None else 0),
        coords.shape[0] if coords is not None else 0,
        ctypes.c_void_p(block_type.data_ptr() if block_type is not None else 0),
        ctypes.c_void_p(block_coord_offset.data_ptr() if block_coord_offset is not None else 0),
        ctypes.c_void_p(bt_n_atoms.data_ptr() if bt_n_atoms is not None else 0),
        bt_n_atoms.shape[0] if bt_n_atoms is not None else 0,
        P,
        B,
        max_dis,
        ctypes.c_void_p(out.data_ptr() if out is not None else 0),
        ctypes.c_void_p(stream),
    )


def test_rejects_inputs_beyond_the_fixed_scratch():
    # checked before any GPU work, so no device is needed
    rc = _noalloc(None, None, None, None, 1, MAX_BLOCKS + 1, 6.0, None, 0)
    assert rc == 4  # TMOL_B200_ERR_CAPACITY
    assert native.load().tmol_b200_status_string(rc) == b"fixed-capacity table overflow"


@pytest.mark.gpu
def test_noalloc_neighbors_match_the_scoring_path(term):
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev).cuda_stream
    # two calls in a row on different batches: the second must not see the
    # first call's scratch contents
    for sizes, seed in (([150, 40, 7, 300, 1], 30), ([20, 3], 40)):
        ps = synthetic_pose_stack(sizes, [seed + k for k in range(len(sizes))])
        args = [a.to(dev) if isinstance(a, torch.Tensor) else a for a in pose_score_args(ps, term)]
        coords = ps.coords.flatten(0, 1).to(dev).contiguous()
        plan = LJLKPlan(coords, args[:-1])
        _, nbr_ref = plan.forward(coords, block_pair=False, want_neighbors=True)
        P, B = ps.n_poses, ps.max_n_blocks
        out = torch.full((P, B, B), -7, dtype=torch.int32, device=dev)
        rc = _noalloc(
            coords,
            args[3].contiguous(),  # first_rot_block_type
            args[0].contiguous(),  # rot_coord_offset
            args[14].contiguous(),  # block-type atom counts
            P,
            B,
            float(args[24]),
            out,
            stream,
        )
        assert rc == 0, native.load().tmol_b200_status_string(rc)
        torch.cuda.synchronize()
        assert numpy.array_equal(out.cpu().numpy(), nbr_ref.cpu().numpy())

        # the promise itself: once the first call has loaded the module, a
        # call leaves the device's free memory and torch's allocations as
        # they were (everything it touches is allocated above)
        free0, _ = torch.cuda.mem_get_info(dev)
        torch_bytes0 = torch.cuda.memory_allocated(dev)
        rc = _noalloc(
            coords, args[3].contiguous(), args[0].contiguous(), args[14].contiguous(),
            P, B, float(args[24]), out, stream,
        )
        torch.cuda.synchronize()
        assert rc == 0
        assert torch.cuda.mem_get_info(dev)[0] == free0
        assert torch.cuda.memory_allocated(dev) == torch_bytes0
        assert numpy.array_equal(out.cpu().numpy(), nbr_ref.cpu().numpy())
