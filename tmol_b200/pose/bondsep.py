"""PoseStack construction steps on the GPU: inter-block bond separation
from the connectivity, and tmol's stacked all-pairs-shortest-paths op.

``pose_bondsep(pose_stack)`` returns ``(inter_block_bondsep [P, B, B, C, C],
min_bondsep [P, B, B])`` as tmol's ``PoseStackBuilder`` and
``BondDependentTerm`` compute them (``tmol/pose/pose_stack_builder.py:436-599,
1230-1343``; ``tmol/score/bond_dependent_term.py:91-100``), from one bounded
search per connection point on the device (``include/tmol_b200_pose.h``).
``stacked_apsp(weights, threshold=-1)`` is tmol's
``tmol.pose.compiled.apsp_ops.stacked_apsp`` (in place on int32 CUDA weights
``[G, N, N]``, -1 = no edge), with the CPU implementation's cutoff rule on
the GPU.  ``connectivity(pose_stack)`` is the C struct that plan creation
from connectivity takes (``LJLKPlan(..., connectivity=...)``).  CUDA tensors
only; there is no CPU path.
"""

import ctypes

import torch

from .. import native


def _i32(t, device):
    if t.device != device:
        raise RuntimeError(f"tensor on {t.device}, expected {device}")
    return t.to(torch.int32).contiguous()


def connectivity(block_type_ind, inter_residue_connections, bt_n_conn, bt_conn_sep):
    """(struct, tensors to keep alive) for ``tmol_b200_pose_connectivity``."""
    device = block_type_ind.device
    if device.type != "cuda":
        raise RuntimeError("tmol_b200 bond separation runs on CUDA tensors only")
    keep = [_i32(t, device) for t in (block_type_ind, inter_residue_connections, bt_n_conn, bt_conn_sep)]
    bti, irc, nc, cs = keep
    P, B = bti.shape
    C = cs.shape[1]
    if tuple(irc.shape) != (P, B, C, 2):
        raise ValueError(f"inter_residue_connections must be [{P}, {B}, {C}, 2]")
    if tuple(cs.shape) != (nc.shape[0], C, C):
        raise ValueError(f"conn_at_intrablock_bond_sep must be [{nc.shape[0]}, {C}, {C}]")
    s = native.PoseConnectivity(P, B, nc.shape[0], C, bti.data_ptr(), irc.data_ptr(), nc.data_ptr(), cs.data_ptr())
    return s, keep


def pose_connectivity(pose_stack):
    pbt = pose_stack.packed_block_types
    return connectivity(
        pose_stack.block_type_ind, pose_stack.inter_residue_connections, pbt.n_conn, pbt.conn_at_intrablock_bond_sep
    )


def bondsep_from_connectivity(block_type_ind, inter_residue_connections, bt_n_conn, bt_conn_sep, dense=True,
                              check=True, out=None):
    """(inter_block_bondsep or None, min_bondsep).  With ``check`` the
    device status is read (one synchronisation) and a bad connectivity
    raises ``NativeError``; without, the status tensor is returned third
    for the caller to read.  ``out`` = (ibb or None, min_bondsep, status)
    reuses buffers."""
    s, keep = connectivity(block_type_ind, inter_residue_connections, bt_n_conn, bt_conn_sep)
    device = block_type_ind.device
    P, B, C = s.n_poses, s.max_n_blocks, s.max_n_conn
    if out is None:
        ibb = torch.empty((P, B, B, C, C), dtype=torch.int32, device=device) if dense else None
        mb = torch.empty((P, B, B), dtype=torch.int32, device=device)
        status = torch.empty(1, dtype=torch.int32, device=device)
    else:
        ibb, mb, status = out
    with torch.cuda.device(device):
        stream = torch.cuda.current_stream(device).cuda_stream
        native.call(
            "tmol_b200_pose_bondsep",
            ctypes.byref(s),
            ctypes.c_void_p(ibb.data_ptr() if ibb is not None else 0),
            ctypes.c_void_p(mb.data_ptr()),
            ctypes.c_void_p(status.data_ptr()),
            ctypes.c_void_p(stream),
        )
    del keep
    if not check:
        return ibb, mb, status
    native.check("tmol_b200_pose_bondsep", int(status.item()))
    return ibb, mb


def pose_bondsep(pose_stack, dense=True):
    pbt = pose_stack.packed_block_types
    return bondsep_from_connectivity(
        pose_stack.block_type_ind,
        pose_stack.inter_residue_connections,
        pbt.n_conn,
        pbt.conn_at_intrablock_bond_sep,
        dense,
    )


def stacked_apsp(weights, threshold=-1):
    """Drop-in for tmol's ``stacked_apsp`` (``tmol/pose/compiled/apsp_ops.py:17-33``):
    all-pairs shortest paths of every graph of ``weights`` [G, N, N] (int32,
    CUDA, -1 = no edge), in place; with a threshold, the CPU op's rule
    (symmetrised edges below it, every farther or unreachable pair at it)."""
    if not isinstance(weights, torch.Tensor) or weights.device.type != "cuda":
        raise RuntimeError("tmol_b200 stacked_apsp runs on CUDA tensors only")
    if weights.dtype != torch.int32 or weights.dim() != 3 or weights.shape[1] != weights.shape[2]:
        raise ValueError("weights must be an int32 [n_graphs, n_nodes, n_nodes] tensor")
    if not weights.is_contiguous():
        raise ValueError("weights must be contiguous (the op works in place)")
    with torch.cuda.device(weights.device):
        stream = torch.cuda.current_stream(weights.device).cuda_stream
        native.call(
            "tmol_b200_apsp_stacked",
            ctypes.c_void_p(weights.data_ptr()),
            int(weights.shape[0]),
            int(weights.shape[1]),
            int(threshold),
            ctypes.c_void_p(stream),
        )
    return weights
