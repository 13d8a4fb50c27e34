"""NumPy restatement of the block-pair screen: candidate features, the MLP's
forward and backward passes and the pinball loss.

Test infrastructure only: tests import this module as the checker of the
GPU screen kernels (``tmol_b200/csrc/screen.cu`` and the candidate kernel in
``tmol_b200/csrc/ljlk.cu``).  The product never does.

The screen has no counterpart in the reference (tmol scores every block
pair whose bounding spheres are within reach,
tmol/score/common/sphere_overlap.impl.hh:287-351), so this oracle is pinned
by float64 central finite differences of its own backward pass, not by
reference outputs.  ``bf16=True`` rounds weights and activations to
bfloat16 at the same points as the GPU kernels (round to nearest even), so
GPU gradients can be compared with it at a tolerance set by fp32
accumulation order; ``bf16=False`` computes in float64 throughout, for the
finite-difference check.
"""

import numpy

N_IN, HID, EMB, N_SCAL = 32, 128, 10, 12


def to_bf16(x):
    """Round float32 values to the nearest bfloat16 (ties to even), returned
    as float32.  Keeps the top 16 bits after adding half an ulp of the kept
    part (plus the kept part's lowest bit, for ties)."""
    a = numpy.ascontiguousarray(numpy.asarray(x, dtype=numpy.float32))
    u = a.view(numpy.uint32).astype(numpy.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(numpy.uint32).view(numpy.float32).reshape(a.shape)


class MLP:
    """Parameters as a dict of arrays (torch Linear layout), see
    ``tmol_b200.screen.mlp``."""

    def __init__(self, params, bf16=True):
        self.bf16 = bf16
        dt = numpy.float64
        self.p = {k: numpy.asarray(v, dtype=numpy.float32 if bf16 else dt) for k, v in params.items()}

    def _r(self, x):
        # rounding point of the GPU path
        if self.bf16:
            return to_bf16(x).astype(numpy.float64)
        return numpy.asarray(x, dtype=numpy.float64)

    def _f32(self, x):
        return numpy.asarray(x, dtype=numpy.float32).astype(numpy.float64) if self.bf16 else x

    def inputs(self, features, pair_bt):
        emb = self.p["emb"]
        x = numpy.concatenate(
            [numpy.asarray(features, numpy.float64), emb[pair_bt[:, 0]].astype(numpy.float64),
             emb[pair_bt[:, 1]].astype(numpy.float64)],
            axis=1,
        )
        return self._r(x)

    def forward(self, features, pair_bt):
        """Predictions [n]; keeps the activations for backward()."""
        p = self.p
        X = self.inputs(features, pair_bt)
        W = {k: self._r(p[k]) for k in ("w1", "w2", "w3", "w4")}
        H1 = self._r(numpy.maximum(self._f32(X @ W["w1"].T + p["b1"]), 0))
        H2 = self._r(numpy.maximum(self._f32(H1 @ W["w2"].T + p["b2"]), 0))
        H3 = self._r(numpy.maximum(self._f32(H2 @ W["w3"].T + p["b3"]), 0))
        pred = self._f32(H3 @ W["w4"].T + p["b4"])[:, 0]
        self.cache = (numpy.asarray(pair_bt), X, H1, H2, H3, W)
        return pred

    def backward(self, dpred):
        """Gradients of sum(dpred * pred) for the last forward()."""
        bt, X, H1, H2, H3, W = self.cache
        g = {}
        dpred = numpy.asarray(dpred, numpy.float64)
        dpb = self._r(dpred)
        g["w4"] = (dpb[None, :] @ H3)
        g["b4"] = numpy.array([dpred.sum()])
        dH = self._f32(dpb[:, None] * W["w4"])
        for wname, bname, H, Hin in (("w3", "b3", H3, H2), ("w2", "b2", H2, H1), ("w1", "b1", H1, X)):
            dZ = numpy.where(H > 0, dH, 0.0)
            dZb = self._r(dZ)
            g[wname] = dZb.T @ Hin
            g[bname] = dZ.sum(0)
            dH = self._f32(dZb @ W[wname])
        dX = dH
        gemb = numpy.zeros(self.p["emb"].shape, numpy.float64)
        numpy.add.at(gemb, bt[:, 0], dX[:, N_SCAL:N_SCAL + EMB])
        numpy.add.at(gemb, bt[:, 1], dX[:, N_SCAL + EMB:])
        g["emb"] = gemb
        return g


def pinball(pred, y, tau):
    """Mean pinball loss and its gradient with respect to pred."""
    r = numpy.asarray(y, numpy.float64) - numpy.asarray(pred, numpy.float64)
    n = len(r)
    loss = numpy.where(r >= 0, tau * r, (tau - 1.0) * r).mean()
    d = numpy.where(r >= 0, -tau, 1.0 - tau) / n
    return loss, d


def _sphere(x):
    c = x.mean(0)
    return c, numpy.sqrt(((x - c) ** 2).sum(1).max())


def candidate_features(coords, block_type, block_offset, bt_n_atoms, nbr, min_bondsep, pose_index):
    """Candidates and features of one pose, as the candidate kernel defines
    them: pairs b1 < b2 with nbr[b1, b2] != 0 and min_bondsep > 4.
    Returns (pairs [n, 2] sorted, features [n, 12] float64).  Sub-spheres:
    atoms [0, 4) and [4, n) (the first part again when n <= 4)."""
    B = block_type.shape[0]
    cen = numpy.zeros((B, 3))
    rad = numpy.zeros(B)
    first = numpy.zeros((B, 3))
    sub = numpy.zeros((B, 2, 4))
    for b in range(B):
        if block_type[b] < 0:
            continue
        x = numpy.asarray(coords[block_offset[b]:block_offset[b] + bt_n_atoms[block_type[b]]], numpy.float64)
        cen[b], rad[b] = _sphere(x)
        first[b] = x[0]
        head = x[: min(4, len(x))]
        tail = x[4:] if len(x) > 4 else head
        for part, xs in enumerate((head, tail)):
            c, r = _sphere(xs)
            sub[b, part, :3] = c
            sub[b, part, 3] = r
    b1, b2 = numpy.nonzero(numpy.triu(nbr, 1) & (min_bondsep > 4))
    d = numpy.linalg.norm(cen[b1] - cen[b2], axis=1)
    cols = [
        d / 10,
        (d - rad[b1] - rad[b2]) / 6,
        rad[b1] / 5,
        rad[b2] / 5,
        numpy.log2(numpy.maximum(b2 - b1, 1)) / 10,
        (numpy.linalg.norm(first[b1] - first[b2], axis=1) - d) / 5,
        (numpy.linalg.norm(first[b1] - cen[b2], axis=1) - d) / 5,
        (numpy.linalg.norm(first[b2] - cen[b1], axis=1) - d) / 5,
    ]
    for i in range(2):
        for j in range(2):
            u, v = sub[b1, i], sub[b2, j]
            cols.append((numpy.linalg.norm(u[:, :3] - v[:, :3], axis=1) - u[:, 3] - v[:, 3]) / 6)
    return numpy.stack([b1, b2], axis=1), numpy.stack(cols, axis=1)
