"""The screen network: 32 -> 128 -> 128 -> 128 -> 1 (ReLU), bf16 weights and
activations, fp32 accumulation, trained with a pinball (quantile) loss and
Adam.  Every step runs on the library's own kernels; torch only holds the
buffers.

Input row (32 values): the 12 candidate features of
``tmol_b200_ljlk_screen_candidates`` followed by the 10-value embeddings of
the two block types.
"""

import ctypes
import math

import numpy
import torch

from .. import native

N_IN, HID, EMB, N_SCAL = 32, 128, 10, 12
PARAM_NAMES = ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4", "emb")
BF16_COPIES = ("w1", "w2", "w3", "w4")


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


class ScreenMLP:
    """Parameters (fp32 masters, bf16 copies of the weight matrices), Adam
    state and the training / inference passes."""

    def __init__(self, n_block_types, device, seed=0):
        self.device = torch.device(device)
        self.n_block_types = int(n_block_types)
        g = torch.Generator().manual_seed(seed)

        def randn(*shape, scale):
            return (torch.randn(*shape, generator=g) * scale).to(self.device)

        self.params = {
            "w1": randn(HID, N_IN, scale=math.sqrt(2.0 / N_IN)),
            "b1": torch.zeros(HID, device=self.device),
            "w2": randn(HID, HID, scale=math.sqrt(2.0 / HID)),
            "b2": torch.zeros(HID, device=self.device),
            "w3": randn(HID, HID, scale=math.sqrt(2.0 / HID)),
            "b3": torch.zeros(HID, device=self.device),
            "w4": randn(1, HID, scale=math.sqrt(1.0 / HID)),
            "b4": torch.zeros(1, device=self.device),
            "emb": randn(self.n_block_types, EMB, scale=0.3),
        }
        self.bf16 = {k: self.params[k].to(torch.bfloat16) for k in BF16_COPIES}
        self.grads = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.adam_m = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.adam_v = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.step = 0
        self._buf = {}
        self._weights_struct = None

    # -- parameters ------------------------------------------------------

    def refresh_bf16(self):
        for k in BF16_COPIES:
            self.bf16[k].copy_(self.params[k])

    def state_dict(self):
        return {k: v.detach().cpu().numpy() for k, v in self.params.items()}

    def load_state_dict(self, state):
        for k in PARAM_NAMES:
            v = torch.as_tensor(numpy.asarray(state[k]), dtype=torch.float32)
            if tuple(v.shape) != tuple(self.params[k].shape):
                raise ValueError(f"{k}: shape {tuple(v.shape)}, expected {tuple(self.params[k].shape)}")
            self.params[k].copy_(v.to(self.device))
        self.refresh_bf16()

    @classmethod
    def load(cls, path, device, block_type_names=None):
        """A trained network from ``path`` (written by
        ``tmol_b200.screen.train``) and its calibrated skip threshold.  With
        ``block_type_names``, checks that the embedding rows follow the same
        block-type order."""
        st = dict(numpy.load(path, allow_pickle=False))
        names = [str(v) for v in st["block_type_names"]]
        if block_type_names is not None and list(block_type_names) != names:
            raise ValueError("the screen's block-type order differs from the packed block types")
        net = cls(len(names), device)
        net.load_state_dict(st)
        return net, float(st["threshold"])

    def weights_struct(self):
        w = native.ScreenWeights()
        for k in BF16_COPIES:
            setattr(w, k, self.bf16[k].data_ptr())
        for k in ("b1", "b2", "b3", "b4", "emb"):
            setattr(w, k, self.params[k].data_ptr())
        return w

    # -- buffers ---------------------------------------------------------

    def _buffers(self, n):
        if self._buf.get("n", 0) < n:
            d, bf, f32 = self.device, torch.bfloat16, torch.float32
            self._buf = dict(
                n=n,
                X=torch.empty((n, N_IN), dtype=bf, device=d),
                H1=torch.empty((n, HID), dtype=bf, device=d),
                H2=torch.empty((n, HID), dtype=bf, device=d),
                H3=torch.empty((n, HID), dtype=bf, device=d),
                pred=torch.empty(n, dtype=f32, device=d),
                dpred=torch.empty(n, dtype=f32, device=d),
                dpred_b=torch.empty(n, dtype=bf, device=d),
                dH=torch.empty((n, HID), dtype=f32, device=d),
                dZ=torch.empty((n, HID), dtype=f32, device=d),
                dZb=torch.empty((n, HID), dtype=bf, device=d),
                dX=torch.empty((n, N_IN), dtype=f32, device=d),
                loss=torch.zeros(1, dtype=f32, device=d),
            )
        return self._buf

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    @staticmethod
    def _gemm(st, A, a_rs, a_cs, B, b_rs, b_cs, M, N, K, C=None, c_rs=0, Cb=None, cb_rs=0, bias=None,
              relu=False, accumulate=False, k_split=1):
        native.call(
            "tmol_b200_screen_gemm",
            _p(A), a_rs, a_cs, _p(B), b_rs, b_cs, _p(C), c_rs, _p(Cb), cb_rs, _p(bias),
            M, N, K, int(relu), int(accumulate), int(k_split), st,
        )

    # -- passes ----------------------------------------------------------

    def forward(self, features, pair_bt, n=None):
        """Predictions [n] (fp32) for the first n rows; keeps the bf16
        activations for backward()."""
        n = features.shape[0] if n is None else n
        b = self._buffers(max(n, 1))
        st = self._stream()
        P, W = self.params, self.bf16
        native.call(
            "tmol_b200_screen_assemble_features", _p(features), _p(pair_bt), _p(P["emb"]), n, _p(b["X"]), st
        )
        # H = relu(X W^T + b): B(k, n) = W[n, k]
        self._gemm(st, b["X"], N_IN, 1, W["w1"], 1, N_IN, n, HID, N_IN, Cb=b["H1"], cb_rs=HID, bias=P["b1"], relu=True)
        self._gemm(st, b["H1"], HID, 1, W["w2"], 1, HID, n, HID, HID, Cb=b["H2"], cb_rs=HID, bias=P["b2"], relu=True)
        self._gemm(st, b["H2"], HID, 1, W["w3"], 1, HID, n, HID, HID, Cb=b["H3"], cb_rs=HID, bias=P["b3"], relu=True)
        self._gemm(st, b["H3"], HID, 1, W["w4"], 1, HID, n, 1, HID, C=b["pred"], c_rs=1, bias=P["b4"])
        self._n = n
        self._bt = pair_bt
        return b["pred"][:n]

    def loss_and_backward(self, target, tau):
        """Mean pinball loss of the last forward() against `target` [n] at
        quantile tau; fills self.grads (overwriting) and returns the loss as
        a device tensor."""
        n = self._n
        b = self._buf
        st = self._stream()
        W = self.bf16
        for g in self.grads.values():
            g.zero_()
        b["loss"].zero_()
        native.call(
            "tmol_b200_screen_pinball",
            _p(b["pred"]), _p(target), n, ctypes.c_float(tau), _p(b["dpred"]), _p(b["dpred_b"]), _p(b["loss"]), st,
        )
        self._backward_from_dpred(st, n)
        return b["loss"]

    def backward(self, dpred):
        """Gradients (into self.grads, overwriting) of sum(dpred * pred) for
        the last forward()."""
        n = self._n
        b = self._buf
        for g in self.grads.values():
            g.zero_()
        b["dpred"][:n].copy_(dpred[:n])
        b["dpred_b"][:n].copy_(dpred[:n])
        self._backward_from_dpred(self._stream(), n)

    def _backward_from_dpred(self, st, n):
        b, W, G = self._buf, self.bf16, self.grads
        ks = max(1, min(1024, n // 512))
        # layer 4: dW4 = dpred^T H3, db4 = sum dpred, dH3 = dpred w4
        self._gemm(st, b["dpred_b"], 0, 1, b["H3"], HID, 1, 1, HID, n, C=G["w4"], c_rs=HID, accumulate=True, k_split=ks)
        native.call("tmol_b200_screen_col_sum", _p(b["dpred"]), n, 1, _p(G["b4"]), st)
        self._gemm(st, b["dpred_b"], 1, 1, W["w4"], 0, 1, n, HID, 1, C=b["dH"], c_rs=HID)
        layers = (("w3", "b3", b["H3"], b["H2"]), ("w2", "b2", b["H2"], b["H1"]), ("w1", "b1", b["H1"], b["X"]))
        for wname, bname, H, Hin in layers:
            k_in = N_IN if wname == "w1" else HID
            native.call("tmol_b200_screen_relu_backward", _p(b["dH"]), _p(H), _p(b["dZb"]), _p(b["dZ"]), n * HID, st)
            # dW = dZ^T Hin: A(m, k) = dZ[k, m], B(k, n) = Hin[k, n]
            self._gemm(st, b["dZb"], 1, HID, Hin, k_in, 1, HID, k_in, n, C=G[wname], c_rs=k_in, accumulate=True,
                       k_split=ks)
            native.call("tmol_b200_screen_col_sum", _p(b["dZ"]), n, HID, _p(G[bname]), st)
            # dHin = dZ W: B(k, n) = W[k, n]
            out = b["dX"] if wname == "w1" else b["dH"]
            self._gemm(st, b["dZb"], HID, 1, W[wname], k_in, 1, n, k_in, HID, C=out, c_rs=k_in)
        native.call("tmol_b200_screen_embedding_backward", _p(b["dX"]), _p(self._bt), n, _p(G["emb"]), st)

    def adam(self, lr, b1=0.9, b2=0.999, eps=1e-8, weight_decay=0.0):
        self.step += 1
        st = self._stream()
        for k, w in self.params.items():
            wd = weight_decay if k.startswith("w") else 0.0
            native.call(
                "tmol_b200_screen_adam",
                _p(w), _p(self.grads[k]), _p(self.adam_m[k]), _p(self.adam_v[k]),
                _p(self.bf16.get(k)), w.numel(),
                ctypes.c_float(lr), ctypes.c_float(b1), ctypes.c_float(b2), ctypes.c_float(eps),
                self.step, ctypes.c_float(wd), st,
            )

    def infer(self, cand, threshold=0.0, mask=None, pred=None):
        """Fused inference over the candidates of
        ``LJLKPlan.screen_candidates``: writes pred (if given) and, if a mask
        is given, clears it and sets the bits of pairs predicted below
        threshold."""
        cap = cand["row"].shape[0]
        if mask is not None and (mask.dtype != torch.int32 or not mask.is_contiguous() or mask.dim() != 2):
            raise ValueError("mask must be a contiguous int32 [rows, words] tensor")
        self._weights_struct = self.weights_struct()
        native.call(
            "tmol_b200_screen_infer",
            ctypes.byref(self._weights_struct),
            _p(cand["features"]), _p(cand["bt"]), _p(cand["row"]), _p(cand["b2"]), _p(cand["count"]),
            int(cap), ctypes.c_float(threshold),
            _p(mask), int(mask.shape[1]) if mask is not None else 0, int(mask.numel()) if mask is not None else 0,
            _p(pred), self._stream(),
        )
