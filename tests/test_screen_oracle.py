"""CPU checks of the screen's NumPy oracle: bfloat16 rounding, the pinball
loss gradient and the MLP backward pass against float64 central finite
differences."""

import numpy
import pytest

from oracle import screen_mlp as sm


def random_params(rng, n_bt=7):
    return {
        "w1": rng.normal(0, (2 / 32) ** 0.5, (128, 32)),
        "b1": rng.normal(0, 0.1, 128),
        "w2": rng.normal(0, (2 / 128) ** 0.5, (128, 128)),
        "b2": rng.normal(0, 0.1, 128),
        "w3": rng.normal(0, (2 / 128) ** 0.5, (128, 128)),
        "b3": rng.normal(0, 0.1, 128),
        "w4": rng.normal(0, (1 / 128) ** 0.5, (1, 128)),
        "b4": rng.normal(0, 0.1, 1),
        "emb": rng.normal(0, 0.3, (n_bt, 10)),
    }


def test_bf16_rounding_known_values():
    x = numpy.array([1.0, 1 + 2**-8, 1 + 3 * 2**-8, 1 + 2**-7, -2.5, 3.0e-3], numpy.float32)
    y = sm.to_bf16(x)
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties go to the even one (1)
    assert y[0] == 1.0 and y[1] == 1.0
    # 1 + 3 * 2^-8 is halfway between 1 + 2^-7 and 1 + 2^-6: even is 1 + 2^-6
    assert y[2] == numpy.float32(1 + 2**-6)
    assert y[3] == numpy.float32(1 + 2**-7)
    assert y[4] == -2.5
    assert abs(y[5] - 3.0e-3) <= 3.0e-3 * 2**-8
    assert (y.view(numpy.uint32) & 0xFFFF).max() == 0


def test_pinball_gradient():
    rng = numpy.random.default_rng(0)
    pred, y = rng.normal(size=50), rng.normal(size=50)
    for tau in (0.5, 0.9):
        loss, d = sm.pinball(pred, y, tau)
        h = 1e-7
        for i in range(5):
            pp = pred.copy()
            pp[i] += h
            pm = pred.copy()
            pm[i] -= h
            fd = (sm.pinball(pp, y, tau)[0] - sm.pinball(pm, y, tau)[0]) / (2 * h)
            assert fd == pytest.approx(d[i], rel=1e-6)
        assert loss >= 0


def test_mlp_backward_matches_finite_differences():
    rng = numpy.random.default_rng(1)
    params = random_params(rng)
    n = 40
    feats = rng.normal(size=(n, 12))
    bt = rng.integers(0, 7, size=(n, 2))
    dpred = rng.normal(size=n)
    net = sm.MLP(params, bf16=False)
    net.forward(feats, bt)
    g = net.backward(dpred)
    h = 1e-6
    for name in ("w1", "b1", "w2", "b3", "w4", "b4", "emb"):
        flat = params[name].reshape(-1)
        for idx in rng.choice(flat.size, size=min(6, flat.size), replace=False):
            pp = {k: v.copy() for k, v in params.items()}
            pp[name].reshape(-1)[idx] += h
            fp = numpy.dot(sm.MLP(pp, bf16=False).forward(feats, bt), dpred)
            pp[name].reshape(-1)[idx] -= 2 * h
            fm = numpy.dot(sm.MLP(pp, bf16=False).forward(feats, bt), dpred)
            fd = (fp - fm) / (2 * h)
            an = g[name].reshape(-1)[idx]
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (name, idx, fd, an)


def test_bf16_mode_is_close_to_float64():
    rng = numpy.random.default_rng(2)
    params = random_params(rng)
    feats = rng.normal(size=(64, 12))
    bt = rng.integers(0, 7, size=(64, 2))
    p64 = sm.MLP(params, bf16=False).forward(feats, bt)
    p16 = sm.MLP(params, bf16=True).forward(feats, bt)
    assert numpy.abs(p64 - p16).max() < 0.05 * (numpy.abs(p64).max() + 1)
