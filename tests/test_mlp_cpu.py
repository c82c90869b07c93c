"""CPU pinning of the guess network's oracle (oracle/mlp_oracle.py).

The FP64 backward pass is checked against central finite differences of the
FP64 loss, so the oracle that later checks the device gradients is itself
verified."""
import numpy as np

from oracle import mlp_oracle as M


def test_layout_size():
    assert M.NPARAM == 9928


def test_fp64_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    P = M.init_params(3)
    x = rng.normal(size=(40, M.IN))
    t = rng.normal(size=(40, M.OUT))
    _, g, _ = M.loss_and_grad(P, x, t, bf=False)
    # probe a spread of real (non-padding) parameters in every block
    idx = [5, 700, 1030, 1100, 3000, 5200, 6000, 9350, 9410, 9411, 9920, 9921]
    h = 1e-6
    for i in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        num = (M.loss_and_grad(Pp, x, t, bf=False)[0] - M.loss_and_grad(Pm, x, t, bf=False)[0]) / (2 * h)
        assert abs(num - g[i]) <= 1e-6 * max(1.0, abs(num)), (i, num, g[i])


def test_padding_gradients_are_zero():
    rng = np.random.default_rng(2)
    P = M.init_params(4)
    _, g, _ = M.loss_and_grad(P, rng.normal(size=(16, M.IN)), rng.normal(size=(16, M.OUT)))
    d = M.unpack(g)
    assert np.all(d["W1"][M.IN:] == 0) and np.all(d["W4"][:, M.OUT:] == 0)
    assert np.all(d["b4"][M.OUT:] == 0)


def test_bf16_rounding():
    # bf16 keeps 7 explicit mantissa bits: the spacing above 1.0 is 2^-7
    v = np.array([1.0, 1 + 2 ** -8, 1 + 3 * 2 ** -8, 1 + 2 ** -9, 3.0e-3, -2.5])
    r = M.bf16(v)
    assert r[0] == 1.0
    assert r[1] == 1.0                # halfway, ties to the even neighbour 1.0
    assert r[2] == 1 + 2 ** -6        # halfway, ties to the even neighbour 1 + 2/128
    assert r[3] == 1.0
    assert abs(r[4] - 3.0e-3) / 3.0e-3 < 2 ** -8
    assert r[5] == -2.5
