"""The learned-guess network's restatement (oracle/mlp_oracle.py): its
backward pass against central differences of its forward pass (FP64, no
bf16 rounding), and the bf16 rounding it applies."""
import numpy as np

import mlp_oracle as M


def _problem(seed=0, n=37, nvars=5):
    rng = np.random.default_rng(seed)
    p = np.zeros(M.N_PARAMS)
    p[M.OFF_W1:M.OFF_B1] = rng.uniform(-0.35, 0.35, M.HID * M.IN)
    p[M.OFF_B1:M.OFF_W2] = rng.uniform(-0.1, 0.1, M.HID)
    p[M.OFF_W2:M.OFF_B2] = rng.uniform(-0.3, 0.3, M.HID * M.HID)
    p[M.OFF_B2:M.OFF_W3] = rng.uniform(-0.1, 0.1, M.HID)
    p[M.OFF_W3:M.OFF_B3] = rng.uniform(-0.3, 0.3, M.OUT * M.HID)
    p[M.OFF_B3:] = rng.uniform(-0.1, 0.1, M.OUT)
    X = rng.standard_normal((n, M.IN))
    T = rng.standard_normal((n, M.OUT))
    return p, X, T, nvars


def test_backward_matches_central_differences():
    p, X, T, nv = _problem()
    loss, g = M.loss_and_grad(p, X, T, nv, rounding=False)
    rng = np.random.default_rng(1)
    idx = np.concatenate([rng.choice(np.arange(s, e), min(12, e - s), replace=False)
                          for s, e in [(M.OFF_W1, M.OFF_B1), (M.OFF_B1, M.OFF_W2), (M.OFF_W2, M.OFF_B2),
                                       (M.OFF_B2, M.OFF_W3), (M.OFF_W3, M.OFF_W3 + nv * M.HID),
                                       (M.OFF_B3, M.OFF_B3 + nv)]])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (M.loss_and_grad(pp, X, T, nv, rounding=False)[0] - M.loss_and_grad(pm, X, T, nv, rounding=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])
    # outputs beyond nvars carry no gradient
    assert np.all(g[M.OFF_W3 + nv * M.HID:M.OFF_B3] == 0) and np.all(g[M.OFF_B3 + nv:] == 0)


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.14159265])
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0 + 4 * 2 ** -8
    assert r[3] == -2.5 and abs(r[4] - 3.140625) < 1e-12
