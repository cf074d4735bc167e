"""The learned initial guess on the GPU: the tcgen05 tensor-core product,
the network's forward and backward kernels against the numpy restatement
(oracle/mlp_oracle.py), training, and the solver's use of the guess with
its zero-guess fallback.

Tolerances: tensor-core product 1e-5 of the largest entry (FP32
accumulation of exact bf16 products); forward 1e-2 of the largest output
with the median entry below 1e-4 (a hidden activation that lands on the
other side of a bf16 rounding boundary moves one output by ~2^-9 of that
unit's contribution); gradient 2e-2 in norm; loss 1e-5.
"""
import numpy as np
import pytest

import mlp_oracle as M
from conftest import rel_err

pytestmark = pytest.mark.gpu


def _params(seed, nvars):
    rng = np.random.default_rng(seed)
    p = np.zeros(M.N_PARAMS, dtype=np.float32)
    p[M.OFF_W1:M.OFF_B1] = rng.uniform(-0.35, 0.35, M.HID * M.IN)
    p[M.OFF_B1:M.OFF_W2] = rng.uniform(-0.1, 0.1, M.HID)
    p[M.OFF_W2:M.OFF_B2] = rng.uniform(-0.3, 0.3, M.HID * M.HID)
    p[M.OFF_B2:M.OFF_W3] = rng.uniform(-0.1, 0.1, M.HID)
    p[M.OFF_W3:M.OFF_W3 + nvars * M.HID] = rng.uniform(-0.3, 0.3, nvars * M.HID)
    p[M.OFF_B3:M.OFF_B3 + nvars] = rng.uniform(-0.1, 0.1, nvars)
    return p


def _features(cb, seed, n):
    rng = np.random.default_rng(seed)
    return cb.to_bf16_bits(rng.standard_normal((n, M.IN)))


@pytest.mark.parametrize("n,k", [(64, 16), (64, 48), (16, 64), (48, 128), (64, 128), (32, 32)])
def test_tcgen05_product(cb, n, k):
    rng = np.random.default_rng(n * 1000 + k)
    a = cb.to_bf16_bits(rng.standard_normal((128, k)))
    b = cb.to_bf16_bits(rng.standard_normal((n, k)))
    d = cb.tc_selftest(a, b)
    ref = M.from_bits(a) @ M.from_bits(b).T
    assert np.abs(d - ref).max() <= 1e-5 * np.abs(ref).max()


@pytest.mark.parametrize("nvars,rows", [(6, 1000), (5, 128), (5, 77)])
def test_forward_matches_oracle(cb, nvars, rows):
    p = _params(3, nvars)
    X = _features(cb, 4, rows)
    with_net = cb.Mlp(nvars, seed=1)
    with_net.set_params(p)
    y = with_net.forward(X)
    y_ref, _ = M.forward(p, M.from_bits(X))
    y_ref = y_ref[:, :nvars]
    err = np.abs(y - y_ref)
    assert err.max() <= 1e-2 * np.abs(y_ref).max()
    assert np.median(err) <= 1e-4 * np.abs(y_ref).max()


@pytest.mark.parametrize("nvars,rows", [(6, 700), (5, 3000)])
def test_gradient_matches_oracle(cb, nvars, rows):
    p = _params(5, nvars)
    X = _features(cb, 6, rows)
    T = np.zeros((rows, M.OUT), dtype=np.float32)
    T[:, :nvars] = np.random.default_rng(7).standard_normal((rows, nvars))
    net = cb.Mlp(nvars, seed=1)
    net.set_params(p)
    loss, g = net.gradient(X, T)
    loss_ref, g_ref = M.loss_and_grad(p, M.from_bits(X), T.astype(np.float64), nvars)
    assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref)
    assert np.linalg.norm(g - g_ref) <= 2e-2 * np.linalg.norm(g_ref)
    for s, e in [(M.OFF_W1, M.OFF_B1), (M.OFF_B1, M.OFF_W2), (M.OFF_W2, M.OFF_B2), (M.OFF_B2, M.OFF_W3),
                 (M.OFF_W3, M.OFF_B3), (M.OFF_B3, M.N_PARAMS)]:
        assert np.linalg.norm(g[s:e] - g_ref[s:e]) <= 3e-2 * max(np.linalg.norm(g_ref[s:e]), 1e-30)


def test_training_fits_a_teacher(cb):
    nvars, rows = 5, 24576
    teacher = _params(11, nvars)
    X = _features(cb, 12, rows)
    T = np.zeros((rows, M.OUT), dtype=np.float32)
    T[:, :nvars] = M.forward(teacher, M.from_bits(X))[0][:, :nvars]
    ds = cb.Dataset(nvars, rows)
    ds.append(X, T)
    assert len(ds) == rows
    net = cb.Mlp(nvars, seed=2)
    loss0, _ = net.gradient(X, T)
    loss = net.train(ds, epochs=60, batch=2048, lr=2e-3)
    loss1, _ = net.gradient(X, T)
    assert loss1 < 0.2 * loss0, (loss0, loss, loss1)


def _run(cb, case, mesh, steps, net=None, ds=None, stride=1):
    its, guess = [], []
    with cb.Solver(mesh, case.cfg, case.bcs) as s:
        s.init_fields()
        if ds is not None:
            s.attach_dataset(ds, stride)
        if net is not None:
            s.attach_guess(net)
        for k in range(steps):
            st = s.newton_step(cb.cases.cfl_at(case.cfg, k + 1))
            its.append(st.krylov_iterations)
            guess.append(st.guess_used)
        U = s.get(cb.FIELD_U)
    return np.array(its), np.array(guess), U


def test_rejected_guess_is_the_zero_guess(cb):
    """A network whose guess is worse than zero is rejected every step and
    the solve is bitwise the zero-guess solve."""
    case = cb.cases.ramp(scale=2)
    case.cfg.pre_freeze = cb.PREFREEZE_CONFIGURED  # the guess from the first step on
    mesh = cb.HostMesh(case.spec)
    p = _params(13, 5)
    p[M.OFF_B3:M.OFF_B3 + 5] = 1e3  # a huge constant update
    net = cb.Mlp(5, seed=1)
    net.set_params(p)
    its0, _, U0 = _run(cb, case, mesh, 6)
    its1, g1, U1 = _run(cb, case, mesh, 6, net=net)
    assert g1[0] == 0 and np.all(g1[1:] == 2)  # no guess before a previous update exists
    assert np.array_equal(its0, its1)
    assert np.array_equal(U0, U1)


def test_solver_collects_trains_and_uses_the_guess(cb):
    """Samples written by the solver train a network whose guess the solver
    accepts; the Krylov iterations of the same steps drop."""
    case = cb.cases.ramp()
    case.cfg.pre_freeze = cb.PREFREEZE_CONFIGURED
    mesh = cb.HostMesh(case.spec)
    steps = 120
    ds = cb.Dataset(5, mesh.n_cells * steps)
    its0, _, _ = _run(cb, case, mesh, steps, ds=ds)
    assert len(ds) == mesh.n_cells * (steps - 1)  # the first step has no previous update
    X, T = ds.read()
    assert np.all(np.isfinite(M.from_bits(X))) and np.all(np.isfinite(T))
    net = cb.Mlp(5, seed=3)
    net.train(ds, epochs=30, batch=4096, lr=2e-3)
    its1, g1, _ = _run(cb, case, mesh, steps, net=net)
    assert (g1 == 1).mean() > 0.5
    assert its1[20:].sum() < its0[20:].sum(), (its0.sum(), its1.sum())


def test_trained_guess_cuts_krylov_work_on_an_unseen_case(cb):
    """Trained on bump flows at M = 0.8 and 0.9 on a coarse mesh, the
    network's guess lowers the Krylov iterations of the M = 0.85 bump on a
    finer mesh, run to a 1e-8 residual drop."""
    ds = cb.Dataset(5, 2_000_000)
    for mach in (0.8, 0.9):
        case = cb.cases.bump(scale=8, mixed=True, mach=mach, iterations=1000)
        mesh = cb.HostMesh(case.spec)
        with cb.Solver(mesh, case.cfg, case.bcs) as s:
            s.init_fields()
            s.attach_dataset(ds, 2)
            assert s.run_steady().converged
    net = cb.Mlp(5, seed=5)
    net.train(ds, epochs=20, batch=8192, lr=1e-3)
    case = cb.cases.bump(scale=4, iterations=2000)
    mesh = cb.HostMesh(case.spec)
    runs = {}
    for learned in (False, True):
        with cb.Solver(mesh, case.cfg, case.bcs) as s:
            s.init_fields()
            if learned:
                s.attach_guess(net)
            runs[learned] = s.run_steady()
            assert runs[learned].converged
    assert runs[True].krylov_iterations_total < 0.95 * runs[False].krylov_iterations_total, (
        runs[False].krylov_iterations_total, runs[True].krylov_iterations_total)


def test_pre_freeze_phase_is_the_fp64_path(cb):
    """CFDG_PREFREEZE_FP64: until the limiter freezes, a mixed-precision
    solver with a learned guess attached takes bitwise the plain FP64
    solver's iterates (FP64 matrix, zero guess); from the freeze on it uses
    the FP32 matrix and the guess."""
    case = cb.cases.ramp(scale=2)
    mesh = cb.HostMesh(case.spec)
    net = cb.Mlp(5, seed=1)
    net.set_params(_params(13, 5))
    F = case.cfg.limiter_freeze
    states = {}
    for name, prec, learned in (("fp64", 0, False), ("mixed", 1, True)):
        case.cfg.precision = prec
        with cb.Solver(mesh, case.cfg, case.bcs) as s:
            s.init_fields()
            if learned:
                s.attach_guess(net)
            guess = []
            for it in range(1, F + 3):
                if it == F:
                    s.freeze_limiter(True)
                guess.append(s.newton_step(cb.cases.cfl_at(case.cfg, it)).guess_used)
                if it == F - 1:
                    states[name] = s.get(cb.FIELD_U)
            states[name + "_after"] = s.get(cb.FIELD_U)
            if learned:
                assert all(g == 0 for g in guess[:F - 1]) and all(g in (1, 2) for g in guess[F - 1:]), guess
    assert np.array_equal(states["fp64"], states["mixed"])
    assert not np.array_equal(states["fp64_after"], states["mixed_after"])
