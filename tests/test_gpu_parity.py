"""GPU parity of the hot path against the reference solver (oracle/_ref),
stage by stage, through the C ABI.

Tolerances (FP64 everywhere): stage outputs 1e-11 relative to the largest
magnitude of each variable; Jacobian blocks 1e-9 relative per block;
SGS level ordering and SpMV 1e-12; the Krylov solution 1e-7 (BiCGSTAB
amplifies round-off of the fused inner products); Newton iterates 1e-8.
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

CASES = {
    "ramp_muscl": lambda cb: cb.cases.ramp(),
    "ramp_first_order": lambda cb: _first_order(cb.cases.ramp()),
    "plate_viscous": lambda cb: cb.cases.plate(scale=8),
    "bump_tets": lambda cb: cb.cases.bump(scale=16, mixed=False),
    "plate_face_stencil": lambda cb: _face_stencil(cb, cb.cases.plate(scale=8)),
}


def _first_order(case):
    case.cfg.reconstruction = 0
    return case


def _face_stencil(cb, case):
    case.cfg.gradient = cb.GRAD_LSQ_FACE
    return case


def _setup(cb, refh, name, level=True):
    case = CASES[name](cb)
    case.cfg.jacobian = cb.JAC_REFERENCE  # the reference's Jacobian
    if level:
        case.cfg.sgs_ordering = cb.SGS_LEVEL
    mesh = cb.HostMesh(case.spec)
    U0 = cb.cases.perturbed_state(case, mesh.n_cells)
    gpu = cb.Solver(mesh, case.cfg, case.bcs)
    ref = refh.RefSolver(mesh, case.cfg, case.bcs)
    gpu.set_state(U0)
    ref.set_state(U0)
    return case, mesh, U0, gpu, ref


@pytest.mark.parametrize("name", list(CASES))
def test_residual_stages(cb, refh, name):
    case, mesh, U0, gpu, ref = _setup(cb, refh, name)
    st = ref.stages()
    gpu.evaluate_residual()
    n, nt = gpu.n_cells, gpu.n_total
    q = gpu.get(cb.FIELD_Q)
    assert rel_err(q, st["q"], nt) < 1e-13  # primitives + BC ghost values
    if case.cfg.reconstruction == 1 or case.cfg.viscous:
        g = gpu.get(cb.FIELD_GRAD)[: 15 * nt]
        assert rel_err(g, st["grad"], nt) < 1e-11  # LSQ gradients + ghost gradients
    if case.cfg.reconstruction == 1:
        phi = gpu.get(cb.FIELD_PHI)
        assert rel_err(phi, st["phi"]) < 1e-9  # limiter values are O(1)
    res = gpu.get(cb.FIELD_RES)
    assert rel_err(res, st["res"], n) < 1e-11
    lam = gpu.get(cb.FIELD_LAM)
    assert rel_err(lam, st["lam"]) < 1e-12


@pytest.mark.parametrize("name", ["ramp_muscl", "plate_viscous", "bump_tets"])
def test_jacobian(cb, refh, name):
    case, mesh, U0, gpu, ref = _setup(cb, refh, name)
    ref.stages()
    alpha_ref, vals_ref = ref.jacobian(7.5)
    gpu.evaluate_residual()
    gpu.compute_dt(7.5)
    gpu.assemble_jacobian()
    assert rel_err(gpu.get(cb.FIELD_ALPHA), alpha_ref) < 1e-13
    vals = gpu.get(cb.FIELD_JAC)
    assert vals.shape == vals_ref.shape
    # per block: diagonal entries are sums of O(1) face terms that cancel to
    # O(1e-14) in places, so summation-order round-off is ~1e-11 of the block
    assert rel_err(vals, vals_ref, 25) < 1e-9
    rhs = gpu.get(cb.FIELD_RHS).reshape(-1, 5)
    res = gpu.get(cb.FIELD_RES).reshape(5, -1).T
    assert np.array_equal(rhs, -res)


def _matrix_from_ref(cb, refh, name, cfl=7.5):
    case, mesh, U0, gpu, ref = _setup(cb, refh, name)
    ref.stages()
    _, vals = ref.jacobian(cfl)
    off, nb = refh.connectivity(mesh, 1)
    n = mesh.n_cells
    row_ptr = np.zeros(n + 1, dtype=np.int32)
    cols = []
    for c in range(n):
        row = sorted([c] + list(nb[off[c]:off[c + 1]]))
        cols.extend(row)
        row_ptr[c + 1] = len(cols)
    return row_ptr, np.array(cols, dtype=np.int32), vals


@pytest.mark.parametrize("name", ["ramp_muscl", "bump_tets"])
def test_spmv_sgs_level_bicgstab(cb, refh, name):
    row_ptr, cols, vals = _matrix_from_ref(cb, refh, name)
    n = len(row_ptr) - 1
    rng = np.random.default_rng(3)
    x = rng.standard_normal(n * 5)
    y0 = rng.standard_normal(n * 5)
    A = cb.Bsr(row_ptr, cols, 5)
    A.set_values(vals)
    for alpha, beta in [(1.0, 0.0), (-0.5, 1.0), (2.0, 0.25), (0.0, 3.0)]:
        y = A.spmv(x, y0, alpha, beta)
        y_ref = refh.bsr_spmv(row_ptr, cols, vals, 5, x, y0, alpha, beta)
        assert rel_err(y, y_ref) < 1e-13
    A.sgs_setup(cb.SGS_LEVEL, 1)
    z = A.sgs_apply(x)
    z_ref = refh.sgs_apply(row_ptr, cols, vals, 5, x)
    assert rel_err(z, z_ref) < 1e-12
    A.sgs_setup(cb.SGS_LEVEL, 2)
    assert rel_err(A.sgs_apply(x), refh.sgs_apply(row_ptr, cols, vals, 5, x, sweeps=2)) < 1e-12
    A.sgs_setup(cb.SGS_LEVEL, 1)
    b = rng.standard_normal(n * 5)
    sol, info = A.bicgstab(b, precond=cb.PC_SGS, rel_tol=1e-10, max_it=200)
    sol_ref, info_ref = refh.bicgstab(row_ptr, cols, vals, 5, b, precond=1, rel_tol=1e-10, max_it=200)
    assert info.status == cb.KRYLOV_CONVERGED and info_ref["status"] == 0
    assert abs(info.iterations - info_ref["iterations"]) <= 1
    assert rel_err(sol, sol_ref) < 1e-7
    # multicolour SGS: a different preconditioner, same solution
    A.sgs_setup(cb.SGS_COLOR, 1)
    sol_c, info_c = A.bicgstab(b, precond=cb.PC_SGS, rel_tol=1e-10, max_it=400)
    assert info_c.status == cb.KRYLOV_CONVERGED
    assert rel_err(sol_c, sol_ref) < 1e-7
    # unpreconditioned
    sol_n, info_n = A.bicgstab(b, precond=cb.PC_NONE, rel_tol=1e-10, max_it=2000)
    sol_nr, info_nr = refh.bicgstab(row_ptr, cols, vals, 5, b, precond=0, rel_tol=1e-10, max_it=2000)
    assert info_n.status == cb.KRYLOV_CONVERGED
    assert rel_err(sol_n, sol_nr) < 1e-6


@pytest.mark.parametrize("name", ["ramp_muscl", "bump_tets"])
def test_gmres_matches_reference_solution(cb, refh, name):
    """Restarted GMRES (the Jacobian-free solves' Krylov method) on the
    reference's matrices: the solution of the reference's BiCGSTAB to the
    tolerance, with SGS (level and multicolour) and without a
    preconditioner, with and without restarts; x0 != 0 is honoured."""
    row_ptr, cols, vals = _matrix_from_ref(cb, refh, name)
    n = len(row_ptr) - 1
    rng = np.random.default_rng(4)
    b = rng.standard_normal(n * 5)
    A = cb.Bsr(row_ptr, cols, 5)
    A.set_values(vals)
    sol_ref, info_ref = refh.bicgstab(row_ptr, cols, vals, 5, b, precond=1, rel_tol=1e-12, max_it=400)
    assert info_ref["status"] == 0
    for ordering, restart in [(cb.SGS_LEVEL, 30), (cb.SGS_COLOR, 30), (cb.SGS_COLOR, 15)]:
        A.sgs_setup(ordering, 1)
        sol, info = A.gmres(b, precond=cb.PC_SGS, rel_tol=1e-10, max_it=2000, restart=restart)
        assert info.status == cb.KRYLOV_CONVERGED, (ordering, restart, info.iterations)
        assert info.final_residual <= 1e-10 * np.linalg.norm(b) * (1 + 1e-9)
        assert rel_err(sol, sol_ref) < 1e-7, (ordering, restart)
        # the true residual agrees with the estimate
        r = b - A.spmv(sol, np.zeros_like(b), 1.0, 0.0)
        assert np.linalg.norm(r) < 1e-8 * np.linalg.norm(b)
    sol_n, info_n = A.gmres(b, precond=cb.PC_NONE, rel_tol=1e-10, max_it=3000, restart=60)
    assert info_n.status == cb.KRYLOV_CONVERGED
    assert rel_err(sol_n, sol_ref) < 1e-6
    # a starting vector near the solution (a looser solve's) needs fewer iterations
    A.sgs_setup(cb.SGS_COLOR, 1)
    _, info_0 = A.gmres(b, precond=cb.PC_SGS, rel_tol=1e-10, max_it=600)
    x0, _ = A.gmres(b, precond=cb.PC_SGS, rel_tol=1e-4, max_it=600)
    sol_g, info_g = A.gmres(b, x0=x0, precond=cb.PC_SGS, rel_tol=1e-10, max_it=600)
    assert info_g.status == cb.KRYLOV_CONVERGED and info_g.initial_residual < info_0.initial_residual
    assert info_g.iterations < info_0.iterations
    assert rel_err(sol_g, sol_ref) < 1e-7


@pytest.mark.parametrize("name", ["ramp_muscl", "plate_viscous", "bump_tets"])
def test_newton_steps_match_reference(cb, refh, name):
    case, mesh, U0, gpu, ref = _setup(cb, refh, name, level=True)
    for k, cfl in enumerate([1.0, 3.0, 10.0]):
        st = gpu.newton_step(cfl)
        l2_ref = ref.newton_step(cfl)
        assert rel_err(np.array(st.l2[:5]), l2_ref) < 1e-9, k
        U = gpu.get(cb.FIELD_U)
        U_ref = ref.get_state().ravel()
        assert rel_err(U, U_ref, mesh.n_cells) < 1e-8, k


def test_bitwise_determinism(cb, refh):
    case = cb.cases.plate(scale=8)
    mesh = cb.HostMesh(case.spec)
    U0 = cb.cases.perturbed_state(case, mesh.n_cells)
    outs = []
    for _ in range(2):
        with cb.Solver(mesh, case.cfg, case.bcs) as s:
            s.set_state(U0)
            for cfl in (1.0, 5.0):
                s.newton_step(cfl)
            outs.append(s.get(cb.FIELD_U))
    assert np.array_equal(outs[0], outs[1])


def test_colour_sgs_newton_converges(cb):
    """Multicolour SGS (a different preconditioner from the reference's
    natural-order sweep) drives the ramp to the same residual level the
    reference reaches in the same number of iterations (rel ~1e-2 at 80)."""
    case = cb.cases.ramp(iterations=100)
    mesh = cb.HostMesh(case.spec)
    with cb.Solver(mesh, case.cfg, case.bcs) as s:
        s.init_fields()
        r = s.run_steady()
        assert not r.blowup
        assert r.rel < 2e-2, r.rel


def test_thin_layer_jacobian_matches_oracle(cb):
    """CFDG_JAC_THIN_LAYER (normal-stress term + no-slip ghost) against the
    oracle restatement of the same variant."""
    import port
    case = cb.cases.plate(scale=8, jacobian=cb.JAC_THIN_LAYER)
    mesh = cb.HostMesh(case.spec)
    U0 = cb.cases.perturbed_state(case, mesh.n_cells)
    ora = port.PortSolver(mesh, case.cfg, case.bcs)
    ora.set_state(U0)
    ora.stages()
    _, vals_ref = ora.jacobian(7.5)
    ref0 = port.PortSolver(mesh, cb.cases.plate(scale=8, jacobian=cb.JAC_REFERENCE).cfg, case.bcs)
    ref0.set_state(U0)
    ref0.stages()
    _, vals0 = ref0.jacobian(7.5)
    assert rel_err(vals_ref, vals0, 25) > 1e-3  # the variants differ
    with cb.Solver(mesh, case.cfg, case.bcs) as s:
        s.set_state(U0)
        s.evaluate_residual()
        s.compute_dt(7.5)
        s.assemble_jacobian()
        assert rel_err(s.get(cb.FIELD_JAC), vals_ref, 25) < 1e-9


def _colour_ordered(row_ptr, cols, vals, bs=5):
    """The matrix with its rows and columns permuted so that the greedy
    colouring (natural order) lists colour 0 first, then colour 1, ..."""
    n = len(row_ptr) - 1
    colour = np.full(n, -1)
    for i in range(n):
        used = {colour[j] for j in cols[row_ptr[i]:row_ptr[i + 1]] if j != i and colour[j] >= 0}
        c = 0
        while c in used:
            c += 1
        colour[i] = c
    order = np.argsort(colour, kind="stable")  # new row -> old row
    new_of = np.empty(n, dtype=np.int64)
    new_of[order] = np.arange(n)
    blocks = vals.reshape(-1, bs, bs)
    rp, cl, vb = np.zeros(n + 1, dtype=np.int32), [], []
    for r, i in enumerate(order):
        ks = np.arange(row_ptr[i], row_ptr[i + 1])
        cnew = new_of[cols[ks]]
        srt = np.argsort(cnew)
        cl.extend(cnew[srt])
        vb.append(blocks[ks[srt]])
        rp[r + 1] = len(cl)
    return rp, np.array(cl, dtype=np.int32), np.concatenate(vb).ravel(), int(colour.max()) + 1


@pytest.mark.parametrize("name", ["ramp_muscl", "bump_tets"])
def test_colour_sgs_split_sweep_matches_sequential_sweep(cb, refh, name):
    """On a colour-ordered matrix the multicolour sweep is the sequential
    sweep (rows of one colour are independent), so the split first sweep
    (forward below the diagonal, backward correction above it) must agree
    with the reference's natural-order SGS to round-off, for one and two
    sweeps.  The multicolour sweep applies the explicit inverse of each
    diagonal block instead of its pivoted LU factors: 1e-10 covers the
    condition number of the blocks times the FP64 rounding."""
    row_ptr, cols, vals = _matrix_from_ref(cb, refh, name)
    rp, cl, vb, ncol = _colour_ordered(row_ptr, cols, vals)
    n = len(rp) - 1
    x = np.random.default_rng(11).standard_normal(n * 5)
    A = cb.Bsr(rp, cl, 5)
    A.set_values(vb)
    for sweeps in (1, 2):
        A.sgs_setup(cb.SGS_COLOR, sweeps)
        z = A.sgs_apply(x)
        z_ref = refh.sgs_apply(rp, cl, vb, 5, x, sweeps=sweeps)
        assert rel_err(z, z_ref) < 1e-10, (sweeps, ncol)
    if name == "bump_tets":
        assert ncol > 2  # more than two colours: the split skips blocks the full sweep reads
    # BiCGSTAB with the split sweep, whose colour-0 pass carries the product
    # A z of those rows: the same solution as the reference's solver
    A.sgs_setup(cb.SGS_COLOR, 1)
    b = np.random.default_rng(12).standard_normal(n * 5)
    sol, info = A.bicgstab(b, precond=cb.PC_SGS, rel_tol=1e-10, max_it=400)
    sol_ref, info_ref = refh.bicgstab(rp, cl, vb, 5, b, precond=1, rel_tol=1e-10, max_it=400)
    assert info.status == cb.KRYLOV_CONVERGED and info_ref["status"] == 0
    assert rel_err(sol, sol_ref) < 1e-7
    assert rel_err(A.spmv(sol, np.zeros_like(b), 1.0, 0.0), b) < 1e-9


@pytest.mark.parametrize("mixed", [False, True])
def test_device_loop_matches_host_loop(cb, mixed):
    """The BiCGSTAB iterations run as one graph launch (conditional while
    node) or one launch sequence per iteration with a host poll: the same
    kernels in the same order, so the Newton iterates are bitwise equal."""
    case = cb.cases.bump(scale=16, mixed=mixed)
    mesh = cb.HostMesh(case.spec)
    outs = []
    for loop in (cb.KRYLOV_DEVICE_LOOP, cb.KRYLOV_HOST_LOOP):
        case.cfg.krylov_loop = loop
        its = []
        with cb.Solver(mesh, case.cfg, case.bcs) as s:
            s.init_fields()
            for k in range(12):
                st = s.newton_step(cb.cases.cfl_at(case.cfg, k + 1))
                its.append(st.krylov_iterations)
            outs.append((its, s.get(cb.FIELD_U)))
    assert outs[0][0] == outs[1][0]
    assert max(outs[0][0]) > 1
    assert np.array_equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("variant", ["isothermal_wall", "heat_flux_wall", "inlet_mach_angles",
                                     "inlet_mach_direction", "farfield_top"])
def test_boundary_variants_match_reference(cb, refh, variant):
    """The boundary kinds and inflow modes beyond the benchmark cases' own
    (isothermal no-slip wall, heat-flux wall with a non-zero gradient,
    subsonic inlet by Mach and angles or Mach and direction, a Riemann far
    field on the plate's top), each swapped into the 1/8 plate: the GPU's
    primitives and ghost values, gradients with ghost gradients, residual,
    and two Newton iterates against the reference build."""
    from test_oracle_cpu import _plate_bc_variant
    case = _plate_bc_variant(cb, variant)
    mesh = cb.HostMesh(case.spec)
    n, nt = mesh.n_cells, mesh.n_cells + mesh.n_faces - mesh.n_inner
    U0 = cb.cases.perturbed_state(case, n, seed=13)
    ref = refh.RefSolver(mesh, case.cfg, case.bcs)
    ref.set_state(U0)
    st = ref.stages()
    with cb.Solver(mesh, case.cfg, case.bcs) as gpu:
        gpu.set_state(U0)
        gpu.evaluate_residual()
        assert rel_err(gpu.get(cb.FIELD_Q), st["q"], nt) < 1e-13
        assert rel_err(gpu.get(cb.FIELD_GRAD)[: 15 * nt], st["grad"], nt) < 1e-11
        assert rel_err(gpu.get(cb.FIELD_RES), st["res"], n) < 1e-11
        for cfl in (2.0, 20.0):
            l2 = np.array(gpu.newton_step(cfl).l2[:5])
            assert rel_err(l2, ref.newton_step(cfl)) < 1e-9
            assert rel_err(gpu.get(cb.FIELD_U), ref.get_state().ravel(), n) < 1e-8
