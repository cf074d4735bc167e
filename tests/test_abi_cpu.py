"""C-ABI checks that need no GPU: the library loads, exports every symbol
include/cfdg.h declares, reports statuses, and refuses to run without a
device instead of falling back to the CPU."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    text = (ROOT / "include" / "cfdg.h").read_text()
    return sorted(set(re.findall(r"CFDG_API\s+[\w\s\*]+?\b(cfdg_\w+)\s*\(", text)))


def test_header_symbols_exported(cb):
    lib = C.CDLL(str(cb.LIB_PATH))
    names = _declared()
    assert len(names) >= 38
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python mirror binds every declared entry point
    assert sorted(cb._SIGS) == names


def test_status_strings_and_version(cb):
    L = cb.lib()
    assert L.cfdg_version() >= 10000
    for code in range(0, -10, -1):
        assert L.cfdg_status_string(code)
    assert L.cfdg_status_string(-99) == b"unknown status"


def test_config_defaults_match_reference(cb):
    cfg = cb.default_config()
    # SolverConfig / linalg::SolverParams defaults (config.hpp:94-136, linalg/config.hpp:14-26)
    assert cfg.cfl == 0.4 and cfg.venkat_k == 0.5 and cfg.residual_tolerance == 1e-10
    assert cfg.lin_rel_tol == 1e-1 and cfg.lin_abs_tol == 1e-15 and cfg.lin_max_iterations == 500
    assert cfg.gamma == 1.4 and cfg.gas_constant == 287.052874 and cfg.prandtl == 0.71
    assert cfg.init_p == 101325.0 and cfg.init_rho == 1.225 and cfg.max_iterations == 10000


def test_python_config_defaults_equal_library(cb):
    # default_config() writes its values without loading the library; they
    # must be cfdg_config_default's, field by field
    lib_cfg = cb.Config()
    cb.lib().cfdg_config_default(C.byref(lib_cfg))
    py_cfg = cb.default_config()
    for name, ctype in cb.Config._fields_:
        a, b = getattr(lib_cfg, name), getattr(py_cfg, name)
        if name == "init_velocity":
            a, b = list(a), list(b)
        assert a == b, name
    assert C.sizeof(cb.Config) == C.sizeof(lib_cfg)


def test_null_arguments_rejected(cb):
    L = cb.lib()
    assert L.cfdg_solver_create(0, None, None, None, 0, None) == cb.ERR_INVALID
    assert L.cfdg_newton_step(None, 1.0, None) == cb.ERR_INVALID
    assert L.cfdg_bsr_spmv(None, None, None, 1.0, 0.0) == cb.ERR_INVALID
    assert L.cfdg_solver_destroy(None) == cb.OK


def test_no_device_is_an_error_not_a_fallback(cb):
    if cb.device_count() > 0:
        pytest.skip("a CUDA device is visible")
    case = cb.cases.ramp()
    mesh = cb.HostMesh(case.spec)
    with pytest.raises(cb.CfdgError) as e:
        cb.Solver(mesh, case.cfg, case.bcs)
    assert e.value.status == cb.ERR_NODEVICE
    with pytest.raises(cb.CfdgError):
        cb.Bsr([0, 1], [0], 5)


def test_mesh_api_errors(cb):
    spec = cb.MeshSpec()
    spec.kind, spec.nx, spec.ny, spec.nz = 7, 2, 2, 2
    with pytest.raises(cb.CfdgError) as e:
        cb.HostMesh(spec)
    assert e.value.status == cb.ERR_INVALID
