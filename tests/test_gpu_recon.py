"""cfdg_gradient / cfdg_limiter on caller-owned device arrays against the
reference's GradientOperator::apply_set and Muscl::compute_limiters (run by
the reference build on the same primitives).  Tolerances as the solver's
own stages: gradients 1e-11, limiter 1e-9, relative to the largest
magnitude of each variable."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,limiter", [("ramp", 1), ("plate_face", 1), ("bump", 1), ("ramp", 2), ("ramp", 3)])
def test_recon_operators_match_reference(cb, refh, name, limiter):
    import torch

    if name == "ramp":
        case = cb.cases.ramp()
    elif name == "plate_face":
        case = cb.cases.plate(scale=8)
        case.cfg.gradient = cb.GRAD_LSQ_FACE
    else:
        case = cb.cases.bump(scale=16, mixed=False)
    case.cfg.limiter = limiter
    mesh = cb.HostMesh(case.spec)
    n = mesh.n_cells
    nt = n + mesh.n_faces - mesh.n_inner
    ref = refh.RefSolver(mesh, case.cfg, case.bcs)
    ref.set_state(cb.cases.perturbed_state(case, n))
    st = ref.stages()
    q = st["q"].reshape(5, nt)[:, :n]
    g_ref = st["grad"].reshape(5, 3, nt)[:, :, :n]
    dev = "cuda:0"
    # seven fields: the five primitives and two of them again (two launches)
    qs = [torch.from_numpy(np.ascontiguousarray(q[v % 5])).to(dev) for v in range(7)]
    gx = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(7)]
    gy = [torch.zeros_like(g) for g in gx]
    gz = [torch.zeros_like(g) for g in gx]
    r = cb.Recon(mesh, case.cfg.gradient, limiter, case.cfg.venkat_k)
    side = torch.cuda.Stream(device=dev)
    r.gradient([t.data_ptr() for t in qs], [t.data_ptr() for t in gx], [t.data_ptr() for t in gy],
               [t.data_ptr() for t in gz], stream=side.cuda_stream)
    side.synchronize()
    for v in range(7):
        got = np.stack([gx[v].cpu().numpy(), gy[v].cpu().numpy(), gz[v].cpu().numpy()])
        assert rel_err(got, g_ref[v % 5]) < 1e-11, v
    # the limiter on the reference's own gradients
    gref = [[torch.from_numpy(np.ascontiguousarray(g_ref[v % 5, d])).to(dev) for v in range(7)] for d in range(3)]
    phi = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(7)]
    r.limiter([t.data_ptr() for t in qs], [t.data_ptr() for t in gref[0]], [t.data_ptr() for t in gref[1]],
              [t.data_ptr() for t in gref[2]], [t.data_ptr() for t in phi])
    torch.cuda.synchronize()
    phi_ref = st["phi"].reshape(5, n)
    for v in range(7):
        assert rel_err(phi[v].cpu().numpy(), phi_ref[v % 5]) < 1e-9, v
    r.close()


def test_recon_rejects_bad_arguments(cb):
    import torch

    case = cb.cases.ramp()
    mesh = cb.HostMesh(case.spec)
    with pytest.raises(cb.CfdgError) as e:
        cb.Recon(mesh, gradient=1)  # Green-Gauss is not on the path
    assert e.value.status == cb.ERR_UNSUPPORTED
    with pytest.raises(cb.CfdgError):
        cb.Recon(mesh, limiter=9)
    r = cb.Recon(mesh)
    t = torch.zeros(mesh.n_cells, dtype=torch.float64, device="cuda:0")
    with pytest.raises(cb.CfdgError):
        r.gradient([t.data_ptr()], [0], [t.data_ptr()], [t.data_ptr()])
    r.close()
