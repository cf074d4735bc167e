"""Device halo packing (cfdg_halo_pack / cfdg_halo_unpack, the device form
of pack_soa_to_aos / unpack_aos_to_soa, src/fields/halo.cpp:26-124) on one
GPU: the ranks of a partition are emulated in one process, each rank's
send buffer packed by the library, the messages routed to the receivers'
buffers as the exchanger's point-to-point operations would, and unpacked
into the ghosts, which must then hold the owning rank's values exactly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,nparts", [("hex", 2), ("hex", 3), ("tet", 4)])
def test_pack_route_unpack_fills_every_ghost(cb, kind, nparts):
    import torch
    case = cb.cases.plate(scale=8) if kind == "hex" else cb.cases.bump(scale=16)
    mesh = cb.HostMesh(case.spec)
    plans = [cb.halo.HaloPlan(mesh, nparts, r) for r in range(nparts)]
    nv = 7
    scales = np.arange(1.0, nv + 1.0)
    fields, sends = [], []
    for p in plans:
        g = torch.from_numpy(p.local_to_global.astype(np.float64)).cuda()
        fs = []
        for s in scales:
            f = torch.full((p.n_local,), float("nan"), dtype=torch.float64, device="cuda")
            f[:p.n_own] = s * g[:p.n_own] + 0.25
            fs.append(f)
        fields.append(fs)
        send = torch.empty(p.n_send * nv, dtype=torch.float64, device="cuda")
        p.pack([f.data_ptr() for f in fs], send.data_ptr(), 0)
        sends.append(send)
    for p, fs in zip(plans, fields):
        recv = torch.empty(p.n_recv * nv, dtype=torch.float64, device="cuda")
        for k, q in enumerate(p.nb_ranks):
            pq = plans[q]
            kk = int(np.where(pq.nb_ranks == p.rank)[0][0])
            seg = sends[q][pq.send_offsets[kk] * nv:pq.send_offsets[kk + 1] * nv]
            recv[p.recv_offsets[k] * nv:p.recv_offsets[k + 1] * nv] = seg
        p.unpack(recv.data_ptr(), [f.data_ptr() for f in fs], 0)
        torch.cuda.synchronize()
        g = p.local_to_global.astype(np.float64)
        for s, f in zip(scales, fs):
            assert np.array_equal(f.cpu().numpy(), s * g + 0.25)


def test_pack_matches_the_numpy_restatement(cb):
    import torch
    mesh = cb.HostMesh(cb.cases.plate(scale=8).spec)
    p = cb.halo.HaloPlan(mesh, 3, 1)
    rng = np.random.default_rng(0)
    host = [rng.standard_normal(p.n_local) for _ in range(5)]
    dev = [torch.from_numpy(h).cuda() for h in host]
    send = torch.empty(p.n_send * 5, dtype=torch.float64, device="cuda")
    p.pack([d.data_ptr() for d in dev], send.data_ptr(), 0)
    torch.cuda.synchronize()
    want = np.stack([h[p.send_owned_local] for h in host], axis=1).ravel()
    assert np.array_equal(send.cpu().numpy(), want)
    with pytest.raises(cb.CfdgError):  # more variables than a message holds
        p.pack([dev[0].data_ptr()] * 33, send.data_ptr(), 0)


def test_block_vector_pack_route_unpack(cb):
    """The Krylov-layout form (x[row*bs + v]): rows packed by the owners
    and unpacked into the receivers' ghost rows."""
    import torch
    mesh = cb.HostMesh(cb.cases.bump(scale=16).spec)
    nparts, bs = 3, 6
    plans = [cb.halo.HaloPlan(mesh, nparts, r) for r in range(nparts)]
    xs, sends = [], []
    for p in plans:
        g = p.local_to_global.astype(np.float64)
        want = (g[:, None] * 10.0 + np.arange(bs)[None, :]).ravel()
        x = torch.full((p.n_local * bs,), float("nan"), dtype=torch.float64, device="cuda")
        x[:p.n_own * bs] = torch.from_numpy(want[:p.n_own * bs]).cuda()
        send = torch.empty(p.n_send * bs, dtype=torch.float64, device="cuda")
        p.pack_blocks(x.data_ptr(), bs, send.data_ptr(), 0)
        xs.append((x, want))
        sends.append(send)
    for p, (x, want) in zip(plans, xs):
        recv = torch.empty(p.n_recv * bs, dtype=torch.float64, device="cuda")
        for k, q in enumerate(p.nb_ranks):
            pq = plans[q]
            kk = int(np.where(pq.nb_ranks == p.rank)[0][0])
            recv[p.recv_offsets[k] * bs:p.recv_offsets[k + 1] * bs] = \
                sends[q][pq.send_offsets[kk] * bs:pq.send_offsets[kk + 1] * bs]
        p.unpack_blocks(recv.data_ptr(), bs, x.data_ptr(), 0)
        torch.cuda.synchronize()
        assert np.array_equal(x.cpu().numpy(), want)
