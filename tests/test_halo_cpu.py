"""Partitions and halo plans (cfdg_halo_*: mesh::MeshPart's halo fields,
include/cfd/mesh/localmesh.hpp:30-32,79-83) and the HaloExchanger phases
over torch.distributed (src/fields/halo.cpp:212-330), on the CPU.

The plans are checked against the mesh's face adjacency for contiguous and
random partitions; the exchange runs as gloo ranks with the message packing
restated in numpy (the library's device packing is tested on the GPU in
tests/test_gpu_halo.py)."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def _mesh(cb, kind):
    case = cb.cases.plate(scale=8) if kind == "hex" else cb.cases.bump(scale=16)
    return cb.HostMesh(case.spec)


def _faces(mesh):
    v = mesh.view
    ni = v.n_inner_faces
    own = np.ctypeslib.as_array(v.face_owner, shape=(v.n_faces,))[:ni].copy()
    nei = np.ctypeslib.as_array(v.face_neigh, shape=(v.n_faces,))[:ni].copy()
    return own, nei


def _parts(n, nparts, how):
    if how == "ranges":
        return None, (np.arange(n, dtype=np.int64) * nparts // n).astype(np.int32)
    rng = np.random.default_rng(nparts)
    p = rng.integers(0, nparts, n).astype(np.int32)
    p[:nparts] = np.arange(nparts)  # every rank owns a cell
    return p, p


@pytest.mark.parametrize("kind", ["hex", "tet"])
@pytest.mark.parametrize("nparts,how", [(2, "ranges"), (3, "ranges"), (4, "random")])
def test_plans_match_the_face_adjacency(cb, kind, nparts, how):
    mesh = _mesh(cb, kind)
    n = mesh.n_cells
    part_arg, part = _parts(n, nparts, how)
    own, nei = _faces(mesh)
    plans = [cb.halo.HaloPlan(mesh, nparts, r, part_arg) for r in range(nparts)]
    owned = np.concatenate([p.local_to_global[:p.n_own] for p in plans])
    assert np.array_equal(np.sort(owned), np.arange(n))  # the owned sets partition the cells
    for p in plans:
        r = p.rank
        g = p.local_to_global
        assert np.all(part[g[:p.n_own]] == r) and np.all(np.diff(g[:p.n_own]) > 0)
        # ghosts: the face neighbours of owned cells that other ranks own
        cut = (part[own] != part[nei]) & ((part[own] == r) | (part[nei] == r))
        other = np.where(part[own[cut]] == r, nei[cut], own[cut])
        assert np.array_equal(np.sort(g[p.n_own:]), np.unique(other))
        assert np.array_equal(p.nb_ranks, np.unique(part[other]))
        assert np.all(p.recv_ghost_local == np.arange(p.n_own, p.n_local))
        assert np.all(p.send_owned_local < p.n_own)
        for k, q in enumerate(p.nb_ranks):
            ghosts = g[p.recv_ghost_local[p.recv_offsets[k]:p.recv_offsets[k + 1]]]
            assert np.all(part[ghosts] == q) and np.all(np.diff(ghosts) > 0)
            # what q sends to r is what r receives from q, in the same order
            pq = plans[q]
            kk = int(np.where(pq.nb_ranks == r)[0][0])
            sent = pq.local_to_global[pq.send_owned_local[pq.send_offsets[kk]:pq.send_offsets[kk + 1]]]
            assert np.array_equal(sent, ghosts)


def test_plan_arguments_are_checked(cb):
    mesh = _mesh(cb, "hex")
    with pytest.raises(cb.CfdgError):
        cb.halo.HaloPlan(mesh, 2, 2)
    with pytest.raises(cb.CfdgError):
        cb.halo.HaloPlan(mesh, 0, 0)
    bad = np.zeros(mesh.n_cells, dtype=np.int32)
    bad[0] = 5
    with pytest.raises(cb.CfdgError):
        cb.halo.HaloPlan(mesh, 2, 0, bad)
    with pytest.raises(cb.CfdgError):  # rank 1 owns nothing
        cb.halo.HaloPlan(mesh, 2, 1, np.zeros(mesh.n_cells, dtype=np.int32))
    one = cb.halo.HaloPlan(mesh, 1, 0)
    assert one.n_own == one.n_local == mesh.n_cells and one.nb_ranks.size == 0


class _NumpyPacker:
    """pack_soa_to_aos / unpack_aos_to_soa (src/fields/halo.cpp:26-124) and
    the vector layout's block packing (vector_layout.hpp:172-260) in numpy."""

    def __init__(self, plan):
        self.plan = plan

    def pack(self, fields, send):
        import torch
        a = np.stack([f.numpy()[self.plan.send_owned_local] for f in fields], axis=1)
        send.copy_(torch.from_numpy(a.ravel()))

    def unpack(self, recv, fields):
        a = recv.numpy().reshape(-1, len(fields))
        for v, f in enumerate(fields):
            f.numpy()[self.plan.recv_ghost_local] = a[:, v]

    def pack_blocks(self, x, bs, send):
        import torch
        send.copy_(torch.from_numpy(x.numpy().reshape(-1, bs)[self.plan.send_owned_local].ravel()))

    def unpack_blocks(self, recv, bs, x):
        x.numpy().reshape(-1, bs)[self.plan.recv_ghost_local] = recv.numpy().reshape(-1, bs)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import __graft_entry__ as ge
    cb = ge.load_package()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mesh = cb.HostMesh(cb.cases.plate(scale=8).spec)
        plan = cb.halo.HaloPlan(mesh, world, rank)
        g = plan.local_to_global.astype(np.float64)

        def field(scale):
            f = torch.full((plan.n_local,), float("nan"), dtype=torch.float64)
            f[:plan.n_own] = torch.from_numpy(scale * g[:plan.n_own] + 1.0)
            return f
        rho, e = field(2.0), field(-3.0)
        gx, gy, gz, phi = field(5.0), field(7.0), field(11.0), field(0.5)
        ex = cb.halo.HaloExchanger(plan, packer=_NumpyPacker(plan))
        ex.register_cell_fields([rho, e])
        ex.register_grad_limiters([gx], [gy], [gz], [phi])
        ex.start_exchange_fields()
        ex.finish_exchange_fields()
        ex.exchange_grad_limiters()
        once = field(13.0)
        ex.exchange_once([once])
        ok = True
        for f, s in ((rho, 2.0), (e, -3.0), (gx, 5.0), (gy, 7.0), (gz, 11.0), (phi, 0.5), (once, 13.0)):
            ok = ok and np.array_equal(f.numpy(), s * g + 1.0)
        # a Krylov-layout block vector (6 entries a row)
        xv = torch.full((plan.n_local * 6,), float("nan"), dtype=torch.float64)
        want = (g[:, None] * 10.0 + np.arange(6)[None, :]).ravel()
        xv[:plan.n_own * 6] = torch.from_numpy(want[:plan.n_own * 6])
        ex.exchange_vector(xv, 6)
        ok = ok and np.array_equal(xv.numpy(), want)
        total = cb.halo.allreduce_sum(torch.tensor([float(plan.n_own)], dtype=torch.float64))
        Path(out_dir, f"r{rank}.txt").write_text(
            f"{int(ok)} {ex.num_registered_fields} {ex.num_registered_grads_and_limiters} {int(total.item())}")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_fills_every_ghost(cb, tmp_path, world):
    import torch.multiprocessing as mp
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    n = cb.HostMesh(cb.cases.plate(scale=8).spec).n_cells
    for r in range(world):
        ok, nf, ng, total = map(int, Path(tmp_path, f"r{r}.txt").read_text().split())
        assert ok == 1 and nf == 2 and ng == 4 and total == n
