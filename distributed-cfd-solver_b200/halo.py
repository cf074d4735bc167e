"""Partitions and halo exchange: the reference's HaloExchanger
(src/fields/halo.cpp:212-330, include/cfd/fields/halo.hpp) over
torch.distributed instead of MPI.

HaloPlan is one rank's part of a partitioned mesh in the layout of
mesh::MeshPart's halo fields (include/cfd/mesh/localmesh.hpp:30-32, 79-83):
owned cells [0, n_own) in ascending global order, then ghost cells grouped by
owning rank; per neighbour rank the owned cells to send and the ghost slots
to fill, both in ascending global id so the two sides agree.

HaloExchanger keeps the reference's phases and calls: cell fields and
gradients + limiters registered once, then start_*/finish_* (or exchange_*)
every iteration, and exchange_once for an unregistered group.  Each phase
sends ONE message per neighbour: the registered variables of every listed
cell, AoS (nvars values a cell), packed and unpacked on the device by the
library (cfdg_halo_pack / cfdg_halo_unpack) and moved by torch.distributed
point-to-point operations (NCCL over NVLink on GPUs).  The solver itself
runs one partition; this is the exchange layer a partitioned run uses.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import (CFDG_HALO_ARRAYS, HostMesh, _dptr_int, _ptr_array, check, lib)


class HaloPlan:
    """cfdg_halo_create: rank `rank` of `nparts` (part: owning rank of every
    global cell, or None for contiguous ranges of the cell order)."""

    def __init__(self, mesh: HostMesh, nparts: int, rank: int, part=None):
        h = C.c_void_p()
        p = None
        if part is not None:
            self._part = np.ascontiguousarray(part, dtype=np.int32)
            if self._part.shape != (mesh.n_cells,):
                raise ValueError("part needs one entry per cell")
            p = _dptr_int(self._part)
        check(lib().cfdg_halo_create(C.byref(mesh.view), nparts, p, rank, C.byref(h)))
        self._h = h
        self.nparts, self.rank = nparts, rank
        sz = (C.c_int64 * 5)()
        check(lib().cfdg_halo_sizes(self._h, sz))
        self.n_own, self.n_local, n_nb, n_send, n_recv = (int(x) for x in sz)
        counts = {"local_to_global": self.n_local, "nb_ranks": n_nb, "send_offsets": n_nb + 1,
                  "send_owned_local": n_send, "recv_offsets": n_nb + 1, "recv_ghost_local": n_recv}
        for name, what in CFDG_HALO_ARRAYS.items():
            a = np.zeros(max(counts[name], 1), dtype=np.int32)
            check(lib().cfdg_halo_get(self._h, what, _dptr_int(a), a.size))
            setattr(self, name, a[:counts[name]])

    @property
    def n_send(self) -> int:
        return int(self.send_owned_local.size)

    @property
    def n_recv(self) -> int:
        return int(self.recv_ghost_local.size)

    def close(self):
        if getattr(self, "_h", None):
            lib().cfdg_halo_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # device side (the library's kernels)
    def pack(self, fields, send, device: int, stream: int = 0):
        """send[i*nvars + v] = fields[v][send_owned_local[i]] (device addresses)."""
        check(lib().cfdg_halo_pack(self._h, device, _ptr_array(fields), len(fields), C.c_void_p(int(send)),
                                   C.c_void_p(stream or None)))

    def unpack(self, recv, fields, device: int, stream: int = 0):
        """fields[v][recv_ghost_local[i]] = recv[i*nvars + v] (device addresses)."""
        check(lib().cfdg_halo_unpack(self._h, device, C.c_void_p(int(recv)), len(fields), _ptr_array(fields),
                                     C.c_void_p(stream or None)))

    def pack_blocks(self, x, bs: int, send, device: int, stream: int = 0):
        """send[i*bs + v] = x[send_owned_local[i]*bs + v] (a block vector, device addresses)."""
        check(lib().cfdg_halo_pack_blocks(self._h, device, C.c_void_p(int(x)), bs, C.c_void_p(int(send)),
                                          C.c_void_p(stream or None)))

    def unpack_blocks(self, recv, bs: int, x, device: int, stream: int = 0):
        """x[recv_ghost_local[i]*bs + v] = recv[i*bs + v] (a block vector, device addresses)."""
        check(lib().cfdg_halo_unpack_blocks(self._h, device, C.c_void_p(int(recv)), bs, C.c_void_p(int(x)),
                                            C.c_void_p(stream or None)))


class DevicePacker:
    """Message packing of CUDA tensors by the library's kernels on the
    current torch stream: fields (SoA phases) and block vectors."""

    def __init__(self, plan: HaloPlan):
        self.plan = plan

    @staticmethod
    def _stream(t):
        import torch
        return t.device.index, torch.cuda.current_stream(t.device.index).cuda_stream

    def pack(self, fields, send):
        dev, st = self._stream(send)
        self.plan.pack([f.data_ptr() for f in fields], send.data_ptr(), dev, st)

    def unpack(self, recv, fields):
        dev, st = self._stream(recv)
        self.plan.unpack(recv.data_ptr(), [f.data_ptr() for f in fields], dev, st)

    def pack_blocks(self, x, bs, send):
        dev, st = self._stream(send)
        self.plan.pack_blocks(x.data_ptr(), bs, send.data_ptr(), dev, st)

    def unpack_blocks(self, recv, bs, x):
        dev, st = self._stream(recv)
        self.plan.unpack_blocks(recv.data_ptr(), bs, x.data_ptr(), dev, st)


class HaloExchanger:
    """HaloExchanger (src/fields/halo.cpp:212-330) over torch.distributed.

    Fields are 1-D float64 tensors of at least plan.n_local entries (local
    cell order), on the device the library packs them on.  `group` is the
    torch.distributed process group (None: the default one).  `packer`
    replaces the device packing (an object with pack(fields, send),
    unpack(recv, fields), pack_blocks(x, bs, send), unpack_blocks(recv, bs,
    x)); the default, DevicePacker, runs the library's kernels and needs
    CUDA tensors."""

    # the reference's message tags: cell fields, gradients + limiters,
    # one-off groups (src/fields/halo.cpp:16-18), block vectors
    # (vector_layout.hpp:215)
    FIELD_TAG, GRAD_LIMITER_TAG, ONCE_TAG, VECTOR_TAG = 4242, 4243, 4244, 4317

    def __init__(self, plan: HaloPlan, group=None, packer=None):
        self.plan = plan
        self.group = group
        self.packer = packer if packer is not None else DevicePacker(plan)
        self._pack, self._unpack = self.packer.pack, self.packer.unpack
        self._phases = {"fields": {"ptrs": [], "tag": self.FIELD_TAG},
                        "grads": {"ptrs": [], "tag": self.GRAD_LIMITER_TAG}}

    # registration (initialisation time)
    def register_cell_fields(self, fields):
        self._register("fields", list(fields))

    def register_grad_limiters(self, grad_x, grad_y, grad_z, limiters=()):
        ptrs = []
        for gx, gy, gz in zip(grad_x, grad_y, grad_z):
            ptrs += [gx, gy, gz]
        self._register("grads", ptrs + list(limiters))

    def _register(self, phase, tensors):
        for t in tensors:
            if t.dim() != 1 or t.numel() < self.plan.n_local:
                raise ValueError("a registered field needs n_local entries (owned + ghost cells)")
        ph = self._phases[phase]
        ph["ptrs"] += tensors
        self._resize(ph)

    def _resize(self, ph):
        import torch
        nv = len(ph["ptrs"])
        like = ph["ptrs"][0]
        ph["send"] = torch.zeros(self.plan.n_send * nv, dtype=torch.float64, device=like.device)
        ph["recv"] = torch.zeros(self.plan.n_recv * nv, dtype=torch.float64, device=like.device)
        ph["reqs"] = []

    @property
    def num_registered_fields(self) -> int:
        return len(self._phases["fields"]["ptrs"])

    @property
    def num_registered_grads_and_limiters(self) -> int:
        return len(self._phases["grads"]["ptrs"])

    # one phase: post receives, pack and send, then wait and unpack
    def _start(self, ph, nv=None, packed=False):
        import torch.distributed as dist
        p = self.plan
        if not p.nb_ranks.size or not ph["ptrs"]:
            return
        if nv is None:
            nv = len(ph["ptrs"])
        if not packed:
            self._pack(ph["ptrs"], ph["send"])
        ops = []
        for k, r in enumerate(p.nb_ranks):
            r0, r1 = int(p.recv_offsets[k]) * nv, int(p.recv_offsets[k + 1]) * nv
            ops.append(dist.P2POp(dist.irecv, ph["recv"][r0:r1], int(r), self.group, ph["tag"]))
        for k, r in enumerate(p.nb_ranks):
            s0, s1 = int(p.send_offsets[k]) * nv, int(p.send_offsets[k + 1]) * nv
            ops.append(dist.P2POp(dist.isend, ph["send"][s0:s1], int(r), self.group, ph["tag"]))
        ph["reqs"] = dist.batch_isend_irecv(ops)

    def _finish(self, ph, unpack=True):
        p = self.plan
        if not p.nb_ranks.size or not ph["ptrs"]:
            return
        for q in ph["reqs"]:
            q.wait()
        ph["reqs"] = []
        if unpack:
            self._unpack(ph["recv"], ph["ptrs"])

    def start_exchange_fields(self):
        self._start(self._phases["fields"])

    def finish_exchange_fields(self):
        self._finish(self._phases["fields"])

    def exchange_fields(self):
        self.start_exchange_fields()
        self.finish_exchange_fields()

    def start_exchange_grad_limiters(self):
        self._start(self._phases["grads"])

    def finish_exchange_grad_limiters(self):
        self._finish(self._phases["grads"])

    def exchange_grad_limiters(self):
        self.start_exchange_grad_limiters()
        self.finish_exchange_grad_limiters()

    def exchange_once(self, fields):
        """Blocking exchange of an unregistered group (its own message and tag)."""
        fields = list(fields)
        if not self.plan.nb_ranks.size or not fields:
            return
        ph = {"ptrs": fields, "tag": self.ONCE_TAG}
        self._resize(ph)
        self._start(ph)
        self._finish(ph)


    def exchange_vector(self, x, bs: int):
        """Ghost rows of a block vector x[row*bs + v] (n_local rows, the
        Krylov vectors' layout) from their owners: the reference vector
        layout's pack_values, post_sr and wait_and_unpack
        (include/cfd/linalg/vector_layout.hpp:172-260)."""
        import torch
        p = self.plan
        if not p.nb_ranks.size:
            return
        if x.dim() != 1 or x.numel() < p.n_local * bs:
            raise ValueError("the vector needs n_local * bs entries")
        ph = {"ptrs": [x], "tag": self.VECTOR_TAG, "reqs": [],
              "send": torch.zeros(p.n_send * bs, dtype=torch.float64, device=x.device),
              "recv": torch.zeros(p.n_recv * bs, dtype=torch.float64, device=x.device)}
        self.packer.pack_blocks(x, bs, ph["send"])
        self._start(ph, nv=bs, packed=True)
        self._finish(ph, unpack=False)
        self.packer.unpack_blocks(ph["recv"], bs, x)


def allreduce_sum(values, group=None):
    """Sum of per-rank partial values over the ranks (the reduction the
    distributed inner products and residual norms need); `values` is a
    float64 tensor, reduced in place and returned."""
    import torch.distributed as dist
    dist.all_reduce(values, op=dist.ReduceOp.SUM, group=group)
    return values
