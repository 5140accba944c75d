"""Blocks spread over ranks, one process and one GPU per rank.

The reference spreads its leaf blocks over MPI processes in contiguous runs
of the leaf list (src/mesh.F90:652-721), fills the ghost cells whose source
block lives on another process from slabs exchanged every stage
(boundaries_*_copy with exchange_real_arrays, src/boundaries.F90:1554,
src/mpitools.F90:1472-1539), and reduces the maximum speed over processes
before each time step (reduce_maximum_real, src/evolution.F90:459-460).
``ShardedSimulation`` does the same over torch.distributed: the library
context of each rank holds its leaves (amun_gpu_set_blocks_sharded), packs
the slabs other ranks need into one device buffer, the slabs go peer to peer
(NCCL send/receive pairs between GPUs, gloo between host processes), and
the library unpacks what arrived into its ghost cells.

One step:

    ms = sim.local_maxspeed()                 # this rank's max |v| + c
    ms = allreduce(ms, MAX)
    t, dt = sim.begin_step(ms, dtnext)        # new_time_step with the global speed
    for s in 1..sim.nstages:
        sim.stage(s)                          # sweeps, combination, local ghost fill
        sim.pack(); exchange(); sim.unpack()  # ghost slabs from other ranks
    sim.end_step()

``advance`` runs that with torch.distributed; the phases are public so that a
caller (or a test) can drive several ranks' contexts itself.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .mesh import UniformMesh
from .params import geometry, to_native


def partition(nleafs: int, nprocs: int) -> np.ndarray:
    """The rank of every leaf: contiguous runs of the leaf list, the first
    nleafs mod nprocs ranks one leaf more (src/mesh.F90:652-721)."""
    if nleafs <= 0 or nprocs <= 0:
        raise ValueError("need leaves and ranks")
    lb = np.full(nprocs, nleafs // nprocs)
    lb[:nleafs % nprocs] += 1
    return np.repeat(np.arange(nprocs, dtype=np.int32), lb)


def halo_plan(mesh, owner: np.ndarray, rank: int):
    """The library's exchange plan for `rank` (host only): (send, recv),
    arrays of rows (peer, this rank's leaf, other leaf, direction, cells) in
    buffer order."""
    L = N.lib()
    desc = mesh.descriptors()
    owner = np.ascontiguousarray(owner, dtype=np.int32)
    cap = 27 * mesh.nblocks
    send = np.zeros((cap, 5), dtype=np.int32)
    recv = np.zeros((cap, 5), dtype=np.int32)
    ns, nr = C.c_int(), C.c_int()
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))  # noqa: E731
    N.check(L.amun_gpu_halo_plan(mesh.nblocks, desc, ip(owner), rank, mesh.ndims, mesh.nc, mesh.ng, cap,
                                 C.byref(ns), ip(send), C.byref(nr), ip(recv)))
    return send[:ns.value].copy(), recv[:nr.value].copy()


class ShardedSimulation:
    """This rank's share of a uniform periodic block mesh (one level)."""

    def __init__(self, params: dict, rank: int, world: int, precision: str = "fp64"):
        import torch
        self.params = dict(params)
        self.params["precision"] = precision
        self.rank, self.world = int(rank), int(world)
        self.L = N.ContextLib()
        self.native = to_native(self.params)
        self.mesh = UniformMesh(geometry(self.params))
        self.nv = (5 if self.native.eqsys in (N.AMUN_EQ_HD, N.AMUN_EQ_SRHD) else 9) - \
            (self.native.eos == N.AMUN_EOS_ISO)
        N.check(self.L.amun_gpu_init(C.byref(self.native)))
        self.owner = partition(self.mesh.nblocks, self.world)
        self.mine = np.flatnonzero(self.owner == self.rank)
        self._desc = self.mesh.descriptors()
        owner = np.ascontiguousarray(self.owner, dtype=np.int32)
        N.check(self.L.amun_gpu_set_blocks_sharded(self.mesh.nblocks, self._desc,
                                                   owner.ctypes.data_as(C.POINTER(C.c_int)), self.rank))
        cap = max(1, self.world)
        npeers = C.c_int()
        ranks = (C.c_int * cap)()
        sn, rn = (C.c_longlong * cap)(), (C.c_longlong * cap)()
        eb = C.c_int()
        N.check(self.L.amun_gpu_halo_peers(cap, C.byref(npeers), ranks, sn, rn, C.byref(eb)))
        self.peers = [(ranks[k], sn[k], rn[k]) for k in range(npeers.value)]
        dtype = torch.float64 if eb.value == 8 else torch.float32
        self.sendbuf = torch.empty(max(1, sum(p[1] for p in self.peers)), dtype=dtype, device="cuda")
        self.recvbuf = torch.empty(max(1, sum(p[2] for p in self.peers)), dtype=dtype, device="cuda")
        n = C.c_int()
        N.check(self.L.amun_gpu_stages(C.byref(n)))
        self.nstages = n.value
        self.time, self.dt = 0.0, 0.0
        # the library launches on the caller's current stream, so that the
        # pack, the transfers and the unpack are ordered on one stream; the
        # legacy default stream (handle 0) would mean the library's own
        # stream, unordered with torch's work, so a new stream replaces it
        cur = torch.cuda.current_stream()
        self.stream = cur if cur.cuda_stream else torch.cuda.Stream()
        N.check(self.L.amun_gpu_set_stream(C.c_void_p(self.stream.cuda_stream)))

    # ---- state -----------------------------------------------------------------
    def set_primitive(self, q: np.ndarray):
        """This rank's blocks of the global primitive field q (NZ, NY, NX, nv):
        u0 = prim2cons(q), upload, ghost fill of the local neighbours (the
        caller then exchanges, as after every stage)."""
        qb = np.ascontiguousarray(self.mesh.to_blocks(np.asarray(q, dtype=np.float64))[self.mine])
        ub = np.empty_like(qb)
        N.check(self.L.amun_gpu_prim2cons(qb.size // self.nv, N.dptr(qb), N.dptr(ub)))
        N.check(self.L.amun_gpu_upload_blocks(0, len(self.mine), N.dptr(ub), N.dptr(qb)))
        N.check(self.L.amun_gpu_boundary_variables())
        N.check(self.L.amun_gpu_set_time(0.0, 0.0))
        self.time = 0.0

    def set_primitive_blocks(self, qb: np.ndarray):
        """This rank's block arrays of primitives (Fortran layout, ghost
        entries ignored) as the state; the caller exchanges afterwards."""
        qb = np.ascontiguousarray(qb, dtype=np.float64)
        ub = np.empty_like(qb)
        N.check(self.L.amun_gpu_prim2cons(qb.size // self.nv, N.dptr(qb), N.dptr(ub)))
        N.check(self.L.amun_gpu_upload_blocks(0, len(self.mine), N.dptr(ub), N.dptr(qb)))
        N.check(self.L.amun_gpu_boundary_variables())
        N.check(self.L.amun_gpu_set_time(0.0, 0.0))
        self.time = 0.0

    def upload_conserved(self, ub: np.ndarray):
        """This rank's conserved block arrays (Fortran layout, host or
        device); primitives and local ghosts are rebuilt on the device, the
        caller exchanges the remote ghosts afterwards."""
        N.check(self.L.amun_gpu_upload_conserved(0, len(self.mine), N.dptr(ub)))

    def download_conserved(self, ub: np.ndarray):
        N.check(self.L.amun_gpu_download_blocks(0, len(self.mine), N.dptr(ub), None))

    def blocks(self):
        """(u0, q) block arrays of this rank's leaves (Fortran layout)."""
        shp = (len(self.mine), self.mesh.km, self.mesh.jm, self.mesh.im, self.nv)
        u, q = np.empty(shp), np.empty(shp)
        N.check(self.L.amun_gpu_download_blocks(0, len(self.mine), N.dptr(u), N.dptr(q)))
        return u, q

    # ---- the phases of one step -------------------------------------------------
    def local_maxspeed(self) -> float:
        ms = C.c_double()
        N.check(self.L.amun_gpu_get_maxspeed(C.byref(ms)))
        return ms.value

    def begin_step(self, global_maxspeed: float, dtnext: float = 1.0e30):
        N.check(self.L.amun_gpu_set_maxspeed(float(global_maxspeed)))
        cm, dt = C.c_double(), C.c_double()
        N.check(self.L.amun_gpu_new_time_step(float(dtnext), C.byref(cm), C.byref(dt)))
        self.dt = dt.value
        return self.time, self.dt

    def stage(self, s: int):
        N.check(self.L.amun_gpu_stage(int(s), self.time, self.dt))

    def pack(self):
        N.check(self.L.amun_gpu_halo_pack(C.c_void_p(self.sendbuf.data_ptr())))

    def unpack(self):
        N.check(self.L.amun_gpu_halo_unpack(C.c_void_p(self.recvbuf.data_ptr())))

    def end_step(self):
        self.time += self.dt
        N.check(self.L.amun_gpu_set_time(self.time, self.dt))

    # ---- with torch.distributed -------------------------------------------------
    def exchange(self, group=None):
        """Pack, one send and one receive per peer, unpack (NCCL orders the
        transfers after the pack on the current stream and the unpack after
        the transfers)."""
        import torch
        import torch.distributed as dist
        self.pack()
        ops, so, ro = [], 0, 0
        for peer, ns, nr in self.peers:
            ops.append(dist.P2POp(dist.isend, self.sendbuf[so:so + ns], peer, group))
            ops.append(dist.P2POp(dist.irecv, self.recvbuf[ro:ro + nr], peer, group))
            so, ro = so + ns, ro + nr
        if ops:
            with torch.cuda.stream(self.stream):
                for req in dist.batch_isend_irecv(ops):
                    req.wait()
        self.unpack()

    def allreduce_maxspeed(self, group=None) -> float:
        import torch
        import torch.distributed as dist
        t = torch.tensor([self.local_maxspeed()], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
        return float(t.item())

    def advance(self, dtnext: float = 1.0e30, group=None):
        """One step of every rank's blocks (all ranks call it together)."""
        self.begin_step(self.allreduce_maxspeed(group), dtnext)
        for s in range(1, self.nstages + 1):
            self.stage(s)
            self.exchange(group)
        self.end_step()
        return self.time, self.dt

    def close(self):
        self.L.amun_gpu_finalize()
        self.L.destroy()
