"""Blocks spread over ranks, tested on host processes (gloo, no GPU).

Each rank advances its share of the leaves with the oracle's per-block
procedures (update_flux, cons2prim, maxspeed) and numpy for the increment and
the SSPRK(2,2) combination, in the reference's operation order
(src/evolution.F90:628-770, 1898-1977).  Its ghost cells come from its own
blocks where the neighbour is local and, where it is not, from the slabs of
the library's exchange plan (amun_gpu_halo_plan), packed and unpacked with
the layout of the device kernels and sent between the processes with
torch.distributed (gloo); the maximum speed is reduced over the ranks before
each step (src/evolution.F90:459-460).  After three steps every rank's
blocks must equal the single-process oracle's bit for bit."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _box(d, nd, nc, ng):
    """ghost-cell ranges (k, j, i) of direction d, and the direction offsets"""
    o = (d % 3 - 1, (d // 3) % 3 - 1, d // 9 - 1)
    rng = []
    for a in (2, 1, 0):
        if a >= nd:
            rng.append(slice(0, 1))
            continue
        lo = 0 if o[a] < 0 else (ng if o[a] == 0 else ng + nc)
        rng.append(slice(lo, lo + (nc if o[a] == 0 else ng)))
    return rng, o


def _shift(rng, o, nc, nd):
    out = []
    for r, a in zip(rng, (2, 1, 0)):
        s = o[a] * nc if a < nd else 0
        out.append(slice(r.start - s, r.stop - s))
    return out


class HostRank:
    """One rank of the sharded step on the host."""

    def __init__(self, p, rank, world):
        import oracle
        from amun_b200.mesh import UniformMesh
        from amun_b200.params import geometry
        from amun_b200.shards import halo_plan, partition
        self.p, self.rank = p, rank
        self.mesh = UniformMesh(geometry(p))
        self.o = oracle.Oracle(p)  # per-block procedures on the same block shape
        self.nv = self.o.nv
        self.owner = partition(self.mesh.nblocks, world)
        self.mine = list(np.flatnonzero(self.owner == rank))
        self.local = {int(g): k for k, g in enumerate(self.mine)}
        self.send, self.recv = halo_plan(self.mesh, self.owner, rank)
        self.nbr = self.mesh.descriptors()
        self.nd, self.nc, self.ng = self.mesh.ndims, self.mesh.nc, self.mesh.ng

    def set_prim(self, q0):
        self.q = self.mesh.to_blocks(q0)[self.mine].copy()
        self.u0 = self.o.prim2cons(self.q)
        self.u1 = np.zeros_like(self.u0)

    def fill_local(self):
        nd, nc, ng = self.nd, self.nc, self.ng
        for k, g in enumerate(self.mine):
            for d in range(27):
                if d == 13 or (nd == 2 and d // 9 != 1):
                    continue
                nb = self.nbr[int(g)].neighbor[d]
                if nb not in self.local:
                    continue
                rng, o = _box(d, nd, nc, ng)
                self.q[k][tuple(rng)] = self.q[self.local[nb]][tuple(_shift(rng, o, nc, nd))]

    def exchange(self, dist):
        nd, nc, ng, nv = self.nd, self.nc, self.ng, self.nv
        import torch
        peers = sorted(set(int(r[0]) for r in self.send) | set(int(r[0]) for r in self.recv))
        out = {p: [] for p in peers}
        for peer, blk, other, d, cells in self.send:
            rng, o = _box(d, nd, nc, ng)
            v = self.q[self.local[int(blk)]][tuple(_shift(rng, o, nc, nd))]  # (lz, ly, lx, nv)
            out[int(peer)].append(np.moveaxis(v, -1, 0).reshape(nv, -1).ravel())
        ins = {p: np.empty(int(sum(r[4] for r in self.recv if r[0] == p)) * nv) for p in peers}
        ops = []
        for p in peers:
            ops.append(dist.P2POp(dist.isend, torch.from_numpy(np.concatenate(out[p])), p))
            ops.append(dist.P2POp(dist.irecv, torch.from_numpy(ins[p]), p))
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        offs = {p: 0 for p in peers}
        for peer, blk, other, d, cells in self.recv:
            p = int(peer)
            seg = ins[p][offs[p]:offs[p] + cells * nv]
            offs[p] += cells * nv
            rng, _ = _box(d, nd, nc, ng)
            shp = tuple(r.stop - r.start for r in rng)
            self.q[self.local[int(blk)]][tuple(rng)] = np.moveaxis(seg.reshape((nv,) + shp), 0, -1)

    def increment(self, f, dx):
        ng, nc, nd = self.ng, self.nc, self.nd
        du = np.zeros(f.shape[:-1])
        s, m = slice(ng - 1, ng + nc + 1), slice(ng - 2, ng + nc)
        ks, km = (s, m) if nd == 3 else (slice(0, 1), slice(0, 1))
        a = (-1.0 / dx[0]) * (f[ks, s, s, :, 0] - f[ks, s, m, :, 0]) - (1.0 / dx[1]) * (f[ks, s, s, :, 1] -
                                                                                         f[ks, m, s, :, 1])
        if nd == 3:
            a = a - (1.0 / dx[2]) * (f[s, s, s, :, 2] - f[m, s, s, :, 2])
        du[ks, s, s] = a
        return du

    def step(self, dist):
        import torch
        ng, nc, nd = self.ng, self.nc, self.nd
        cm = max(np.finfo(float).tiny, max(self.o.maxspeed(qb) for qb in self.q))
        t = torch.tensor([cm], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        cmax = float(t.item())
        m = self.mesh
        dxs = (m.dx, m.dy, m.dz)
        dx_min = min(m.dx, m.dy) if nd == 2 else min(min(m.dx, m.dy), m.dz)
        dt = self.p["cfl"] * dx_min / max(cmax + 2.0 * 0.0 / dx_min, np.finfo(float).tiny)
        inner = (slice(ng, ng + nc),) * 2
        inner = ((slice(ng, ng + nc),) if nd == 3 else (slice(0, 1),)) + inner
        for stage in (1, 2):
            for k in range(len(self.mine)):
                du = self.increment(self.o.update_flux(self.q[k]), dxs)
                if stage == 1:
                    self.u1[k] = self.u0[k] + dt * du
                    u = self.u1[k]
                else:
                    self.u0[k] = 0.5 * (self.u0[k] + self.u1[k] + dt * du)
                    u = self.u0[k]
                self.q[k][inner] = self.o.cons2prim(u[inner])
            self.fill_local()
            self.exchange(dist)
        return dt


def _rank_main(rank, world, port, p, q0, ref_q, ref_u):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r = HostRank(p, rank, world)
        r.set_prim(q0)
        r.fill_local()
        r.exchange(dist)
        for _ in range(3):
            r.step(dist)
        qb = r.mesh.to_blocks(ref_q)[r.mine]
        ub = r.mesh.to_blocks(ref_u)[r.mine]
        ng, nc, nd = r.ng, r.nc, r.nd
        inner = ((slice(ng, ng + nc),) if nd == 3 else (slice(0, 1),)) + (slice(ng, ng + nc),) * 2
        for k in range(len(r.mine)):
            assert np.array_equal(r.q[k][inner], qb[k][inner]), f"rank {rank} block {r.mine[k]}: primitives differ"
            assert np.array_equal(r.u0[k][inner], ub[k][inner]), f"rank {rank} block {r.mine[k]}: conserved differ"
        # every ghost cell equals the single-process state's (periodic wrap)
        for k in range(len(r.mine)):
            assert np.array_equal(r.q[k], qb[k]), f"rank {rank} block {r.mine[k]}: ghost cells differ"
    finally:
        dist.destroy_process_group()


CASES = [
    # (ndims, blocks per direction, ncells, ranks)
    (2, (4, 2, 1), 8, 2),
    (2, (4, 2, 1), 8, 3),
    (3, (2, 2, 2), 8, 2),
    (3, (2, 2, 2), 8, 4),
]


@pytest.mark.parametrize("nd,nb,n,world", CASES)
def test_sharded_steps_match_single_process_oracle(oracle_mod, nd, nb, n, world):
    import torch.multiprocessing as mp
    from helpers import params
    from amun_b200 import problems
    from amun_b200.mesh import UniformMesh
    from amun_b200.params import geometry
    kw = dict(ncells=n, nghosts=2, xblocks=nb[0], yblocks=nb[1], xmin=-0.5, xmax=0.5, ymin=-0.5, ymax=0.5)
    if nd == 3:
        kw.update(zblocks=nb[2], zmin=-0.5, zmax=0.5)
    p = params("hd", "tvd", "hllc", "rk2", ndims=nd, **kw)
    mesh = UniformMesh(geometry(p))
    q0 = problems.blast(mesh, 5, 5.0 / 3.0, ratio=10.0, radius=0.3, csnd=np.sqrt(5.0 / 3.0))
    o = oracle_mod.Oracle(p)
    o.set_prim(q0)
    for _ in range(3):
        o.advance(1.0e30)
    mp.spawn(_rank_main, args=(world, _free_port(), p, q0, o.prim(), o.cons()), nprocs=world, join=True)


def test_partition_follows_the_reference():
    """Contiguous runs of the leaf list, the first nleafs mod nprocs ranks
    one leaf more (src/mesh.F90:652-721)."""
    from amun_b200.shards import partition
    assert partition(8, 3).tolist() == [0, 0, 0, 1, 1, 1, 2, 2]
    assert partition(7, 2).tolist() == [0, 0, 0, 0, 1, 1, 1]
    assert partition(4, 4).tolist() == [0, 1, 2, 3]
    assert partition(1, 1).tolist() == [0]


def test_halo_plan_pairs_up():
    """Every rank's outgoing slabs to a peer are exactly that peer's incoming
    slabs, in the same order and with the same sizes."""
    from amun_b200.mesh import UniformMesh
    from amun_b200.params import geometry
    from amun_b200.shards import halo_plan, partition
    from helpers import params
    p = params("hd", "tvd", "hllc", "rk2", ndims=3, ncells=8, nghosts=2, xblocks=3, yblocks=2, zblocks=2)
    mesh = UniformMesh(geometry(p))
    world = 5
    owner = partition(mesh.nblocks, world)
    plans = [halo_plan(mesh, owner, r) for r in range(world)]
    for r in range(world):
        send, _ = plans[r]
        for peer in set(int(x) for x in send[:, 0]):
            out = send[send[:, 0] == peer][:, [2, 1, 3, 4]]  # receiving leaf, sending leaf, dir, cells
            _, recv = plans[peer]
            inc = recv[recv[:, 0] == r][:, [1, 2, 3, 4]]
            assert np.array_equal(out, inc)
        # every remote face/edge/corner of the rank's leaves is received once
        _, recv = plans[r]
        mine = set(np.flatnonzero(owner == r).tolist())
        desc = mesh.descriptors()
        want = sorted((b, d) for b in mine for d in range(27)
                      if d != 13 and owner[desc[b].neighbor[d]] != r)
        assert sorted((int(x[1]), int(x[3])) for x in recv) == want
