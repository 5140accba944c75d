"""Blocks spread over ranks on one GPU: one library context per rank in one
process, the ranks' halo buffers routed between them by device copies in
place of the network (nothing waits on another launch).  After three steps
every rank's blocks, ghost cells included, must equal a single context's
run over the whole mesh bit for bit -- the sweeps and the fused stage
kernel, FP64 and FP32 bulk.  The ranks and the routing copies share one
stream and nothing synchronises between them, as on the real exchange."""
import numpy as np
import pytest

from helpers import params
from amun_b200 import problems

pytestmark = pytest.mark.gpu


def _route(ranks):
    """Copy every rank's send segment for each peer into that peer's receive
    segment for the sender (both ordered by ascending peer rank)."""
    offs = []
    for r in ranks:
        so, ro, s_at, r_at = 0, 0, {}, {}
        for peer, ns, nr in r.peers:
            s_at[peer] = (so, ns)
            r_at[peer] = (ro, nr)
            so, ro = so + ns, ro + nr
        offs.append((s_at, r_at))
    for k, r in enumerate(ranks):
        for peer, _, _ in r.peers:
            so, ns = offs[k][0][peer]
            ro, nr = offs[peer][1][k]
            assert ns == nr
            ranks[peer].recvbuf[ro:ro + nr].copy_(r.sendbuf[so:so + ns])


def _step(ranks):
    ms = max(r.local_maxspeed() for r in ranks)
    for r in ranks:
        r.begin_step(ms)
    for s in range(1, ranks[0].nstages + 1):
        for r in ranks:
            r.stage(s)
            r.pack()
        _route(ranks)
        for r in ranks:
            r.unpack()
    for r in ranks:
        r.end_step()


@pytest.mark.parametrize("prec,fused,world,nd", [("fp64", 0, 2, 3), ("fp64", 1, 3, 3), ("fp32", 0, 2, 2),
                                                  ("fp32", 1, 2, 3)])
def test_sharded_ranks_match_one_context(prec, fused, world, nd):
    import torch
    from amun_b200.shards import ShardedSimulation
    from amun_b200.solver import Simulation
    kw = dict(ncells=16, xblocks=3, yblocks=2, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0)
    if nd == 3:
        kw.update(zblocks=2, zmin=0.0, zmax=1.0)
    p = params("mhd", "weno5z", "hlld", "rk3", ndims=nd, **kw)
    full = Simulation(p, precision=prec)
    with torch.cuda.stream(torch.cuda.Stream()):
        ranks = [ShardedSimulation(p, r, world, precision=prec) for r in range(world)]
        _run(full, ranks, fused)


def _run(full, ranks, fused):
    import torch
    try:
        q0 = problems.turbulence(full.mesh, 5.0 / 3.0, seed=5)
        full.set_stage_kernel(fused, 8)
        full.set_primitive(q0)
        for r in ranks:
            r.L.amun_gpu_set_stage_kernel(fused, 8, None)
            r.set_primitive(q0)
            r.pack()
        _route(ranks)
        for r in ranks:
            r.unpack()
        for _ in range(3):
            full.advance(1.0e30)
            _step(ranks)
        torch.cuda.synchronize()
        uf, qf = full.download_blocks()
        for r in ranks:
            u, q = r.blocks()
            assert np.array_equal(q, qf[r.mine]), f"rank {r.rank}: primitives (ghosts included) differ"
            assert np.array_equal(u, uf[r.mine]), f"rank {r.rank}: conserved state differs"
            assert abs(r.time - full.status()["time"]) == 0.0
    finally:
        full.close()
        for r in ranks:
            r.close()
