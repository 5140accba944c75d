"""amun_gpu_update_flux_block_noalloc against amun_gpu_update_flux_block.

The allocation-free entry point takes device arrays and uses the library's
fixed device scratch; on the same block it must give the same fluxes as the
allocating entry point, call after call, and reject what does not fit."""
import ctypes as C

import numpy as np
import pytest

from helpers import params
from amun_b200 import problems

pytestmark = pytest.mark.gpu

# (system, reconstruction, solver, ndims, ncells, extra parameters): WENO3
# reads the cell sizes (dx), the relativistic 4-vector case uses the larger
# line scratch of the 4-vector states
CASES = [
    ("mhd", "weno5z", "hlld", 3, 16, {}),
    ("hd", "tvd", "hllc", 2, 32, {}),
    ("mhd", "weno3", "hlld", 2, 32, {"nghosts": 2}),
    ("hd", "limo3", "hllc", 3, 16, {"nghosts": 2}),
    ("srmhd", "tvd", "hllc", 3, 16, {"state_variables": "4vec", "gamma": 4.0 / 3.0, "xmin": 0.0, "xmax": 1.0,
                                     "ymin": 0.0, "ymax": 1.0, "zmin": 0.0, "zmax": 1.0}),
]


def _inputs(sim, eq, seed):
    if eq == "mhd":
        q = problems.turbulence(sim.mesh, 5.0 / 3.0, seed=seed)
    elif eq == "srmhd":
        q = problems.srmhd_turbulence(sim.mesh, seed=seed, lorentz_max=4.0)
    else:
        q = problems.blast(sim.mesh, 5, 5.0 / 3.0, ratio=10.0 + seed, radius=0.2)
    return np.ascontiguousarray(sim.mesh.to_blocks(q)[0])


@pytest.mark.parametrize("eq,rec,rs,nd,n,kw", CASES)
def test_noalloc_matches_allocating_entry(eq, rec, rs, nd, n, kw):
    import torch
    from amun_b200.solver import Simulation
    sim = Simulation(params(eq, rec, rs, "rk2", ndims=nd, ncells=n, **kw))
    try:
        sim.set_cmax(1.7)
        L = sim.L
        dx = np.array([sim.mesh.dx, sim.mesh.dy, sim.mesh.dz][:nd])
        for call, seed in enumerate((1, 2)):
            q = _inputs(sim, eq, seed)
            ref = sim.update_flux_block(q)
            qd = torch.from_numpy(q).cuda()
            fd = torch.full(ref.shape, float("nan"), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
            rc = L.amun_gpu_update_flux_block_noalloc(dx.ctypes.data_as(C.POINTER(C.c_double)),
                                                      qd.data_ptr(), fd.data_ptr())
            torch.cuda.synchronize()
            free1 = torch.cuda.mem_get_info()[0]
            assert rc == 0, L.amun_gpu_last_error().decode()
            out = fd.cpu().numpy()
            # same kernels, same FP64 arithmetic: bit-identical
            assert np.array_equal(out, ref), f"call {call}: max diff {np.nanmax(np.abs(out - ref))}"
            if call == 1:
                assert free1 == free0, "device memory changed during the call"
    finally:
        sim.close()


def test_noalloc_needs_dx_where_the_method_reads_it():
    """WENO3 and LimO3 divide by the cell size: a null dx is refused before
    anything is queued, as the allocating entry point refuses it."""
    import torch
    from amun_b200.solver import Simulation
    sim = Simulation(params("hd", "weno3", "hllc", "rk2", ndims=2, ncells=16, nghosts=2))
    try:
        L = sim.L
        shp = (1, sim.mesh.jm, sim.mesh.im, 5)
        qd = torch.ones(shp, dtype=torch.float64, device="cuda")
        fd = torch.zeros(shp + (2,), dtype=torch.float64, device="cuda")
        rc = L.amun_gpu_update_flux_block_noalloc(None, qd.data_ptr(), fd.data_ptr())
        assert rc == 902
        assert b"dx" in L.amun_gpu_last_error()
    finally:
        sim.close()


def test_noalloc_reports_positivity_events():
    """TVD positivity events (a non-positive density or pressure) found by the
    allocation-free call are added to the status counter like the allocating
    call's."""
    import torch
    from amun_b200.solver import Simulation
    sim = Simulation(params("hd", "tvd", "hllc", "rk2", ndims=2, ncells=16))
    try:
        L = sim.L
        q = np.ascontiguousarray(sim.mesh.to_blocks(problems.blast(sim.mesh, 5, 5.0 / 3.0, ratio=10.0,
                                                                   radius=0.2))[0])
        q[..., 5, 6, 0] = -1.0  # one cell with a negative density
        before = sim.status()["nonpositive"]
        sim.update_flux_block(q)
        mid = sim.status()["nonpositive"]
        assert mid > before
        dx = np.full(2, sim.mesh.dx)
        qd = torch.from_numpy(q).cuda()
        fd = torch.zeros(q.shape + (2,), dtype=torch.float64, device="cuda")
        rc = L.amun_gpu_update_flux_block_noalloc(dx.ctypes.data_as(C.POINTER(C.c_double)), qd.data_ptr(),
                                                  fd.data_ptr())
        assert rc == 0, L.amun_gpu_last_error().decode()
        torch.cuda.synchronize()
        assert sim.status()["nonpositive"] - mid == mid - before
    finally:
        sim.close()


def test_noalloc_rejects_oversize_and_host_pointers():
    import torch
    from amun_b200.solver import Simulation
    # 40^3 cells with ghosts: the face states alone exceed the fixed scratch
    sim = Simulation(params("mhd", "weno5z", "hlld", "rk2", ndims=3, ncells=32))
    try:
        L = sim.L
        dx = np.full(3, sim.mesh.dx)
        shp = (sim.mesh.km, sim.mesh.jm, sim.mesh.im, 9)
        qd = torch.ones(shp, dtype=torch.float64, device="cuda")
        fd = torch.zeros(shp + (3,), dtype=torch.float64, device="cuda")
        rc = L.amun_gpu_update_flux_block_noalloc(dx.ctypes.data_as(C.POINTER(C.c_double)),
                                                  qd.data_ptr(), fd.data_ptr())
        assert rc == 904
        assert b"fixed limit" in L.amun_gpu_last_error()
    finally:
        sim.close()
    sim = Simulation(params("hd", "tvd", "hllc", "rk2", ndims=2, ncells=16))
    try:
        L = sim.L
        dx = np.full(2, sim.mesh.dx)
        q = np.ones((1, sim.mesh.jm, sim.mesh.im, 5))
        f = np.zeros(q.shape + (2,))
        rc = L.amun_gpu_update_flux_block_noalloc(dx.ctypes.data_as(C.POINTER(C.c_double)),
                                                  q.ctypes.data, f.ctypes.data)
        assert rc == 902
        assert b"device memory" in L.amun_gpu_last_error()
    finally:
        sim.close()
