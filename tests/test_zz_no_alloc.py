"""artss_residual_norm_static: the residual norm for callers that cannot
allocate device memory (a host code whose allocator owns the GPU, a memory
pool that must not grow).  It keeps its partial sums in a fixed device array
of the library instead of context memory; its results must equal those of
artss_residual_norm, which uses context scratch, on two calls in a row, and
the same norms computed on the CPU from the downloaded arrays.

Collected last on purpose (file name), so that a run stopping at the first
failure has run every other test first."""
import ctypes as C

import numpy as np
import pytest

import artss_b200 as A
from artss_b200 import scenes

pytestmark = pytest.mark.gpu
TOL = 1e-10
_D = C.POINTER(C.c_double)


def _static_fn():
    lib = A.load_cuda()
    f = lib.artss_residual_norm_static
    f.argtypes = [C.POINTER(A.GridDesc), C.c_void_p, _D, _D, C.c_void_p, _D, _D]
    f.restype = C.c_int
    return lib, f


def _norms(sim, lib, f, grid, flags_ptr):
    p = C.cast(C.c_void_p(sim.device_pointer("p")), _D)
    b = C.cast(C.c_void_p(sim.device_pointer("rhs")), _D)
    r_ctx, b_ctx = C.c_double(), C.c_double()
    A.cuda_check(lib.artss_residual_norm(sim.context, p, b, C.byref(r_ctx), C.byref(b_ctx)), "residual_norm")
    r_st, b_st = C.c_double(), C.c_double()
    A.cuda_check(f(C.byref(grid), flags_ptr, p, b, lib.artss_ctx_stream(sim.context), C.byref(r_st), C.byref(b_st)),
                 "residual_norm_static")
    return (r_ctx.value, b_ctx.value), (r_st.value, b_st.value)


def _check(ref, got):
    for x, y in zip(ref, got):
        assert np.isfinite(y)
        assert abs(x - y) <= TOL * max(abs(x), 1e-300), (ref, got)


def _cpu_norms(sim, grid, inner):
    """||b - A p||_2 over the inner cells and ||b||_2, the 7-point Laplacian
    of VCycleMG.cpp:186-194 evaluated in numpy on the downloaded arrays"""
    p, b = sim.field("p"), sim.field("rhs")
    nj, nk = grid.Nx[0], grid.Nx[0] * grid.Ny[0]
    rx, ry, rz = (1.0 / (grid.dx[0] * grid.dx[0]), 1.0 / (grid.dy[0] * grid.dy[0]), 1.0 / (grid.dz[0] * grid.dz[0]))
    q = inner
    r = b[q] - (rx * (p[q - 1] - 2 * p[q] + p[q + 1]) + ry * (p[q - nj] - 2 * p[q] + p[q + nj]) +
                rz * (p[q - nk] - 2 * p[q] + p[q + nk]))
    return float(np.sqrt(np.sum(r * r))), float(np.sqrt(np.sum(b[q] * b[q])))


def test_static_residual_norm_box(tmp_path):
    """obstacle-free box: flags = NULL (every computational-domain cell is inner)"""
    lib, f = _static_fn()
    xml = scenes.write(scenes.plume_box(n=32, steps=4, n_level=3), str(tmp_path / "box.xml"))
    geom = A.Geometry(xml)
    grid = geom.grid_desc()
    inner = geom.list("inner", 0)
    with A.Simulation(xml) as sim:
        for _ in range(2):
            sim.run(1)
            ref, got = _norms(sim, lib, f, grid, None)
            assert ref[1] > 0
            _check(ref, got)
            _check(_cpu_norms(sim, grid, inner), got)


def test_static_residual_norm_with_obstacle(tmp_path):
    """channel with a cube: the caller passes its own device array of inner flags"""
    torch = pytest.importorskip("torch")
    lib, f = _static_fn()
    xml = scenes.write(scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=4, n_level=3), str(tmp_path / "ch.xml"))
    geom = A.Geometry(xml)
    grid = geom.grid_desc()
    n = grid.Nx[0] * grid.Ny[0] * grid.Nz[0]
    flags = np.zeros(n, np.uint8)
    flags[geom.list("inner", 0)] = 1
    d_flags = torch.from_numpy(flags).to("cuda:0")
    with A.Simulation(xml) as sim:
        for _ in range(2):
            sim.run(1)
            torch.cuda.synchronize()
            ref, got = _norms(sim, lib, f, grid, C.c_void_p(d_flags.data_ptr()))
            _check(ref, got)
            _check(_cpu_norms(sim, grid, geom.list("inner", 0)), got)


def _grid(nx, ny, nz, d=1.0):
    grid = A.GridDesc()
    grid.n_levels = 0
    grid.Nx[0], grid.Ny[0], grid.Nz[0] = nx + 2, ny + 2, nz + 2
    grid.i1[0], grid.i2[0] = 1, nx
    grid.j1[0], grid.j2[0] = 1, ny
    grid.k1[0], grid.k2[0] = 1, nz
    grid.dx[0] = grid.dy[0] = grid.dz[0] = d
    return grid


def _device_arrays(grid):
    """zero device arrays p, b covering the whole described grid, so that no
    access could leave them even if a size check were missing"""
    torch = pytest.importorskip("torch")
    n = grid.Nx[0] * grid.Ny[0] * grid.Nz[0]
    p = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    b = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    return p, b, C.cast(C.c_void_p(p.data_ptr()), _D), C.cast(C.c_void_p(b.data_ptr()), _D)


def test_static_residual_norm_rejects_oversized_grid():
    lib, f = _static_fn()
    grid = _grid(64 * 200, 4 * 50, 1)  # 10000 tiles of 64x4 cells per plane: above the 8192 limit
    keep = _device_arrays(grid)
    r, bn = C.c_double(), C.c_double()
    st = f(C.byref(grid), None, keep[2], keep[3], None, C.byref(r), C.byref(bn))
    assert st == -6
    assert b"too large" in lib.artss_last_error()


@pytest.mark.parametrize("d", [0.0, -1.0, float("inf"), float("nan")])
def test_static_residual_norm_rejects_bad_spacing(d):
    lib, f = _static_fn()
    grid = _grid(8, 8, 8)
    grid.dy[0] = d
    keep = _device_arrays(grid)
    r, bn = C.c_double(), C.c_double()
    st = f(C.byref(grid), None, keep[2], keep[3], None, C.byref(r), C.byref(bn))
    assert st == -1
    assert b"spacing" in lib.artss_last_error()
