"""Mixed-precision pressure solve (FP32 V-cycles inside FP64 defect
correction) against the plain FP64 VCycleMG iterated to a relative tolerance.

The mixed solver's claim, ||b - A p|| <= 1e-8 ||b||, is checked on the CPU
with the oracle's boundary program and a numpy Laplacian, and its solution is
compared with a plain FP64 solve taken to 1e-11.  Right-hand sides are
seeded N(0, 1) fields made consistent with the discrete operator
(artss_b200.consistent_rhs)."""
import ctypes as C

import numpy as np
import pytest

import artss_b200 as A
from artss_b200 import scenes
from tests import cabi, oracle

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle.available(), reason="oracle not built")]

FT_P = 4


def residual_cpu(osc, geom, p, b):
    """b - A p on the level-0 inner cells, FP64, after the oracle's pressure
    boundary program (VCycleMG.cpp:186-194 arithmetic)."""
    d = geom.grid_desc()
    q = p.copy()
    oracle.lib().oracle_apply_bc(osc.ptr, oracle.p(q), 0, FT_P)
    inner = geom.list("inner", 0)
    nj, nk = d.Nx[0], d.Nx[0] * d.Ny[0]
    rx, ry, rz = 1 / d.dx[0] ** 2, 1 / d.dy[0] ** 2, 1 / d.dz[0] ** 2
    c = 2 * q[inner]
    lap = (rx * (q[inner - 1] - c + q[inner + 1]) + ry * (q[inner - nj] - c + q[inner + nj]) +
           rz * (q[inner - nk] - c + q[inner + nk]))
    return b[inner] - lap


def solve_pair(sc, seed, mixed_flags, rel_tol=1e-8, w=0.6666666667):
    import tempfile, os
    xml = scenes.write(sc, os.path.join(tempfile.mkdtemp(), "poisson.xml"))
    geom = A.Geometry(xml)
    ctx = cabi.Context(geom)
    osc = oracle.OracleScene(geom)
    try:
        n = ctx.size()
        inner = geom.list("inner", 0)
        b_raw = scenes.poisson_rhs(inner, n, seed)
        db, b = A.consistent_rhs(ctx, b_raw, sc.n_level)
        # consistent: close to the drawn field, and A p_inf as the CPU computes it
        assert np.linalg.norm(b[inner] - b_raw[inner]) <= 1e-2 * np.linalg.norm(b_raw[inner])
        # plain FP64 reference V-cycle, taken far below the target tolerance
        cfg = A.MgCfg(sc.n_level, 2, 100, 2, 1e-30, 0, 0, 100, 1e-30, 0.6666666667)
        mg = C.c_void_p()
        A.cuda_check(ctx.lib.artss_mg_create(ctx.h, C.byref(cfg), C.byref(mg)), "mg")
        dp_ref = ctx.field(np.zeros(n))
        ref_stats = A.SolveStats()
        A.cuda_check(ctx.lib.artss_mg_solve_rel(mg, dp_ref, db, 1e-11, 2000, C.byref(ref_stats)), "plain")
        ctx.lib.artss_mg_destroy(mg)
        p_ref = ctx.download(dp_ref)
        # mixed precision to the target tolerance
        mcfg = A.MixedCfg(sc.n_level, 2, 1, mixed_flags, w, 0.0, 1e-3, 40, rel_tol, 200)
        mx = C.c_void_p()
        A.cuda_check(ctx.lib.artss_mixed_create(ctx.h, C.byref(mcfg), C.byref(mx)), "mixed")
        dp = ctx.field(np.zeros(n))
        st = A.SolveStats()
        A.cuda_check(ctx.lib.artss_mixed_solve(mx, dp, db, C.byref(st)), "mixed solve")
        # a second solve from the same start reuses the batch hint
        dp2 = ctx.field(np.zeros(n))
        st2 = A.SolveStats()
        A.cuda_check(ctx.lib.artss_mixed_solve(mx, dp2, db, C.byref(st2)), "mixed solve 2")
        ctx.lib.artss_mixed_destroy(mx)
        p = ctx.download(dp)
        p2 = ctx.download(dp2)
        return geom, osc, b, inner, p, p2, p_ref, st, st2, ref_stats
    finally:
        ctx.close()


@pytest.mark.parametrize("seed,n_level", [(0, 3), (1, 3), (2, 3), (3, 4)])
def test_mixed_neumann_boxes(seed, n_level):
    """n_level 4 puts the coarse solve on a 4^3 level: a cluster of 6 blocks."""
    sc = scenes.poisson_boxes(n=32, seed=seed, n_level=n_level)
    geom, osc, b, inner, p, p2, p_ref, st, st2, ref = solve_pair(sc, seed, A.MIXED_REMOVE_MEAN)
    assert 0 < st.cycles < 200 and st.rel_residual <= 1e-8
    assert st2.cycles == st.cycles and np.array_equal(p, p2)
    r = residual_cpu(osc, geom, p, b)
    assert np.linalg.norm(r) <= 1.0000001e-8 * np.linalg.norm(b[inner])
    assert abs(p[inner].mean()) <= 1e-12 * np.abs(p[inner]).max()
    # both solve the same singular system: compare up to the constant
    d = (p[inner] - p[inner].mean()) - (p_ref[inner] - p_ref[inner].mean())
    assert np.abs(d).max() <= 1e-5 * np.abs(p_ref[inner]).max()
    assert ref.rel_residual <= 1e-11


def test_mixed_dirichlet_channel():
    """Outflow with Dirichlet p = 0 (no mean removal) and an obstacle."""
    sc = scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=1, n_level=3)
    geom, osc, b, inner, p, p2, p_ref, st, st2, ref = solve_pair(sc, 7, 0)
    assert 0 < st.cycles < 200 and st.rel_residual <= 1e-8
    r = residual_cpu(osc, geom, p, b)
    assert np.linalg.norm(r) <= 1.0000001e-8 * np.linalg.norm(b[inner])
    d = p[inner] - p_ref[inner]
    assert np.abs(d).max() <= 1e-5 * np.abs(p_ref[inner]).max()


@pytest.mark.parametrize("case", ["neumann_boxes", "dirichlet_channel"])
def test_mixed_rbgs_smoother(case):
    """Red-black Gauss-Seidel smoothing (MIXED_RBGS, w = 1) meets the same
    residual claim as the Jacobi smoother, agrees with the plain FP64 solve,
    and takes fewer defect-correction cycles."""
    if case == "neumann_boxes":
        sc, seed, flags = scenes.poisson_boxes(n=32, seed=5, n_level=4), 5, A.MIXED_REMOVE_MEAN
    else:
        sc, seed, flags = scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=1, n_level=3), 7, 0
    geom, osc, b, inner, p, p2, p_ref, st, st2, ref = solve_pair(sc, seed, flags | A.MIXED_RBGS, w=1.0)
    assert 0 < st.cycles < 200 and st.rel_residual <= 1e-8
    assert st2.cycles == st.cycles and np.array_equal(p, p2)
    r = residual_cpu(osc, geom, p, b)
    assert np.linalg.norm(r) <= 1.0000001e-8 * np.linalg.norm(b[inner])
    if flags & A.MIXED_REMOVE_MEAN:
        d = (p[inner] - p[inner].mean()) - (p_ref[inner] - p_ref[inner].mean())
    else:
        d = p[inner] - p_ref[inner]
    assert np.abs(d).max() <= 1e-5 * np.abs(p_ref[inner]).max()
    jac = solve_pair(sc, seed, flags)[7]
    print(f"{case}: cycles red-black GS {st.cycles}, weighted Jacobi {jac.cycles}")
    assert st.cycles < jac.cycles


@pytest.mark.parametrize("case", ["neumann_boxes", "dirichlet_channel"])
def test_mixed_boundary_writes_match_launched_programs(case):
    """By default the FP32 sweeps write the boundary cells their stencils read
    (x_t = +-x_root of the homogeneous pressure program) with each inner
    value instead of launching the program after every sweep
    (MIXED_BC_LAUNCH): the same values, so the solves are bit-identical,
    cycle for cycle."""
    if case == "neumann_boxes":
        sc, seed, flags = scenes.poisson_boxes(n=32, seed=6, n_level=4), 6, A.MIXED_REMOVE_MEAN
    else:
        sc, seed, flags = scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=1, n_level=3), 7, 0
    folded = solve_pair(sc, seed, flags)
    launched = solve_pair(sc, seed, flags | A.MIXED_BC_LAUNCH)
    assert folded[7].cycles == launched[7].cycles
    assert np.array_equal(folded[4], launched[4])


@pytest.mark.parametrize("case", ["neumann_boxes", "dirichlet_channel"])
def test_mixed_block_coarse_matches_cluster(case):
    """The coarsest level solved by one block (shared memory, block barriers;
    the default where the level fits) and by the thread-block cluster
    (MIXED_CLUSTER_COARSE) compute the same iterates; only the order of the
    residual sums that stop the coarse loop differs."""
    if case == "neumann_boxes":
        sc, seed, flags = scenes.poisson_boxes(n=32, seed=8, n_level=3), 8, A.MIXED_REMOVE_MEAN
    else:
        sc, seed, flags = scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=1, n_level=3), 7, 0
    block = solve_pair(sc, seed, flags)
    cluster = solve_pair(sc, seed, flags | A.MIXED_CLUSTER_COARSE)
    inner = block[3]
    assert block[7].cycles == cluster[7].cycles and block[7].rel_residual <= 1e-8
    p_b, p_c = block[4][inner], cluster[4][inner]
    assert np.abs(p_b - p_c).max() <= 1e-9 * np.abs(p_c).max()


@pytest.mark.parametrize("case", ["neumann_boxes", "dirichlet_channel"])
def test_mixed_coarse_column_prolongation_matches_fine(case):
    """The prolongation by coarse columns (a register window of 27 coarse
    values, 8 children per coarse cell; the default) and by fine cells
    (MIXED_FINE_PROLONG) evaluate the same expression for every fine cell: the
    solves are bit-identical, cycle for cycle."""
    if case == "neumann_boxes":
        sc, seed, flags = scenes.poisson_boxes(n=32, seed=9, n_level=4), 9, A.MIXED_REMOVE_MEAN
    else:
        sc, seed, flags = scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=1, n_level=3), 7, 0
    column = solve_pair(sc, seed, flags)
    fine = solve_pair(sc, seed, flags | A.MIXED_FINE_PROLONG)
    assert column[7].cycles == fine[7].cycles
    assert np.array_equal(column[4], fine[4])
