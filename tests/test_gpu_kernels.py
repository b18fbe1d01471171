"""Kernel-level parity through the C ABI: every entry point of
include/artss_cuda.h against the C oracle (oracle/artss_oracle.c, pinned to
the reference build by test_oracle.py) on seeded random inputs, on a scene
with an obstacle and three multigrid levels.  Integer/index work and every
field value must match exactly; only loop-termination residuals are reduced
in a different order."""
import ctypes as C

import numpy as np
import pytest

import artss_b200 as A
from artss_b200 import scenes
from tests import cabi, oracle

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle.available(), reason="oracle not built")]

_D = C.POINTER(C.c_double)
FT = {"u": 1, "v": 2, "w": 3, "p": 4, "T": 5, "nu": 6}


@pytest.fixture(scope="module")
def env(tmp_path_factory):
    sc = scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=1, n_level=3)
    xml = scenes.write(sc, str(tmp_path_factory.mktemp("k") / "ch.xml"))
    geom = A.Geometry(xml)
    ctx = cabi.Context(geom)
    osc = oracle.OracleScene(geom)
    yield sc, geom, ctx, osc
    ctx.close()


def rnd(seed, n, lo=-1.0, hi=1.0):
    return np.random.default_rng(seed).uniform(lo, hi, n)


def P(a):
    return oracle.p(a)


def test_boundary_programs(env):
    sc, geom, ctx, osc = env
    L = oracle.lib()
    for level in range(geom.levels + 1):
        n = ctx.size(level)
        for name, ft in FT.items():
            if geom.boundary_program(level, ft).size == 0:
                continue
            x = rnd(level * 10 + ft, n)
            d = ctx.field(x, level)
            A.cuda_check(ctx.lib.artss_apply_boundary(ctx.h, d, level, ft), "bc")
            ref = x.copy()
            L.oracle_apply_bc(osc.ptr, P(ref), level, ft)
            assert np.array_equal(ctx.download(d, level), ref), f"level {level} field {name}"
            assert ctx.lib.artss_boundary_program_waves(ctx.h, level, ft) == 1


def test_advect(env):
    sc, geom, ctx, osc = env
    n = ctx.size()
    u, v, w = rnd(1, n, -150, 150), rnd(2, n, -150, 150), rnd(3, n, -150, 150)
    src, out0 = rnd(4, n), rnd(5, n)
    du, dv, dw, ds, do = (ctx.field(a) for a in (u, v, w, src, out0))
    A.cuda_check(ctx.lib.artss_advect_sl(ctx.h, do, ds, du, dv, dw, sc.dt, FT["T"]), "advect")
    ref = out0.copy()
    oracle.lib().oracle_advect(osc.ptr, P(ref), P(src), P(u), P(v), P(w), sc.dt, FT["T"])
    assert np.array_equal(ctx.download(do), ref)
    # fused u,v,w: each output advected by (u,v,w), the inputs being the velocities
    o1, o2, o3 = ctx.field(out0), ctx.field(out0), ctx.field(out0)
    A.cuda_check(ctx.lib.artss_advect_sl_uvw(ctx.h, o1, o2, o3, du, dv, dw, du, dv, dw, sc.dt), "uvw")
    for o, a, ft in ((o1, u, 1), (o2, v, 2), (o3, w, 3)):
        ref = out0.copy()
        oracle.lib().oracle_advect(osc.ptr, P(ref), P(a), P(u), P(v), P(w), sc.dt, ft)
        assert np.array_equal(ctx.download(o), ref)


def test_dynamic_smagorinsky(env):
    """DynamicSmagorinsky (filters, Leonard stress, dynamic coefficient, the
    in-place list-order averaging run as hyperplanes, the clamp) against the
    oracle's loop-by-loop restatement, bit for bit, twice in a row (the work
    fields persist in the context)."""
    sc, geom, ctx, osc = env
    n = ctx.size()
    for seed in (41, 42):
        u, v, w = rnd(seed, n), rnd(seed + 10, n), rnd(seed + 20, n)
        du, dv, dw = (ctx.field(a) for a in (u, v, w))
        ev0 = rnd(seed + 30, n)
        dev = ctx.field(ev0)
        # nu large enough that some cells take the clamp
        nu = 1e-3
        A.cuda_check(ctx.lib.artss_turb_dynamic_smagorinsky(ctx.h, dev, du, dv, dw, nu), "dynamic smagorinsky")
        ref = ev0.copy()
        oracle.lib().oracle_dynamic_smagorinsky(osc.ptr, P(ref), P(u), P(v), P(w), nu)
        got = ctx.download(dev)
        assert np.array_equal(got, ref)
        inner = geom.list("inner", 0)
        assert (got[inner] == 0).any() and (got[inner] != 0).any()


def test_smagorinsky_divergence_projection_sources(env):
    sc, geom, ctx, osc = env
    L = oracle.lib()
    n = ctx.size()
    u, v, w, p = rnd(11, n), rnd(12, n), rnd(13, n), rnd(14, n)
    du, dv, dw, dp = (ctx.field(a) for a in (u, v, w, p))
    ev0 = rnd(15, n)
    dev = ctx.field(ev0)
    A.cuda_check(ctx.lib.artss_turb_const_smagorinsky(ctx.h, dev, du, dv, dw, 0.2), "smag")
    ref = ev0.copy()
    L.oracle_smagorinsky(osc.ptr, P(ref), P(u), P(v), P(w), 0.2)
    assert np.array_equal(ctx.download(dev), ref)

    rhs0 = rnd(16, n)
    drhs = ctx.field(rhs0)
    A.cuda_check(ctx.lib.artss_divergence(ctx.h, drhs, du, dv, dw), "div")
    ref = rhs0.copy()
    L.oracle_divergence(osc.ptr, P(ref), P(u), P(v), P(w))
    assert np.array_equal(ctx.download(drhs), ref)

    o = [rnd(17 + k, n) for k in range(3)]
    do = [ctx.field(a) for a in o]
    A.cuda_check(ctx.lib.artss_projection(ctx.h, do[0], do[1], do[2], du, dv, dw, dp), "proj")
    ref = [a.copy() for a in o]
    L.oracle_projection(osc.ptr, P(ref[0]), P(ref[1]), P(ref[2]), P(u), P(v), P(w), P(p))
    for k in range(3):
        assert np.array_equal(ctx.download(do[k]), ref[k])

    T, Ta, f0 = rnd(21, n, 290, 310), rnd(22, n, 290, 300), rnd(23, n)
    dT, dTa, df = ctx.field(T), ctx.field(Ta), ctx.field(f0)
    A.cuda_check(ctx.lib.artss_buoyancy_force(ctx.h, df, dT, dTa, sc.beta, sc.g), "buoy")
    ref = f0.copy()
    L.oracle_buoyancy(osc.ptr, P(ref), P(T), P(Ta), sc.beta, sc.g)
    assert np.array_equal(ctx.download(df), ref)

    S = rnd(24, n, 0, 50)
    dS = ctx.field(S)
    A.cuda_check(ctx.lib.artss_add_source(ctx.h, dT, dS, sc.dt, FT["T"]), "source")
    ref = T.copy()
    L.oracle_add_source(osc.ptr, P(ref), P(S), sc.dt, FT["T"])
    assert np.array_equal(ctx.download(dT), ref)


@pytest.mark.parametrize("method", ["cgs", "jacobi"])
@pytest.mark.parametrize("turbulent", [False, True])
@pytest.mark.parametrize("scratch", [0, 1])
def test_diffusion(env, method, turbulent, scratch):
    if method == "jacobi" and scratch:
        pytest.skip("the Jacobi solver always keeps its input")
    sc, geom, ctx, osc = env
    n = ctx.size()
    out0, in0, b = rnd(31, n, 290, 300), rnd(32, n, 290, 300), rnd(33, n, 290, 300)
    ev = rnd(34, n, 0, 1e-3)
    dout, din, db, dev = ctx.field(out0), ctx.field(in0), ctx.field(b), ctx.field(ev)
    cfg = A.IterCfg(9, 1e-12, 1.0)
    stats = A.IterStats()
    D = 4.2e-5
    evp = dev if turbulent else None
    if method == "cgs":
        A.cuda_check(ctx.lib.artss_diffuse_cgs(ctx.h, dout, din, db, D, evp, sc.dt, FT["T"], C.byref(cfg), scratch,
                                               C.byref(stats)), "cgs")
        fn = oracle.lib().oracle_diffuse_cgs
    else:
        A.cuda_check(ctx.lib.artss_diffuse_jacobi(ctx.h, dout, din, db, D, evp, sc.dt, FT["T"], C.byref(cfg),
                                                  C.byref(stats)), "jacobi")
        fn = oracle.lib().oracle_diffuse_jacobi
    ro, ri = out0.copy(), in0.copy()
    res = C.c_double()
    its = fn(osc.ptr, P(ro), P(ri), P(b), D, P(ev) if turbulent else None, sc.dt, FT["T"], 9, 1e-12, 1.0,
             C.byref(res))
    assert stats.iterations == its and its >= 3
    assert np.array_equal(ctx.download(dout), ro)
    if not scratch:
        assert np.array_equal(ctx.download(din), ri)
    assert abs(stats.residual - res.value) <= 1e-12 * res.value


# coarse solve: "cluster" = one thread-block cluster (Jacobi: pipelined, one
# cluster barrier per sweep), "cluster3" = the cluster with three barriers per
# sweep, "block" = one block, "multi" = separate multi-block launches per sweep
COARSE_FLAGS = {"cluster": 0, "cluster3": 4, "block": 2, "multi": 1}


@pytest.mark.parametrize("smoother", [0, 1])
@pytest.mark.parametrize("coarse", list(COARSE_FLAGS))
@pytest.mark.parametrize("first_step", [1, 0])
def test_vcycle_mg(env, smoother, coarse, first_step):
    sc, geom, ctx, osc = env
    n = ctx.size()
    p0, rhs = rnd(41, n), rnd(42, n)
    cfg = A.MgCfg(3, 2, 3, 2, 1e-30, smoother, COARSE_FLAGS[coarse], 40, 1e-9, 0.6666666667)
    mg = C.c_void_p()
    A.cuda_check(ctx.lib.artss_mg_create(ctx.h, C.byref(cfg), C.byref(mg)), "mg")
    try:
        dp, drhs = ctx.field(p0), ctx.field(rhs)
        st = A.MgStats()
        A.cuda_check(ctx.lib.artss_mg_pressure(mg, dp, drhs, first_step, C.byref(st)), "pressure")
        ocfg = oracle.MgCfg(3, 2, 3, 2, 1e-30, smoother, 0, 40, 1e-9, 0.6666666667)
        om = oracle.lib().oracle_mg_create(osc.ptr, C.byref(ocfg))
        ref = p0.copy()
        res = C.c_double()
        cyc = oracle.lib().oracle_mg_pressure(om, P(ref), P(rhs), first_step, C.byref(res))
        oracle.lib().oracle_mg_destroy(om)
        assert st.cycles == cyc
        assert np.array_equal(ctx.download(dp), ref)
    finally:
        ctx.lib.artss_mg_destroy(mg)


@pytest.mark.parametrize("coarse", ["cluster", "cluster3"])
def test_coarse_solve_stops_early(env, coarse):
    """Coarse solves that stop on the tolerance after odd and even sweep
    counts: the reference leaves iterate it (odd) or it-1 (even) in out, and
    the pipelined kernel decides one sweep late, so both parities must still
    give the reference's pressure."""
    sc, geom, ctx, osc = env
    n = ctx.size()
    p0, rhs = rnd(45, n), rnd(46, n)
    seen = set()
    # 1, 2, 3, 6, 13 and 23 sweeps on this scene, then the 200-sweep cap
    for tol in (100.0, 30.0, 20.0, 10.0, 5.0, 3.0, 1e-30):
        cfg = A.MgCfg(3, 1, 1, 2, 1e-30, 0, COARSE_FLAGS[coarse], 200, tol, 0.6666666667)
        mg = C.c_void_p()
        A.cuda_check(ctx.lib.artss_mg_create(ctx.h, C.byref(cfg), C.byref(mg)), "mg")
        try:
            dp, drhs = ctx.field(p0), ctx.field(rhs)
            st = A.MgStats()
            A.cuda_check(ctx.lib.artss_mg_pressure(mg, dp, drhs, 0, C.byref(st)), "pressure")
            ocfg = oracle.MgCfg(3, 1, 1, 2, 1e-30, 0, 0, 200, tol, 0.6666666667)
            om = oracle.lib().oracle_mg_create(osc.ptr, C.byref(ocfg))
            ref = p0.copy()
            res = C.c_double()
            oracle.lib().oracle_mg_pressure(om, P(ref), P(rhs), 0, C.byref(res))
            sweeps = oracle.lib().oracle_mg_last_coarse_iterations(om)
            oracle.lib().oracle_mg_destroy(om)
            seen.add(sweeps % 2)
            assert np.array_equal(ctx.download(dp), ref), (tol, sweeps)
        finally:
            ctx.lib.artss_mg_destroy(mg)
    assert seen == {0, 1}


@pytest.mark.parametrize("scratch", [0, 1])
def test_cgs_iteration_parity(env, scratch):
    """Solves of 3..6 iterations in a row: the sweep alternates between out and
    in, so each length ends in either array depending on the previous length;
    out (and in, when kept) must always match the in-place reference."""
    sc, geom, ctx, osc = env
    n = ctx.size()
    for its_req in (3, 4, 4, 5, 6, 3):
        out0, in0, b = rnd(51, n, 290, 300), rnd(52 + its_req, n, 290, 300), rnd(53, n, 290, 300)
        ev = rnd(54, n, 0, 1e-3)
        dout, din, db, dev = ctx.field(out0), ctx.field(in0), ctx.field(b), ctx.field(ev)
        cfg = A.IterCfg(its_req, 1e-300, 1.0)
        stats = A.IterStats()
        A.cuda_check(ctx.lib.artss_diffuse_cgs(ctx.h, dout, din, db, 4.2e-5, dev, sc.dt, FT["u"], C.byref(cfg),
                                               scratch, C.byref(stats)), "cgs")
        ro, ri = out0.copy(), in0.copy()
        res = C.c_double()
        its = oracle.lib().oracle_diffuse_cgs(osc.ptr, P(ro), P(ri), P(b), 4.2e-5, P(ev), sc.dt, FT["u"], its_req,
                                              1e-300, 1.0, C.byref(res))
        assert stats.iterations == its == its_req
        assert np.array_equal(ctx.download(dout), ro)
        if not scratch:
            assert np.array_equal(ctx.download(din), ri)


@pytest.mark.parametrize("turbulent", [False, True])
def test_cgs_odd_pitch(tmp_path, turbulent):
    """An odd row pitch (nx + 2 odd) rules out TMA plane loads; the cp.async
    variant of the sweep must give the same values."""
    sc = scenes.channel_with_cube(nx=63, ny=20, nz=19, steps=1, n_level=1)
    geom = A.Geometry(scenes.write(sc, str(tmp_path / "odd.xml")))
    ctx = cabi.Context(geom)
    try:
        osc = oracle.OracleScene(geom)
        n = ctx.size()
        assert (geom.grid_desc().Nx[0] % 2) == 1
        out0, in0, b, ev = rnd(61, n, 290, 300), rnd(62, n, 290, 300), rnd(63, n, 290, 300), rnd(64, n, 0, 1e-3)
        dout, din, db, dev = ctx.field(out0), ctx.field(in0), ctx.field(b), ctx.field(ev)
        cfg = A.IterCfg(5, 1e-300, 1.0)
        stats = A.IterStats()
        A.cuda_check(ctx.lib.artss_diffuse_cgs(ctx.h, dout, din, db, 4.2e-5, dev if turbulent else None, sc.dt,
                                               FT["v"], C.byref(cfg), 0, C.byref(stats)), "cgs")
        ro, ri = out0.copy(), in0.copy()
        res = C.c_double()
        its = oracle.lib().oracle_diffuse_cgs(osc.ptr, P(ro), P(ri), P(b), 4.2e-5, P(ev) if turbulent else None,
                                              sc.dt, FT["v"], 5, 1e-300, 1.0, C.byref(res))
        assert stats.iterations == its == 5
        assert np.array_equal(ctx.download(dout), ro)
        assert np.array_equal(ctx.download(din), ri)
    finally:
        ctx.close()


@pytest.mark.parametrize("turbulent", [False, True])
def test_explicit_diffusion(env, turbulent):
    """ExplicitDiffuse (laminar and the reference's turbulent form) + the
    boundary program, against the oracle, bit for bit."""
    sc, geom, ctx, osc = env
    n = ctx.size()
    out0, in0, ev = rnd(111, n, 290, 300), rnd(112, n, 290, 300), rnd(113, n, 0, 1e-3)
    dout, din, dev = ctx.field(out0), ctx.field(in0), ctx.field(ev)
    A.cuda_check(ctx.lib.artss_diffuse_explicit(ctx.h, dout, din, 3.1e-5, dev if turbulent else None, sc.dt,
                                                FT["v"]), "explicit")
    ref = out0.copy()
    oracle.lib().oracle_diffuse_explicit(osc.ptr, P(ref), P(in0), 3.1e-5, P(ev) if turbulent else None, sc.dt, FT["v"])
    assert np.array_equal(ctx.download(dout), ref)
    assert np.array_equal(ctx.download(din), in0)


def test_dissipate(env):
    """ISource::dissipate (viscous heating of T from u, v, w) + the boundary
    program, against the oracle, bit for bit."""
    sc, geom, ctx, osc = env
    n = ctx.size()
    T, u, v, w = rnd(121, n, 290, 300), rnd(122, n), rnd(123, n), rnd(124, n)
    dT, du, dv, dw = ctx.field(T), ctx.field(u), ctx.field(v), ctx.field(w)
    A.cuda_check(ctx.lib.artss_dissipate(ctx.h, dT, du, dv, dw, 3.1e-5, sc.dt, FT["T"]), "dissipate")
    ref = T.copy()
    oracle.lib().oracle_dissipate(osc.ptr, P(ref), P(u), P(v), P(w), 3.1e-5, sc.dt, FT["T"])
    assert np.array_equal(ctx.download(dT), ref)


@pytest.mark.parametrize("turbulent", [False, True])
def test_cgs_mixed_precision(env, turbulent):
    """FP32 sweeps inside FP64 defect correction: the same iterations as the
    reference's FP64 sweep (oracle), values within the FP32 rounding of the
    corrections (1e-8 relative here)."""
    sc, geom, ctx, osc = env
    n = ctx.size()
    out0, in0, b, ev = rnd(131, n, 290, 300), rnd(132, n, 290, 300), rnd(133, n, 290, 300), rnd(134, n, 0, 1e-3)
    dout, din, db, dev = ctx.field(out0), ctx.field(in0), ctx.field(b), ctx.field(ev)
    cfg = A.IterCfg(5, 1e-300, 1.0)
    stats = A.IterStats()
    A.cuda_check(ctx.lib.artss_diffuse_cgs_mixed(ctx.h, dout, din, db, 4.2e-5, dev if turbulent else None, sc.dt,
                                                 FT["u"], C.byref(cfg), 0, C.byref(stats)), "cgs mixed")
    ro, ri = out0.copy(), in0.copy()
    res = C.c_double()
    its = oracle.lib().oracle_diffuse_cgs(osc.ptr, P(ro), P(ri), P(b), 4.2e-5, P(ev) if turbulent else None, sc.dt,
                                          FT["u"], 5, 1e-300, 1.0, C.byref(res))
    assert stats.iterations == its == 5
    got = ctx.download(dout)
    err = float(np.max(np.abs(got - ro)) / np.max(np.abs(ro)))
    assert err <= 1e-8, err
    assert np.array_equal(ctx.download(din), got)  # in = out as the reference leaves them
    # the stopping measure ||rb (x_new - x)||, taken while it is well above round-off
    dout, din = ctx.field(out0), ctx.field(in0)
    cfg2 = A.IterCfg(2, 1e-300, 1.0)
    A.cuda_check(ctx.lib.artss_diffuse_cgs_mixed(ctx.h, dout, din, db, 4.2e-5, dev if turbulent else None, sc.dt,
                                                 FT["u"], C.byref(cfg2), 0, C.byref(stats)), "cgs mixed")
    ro, ri = out0.copy(), in0.copy()
    oracle.lib().oracle_diffuse_cgs(osc.ptr, P(ro), P(ri), P(b), 4.2e-5, P(ev) if turbulent else None, sc.dt,
                                    FT["u"], 2, 1e-300, 1.0, C.byref(res))
    assert res.value > 1e-6
    assert abs(stats.residual - res.value) <= 1e-6 * res.value, (stats.residual, res.value)


def _sweep_scenes():
    """a channel with a cube (obstacle planes take the flag path of the
    row-pair sweep); odd sizes with a box that touches the x-y edges of the
    inner box (partial 64 x 8 tiles, segments that cross tile columns); a
    domain wider than one tile in x with a box spanning two tile columns"""
    return {
        "channel_cube": scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=1, n_level=1),
        "odd_edges": scenes.channel_with_cube(nx=70, ny=20, nz=19, steps=1, n_level=1,
                                              obstacles=[scenes.Box(0.1, 0.4, 0.2, 0.6, 1.0, 1.6, name="edge")]),
        "wide": scenes.channel_with_cube(nx=130, ny=18, nz=13, steps=1, n_level=1,
                                         obstacles=[scenes.Box(2.9, 3.5, 1.2, 1.6, 0.4, 2.0, name="mid")]),
    }


@pytest.mark.parametrize("scene", list(_sweep_scenes().keys()))
@pytest.mark.parametrize("turbulent", [False, True])
def test_cgs_every_sweep_variant(tmp_path, scene, turbulent):
    """Each sweep variant (two-phase and one-phase kernels at every z-depth,
    the row-pair kernel with persistent blocks on 64 x 8, 64 x 6 and 64 x 16
    tiles, two or one blocks per multiprocessor), pinned, gives the oracle's
    colored Gauss-Seidel iterations bit for bit."""
    sc = _sweep_scenes()[scene]
    geom = A.Geometry(scenes.write(sc, str(tmp_path / f"{scene}.xml")))
    ctx = cabi.Context(geom)
    try:
        osc = oracle.OracleScene(geom)
        n = ctx.size()
        out0, in0, b, ev = rnd(91, n, 290, 300), rnd(92, n, 290, 300), rnd(93, n, 290, 300), rnd(94, n, 0, 1e-3)
        ro, ri = out0.copy(), in0.copy()
        res = C.c_double()
        oracle.lib().oracle_diffuse_cgs(osc.ptr, P(ro), P(ri), P(b), 4.2e-5, P(ev) if turbulent else None, sc.dt,
                                        FT["u"], 5, 1e-300, 1.0, C.byref(res))
        for v in range(9):
            A.cuda_check(ctx.lib.artss_ctx_sweep_variant(ctx.h, v), "variant")
            dout, din, db, dev = ctx.field(out0), ctx.field(in0), ctx.field(b), ctx.field(ev)
            cfg = A.IterCfg(5, 1e-300, 1.0)
            stats = A.IterStats()
            A.cuda_check(ctx.lib.artss_diffuse_cgs(ctx.h, dout, din, db, 4.2e-5, dev if turbulent else None, sc.dt,
                                                   FT["u"], C.byref(cfg), 0, C.byref(stats)), f"cgs variant {v}")
            assert stats.iterations == 5
            assert np.array_equal(ctx.download(dout), ro), f"variant {v}: out"
            assert np.array_equal(ctx.download(din), ri), f"variant {v}: in"
            assert abs(stats.residual - res.value) <= 1e-12 * max(res.value, 1e-300), f"variant {v}: residual"
        A.cuda_check(ctx.lib.artss_ctx_sweep_variant(ctx.h, -1), "variant")
    finally:
        ctx.close()


@pytest.mark.parametrize("autotune", [0, 1])
def test_cgs_autotune(env, autotune):
    """Every z-depth of the sweep gives the same result; the tuner records one."""
    sc, geom, ctx, osc = env
    A.cuda_check(ctx.lib.artss_ctx_autotune(ctx.h, autotune), "autotune")
    n = ctx.size()
    out0, in0, b, ev = rnd(71, n, 290, 300), rnd(72, n, 290, 300), rnd(73, n, 290, 300), rnd(74, n, 0, 1e-3)
    dout, din, db, dev = ctx.field(out0), ctx.field(in0), ctx.field(b), ctx.field(ev)
    cfg = A.IterCfg(4, 1e-300, 1.0)
    stats = A.IterStats()
    A.cuda_check(ctx.lib.artss_diffuse_cgs(ctx.h, dout, din, db, 4.2e-5, dev, sc.dt, FT["w"], C.byref(cfg), 0,
                                           C.byref(stats)), "cgs")
    ro, ri = out0.copy(), in0.copy()
    res = C.c_double()
    oracle.lib().oracle_diffuse_cgs(osc.ptr, P(ro), P(ri), P(b), 4.2e-5, P(ev), sc.dt, FT["w"], 4, 1e-300, 1.0,
                                    C.byref(res))
    assert np.array_equal(ctx.download(dout), ro)
    assert np.array_equal(ctx.download(din), ri)
    depth = ctx.lib.artss_cgs_sweep_depth(ctx.h, 1)
    assert depth in ((8, 16, 32, -1) if autotune else (0,))
    A.cuda_check(ctx.lib.artss_ctx_autotune(ctx.h, 1), "autotune")


def test_vcycle_graph_replay(env):
    """Later-step pressure calls run as a captured graph; replaying it on the
    same arrays gives the eager result again, and launches are still counted."""
    sc, geom, ctx, osc = env
    n = ctx.size()
    p0, rhs = rnd(81, n), rnd(82, n)
    cfg = A.MgCfg(3, 2, 3, 2, 1e-30, 0, 0, 40, 1e-9, 0.6666666667)
    mg = C.c_void_p()
    A.cuda_check(ctx.lib.artss_mg_create(ctx.h, C.byref(cfg), C.byref(mg)), "mg")
    try:
        dp, drhs = ctx.field(p0), ctx.field(rhs)
        st = A.MgStats()
        outs = []
        for _ in range(3):
            ctx.upload(dp, p0)
            l0 = ctx.lib.artss_ctx_kernel_launches(ctx.h)
            A.cuda_check(ctx.lib.artss_mg_pressure(mg, dp, drhs, 0, C.byref(st)), "pressure")
            assert ctx.lib.artss_ctx_kernel_launches(ctx.h) - l0 > 20
            outs.append(ctx.download(dp))
        ocfg = oracle.MgCfg(3, 2, 3, 2, 1e-30, 0, 0, 40, 1e-9, 0.6666666667)
        om = oracle.lib().oracle_mg_create(osc.ptr, C.byref(ocfg))
        ref = p0.copy()
        res = C.c_double()
        oracle.lib().oracle_mg_pressure(om, P(ref), P(rhs), 0, C.byref(res))
        oracle.lib().oracle_mg_destroy(om)
        for o in outs:
            assert np.array_equal(o, ref)
    finally:
        ctx.lib.artss_mg_destroy(mg)
