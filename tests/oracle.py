"""ctypes access to the C oracle (oracle/artss_oracle.c, built as
oracle/_ref/liboracle.so) and an NSTempTurbSolver timestep orchestrated from
its kernels in the order of ARTSS src/solver/NSTempTurbSolver.cpp:94-248,
SolverController::update_sources and FieldController::update_data.

Test infrastructure: the checker for the B200 kernels, never the product."""
from __future__ import annotations

import ctypes as C
import math
import os
from typing import Dict

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "liboracle.so")
ML = 8
_D = C.POINTER(C.c_double)


class OracleBc(C.Structure):
    _fields_ = [("target", C.c_int64), ("source", C.c_int64), ("value", C.c_double), ("sign", C.c_int32),
                ("reserved", C.c_int32)]


class Scene(C.Structure):
    _fields_ = ([("levels", C.c_int32)] +
                [(f, C.c_int64 * (ML + 1)) for f in ("Nx", "Ny", "Nz", "i1", "i2", "j1", "j2", "k1", "k2")] +
                [(f, C.c_double * (ML + 1)) for f in ("dx", "dy", "dz")] +
                [("inner", C.POINTER(C.c_int64) * (ML + 1)), ("n_inner", C.c_int64 * (ML + 1)),
                 ("domain", C.POINTER(C.c_int64) * (ML + 1)), ("n_domain", C.c_int64 * (ML + 1)),
                 ("bc", (C.POINTER(OracleBc) * 7) * (ML + 1)), ("n_bc", (C.c_int64 * 7) * (ML + 1))])


class MgCfg(C.Structure):
    _fields_ = [("n_level", C.c_int32), ("n_cycle", C.c_int32), ("max_cycle", C.c_int32), ("n_relax", C.c_int32),
                ("tol_res", C.c_double), ("smoother", C.c_int32), ("reserved", C.c_int32),
                ("smoother_max_iter", C.c_int64), ("smoother_tol_res", C.c_double), ("smoother_w", C.c_double)]


def available() -> bool:
    return os.path.exists(LIB)


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB)
        S = C.POINTER(Scene)
        sig = {
            "oracle_apply_bc": [S, _D, C.c_int, C.c_int],
            "oracle_advect": [S, _D, _D, _D, _D, _D, C.c_double, C.c_int],
            "oracle_smagorinsky": [S, _D, _D, _D, _D, C.c_double],
            "oracle_divergence": [S, _D, _D, _D, _D],
            "oracle_projection": [S, _D, _D, _D, _D, _D, _D, _D],
            "oracle_buoyancy": [S, _D, _D, _D, C.c_double, C.c_double],
            "oracle_add_source": [S, _D, _D, C.c_double, C.c_int],
            "oracle_diffuse_explicit": [S, _D, _D, C.c_double, _D, C.c_double, C.c_int],
            "oracle_dissipate": [S, _D, _D, _D, _D, C.c_double, C.c_double, C.c_int],
            "oracle_dynamic_smagorinsky": [S, _D, _D, _D, _D, C.c_double],
        }
        for fn, a in sig.items():
            getattr(L, fn).argtypes = a
            getattr(L, fn).restype = None
        for fn in ("oracle_diffuse_cgs", "oracle_diffuse_jacobi"):
            getattr(L, fn).argtypes = [S, _D, _D, _D, C.c_double, _D, C.c_double, C.c_int, C.c_int64, C.c_double,
                                       C.c_double, _D]
            getattr(L, fn).restype = C.c_int64
        L.oracle_mg_create.argtypes = [S, C.POINTER(MgCfg)]
        L.oracle_mg_create.restype = C.c_void_p
        L.oracle_mg_destroy.argtypes = [C.c_void_p]
        L.oracle_mg_pressure.argtypes = [C.c_void_p, _D, _D, C.c_int, _D]
        L.oracle_mg_pressure.restype = C.c_int64
        L.oracle_mg_last_coarse_iterations.argtypes = [C.c_void_p]
        L.oracle_mg_last_coarse_iterations.restype = C.c_int64
        _lib = L
    return _lib


def p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


class OracleScene:
    """oracle_scene built from the host geometry (artss_b200.Geometry), whose
    lists and boundary programs are pinned bit-exact to the reference."""

    def __init__(self, geom):
        self.geom = geom
        s = Scene()
        d = geom.grid_desc()
        s.levels = d.n_levels
        for f in ("Nx", "Ny", "Nz", "i1", "i2", "j1", "j2", "k1", "k2", "dx", "dy", "dz"):
            getattr(s, f)[:] = list(getattr(d, f))
        self._keep = []
        for l in range(d.n_levels + 1):
            inner = np.ascontiguousarray(geom.list("inner", l))
            dom = np.ascontiguousarray(geom.list("domain", l))
            self._keep += [inner, dom]
            s.inner[l] = inner.ctypes.data_as(C.POINTER(C.c_int64))
            s.n_inner[l] = inner.size
            s.domain[l] = dom.ctypes.data_as(C.POINTER(C.c_int64))
            s.n_domain[l] = dom.size
            for ft in range(7):
                prog = geom.boundary_program(l, ft)
                if prog.size:
                    arr = (OracleBc * prog.size)()
                    C.memmove(arr, prog.ctypes.data, prog.nbytes)
                    self._keep.append(arr)
                    s.bc[l][ft] = C.cast(arr, C.POINTER(OracleBc))
                    s.n_bc[l][ft] = prog.size
        self.s = s
        self.ptr = C.byref(s)
        self.size0 = d.Nx[0] * d.Ny[0] * d.Nz[0]

    def size(self, level: int = 0) -> int:
        return self.s.Nx[level] * self.s.Ny[level] * self.s.Nz[level]


FT = {"u": 1, "v": 2, "w": 3, "p": 4, "T": 5, "nu": 6}


class NSTempTurbOracle:
    """One NSTempTurbSolver timestep from the oracle kernels, starting from a
    reference set-up state (fields of the reference's step-0 dump)."""

    def __init__(self, sc: OracleScene, scene, state: Dict[str, np.ndarray], gauss_spatial: np.ndarray):
        self.sc = sc
        self.sp = scene  # artss_b200.scenes.Scene (physical parameters)
        self.f = {k: np.ascontiguousarray(v, dtype=np.float64).copy() for k, v in state.items()}
        n = sc.size0
        for k in ("u0", "v0", "w0", "u_tmp", "v_tmp", "w_tmp", "T0", "T_tmp", "kappa_t", "p0"):
            self.f.setdefault(k, np.zeros(n))
        # FieldController::update_data after set-up
        for a in ("u", "v", "w", "T"):
            self.f[a + "0"][:] = self.f[a]
            self.f[a + "_tmp"][:] = self.f[a]
        self.spatial = np.ascontiguousarray(gauss_spatial)
        cfg = MgCfg(scene.n_level, scene.n_cycle, scene.max_cycle, scene.n_relax, scene.mg_tol,
                    0 if scene.smoother == "Jacobi" else 1, 0, scene.smoother_max_iter, scene.smoother_tol,
                    scene.smoother_w)
        self.mg = lib().oracle_mg_create(sc.ptr, C.byref(cfg))
        self.step_index = 1

    def close(self):
        if self.mg:
            lib().oracle_mg_destroy(self.mg)
            self.mg = None

    def _couple(self, names):
        for a in names:
            self.f[a + "0"][:] = self.f[a]
            self.f[a + "_tmp"][:] = self.f[a]

    def _diffuse(self, out, inn, b, D, ev, ft):
        L = lib()
        s = self.sp
        res = C.c_double()
        fn = L.oracle_diffuse_cgs if s.diffusion == "ColoredGaussSeidel" else L.oracle_diffuse_jacobi
        return fn(self.sc.ptr, p(self.f[out]), p(self.f[inn]), p(self.f[b]), D, p(self.f[ev]), s.dt, FT[out[0]],
                  s.diff_max_iter, s.diff_tol, 1.0, C.byref(res))

    def step(self):
        L = lib()
        f, s, S = self.f, self.sp, self.sc.ptr
        t = self.step_index * s.dt
        for a in ("u", "v", "w"):
            L.oracle_advect(S, p(f[a]), p(f[a + "0"]), p(f["u0"]), p(f["v0"]), p(f["w0"]), s.dt, FT[a])
        self._couple("uvw")
        L.oracle_smagorinsky(S, p(f["nu_t"]), p(f["u"]), p(f["v"]), p(f["w"]), s.cs)
        for a in ("u", "v", "w"):
            self._diffuse(a, a + "0", a + "_tmp", s.nu, "nu_t", FT[a])
        self._couple("uvw")
        axis = "xyz".index(s.buoyancy_dir)
        a = "uvw"[axis]
        L.oracle_add_source(S, p(f[a]), p(f["f_" + "xyz"[axis]]), s.dt, FT[a])
        self._couple("uvw")
        L.oracle_divergence(S, p(f["rhs"]), p(f["u_tmp"]), p(f["v_tmp"]), p(f["w_tmp"]))
        res = C.c_double()
        first = int(round(t / s.dt)) == 1
        L.oracle_mg_pressure(self.mg, p(f["p"]), p(f["rhs"]), 1 if first else 0, C.byref(res))
        L.oracle_projection(S, p(f["u"]), p(f["v"]), p(f["w"]), p(f["u_tmp"]), p(f["v_tmp"]), p(f["w_tmp"]),
                            p(f["p"]))
        L.oracle_advect(S, p(f["T"]), p(f["T0"]), p(f["u"]), p(f["v"]), p(f["w"]), s.dt, FT["T"])
        self._couple(["T"])
        f["kappa_t"][:] = f["nu_t"] * (1. / s.pr_t)
        self._diffuse("T", "T0", "T_tmp", s.kappa, "kappa_t", FT["T"])
        self._couple(["T"])
        L.oracle_add_source(S, p(f["T"]), p(f["S_T"]), s.dt, FT["T"])
        self._couple(["T"])
        # SolverController::update_sources(t): buoyancy from T, S_T = spatial * tanh(t / tau)
        L.oracle_buoyancy(S, p(f["f_" + "xyz"[axis]]), p(f["T"]), p(f["T_a"]), s.beta, s.g)
        f["S_T"][:] = self.spatial * math.tanh(t / s.tau)
        f["p0"][:] = f["p"]
        self._couple("uvw")
        self._couple(["T"])
        self.step_index += 1
