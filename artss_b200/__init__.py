"""artss_b200 -- the ARTSS fractional-step timestep on NVIDIA B200.

Python access to the two native libraries of this package:

* ``libartss_host.so``: C++ host runtime (ARTSS XML reader, geometry and index
  lists, plugin classes, SolverController / TimeIntegration), ``include/artss_host.h``;
* ``libartss_cuda.so``: the sm_100a kernels behind the plugin interfaces,
  ``include/artss_cuda.h``.

There is no CPU implementation of the timestep: a missing library raises
:class:`NativeLibraryMissing`, and a machine without a CUDA device makes
:class:`Simulation` raise.  :class:`Geometry` (index lists and boundary
assignments) runs on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional

import numpy as np

__all__ = ["Geometry", "Simulation", "NativeLibraryMissing", "ArtssError", "library_path", "FIELD_TYPES",
           "PATCHES", "load_cuda", "load_host"]

HERE = os.path.dirname(os.path.abspath(__file__))
FIELD_TYPES = {"rho": 0, "u": 1, "v": 2, "w": 3, "p": 4, "T": 5, "nu": 6}
PATCHES = ["left", "right", "bottom", "top", "front", "back"]
MAX_LEVEL = 8


class NativeLibraryMissing(RuntimeError):
    pass


class ArtssError(RuntimeError):
    pass


def library_path(name: str) -> str:
    return os.path.join(HERE, name)


class GridDesc(C.Structure):
    _fields_ = [("n_levels", C.c_int32), ("reserved", C.c_int32)] + [
        (f, C.c_int64 * (MAX_LEVEL + 1)) for f in ("Nx", "Ny", "Nz", "i1", "i2", "j1", "j2", "k1", "k2")
    ] + [(f, C.c_double * (MAX_LEVEL + 1)) for f in ("dx", "dy", "dz")]


class BcAssign(C.Structure):
    _fields_ = [("target", C.c_int64), ("source", C.c_int64), ("value", C.c_double), ("sign", C.c_int32),
                ("reserved", C.c_int32)]


class IterCfg(C.Structure):
    _fields_ = [("max_iter", C.c_int64), ("tol_res", C.c_double), ("w", C.c_double)]


class IterStats(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("residual", C.c_double)]


class MgCfg(C.Structure):
    _fields_ = [("n_level", C.c_int32), ("n_cycle", C.c_int32), ("max_cycle", C.c_int32), ("n_relax", C.c_int32),
                ("tol_res", C.c_double), ("smoother", C.c_int32), ("flags", C.c_int32),
                ("smoother_max_iter", C.c_int64), ("smoother_tol_res", C.c_double), ("smoother_w", C.c_double)]


class MgStats(C.Structure):
    _fields_ = [("cycles", C.c_int64), ("coarse_iterations", C.c_int64), ("residual", C.c_double)]


class MixedCfg(C.Structure):
    _fields_ = [("n_level", C.c_int32), ("n_relax", C.c_int32), ("coarse_smoother", C.c_int32), ("flags", C.c_int32),
                ("w", C.c_double), ("coarse_w", C.c_double), ("coarse_rel_tol", C.c_double),
                ("coarse_max_iter", C.c_int64), ("rel_tol", C.c_double), ("max_cycles", C.c_int64)]


class SolveStats(C.Structure):
    _fields_ = [("cycles", C.c_int64), ("residual", C.c_double), ("rel_residual", C.c_double), ("b_norm", C.c_double)]


MIXED_REMOVE_MEAN = 1
MIXED_RBGS = 2
MIXED_BC_LAUNCH = 4
MIXED_CLUSTER_COARSE = 8
MIXED_FINE_PROLONG = 16


class ConvDesc(C.Structure):
    _fields_ = [("D", C.c_int32), ("H", C.c_int32), ("W", C.c_int32), ("cin", C.c_int32), ("cout", C.c_int32),
                ("relu", C.c_int32)]

BC_DTYPE = np.dtype([("target", "<i8"), ("source", "<i8"), ("value", "<f8"), ("sign", "<i4"), ("reserved", "<i4")])

_cuda: Optional[C.CDLL] = None
_host: Optional[C.CDLL] = None

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I64P = C.POINTER(C.c_int64)


def _load(name: str) -> C.CDLL:
    path = library_path(name)
    if not os.path.exists(path):
        raise NativeLibraryMissing(f"{path} is not built; run `make -C {HERE}` or __graft_entry__.build()")
    return C.CDLL(path, mode=C.RTLD_GLOBAL)


def load_cuda() -> C.CDLL:
    """libartss_cuda.so with argument types of include/artss_cuda.h."""
    global _cuda
    if _cuda is None:
        lib = _load("libartss_cuda.so")
        sig = {
            "artss_ctx_create": ([C.POINTER(GridDesc), C.c_int, C.POINTER(_P)], C.c_int),
            "artss_ctx_destroy": ([_P], C.c_int),
            "artss_ctx_stream": ([_P], _P),
            "artss_ctx_sync": ([_P], C.c_int),
            "artss_last_error": ([], C.c_char_p),
            "artss_ctx_kernel_launches": ([_P], C.c_int64),
            "artss_field_alloc": ([_P, C.c_int, C.POINTER(_D)], C.c_int),
            "artss_field_free": ([_P, _D], C.c_int),
            "artss_field_size": ([_P, C.c_int], C.c_int64),
            "artss_upload": ([_P, _D, _D, C.c_int64], C.c_int),
            "artss_download": ([_P, _D, _D, C.c_int64], C.c_int),
            "artss_upload_async": ([_P, _D, _D, C.c_int64], C.c_int),
            "artss_download_async": ([_P, _D, _D, C.c_int64], C.c_int),
            "artss_io_in": ([_P, C.c_int, C.POINTER(_D), C.POINTER(_D), C.c_int64], C.c_int),
            "artss_io_out": ([_P, C.c_int, C.POINTER(_D), C.POINTER(_D), C.c_int64], C.c_int),
            "artss_io_sync": ([_P], C.c_int),
            "artss_set_cell_lists": ([_P, C.c_int, _I64P, C.c_int64, _I64P, C.c_int64], C.c_int),
            "artss_get_cell_flags": ([_P, C.c_int, C.POINTER(C.c_uint8), C.c_int64], C.c_int),
            "artss_set_boundary_program": ([_P, C.c_int, C.c_int, C.POINTER(BcAssign), C.c_int64], C.c_int),
            "artss_boundary_program_waves": ([_P, C.c_int, C.c_int], C.c_int),
            "artss_apply_boundary": ([_P, _D, C.c_int, C.c_int], C.c_int),
            "artss_fill": ([_P, _D, C.c_int, C.c_double], C.c_int),
            "artss_copy": ([_P, _D, _D, C.c_int], C.c_int),
            "artss_add_field": ([_P, _D, _D, C.c_int], C.c_int),
            "artss_add_scalar": ([_P, _D, C.c_double, C.c_int], C.c_int),
            "artss_scale": ([_P, _D, C.c_double, C.c_int], C.c_int),
            "artss_scale_copy": ([_P, _D, _D, C.c_double, C.c_int], C.c_int),
            "artss_couple": ([_P] + [_D] * 9, C.c_int),
            "artss_advect_sl": ([_P, _D, _D, _D, _D, _D, C.c_double, C.c_int], C.c_int),
            "artss_advect_sl_uvw": ([_P] + [_D] * 9 + [C.c_double], C.c_int),
            "artss_turb_const_smagorinsky": ([_P, _D, _D, _D, _D, C.c_double], C.c_int),
            "artss_turb_dynamic_smagorinsky": ([_P, _D, _D, _D, _D, C.c_double], C.c_int),
            "artss_diffuse_cgs": ([_P, _D, _D, _D, C.c_double, _D, C.c_double, C.c_int, C.POINTER(IterCfg), C.c_int,
                                   C.POINTER(IterStats)], C.c_int),
            "artss_diffuse_jacobi": ([_P, _D, _D, _D, C.c_double, _D, C.c_double, C.c_int, C.POINTER(IterCfg),
                                      C.POINTER(IterStats)], C.c_int),
            "artss_diffuse_cgs_mixed": ([_P, _D, _D, _D, C.c_double, _D, C.c_double, C.c_int, C.POINTER(IterCfg),
                                         C.c_int, C.POINTER(IterStats)], C.c_int),
            "artss_divergence": ([_P, _D, _D, _D, _D], C.c_int),
            "artss_projection": ([_P] + [_D] * 7, C.c_int),
            "artss_buoyancy_force": ([_P, _D, _D, _D, C.c_double, C.c_double], C.c_int),
            "artss_add_source": ([_P, _D, _D, C.c_double, C.c_int], C.c_int),
            "artss_diffuse_explicit": ([_P, _D, _D, C.c_double, _D, C.c_double, C.c_int], C.c_int),
            "artss_dissipate": ([_P, _D, _D, _D, _D, C.c_double, C.c_double, C.c_int], C.c_int),
            "artss_mg_create": ([_P, C.POINTER(MgCfg), C.POINTER(_P)], C.c_int),
            "artss_mg_destroy": ([_P], C.c_int),
            "artss_mg_pressure": ([_P, _D, _D, C.c_int, C.POINTER(MgStats)], C.c_int),
            "artss_mg_set_rhs": ([_P, _D, _D], C.c_int),
            "artss_mg_vcycle": ([_P, _D], C.c_int),
            "artss_residual_norm": ([_P, _D, _D, _D, _D], C.c_int),
            "artss_mg_solve_rel": ([_P, _D, _D, C.c_double, C.c_int64, C.POINTER(SolveStats)], C.c_int),
            "artss_mixed_create": ([_P, C.POINTER(MixedCfg), C.POINTER(_P)], C.c_int),
            "artss_mixed_destroy": ([_P], C.c_int),
            "artss_mixed_solve": ([_P, _D, _D, C.POINTER(SolveStats)], C.c_int),
            "artss_laplacian": ([_P, _D, _D, C.c_int], C.c_int),
            "artss_cgs_sweep_variant": ([_P, C.c_int], C.c_int),
            "artss_ctx_sweep_variant": ([_P, C.c_int], C.c_int),
            "artss_ctx_autotune": ([_P, C.c_int], C.c_int),
            "artss_ctx_pdl": ([_P, C.c_int], C.c_int),
            "artss_ctx_stage_timing": ([_P, C.c_int], C.c_int),
            "artss_ctx_stage_mark": ([_P, C.c_int], C.c_int),
            "artss_ctx_stage_read": ([_P, C.POINTER(C.c_double), C.c_int], C.c_int),
            "artss_conv3d_fwd": ([_P, C.POINTER(ConvDesc), _P, _P, _P, _P], C.c_int),
            "artss_nn_check": ([_P], C.c_int),
            "artss_conv3d_wgrad": ([_P, C.POINTER(ConvDesc), _P, _P, _P], C.c_int),
            "artss_nn_zero": ([_P, _P, C.c_int64], C.c_int),
            "artss_nn_relu_bwd": ([_P, _P, _P, C.c_int64], C.c_int),
            "artss_nn_pool2": ([_P, _P, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
            "artss_nn_up2": ([_P, _P, _P] + [C.c_int] * 7, C.c_int),
            "artss_nn_copy_channels": ([_P, _P, C.c_int, C.c_int, _P, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_int],
                                       C.c_int),
            "artss_nn_bias_grad": ([_P, _P, _P, C.c_int64, C.c_int], C.c_int),
            "artss_nn_pack_weights": ([_P, _P, _P, C.c_int, C.c_int, C.c_int], C.c_int),
            "artss_nn_adam": ([_P, _P, _P, _P, _P, C.c_int64, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int],
                              C.c_int),
            "artss_nn_inputs": ([_P, C.c_int, _P, _P, C.c_double, C.c_double, _P, C.c_int], C.c_int),
            "artss_nn_apply": ([_P, C.c_int, _P, C.c_int, _P, C.c_double, _P], C.c_int),
            "artss_nn_target": ([_P, C.c_int, _P, _P, C.c_double, _P], C.c_int),
            "artss_coarse_project": ([_P, _D, C.c_int], C.c_int),
            "artss_nn_mse": ([_P, _P, C.c_int, _P, _P, _P, C.c_int64, C.c_float, _P, C.c_int], C.c_int),
            "artss_cgs_sweep_depth": ([_P, C.c_int], C.c_int),
            "artss_ctx_profile": ([_P, C.c_uint64], C.c_int),
            "artss_ctx_profile_read": ([_P, _I64P, _D, C.c_int], C.c_int),
            "artss_ctx_profile_reset": ([_P], C.c_int),
            "artss_kernel_family_name": ([C.c_int], C.c_char_p),
        }
        for fn, (args, res) in sig.items():
            f = getattr(lib, fn)
            f.argtypes = args
            f.restype = res
        _cuda = lib
    return _cuda


def load_host() -> C.CDLL:
    """libartss_host.so with argument types of include/artss_host.h."""
    global _host
    if _host is None:
        load_cuda()
        lib = _load("libartss_host.so")
        sig = {
            "artss_host_last_error": ([], C.c_char_p),
            "artss_geom_create": ([C.c_char_p, C.POINTER(_P)], C.c_int),
            "artss_geom_destroy": ([_P], None),
            "artss_geom_levels": ([_P], C.c_int),
            "artss_geom_obstacles": ([_P], C.c_int),
            "artss_geom_list": ([_P, C.c_char_p, C.c_int, C.POINTER(_I64P), _I64P], C.c_int),
            "artss_geom_dims": ([_P, C.c_int, _I64P], C.c_int),
            "artss_geom_boundary_program": ([_P, C.c_int, C.c_int, C.POINTER(C.POINTER(BcAssign)), _I64P], C.c_int),
            "artss_geom_grid_desc": ([_P, C.POINTER(GridDesc)], C.c_int),
            "artss_sim_create": ([C.c_char_p, C.c_int, C.POINTER(_P)], C.c_int),
            "artss_sim_destroy": ([_P], None),
            "artss_sim_run": ([_P, C.c_int64, _I64P], C.c_int),
            "artss_sim_set_graphs": ([_P, C.c_int], C.c_int),
            "artss_sim_graph_steps": ([_P], C.c_int64),
            "artss_sim_step_io": ([_P, C.c_int, C.POINTER(C.c_char_p), C.POINTER(_D), C.c_int,
                                   C.POINTER(C.c_char_p), C.POINTER(_D)], C.c_int),
            "artss_sim_step_io_async": ([_P, C.c_int, C.POINTER(C.c_char_p), C.POINTER(_D), C.c_int,
                                         C.POINTER(C.c_char_p), C.POINTER(_D)], C.c_int),
            "artss_sim_io_sync": ([_P], C.c_int),
            "artss_sim_finished": ([_P], C.c_int),
            "artss_sim_time": ([_P], C.c_double),
            "artss_sim_step_index": ([_P], C.c_int64),
            "artss_sim_save": ([_P, C.c_char_p], C.c_int),
            "artss_sim_write_dat": ([_P, C.c_char_p, C.c_char_p], C.c_int),
            "artss_sim_write_vtk": ([_P, C.c_char_p], C.c_int),
            "artss_sim_output_wait": ([_P], C.c_int),
            "artss_sim_cfl": ([_P, C.POINTER(C.c_double)], C.c_int),
            "artss_sim_restore": ([_P, C.c_char_p], C.c_int),
            "artss_sim_inner_cells": ([_P], C.c_int64),
            "artss_sim_get_field": ([_P, C.c_char_p, _D, C.c_int64], C.c_int),
            "artss_sim_set_field": ([_P, C.c_char_p, _D, C.c_int64], C.c_int),
            "artss_sim_field_size": ([_P], C.c_int64),
            "artss_sim_field_device": ([_P, C.c_char_p], _D),
            "artss_sim_context": ([_P], _P),
            "artss_sim_last_stats": ([_P, _I64P, _I64P, _D], C.c_int),
            "artss_sim_pressure": ([_P, C.c_int, _I64P, _D], C.c_int),
            "artss_sim_mg": ([_P], _P),
        }
        for fn, (args, res) in sig.items():
            f = getattr(lib, fn)
            f.argtypes = args
            f.restype = res
        _host = lib
    return _host


def _host_check(st: int, what: str) -> None:
    if st != 0:
        msg = load_host().artss_host_last_error().decode(errors="replace")
        raise ArtssError(f"{what}: {msg} (status {st})")


def cuda_check(st: int, what: str) -> None:
    if st != 0:
        msg = load_cuda().artss_last_error().decode(errors="replace")
        raise ArtssError(f"{what}: {msg} (status {st})")


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_D)


class Geometry:
    """Index lists and boundary assignments of an ARTSS XML scene (CPU)."""

    def __init__(self, xml_path: str):
        self._lib = load_host()
        self._h = _P()
        _host_check(self._lib.artss_geom_create(os.fsencode(xml_path), C.byref(self._h)), "geometry")

    def close(self) -> None:
        if self._h:
            self._lib.artss_geom_destroy(self._h)
            self._h = _P()

    __del__ = close

    @property
    def levels(self) -> int:
        return self._lib.artss_geom_levels(self._h)

    @property
    def obstacles(self) -> int:
        return self._lib.artss_geom_obstacles(self._h)

    def dims(self, level: int = 0):
        d = (C.c_int64 * 3)()
        _host_check(self._lib.artss_geom_dims(self._h, level, d), "dims")
        return tuple(int(x) for x in d)

    def list(self, name: str, level: int = 0) -> np.ndarray:
        p = _I64P()
        n = C.c_int64()
        _host_check(self._lib.artss_geom_list(self._h, name.encode(), level, C.byref(p), C.byref(n)), name)
        if n.value == 0:
            return np.zeros(0, np.int64)
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy()

    def boundary_program(self, level: int, field_type) -> np.ndarray:
        ft = FIELD_TYPES[field_type] if isinstance(field_type, str) else int(field_type)
        p = C.POINTER(BcAssign)()
        n = C.c_int64()
        _host_check(self._lib.artss_geom_boundary_program(self._h, level, ft, C.byref(p), C.byref(n)), "program")
        if n.value == 0:
            return np.zeros(0, BC_DTYPE)
        raw = C.string_at(C.cast(p, C.c_void_p), n.value * C.sizeof(BcAssign))
        return np.frombuffer(raw, dtype=BC_DTYPE).copy()

    def grid_desc(self) -> GridDesc:
        d = GridDesc()
        _host_check(self._lib.artss_geom_grid_desc(self._h, C.byref(d)), "grid")
        return d


class Simulation:
    """One ARTSS scene on a B200: ``Simulation(xml).run(steps)``."""

    def __init__(self, xml_path: str, device: int = 0):
        self._lib = load_host()
        self._h = _P()
        _host_check(self._lib.artss_sim_create(os.fsencode(xml_path), device, C.byref(self._h)), "simulation")
        self.size = int(self._lib.artss_sim_field_size(self._h))

    def close(self) -> None:
        h = getattr(self, "_h", None)
        self._h = None
        if h:
            try:
                self._lib.artss_sim_destroy(h)
            except TypeError:  # interpreter shutdown: ctypes objects already torn down
                pass

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self, steps: int = -1) -> int:
        done = C.c_int64()
        _host_check(self._lib.artss_sim_run(self._h, steps, C.byref(done)), "run")
        return done.value

    def cfl(self) -> float:
        """Analysis::calc_CFL of the current velocity (device max-reduction)."""
        out = C.c_double()
        _host_check(self._lib.artss_sim_cfl(self._h, C.byref(out)), "cfl")
        return out.value

    def write_dat(self, field: str, path: str) -> None:
        """Queue Analysis::write_file of one field (written beside later steps)."""
        _host_check(self._lib.artss_sim_write_dat(self._h, field.encode(), os.fsencode(path)), "write_dat")

    def write_vtk(self, path: str) -> None:
        """Queue VTKWriter::write_numerical (written beside later steps)."""
        _host_check(self._lib.artss_sim_write_vtk(self._h, os.fsencode(path)), "write_vtk")

    def output_wait(self) -> None:
        """Every queued output file is written."""
        _host_check(self._lib.artss_sim_output_wait(self._h), "output_wait")

    def save(self, path: str) -> None:
        """Checkpoint: every field, the step index and the time into one raw
        file (artss_sim_save)."""
        _host_check(self._lib.artss_sim_save(self._h, os.fsencode(path)), "save")

    def restore(self, path: str) -> None:
        """Rollback to a checkpoint of this scene (artss_sim_restore); the run
        continues from the saved step."""
        _host_check(self._lib.artss_sim_restore(self._h, os.fsencode(path)), "restore")

    def set_graphs(self, enable: bool = True) -> None:
        """Whole-step CUDA graphs: from the third step on each step is one
        graph launch (solver loops as device-decided conditional nodes)."""
        _host_check(self._lib.artss_sim_set_graphs(self._h, 1 if enable else 0), "graphs")

    @property
    def graph_steps(self) -> int:
        """Steps run as one graph launch so far."""
        return int(self._lib.artss_sim_graph_steps(self._h))

    def step_io(self, inputs: Dict[str, int], outputs: Dict[str, int]) -> None:
        """One timestep with host transfers overlapped with it: `inputs` and
        `outputs` map field names to host addresses of Nx*Ny*Nz doubles
        (page-locked for overlap); inputs are set before they are read,
        outputs read back after their last write of the step."""
        names_in = [k.encode() for k in inputs]
        names_out = [k.encode() for k in outputs]
        a_in = (C.c_char_p * len(names_in))(*names_in)
        a_out = (C.c_char_p * len(names_out))(*names_out)
        p_in = (_D * len(inputs))(*[C.cast(C.c_void_p(v), _D) for v in inputs.values()])
        p_out = (_D * len(outputs))(*[C.cast(C.c_void_p(v), _D) for v in outputs.values()])
        _host_check(self._lib.artss_sim_step_io(self._h, len(names_in), a_in, p_in, len(names_out), a_out, p_out),
                    "step_io")

    def step_io_async(self, inputs: Dict[str, int], outputs: Dict[str, int]) -> None:
        """step_io pipelined: returns once the uploads, the step and the
        read-back are enqueued; inputs go up while the previous call's outputs
        come down.  The host arrays of a call may be reused once the call two
        after it has returned, or after io_sync()."""
        names_in = [k.encode() for k in inputs]
        names_out = [k.encode() for k in outputs]
        a_in = (C.c_char_p * len(names_in))(*names_in)
        a_out = (C.c_char_p * len(names_out))(*names_out)
        p_in = (_D * len(inputs))(*[C.cast(C.c_void_p(v), _D) for v in inputs.values()])
        p_out = (_D * len(outputs))(*[C.cast(C.c_void_p(v), _D) for v in outputs.values()])
        _host_check(self._lib.artss_sim_step_io_async(self._h, len(names_in), a_in, p_in, len(names_out), a_out,
                                                      p_out), "step_io_async")

    def io_sync(self) -> None:
        """Waits for every transfer and step enqueued by step_io_async."""
        _host_check(self._lib.artss_sim_io_sync(self._h), "io_sync")

    @property
    def finished(self) -> bool:
        return bool(self._lib.artss_sim_finished(self._h))

    @property
    def time(self) -> float:
        return self._lib.artss_sim_time(self._h)

    @property
    def step_index(self) -> int:
        return self._lib.artss_sim_step_index(self._h)

    @property
    def inner_cells(self) -> int:
        return self._lib.artss_sim_inner_cells(self._h)

    @property
    def context(self):
        return self._lib.artss_sim_context(self._h)

    def field(self, name: str) -> np.ndarray:
        out = np.empty(self.size, np.float64)
        _host_check(self._lib.artss_sim_get_field(self._h, name.encode(), dptr(out), self.size), name)
        return out

    def set_field(self, name: str, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        _host_check(self._lib.artss_sim_set_field(self._h, name.encode(), dptr(v), v.size), name)

    def device_pointer(self, name: str) -> int:
        p = self._lib.artss_sim_field_device(self._h, name.encode())
        return C.cast(p, C.c_void_p).value or 0

    def stats(self) -> Dict[str, object]:
        it = (C.c_int64 * 4)()
        cyc = C.c_int64()
        res = C.c_double()
        _host_check(self._lib.artss_sim_last_stats(self._h, it, C.byref(cyc), C.byref(res)), "stats")
        return {"diffusion_iterations": list(it), "mg_cycles": cyc.value, "mg_residual": res.value}

    def pressure(self, first_step: bool = True):
        cyc = C.c_int64()
        res = C.c_double()
        _host_check(self._lib.artss_sim_pressure(self._h, 1 if first_step else 0, C.byref(cyc), C.byref(res)),
                    "pressure")
        return cyc.value, res.value

    def kernel_launches(self) -> int:
        return int(load_cuda().artss_ctx_kernel_launches(self.context))


class Context:
    """A device context built directly through the C ABI (include/artss_cuda.h),
    the way a reference-side integration would: grid descriptor, the level
    lists and the ordered boundary assignments of a Geometry, and device
    arrays allocated by the library."""

    def __init__(self, geom: "Geometry", device: int = 0):
        self.lib = load_cuda()
        self.geom = geom
        self.grid = geom.grid_desc()
        self.h = C.c_void_p()
        cuda_check(self.lib.artss_ctx_create(C.byref(self.grid), device, C.byref(self.h)), "ctx")
        self.fields = []
        for l in range(self.grid.n_levels + 1):
            inner = np.ascontiguousarray(geom.list("inner", l))
            dom = np.ascontiguousarray(geom.list("domain", l))
            cuda_check(self.lib.artss_set_cell_lists(self.h, l, inner.ctypes.data_as(_I64P), inner.size,
                                                       dom.ctypes.data_as(_I64P), dom.size), "lists")
            for ft in range(7):
                prog = geom.boundary_program(l, ft)
                if prog.size:
                    arr = (BcAssign * prog.size)()
                    C.memmove(arr, prog.ctypes.data, prog.nbytes)
                    cuda_check(self.lib.artss_set_boundary_program(self.h, l, ft, arr, prog.size), "bc")

    def size(self, level: int = 0) -> int:
        g = self.grid
        return g.Nx[level] * g.Ny[level] * g.Nz[level]

    def field(self, values=None, level: int = 0):
        p = _D()
        cuda_check(self.lib.artss_field_alloc(self.h, level, C.byref(p)), "alloc")
        self.fields.append(p)
        if values is not None:
            self.upload(p, values)
        return p

    def upload(self, p, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        cuda_check(self.lib.artss_upload(self.h, p, v.ctypes.data_as(_D), v.size), "upload")

    def download(self, p, level: int = 0) -> np.ndarray:
        out = np.empty(self.size(level))
        cuda_check(self.lib.artss_download(self.h, out.ctypes.data_as(_D), p, out.size), "download")
        return out

    def close(self):
        if self.h:
            self.lib.artss_ctx_destroy(self.h)
            self.h = C.c_void_p()


def consistent_rhs(ctx: Context, b: np.ndarray, n_level: int, cycles: int = 40):
    """A right-hand side in the range of the level-0 pressure operator A close
    to `b`: b' = A p_inf, where p_inf is what `cycles` mixed-precision V-cycles
    reach from p = 0 (their residual stalls at the part of b outside the range
    of A).  Pure-Neumann scenes with obstacles need this, since the reference's
    obstacle boundary programs make A non-symmetric and a mean-free b is not
    solvable to a small residual.  Returns (device array, host copy)."""
    lib = ctx.lib
    db = ctx.field(b)
    dp = ctx.field(np.zeros(ctx.size()))
    # no mean removal: A p_inf must not change where A 1 != 0 (Dirichlet boundaries)
    cfg = MixedCfg(n_level, 2, 1, 0, 0.6666666667, 0.0, 1e-3, 40, 0.0, cycles)
    mx = C.c_void_p()
    cuda_check(lib.artss_mixed_create(ctx.h, C.byref(cfg), C.byref(mx)), "mixed")
    try:
        st = SolveStats()
        cuda_check(lib.artss_mixed_solve(mx, dp, db, C.byref(st)), "mixed solve")
    finally:
        lib.artss_mixed_destroy(mx)
    out = ctx.field(np.zeros(ctx.size()))
    cuda_check(lib.artss_laplacian(ctx.h, out, dp, 0), "laplacian")
    return out, ctx.download(out)
