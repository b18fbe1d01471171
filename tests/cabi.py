"""A device context built directly through the C ABI (include/artss_cuda.h),
the way a reference-side integration would: grid descriptor, the level lists
and the ordered boundary assignments of artss_b200.Geometry.  Used by the
kernel-level GPU tests."""
from __future__ import annotations

import ctypes as C

import numpy as np

import artss_b200 as A

_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)


class Context:
    def __init__(self, geom: "A.Geometry", device: int = 0):
        self.lib = A.load_cuda()
        self.geom = geom
        self.grid = geom.grid_desc()
        self.h = C.c_void_p()
        A.cuda_check(self.lib.artss_ctx_create(C.byref(self.grid), device, C.byref(self.h)), "ctx")
        self.fields = []
        for l in range(self.grid.n_levels + 1):
            inner = np.ascontiguousarray(geom.list("inner", l))
            dom = np.ascontiguousarray(geom.list("domain", l))
            A.cuda_check(self.lib.artss_set_cell_lists(self.h, l, inner.ctypes.data_as(_I64), inner.size,
                                                       dom.ctypes.data_as(_I64), dom.size), "lists")
            for ft in range(7):
                prog = geom.boundary_program(l, ft)
                if prog.size:
                    arr = (A.BcAssign * prog.size)()
                    C.memmove(arr, prog.ctypes.data, prog.nbytes)
                    A.cuda_check(self.lib.artss_set_boundary_program(self.h, l, ft, arr, prog.size), "bc")

    def size(self, level: int = 0) -> int:
        g = self.grid
        return g.Nx[level] * g.Ny[level] * g.Nz[level]

    def field(self, values=None, level: int = 0):
        p = _D()
        A.cuda_check(self.lib.artss_field_alloc(self.h, level, C.byref(p)), "alloc")
        self.fields.append(p)
        if values is not None:
            self.upload(p, values)
        return p

    def upload(self, p, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        A.cuda_check(self.lib.artss_upload(self.h, p, v.ctypes.data_as(_D), v.size), "upload")

    def download(self, p, level: int = 0) -> np.ndarray:
        out = np.empty(self.size(level))
        A.cuda_check(self.lib.artss_download(self.h, out.ctypes.data_as(_D), p, out.size), "download")
        return out

    def close(self):
        if self.h:
            self.lib.artss_ctx_destroy(self.h)
            self.h = C.c_void_p()
