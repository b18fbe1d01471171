"""The drop-in boundary: both shared libraries load without a GPU and export
every function that include/artss_cuda.h and include/artss_host.h declare
(no compute call is made)."""
import ctypes
import os
import re

import pytest

from artss_b200 import library_path

HERE = os.path.dirname(os.path.abspath(__file__))
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

# a declaration: return type, the artss_ name, an opening parenthesis
_DECL = re.compile(r"^\s*(?:[A-Za-z_][\w ]*[\w*]\s*\**\s*)\b(artss_\w+)\s*\(", re.M)


def declared(header: str):
    with open(os.path.join(INCLUDE, header)) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)  # comments
    text = re.sub(r"//[^\n]*", "", text)
    text = re.sub(r"^\s*#.*$", "", text, flags=re.M)  # preprocessor lines (macros)
    names = set(_DECL.findall(text))
    # struct / typedef names are types, not functions
    return sorted(n for n in names if not re.search(r"\b(struct|typedef)\s+" + n + r"\b", text))


@pytest.mark.parametrize("header,lib", [("artss_cuda.h", "libartss_cuda.so"), ("artss_host.h", "libartss_host.so")])
def test_library_exports_every_declared_function(header, lib):
    names = declared(header)
    assert len(names) > 10, names
    so = ctypes.CDLL(library_path(lib))
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, f"{lib} lacks {missing}"


def test_pipelined_transfer_entry_points_declared():
    # the step-overlapping transfers and programmatic launch switch are part of the boundary
    cuda = declared("artss_cuda.h")
    host = declared("artss_host.h")
    for n in ("artss_io_in", "artss_io_out", "artss_io_sync", "artss_ctx_pdl", "artss_copy_upload"):
        assert n in cuda, n
    for n in ("artss_sim_step_io", "artss_sim_step_io_async", "artss_sim_io_sync", "artss_sim_set_graphs"):
        assert n in host, n


def test_integration_index_lists_every_entry_point():
    """The integration guide's entry-point index names every declared
    function (the network kernels by their artss_nn_ prefix)."""
    with open(os.path.join(os.path.dirname(HERE), "INTEGRATION.md")) as f:
        text = f.read()
    assert "## 7. Entry-point index" in text
    index = text.split("## 7. Entry-point index", 1)[1]
    listed = set(re.findall(r"`(artss_\w+)`", index))
    missing = [n for h in ("artss_cuda.h", "artss_host.h") for n in declared(h)
               if n not in listed and not (n.startswith("artss_nn_") and "artss_nn_*" in index)]
    assert not missing, missing


def test_geometry_entry_points_report_bad_arguments(tmp_path):
    """The CPU-only geometry functions of the host library return
    ARTSS_ERR_ARG (-1) with a message for unusable arguments and a file the
    settings reader refuses, and ARTSS_OK for a valid call."""
    import ctypes as C
    from artss_b200 import scenes
    lib = C.CDLL(library_path("libartss_host.so"))
    lib.artss_host_last_error.restype = C.c_char_p
    lib.artss_geom_create.argtypes = [C.c_char_p, C.POINTER(C.c_void_p)]
    lib.artss_geom_list.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.POINTER(C.POINTER(C.c_int64)),
                                    C.POINTER(C.c_int64)]
    lib.artss_geom_boundary_program.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p),
                                                C.POINTER(C.c_int64)]
    lib.artss_geom_destroy.argtypes = [C.c_void_p]
    err = lambda: lib.artss_host_last_error().decode()  # noqa: E731

    h = C.c_void_p()
    assert lib.artss_geom_create(str(tmp_path / "absent.xml").encode(), C.byref(h)) == -1
    assert lib.artss_geom_create(None, C.byref(h)) == -1 and "null" in err()
    xml = scenes.write(scenes.plume_box(n=16, steps=1, n_level=2), str(tmp_path / "box.xml"))
    assert lib.artss_geom_create(xml.encode(), C.byref(h)) == 0
    try:
        data, n = C.POINTER(C.c_int64)(), C.c_int64()
        assert lib.artss_geom_list(h, b"inner", 0, C.byref(data), C.byref(n)) == 0 and n.value == 16 ** 3
        assert lib.artss_geom_list(h, b"nonsense", 0, C.byref(data), C.byref(n)) == -1
        assert "unknown list 'nonsense'" in err()
        assert lib.artss_geom_list(h, b"inner", 3, C.byref(data), C.byref(n)) == -1 and "level" in err()
        assert lib.artss_geom_list(h, b"inner", -1, C.byref(data), C.byref(n)) == -1
        assert lib.artss_geom_list(h, None, 0, C.byref(data), C.byref(n)) == -1
        ops, m = C.c_void_p(), C.c_int64()
        assert lib.artss_geom_boundary_program(h, 0, 4, C.byref(ops), C.byref(m)) == 0 and m.value > 0
        assert lib.artss_geom_boundary_program(h, 0, 7, C.byref(ops), C.byref(m)) == -1
        assert lib.artss_geom_boundary_program(h, 9, 4, C.byref(ops), C.byref(m)) == -1
    finally:
        lib.artss_geom_destroy(h)
