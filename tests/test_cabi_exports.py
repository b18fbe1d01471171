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
    """The entry-point index of INTEGRATION.md names every declared function
    (the network kernels by their artss_nn_ prefix)."""
    with open(os.path.join(os.path.dirname(HERE), "INTEGRATION.md")) as f:
        text = f.read()
    assert "## 7. Entry-point index" in text
    index = text.split("## 7. Entry-point index", 1)[1]
    listed = set(re.findall(r"`(artss_\w+)`", index))
    missing = [n for h in ("artss_cuda.h", "artss_host.h") for n in declared(h)
               if n not in listed and not (n.startswith("artss_nn_") and "artss_nn_*" in index)]
    assert not missing, missing
