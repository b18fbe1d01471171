"""Every XML configuration the reference ships (tests/, examples/,
data_assimilation/example/), read by both sides: the reference build and
this library must accept the same files, reject the same files with the same
message, and build identical index lists for every level and obstacle.

Runs where the reference source tree and its oracle build are present
(ARTSS_REFERENCE_DIR, default /root/reference); skipped elsewhere.  CPU only:
the geometry and lists are host code."""
import glob
import os
import subprocess

import numpy as np
import pytest

import artss_b200 as A
from tests import refdriver

REFERENCE = os.environ.get("ARTSS_REFERENCE_DIR", "/root/reference")


def _configs():
    return sorted(os.path.relpath(p, REFERENCE) for p in glob.glob(os.path.join(REFERENCE, "**", "*.xml"),
                                                                   recursive=True))


def _names(g):
    names = ["inner", "domain"] + ["bnd_" + p for p in A.PATCHES]
    if g.obstacles:
        names += ["obst"] + [f"obst{i}_{p}" for i in range(g.obstacles) for p in A.PATCHES]
    return names


def test_reference_tree_holds_configs():
    if not os.path.isdir(REFERENCE):
        pytest.skip("reference source tree not present")
    assert len(_configs()) >= 20


@pytest.mark.parametrize("rel", _configs() if os.path.isdir(REFERENCE) else [])
def test_reference_config_accepted_alike_with_identical_lists(tmp_path, rel):
    if not refdriver.available():
        pytest.skip("reference oracle not built (oracle/Makefile)")
    path = os.path.join(REFERENCE, rel)
    ref = subprocess.run([refdriver.DRIVER, path, "--steps", "0", "--dump", str(tmp_path), "--lists"],
                         capture_output=True, text=True, timeout=900)
    try:
        g = A.Geometry(path)
        ours = None
    except A.ArtssError as e:
        g, ours = None, str(e)
    if ref.returncode != 0:
        # the reference's own rejection (config_error caught by the driver)
        msg = ref.stderr.strip().splitlines()[-1]
        assert msg.startswith("reference error: "), ref.stderr
        assert ours is not None, f"{rel}: the reference rejects it ({msg}), this library accepts it"
        assert msg[len("reference error: "):] in ours, f"{rel}: reference '{msg}' vs ours '{ours}'"
        return
    assert ours is None, f"{rel}: the reference accepts it, this library rejects it: {ours}"
    for level in range(g.levels + 1):
        for n in _names(g):
            np.testing.assert_array_equal(g.list(n, level), refdriver.ref_list(str(tmp_path), n, level),
                                          err_msg=f"{rel}: {n} level {level}")
