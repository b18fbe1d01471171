"""Runs the reference oracle (oracle/_ref/artss_ref_driver, the ARTSS serial
build plus a dump driver, see oracle/Makefile) and loads what it dumps.
Test infrastructure only."""
from __future__ import annotations

import json
import os
import subprocess
from typing import Dict, List, Optional

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "artss_ref_driver")
FIELDS = ["u", "v", "w", "p", "T", "nu_t", "rhs", "kappa_t", "S_T", "f_x", "f_y", "f_z", "T_a"]


def available() -> bool:
    return os.access(DRIVER, os.X_OK)


def run(xml: str, out_dir: str, steps: int, every: int = 1, lists: bool = False, timeout: float = 600,
        fields: Optional[List[str]] = None) -> str:
    """Runs the reference for `steps` steps and dumps the fields (all, or
    only `fields`) at step 0 and every `every`-th step."""
    os.makedirs(out_dir, exist_ok=True)
    cmd = [DRIVER, xml, "--steps", str(steps), "--dump", out_dir, "--every", str(every)]
    if lists:
        cmd.append("--lists")
    if fields:
        cmd += ["--fields", ",".join(fields)]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, timeout=timeout)
    return out_dir


def timing(xml: str, steps: int, timeout: float = 3600) -> Dict:
    r = subprocess.run([DRIVER, xml, "--steps", str(steps), "--time"], check=True, capture_output=True, text=True,
                       timeout=timeout)
    return json.loads(r.stdout.strip().splitlines()[-1])


def mg_solve(xml: str, rhs_file: str, tol: float, max_cycles: int = 1000, dump: Optional[str] = None,
             timeout: float = 3600) -> Dict:
    cmd = [DRIVER, xml, "--mg-rhs", rhs_file, "--mg-rel-tol", repr(tol), "--mg-max-cycles", str(max_cycles)]
    if dump:
        cmd += ["--dump", dump]
    r = subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=timeout)
    return json.loads(r.stdout.strip().splitlines()[-1])


def field(out_dir: str, step: int, name: str) -> np.ndarray:
    return np.fromfile(os.path.join(out_dir, f"step{step:05d}_{name}.f64"), dtype=np.float64)


def ref_list(out_dir: str, name: str, level: int) -> np.ndarray:
    return np.fromfile(os.path.join(out_dir, "lists", f"{name}_L{level}.u64"), dtype=np.int64)


def rel_max_err(a: np.ndarray, b: np.ndarray, mask: Optional[np.ndarray] = None) -> float:
    """max|a-b| / max(max|b|, tiny) over the masked cells.  NaNs must sit on
    the same cells in both (the reference produces them in some scenes, e.g.
    DynamicSmagorinsky's 0/0 coefficient where the filtered strain vanishes);
    otherwise the error is infinite.  The other cells are compared as usual."""
    if mask is not None:
        a = a[mask]
        b = b[mask]
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return float("inf")
    a, b = a[~na], b[~nb]
    if a.size == 0:
        return 0.0
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) / scale
