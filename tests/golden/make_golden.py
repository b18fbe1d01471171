"""Generates the committed golden fixtures from the reference serial build
(oracle/_ref/artss_ref_driver, built by oracle/Makefile from the ARTSS
sources).  Run from the repository root: `python tests/golden/make_golden.py`.

Fixtures
  smoke_box16_step2.npz   u,v,w,p,T,nu_t after 2 steps of scenes.plume_box(n=16, steps=2, n_level=2)
  lists_room32.npz        every index list of scenes.room_with_door(n=32, n_level=2)
  box16_steps.npz         u,v,w,p,T,nu_t after steps 1..4 of scenes.plume_box(n=16, steps=4, n_level=2)
"""
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from artss_b200 import scenes  # noqa: E402
from tests import refdriver  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
FIELDS = ["u", "v", "w", "p", "T", "nu_t"]
PATCHES = ["left", "right", "bottom", "top", "front", "back"]


def main():
    assert refdriver.available(), "build oracle/_ref first (make -C oracle ref)"
    with tempfile.TemporaryDirectory() as tmp:
        xml = scenes.write(scenes.plume_box(n=16, steps=2, n_level=2), os.path.join(tmp, "smoke.xml"))
        d = refdriver.run(xml, os.path.join(tmp, "smoke"), steps=2)
        np.savez_compressed(os.path.join(HERE, "smoke_box16_step2.npz"),
                            **{f: refdriver.field(d, 2, f) for f in FIELDS})

        xml = scenes.write(scenes.plume_box(n=16, steps=4, n_level=2), os.path.join(tmp, "box16.xml"))
        d = refdriver.run(xml, os.path.join(tmp, "box16"), steps=4)
        np.savez_compressed(os.path.join(HERE, "box16_steps.npz"),
                            **{f"{f}_{s}": refdriver.field(d, s, f) for f in FIELDS for s in range(0, 5)})

        sc = scenes.room_with_door(n=32, steps=0, n_level=2)
        xml = scenes.write(sc, os.path.join(tmp, "room.xml"))
        d = refdriver.run(xml, os.path.join(tmp, "room"), steps=0, lists=True)
        lists = {}
        for level in range(3):
            names = ["inner", "domain", "obst"] + ["bnd_" + p for p in PATCHES]
            names += [f"obst{i}_{p}" for i in range(7) for p in PATCHES]
            for n in names:
                lists[f"{n}_L{level}"] = refdriver.ref_list(d, n, level)
        np.savez_compressed(os.path.join(HERE, "lists_room32.npz"), **lists)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
