"""Bit-exact index lists ("GPU lists") of the host geometry against the
reference's Multigrid/Domain/Obstacle construction.

The golden fixture pins the room scene (seven touching walls: boundary-patch
trimming and neighbouring-obstacle constraint removal); with the reference
oracle built, every list of several more scenes is compared directly."""
import os

import numpy as np
import pytest

import artss_b200 as A
from artss_b200 import scenes
from tests import refdriver

HERE = os.path.dirname(os.path.abspath(__file__))
PATCHES = A.PATCHES


def all_names(g):
    names = ["inner", "domain"] + ["bnd_" + p for p in PATCHES]
    if g.obstacles:
        names += ["obst"] + [f"obst{i}_{p}" for i in range(g.obstacles) for p in PATCHES]
    return names


def test_room_lists_match_golden(tmp_path):
    gold = np.load(os.path.join(HERE, "golden", "lists_room32.npz"))
    xml = scenes.write(scenes.room_with_door(n=32, steps=0, n_level=2), str(tmp_path / "room.xml"))
    g = A.Geometry(xml)
    assert g.levels == 2 and g.obstacles == 7
    for level in range(3):
        for n in all_names(g):
            np.testing.assert_array_equal(g.list(n, level), gold[f"{n}_L{level}"], err_msg=f"{n} level {level}")


def _scene_set():
    return {
        "box16": scenes.plume_box(n=16, steps=0, n_level=2),
        "box64": scenes.plume_box(n=64, steps=0, n_level=4),
        "channel": scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=0, n_level=3),
        "room64": scenes.room_with_door(n=64, steps=0, n_level=3),
        "odd_sizes": scenes.plume_box(n=24, steps=0, n_level=3),
    }


@pytest.mark.parametrize("name", list(_scene_set().keys()))
def test_lists_match_reference(tmp_path, name):
    if not refdriver.available():
        pytest.skip("reference oracle not built")
    xml = scenes.write(_scene_set()[name], str(tmp_path / f"{name}.xml"))
    d = refdriver.run(xml, str(tmp_path / "ref"), steps=0, lists=True)
    g = A.Geometry(xml)
    for level in range(g.levels + 1):
        for n in all_names(g):
            np.testing.assert_array_equal(g.list(n, level), refdriver.ref_list(d, n, level),
                                          err_msg=f"{name}: {n} level {level}")


def test_random_obstacle_scenes_match_reference(tmp_path):
    """Seeded scenes of 1-6 separated boxes (edges 4-12 cells)."""
    if not refdriver.available():
        pytest.skip("reference oracle not built")
    for seed in range(4):
        n = 32
        boxes = scenes.random_boxes((n, n, n), 4, 12, 1 + seed % 6, seed, (2.4 / n,) * 3, levels=2)
        sc = scenes.plume_box(n=n, steps=0, n_level=2, obstacles=boxes, obstacle_bcs=scenes.solid_obstacle_bcs())
        xml = scenes.write(sc, str(tmp_path / f"r{seed}.xml"))
        d = refdriver.run(xml, str(tmp_path / f"r{seed}"), steps=0, lists=True)
        g = A.Geometry(xml)
        for level in range(g.levels + 1):
            for nm in all_names(g):
                np.testing.assert_array_equal(g.list(nm, level), refdriver.ref_list(d, nm, level),
                                              err_msg=f"seed {seed}: {nm} level {level}")


def test_overlapping_obstacles_rejected(tmp_path):
    sc = scenes.plume_box(n=16, steps=0, n_level=1, obstacles=[
        scenes.Box(0.3, 0.9, 0.3, 0.9, 0.3, 0.9, "a"), scenes.Box(0.6, 1.2, 0.6, 1.2, 0.6, 1.2, "b")],
        obstacle_bcs=scenes.solid_obstacle_bcs())
    xml = scenes.write(sc, str(tmp_path / "ov.xml"))
    with pytest.raises(A.ArtssError, match="overlap"):
        A.Geometry(xml)


def test_multigrid_kat_8x12x4():
    """Known-answer sizes of ARTSS gtests/domain/Multigrid.cpp:30-97 (8x12x4
    cells, 2 levels): domain-inner list 384/48/6 cells."""
    import tempfile
    sc = scenes.Scene(solver="PressureSolver", nx=8, ny=12, nz=4, X=(0, 8), Y=(0, 12), Z=(0, 4), n_level=2,
                      boundaries=[("p", "front,back,bottom,top,left,right", "dirichlet", 0.0)], ic="Zero",
                      noise=False, steps=1)
    with tempfile.TemporaryDirectory() as tmp:
        g = A.Geometry(scenes.write(sc, os.path.join(tmp, "kat.xml")))
        assert [g.list("inner", l).size for l in range(3)] == [384, 48, 6]
        assert g.list("domain", 0).size == 10 * 14 * 6


def test_dynamic_adaption_rejected_like_the_reference(tmp_path):
    """ARTSS's settings parser refuses <adaption dynamic="Yes"> (Settings.cpp:512-524,
    issue #178), so no reference run ever reaches its Adaption classes; this
    library refuses it with the same message."""
    sc = scenes.layered_channel(steps=0, adaption={"buffer": 14, "check_value": 335.0, "timestep": 1,
                                                   "expansion_size": 1})
    xml = scenes.write(sc, str(tmp_path / "adaption.xml"))
    msg = "handling of adaption is not fully implemented yet. Please check issue #178"
    with pytest.raises(A.ArtssError, match="issue #178"):
        A.Geometry(xml)
    if refdriver.available():
        import subprocess
        r = subprocess.run([refdriver.DRIVER, xml, "--steps", "0"], capture_output=True, text=True, timeout=300)
        assert r.returncode != 0 and msg in r.stderr


@pytest.mark.parametrize("name", ["layered_channel", "inset_box"])
def test_computational_domain_lists_match_reference(tmp_path, name):
    """A computational domain inside the physical one: lists of every level."""
    if not refdriver.available():
        pytest.skip("reference oracle not built")
    sc = getattr(scenes, name)(steps=0)
    xml = scenes.write(sc, str(tmp_path / f"{name}.xml"))
    d = refdriver.run(xml, str(tmp_path / "ref"), steps=0, lists=True)
    g = A.Geometry(xml)
    for level in range(g.levels + 1):
        for n in all_names(g):
            np.testing.assert_array_equal(g.list(n, level), refdriver.ref_list(d, n, level),
                                          err_msg=f"{name}: {n} level {level}")


def _inset(n, before, after, levels, h=0.1):
    """A computational domain of n cells of h per axis with `before` and
    `after` physical cells on either side of it."""
    ext = [(0.0, (before[a] + n[a] + after[a]) * h) for a in range(3)]
    cd = tuple((before[a] * h, (before[a] + n[a]) * h) for a in range(3))
    return scenes.Scene(steps=0, n_level=levels, boundaries=scenes.closed_box_bcs(), nx=n[0], ny=n[1], nz=n[2],
                        X=ext[0], Y=ext[1], Z=ext[2], cd=cd, noise=False,
                        source_pos=tuple((cd[a][0] + cd[a][1]) / 2 for a in range(3)))


@pytest.mark.parametrize("shape,axis,coarse,overrun", [
    (((12, 8, 8), (5, 0, 0), (1, 0, 0)), "x", "6 cells, index range 3..9", True),
    (((8, 24, 8), (0, 3, 0), (0, 0, 0)), "y", "12 cells, index range 3..13", False),
])
def test_computational_domain_between_coarse_cells_refused(tmp_path, shape, axis, coarse, overrun):
    """A computational domain whose bounds fall between the cells of a coarse
    level: the level's index range and its cell count differ by one.  The
    reference sizes its lists by the count and fills them over the range
    (Domain.cpp:40-54, 191-203) -- it writes past its inner list (glibc aborts)
    or leaves zero entries in it; this library refuses the file."""
    xml = scenes.write(_inset(*shape, levels=1), str(tmp_path / "cd.xml"))
    with pytest.raises(A.ArtssError, match=f"fall between the cells of multigrid level 1 on axis {axis} \\({coarse}\\)"):
        A.Geometry(xml)
    if refdriver.available():
        import subprocess
        r = subprocess.run([refdriver.DRIVER, xml, "--steps", "0", "--dump", str(tmp_path), "--lists"],
                           capture_output=True, text=True, timeout=300)
        if overrun:
            assert r.returncode != 0 and "reference error" not in r.stderr, r.stderr
        else:
            assert r.returncode == 0, r.stderr
            assert (refdriver.ref_list(str(tmp_path), "inner", 1) == 0).sum() == 16


def test_computational_domain_off_coarse_cells_lists_match_reference(tmp_path):
    """Odd margins whose coarse-level rounding still gives the level's cell
    count are accepted, with the reference's lists on every level."""
    if not refdriver.available():
        pytest.skip("reference oracle not built")
    for i, shape in enumerate([((12, 8, 8), (3, 0, 0), (3, 0, 0)), ((16, 8, 8), (3, 2, 2), (1, 2, 2)),
                               ((12, 12, 8), (2, 3, 2), (2, 1, 2))]):
        xml = scenes.write(_inset(*shape, levels=1), str(tmp_path / f"cd{i}.xml"))
        d = refdriver.run(xml, str(tmp_path / f"ref{i}"), steps=0, lists=True)
        g = A.Geometry(xml)
        for level in range(g.levels + 1):
            for n in all_names(g):
                np.testing.assert_array_equal(g.list(n, level), refdriver.ref_list(d, n, level),
                                              err_msg=f"{shape}: {n} level {level}")


_OFFSET_NEIGHBOURS = [  # two obstacles side by side, offset across the shared face (cell index ranges)
    [((7, 7), (9, 10), (2, 3)), ((8, 9), (9, 11), (2, 2))],
    [((4, 6), (4, 5), (7, 8)), ((3, 6), (6, 8), (7, 7))],
    [((7, 10), (7, 7), (9, 9)), ((8, 10), (7, 9), (10, 10))],
    [((4, 5), (8, 9), (6, 7)), ((6, 7), (8, 10), (6, 6))],
    [((7, 9), (7, 8), (8, 10)), ((10, 11), (7, 9), (8, 8))],
]


def _offset_scene(cells, levels):
    h = 0.1
    boxes = [scenes.Box(round((c[0][0] - 1) * h, 10), round(c[0][1] * h, 10), round((c[1][0] - 1) * h, 10),
                        round(c[1][1] * h, 10), round((c[2][0] - 1) * h, 10), round(c[2][1] * h, 10), f"b{i}")
             for i, c in enumerate(cells)]
    return scenes.Scene(steps=0, n_level=levels, nx=12, ny=12, nz=12, X=(0.0, 1.2), Y=(0.0, 1.2), Z=(0.0, 1.2),
                        obstacles=boxes, obstacle_bcs=scenes.solid_obstacle_bcs(), boundaries=scenes.closed_box_bcs(),
                        noise=False, source_pos=(0.3, 0.3, 0.9))


def test_offset_neighbour_removal_known_answer(tmp_path):
    """Obstacle::circular_constraints walks both obstacles' facing patches in
    one loop (Obstacle.cpp:734-771); a removal rectangle that is empty on the
    outer axis gives up its first matching cell only while that joint loop
    runs.  Here obstacle 0's right patch keeps (7,10,2): the reference build
    gives [539, 721, 735] (two independent walks would also drop 539)."""
    xml = scenes.write(_offset_scene(_OFFSET_NEIGHBOURS[0], 1), str(tmp_path / "n.xml"))
    g = A.Geometry(xml)
    np.testing.assert_array_equal(g.list("obst0_right", 0), [539, 721, 735])


@pytest.mark.parametrize("case", range(len(_OFFSET_NEIGHBOURS)))
def test_offset_neighbour_lists_match_reference(tmp_path, case):
    if not refdriver.available():
        pytest.skip("reference oracle not built")
    xml = scenes.write(_offset_scene(_OFFSET_NEIGHBOURS[case], 2), str(tmp_path / "n.xml"))
    d = refdriver.run(xml, str(tmp_path / "ref"), steps=0, lists=True)
    g = A.Geometry(xml)
    for level in range(g.levels + 1):
        for n in all_names(g):
            np.testing.assert_array_equal(g.list(n, level), refdriver.ref_list(d, n, level),
                                          err_msg=f"case {case}: {n} level {level}")


@pytest.mark.parametrize("case", ["no_layers", "missing_border", "missing_value"])
def test_malformed_layers_rejected_like_the_reference(tmp_path, case):
    """LayersT parameters are read as in parse_layers_parameters
    (Settings.cpp:302-321): at least one layer, value_1 .. value_n and
    border_1 .. border_{n-1}; a malformed set is refused with the reference's
    message."""
    params = dict(scenes.layered_channel(steps=0).ic_params)
    if case == "no_layers":
        params["n_layers"] = 0
        msg = "Numbers of layers has to be at least 1. Current value: 0"
    elif case == "missing_border":
        del params["border_2"]
        msg = "Value border_2 is for initial_conditions/LayersT required."
    else:
        del params["value_4"]
        msg = "Value value_4 is for initial_conditions/LayersT required."
    sc = scenes.layered_channel(steps=0, ic_params=params)
    xml = scenes.write(sc, str(tmp_path / f"{case}.xml"))
    with pytest.raises(A.ArtssError) as e:
        A.Geometry(xml)
    assert msg in str(e.value)
    if refdriver.available():
        import subprocess
        r = subprocess.run([refdriver.DRIVER, xml, "--steps", "0"], capture_output=True, text=True, timeout=300)
        assert r.returncode != 0 and msg in r.stderr, r.stderr


@pytest.mark.parametrize("section,accepted", [
    ('<data_assimilation enabled="Yes" class_name="TemperatureSourceChanger" />', True),
    ('<data_assimilation enabled="Yes" />', False),
    ('<data_assimilation enabled="Yes" class_name="ObstacleChanger" load_data="Yes" file="x" />', False),
])
def test_data_assimilation_section_read_like_the_reference(tmp_path, section, accepted):
    """The data-assimilation section is parsed as in parse_assimilation_parameters
    (Settings.cpp:971-989): class_name is required when enabled, file and time
    when load_data is set; an accepted section leaves the scene as it is."""
    sc = scenes.plume_box(n=16, steps=0, n_level=2)
    text = scenes.to_xml(sc)
    assert '<data_assimilation enabled="No" />' in text
    xml = str(tmp_path / "da.xml")
    with open(xml, "w") as f:
        f.write(text.replace('<data_assimilation enabled="No" />', section))
    ref_rc = None
    if refdriver.available():
        import subprocess
        r = subprocess.run([refdriver.DRIVER, xml, "--steps", "0"], capture_output=True, text=True, timeout=300)
        ref_rc, ref_err = r.returncode, r.stderr
    if accepted:
        g = A.Geometry(xml)
        assert g.levels == 2
        if ref_rc is not None:
            assert ref_rc == 0, ref_err
    else:
        msg = ("Value class_name is for data_assimilation required." if "class_name" not in section
               else "Value time is for data_assimilation required.")
        with pytest.raises(A.ArtssError) as e:
            A.Geometry(xml)
        assert msg in str(e.value)
        if ref_rc is not None:
            assert ref_rc != 0 and msg in ref_err, ref_err


def test_obstacle_boundary_error_names_the_obstacle(tmp_path):
    """A missing boundary attribute inside an obstacle is reported under the
    reference's context, obstacles/obstacle/boundaries (<name>)/boundary
    (Settings.cpp:424-429)."""
    text = scenes.to_xml(scenes.room_with_door(n=16, steps=0, n_level=2))
    i = text.index('<obstacle name="')
    name = text[i + len('<obstacle name="'):text.index('"', i + len('<obstacle name="'))]
    j = text.index("<boundary ", i)
    k = text.index(' type="', j)
    end = text.index('"', k + len(' type="'))
    xml = str(tmp_path / "room.xml")
    with open(xml, "w") as f:
        f.write(text[:k] + text[end + 1:])
    msg = f"Value type is for obstacles/obstacle/boundaries ({name})/boundary required."
    with pytest.raises(A.ArtssError) as e:
        A.Geometry(xml)
    assert msg in str(e.value)
    if refdriver.available():
        import subprocess
        r = subprocess.run([refdriver.DRIVER, xml, "--steps", "0"], capture_output=True, text=True, timeout=300)
        assert r.returncode != 0 and msg in r.stderr, r.stderr


def test_non_numeric_initial_condition_parameter_rejected_like_the_reference(tmp_path):
    """An initial-condition parameter that is not a number counts as missing
    (get_required_real, Settings.cpp:81-88): the file is refused while it is
    read, with the reference's message."""
    sc = scenes.ns_scene("channel", n=16, steps=0)
    text = scenes.to_xml(sc)
    i = text.index("<u_lin>")
    j = text.index("</u_lin>", i)
    xml = str(tmp_path / "drift.xml")
    with open(xml, "w") as f:
        f.write(text[:i] + "<u_lin> fast " + text[j:])
    msg = "Value u_lin is for initial_conditions/Drift required."
    with pytest.raises(A.ArtssError) as e:
        A.Geometry(xml)
    assert msg in str(e.value)
    if refdriver.available():
        import subprocess
        r = subprocess.run([refdriver.DRIVER, xml, "--steps", "0"], capture_output=True, text=True, timeout=300)
        assert r.returncode != 0 and msg in r.stderr, r.stderr


def _gtest_scene(tmp_path, pd, cd, n, levels=1, boxes=()):
    """A scene with the domain parameters of a reference gtest (physical
    domain pd, computational domain cd, n inner cells)."""
    sc = scenes.Scene(solver="PressureSolver", nx=n[0], ny=n[1], nz=n[2], X=pd[0], Y=pd[1], Z=pd[2],
                      cd=None if cd == pd else cd, n_level=levels, ic="Zero", noise=False, steps=1,
                      boundaries=[("p", "front,back,bottom,top,left,right", "dirichlet", 0.0)],
                      obstacles=list(boxes), obstacle_bcs=[("p", "front,back,bottom,top,left,right", "neumann", 0.0)])
    return A.Geometry(scenes.write(sc, str(tmp_path / "gtest.xml")))


def _sizes(g, level):
    return {p: len(g.list("bnd_" + p, level)) for p in PATCHES}, len(g.list("domain", level)), len(g.list("inner", level))


_GT_PD = ((0.0, 5.0), (0.0, 10.0), (0.0, 15.0))


def test_domain_sizes_known_answers(tmp_path):
    """ARTSS gtests/domain/Domain.cpp:13-129: patch, domain-list and inner-list
    sizes without and with a computational domain, on level 1, and with a
    3x3x1 obstacle in the corner (cells 162-178)."""
    full = {"left": 12 * 22, "right": 12 * 22, "front": 7 * 22, "back": 7 * 22, "bottom": 7 * 12, "top": 7 * 12}
    assert _sizes(_gtest_scene(tmp_path, _GT_PD, _GT_PD, (5, 20, 10)), 0) == (full, 1848, 1000)
    g = _gtest_scene(tmp_path, ((0.0, 10.0), (0.0, 11.0), (0.0, 15.0)), _GT_PD, (5, 20, 10))
    assert _sizes(g, 0) == (full, 1848, 1000)
    g = _gtest_scene(tmp_path, _GT_PD, _GT_PD, (8, 12, 4))
    assert _sizes(g, 1) == ({"left": 32, "right": 32, "bottom": 24, "top": 24, "front": 48, "back": 48}, 192, 48)
    g = _gtest_scene(tmp_path, _GT_PD, _GT_PD, (5, 20, 10), boxes=[scenes.Box(0.0, 3.0, 0.0, 1.5, 0.0, 1.5, "corner")])
    np.testing.assert_array_equal(g.list("obst", 0), [162, 163, 164, 169, 170, 171, 176, 177, 178])
    assert _sizes(g, 0) == (full, 1839, 991)


def test_domain_indices_known_answers(tmp_path):
    """ARTSS gtests/domain/Domain.cpp:215-390: sorted lists, and the first and
    last index of the inner list and of every boundary patch, for a
    computational domain inside a physical one (z from -1.5) and without."""
    def ends(g, name):
        L = g.list(name, 0)
        assert np.all(np.diff(L) > 0), name
        return int(L[0]), int(L[-1])
    g = _gtest_scene(tmp_path, ((0.0, 7.0), (0.0, 15.0), (-1.5, 30.0)), _GT_PD, (5, 20, 10))
    assert ends(g, "inner") == (586, 3353)
    assert ends(g, "bnd_left") == (288, 3645) and ends(g, "bnd_right") == (294, 3651)
    assert ends(g, "bnd_bottom") == (288, 3462) and ends(g, "bnd_top") == (477, 3651)
    assert ends(g, "bnd_front") == (288, 483) and ends(g, "bnd_back") == (3456, 3651)
    g = _gtest_scene(tmp_path, _GT_PD, _GT_PD, (5, 20, 10))
    assert ends(g, "inner") == (162, 1685)
    assert ends(g, "bnd_left") == (0, 1841) and ends(g, "bnd_right") == (6, 1847)
    assert ends(g, "bnd_bottom") == (0, 1700) and ends(g, "bnd_top") == (147, 1847)
    assert ends(g, "bnd_front") == (0, 153) and ends(g, "bnd_back") == (1694, 1847)
    assert ends(g, "domain") == (0, 1847)


def test_domain_data_known_answers(tmp_path):
    """ARTSS gtests/domain/DomainData.cpp:23-310: cells per level (with and
    without ghost layer), spacings and the computational domain's index range,
    without and with a computational domain inside the physical one."""
    pd = ((0.0, 1.0), (-1.0, 1.2), (-0.3, 0.3))
    d = _gtest_scene(tmp_path, pd, pd, (10, 11, 12)).grid_desc()
    assert (d.Nx[0], d.Ny[0], d.Nz[0]) == (12, 13, 14) and d.Nx[0] * d.Ny[0] * d.Nz[0] == 2184
    assert (d.dx[0], d.dy[0], d.dz[0]) == pytest.approx((0.1, 0.2, 0.05), rel=1e-15)
    assert (d.i1[0], d.j1[0], d.k1[0], d.i2[0], d.j2[0], d.k2[0]) == (1, 1, 1, 10, 11, 12)

    pd = ((0.0, 1.2), (-1.0, -0.2), (-0.3, 0.3))
    d = _gtest_scene(tmp_path, pd, pd, (24, 4, 1), levels=2).grid_desc()
    assert [(d.i2[l] - d.i1[l] + 1, d.j2[l] - d.j1[l] + 1, d.k2[l] - d.k1[l] + 1) for l in range(3)] == \
        [(24, 4, 1), (12, 2, 1), (6, 1, 1)]
    assert [(d.Nx[l], d.Ny[l], d.Nz[l]) for l in range(3)] == [(26, 6, 3), (14, 4, 3), (8, 3, 3)]
    for l, h in enumerate([(0.05, 0.2, 0.6), (0.1, 0.4, 0.6), (0.2, 0.8, 0.6)]):
        assert (d.dx[l], d.dy[l], d.dz[l]) == pytest.approx(h, rel=1e-15), l

    cd = ((0.0, 1.0), (-1.0, 1.2), (-0.3, 0.3))
    d = _gtest_scene(tmp_path, ((0.0, 1.0), (-1.2, 1.4), (-0.4, 0.4)), cd, (10, 11, 12), levels=2).grid_desc()
    assert (d.i1[0], d.j1[0], d.k1[0], d.i2[0], d.j2[0], d.k2[0]) == (1, 2, 3, 10, 12, 14)
