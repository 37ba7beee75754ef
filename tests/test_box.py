"""Axis-aligned box obstacle (src/physics/StaticAxisAlignedBox.cpp:41-201,
JSON reader src/scene_building.cpp:205-211).

A vertex touches the box when it lies inside it (no margin); the contact side
is the first of TOP (+y), BOTTOM (-y), LEFT (-x), RIGHT (+x), FRONT (+z),
BACK (-z) at the smallest distance, and the normal is that side's axis vector.
Expected values are derived here from those rules, not from the oracle."""
import numpy as np
import pytest

from climatenet_b200 import abi, native, scenes
from oracle import oracle as orc


def box_side(x, corner, size):
    """The reference's nearest side for a point inside the box: (axis, sign, distance)."""
    rel = (x - corner) - 0.5 * size
    sides = [(1, 1.0), (1, -1.0), (0, -1.0), (0, 1.0), (2, 1.0), (2, -1.0)]
    best = None
    for ax, sg in sides:
        d = abs(rel[ax] - sg * 0.5 * size[ax])
        if best is None or d < best[2]:
            best = (ax, sg, d)
    return best


def inside(x, corner, size):
    rel = (x - corner) - 0.5 * size
    return bool(np.all(np.abs(rel) <= size / 2))


def triangle_on_box(v0=(0.0, 0.0, 0.0), mu=0.3, corner=(-1.0, -1.0, -1.0), size=(2.0, 2.0, 1.002)):
    pos = np.array([[0.0, 0.0, 0.0], [0.1, 0.0, 0.0], [0.0, 0.1, 0.0]])
    s = scenes.Scene(friction=((mu,),))
    s.add_mesh(pos, np.array([[0, 1, 2]]), area_density=2.0, bending=1e-3, stretching=100.0)
    s.add_box(corner, size)
    s.vel = np.tile(np.asarray(v0, dtype=float), (3, 1))
    return s


def test_box_top_face_contact_normal_and_stick():
    # the cloth lies 2 mm below the +z face: FRONT side, normal +z, gap -2 mm
    dt, g = 1e-3, 9.81
    o = orc.Oracle(triangle_on_box(), abi.params(time_step=dt, iterations=10))
    o.step(1)
    c = o.contacts()
    assert list(c["vertex"]) == [0, 1, 2]
    assert np.allclose(c["normal"], [[0.0, 0.0, 1.0]] * 3, rtol=0, atol=0)
    q, v = o.state()
    assert np.abs(v).max() < 1e-12
    m = o.masses()
    assert np.allclose(c["force"][:, 0], m * dt * g, rtol=1e-10)


def test_box_slip_on_top_face():
    dt, g, mu, u = 1e-3, 9.81, 0.3, 0.5
    o = orc.Oracle(triangle_on_box(v0=(u, 0, 0), mu=mu), abi.params(time_step=dt, iterations=10))
    o.step(1)
    _, v = o.state()
    assert np.allclose(v[:, 0], u - mu * g * dt, rtol=0, atol=1e-12)
    assert np.abs(v[:, 1:]).max() < 1e-12


def test_box_has_no_margin_and_picks_first_nearest_side():
    corner, size = np.array([0.0, 0.0, 0.0]), np.array([1.0, 1.0, 1.0])
    pts = np.array([
        [0.5, 0.5, 1.0 + 1e-9],   # just above the box: no contact
        [0.5, 0.99, 0.5],         # nearest to +y (TOP)
        [0.02, 0.5, 0.5],         # nearest to -x (LEFT)
        [0.5, 0.5, 0.5],          # centre: all six sides tie -> TOP, the first
        [0.97, 0.5, 0.04],        # -z (BACK) at 0.04 vs +x (RIGHT) at 0.03 -> RIGHT
        [0.2, 0.3, 0.995],        # +z (FRONT)
    ])
    tri = np.array([[0, 1, 2], [3, 4, 5]])
    s = scenes.Scene(friction=((0.3,),))
    s.add_mesh(pts, tri, area_density=1.0, bending=1e-3, stretching=1.0)
    s.add_box(corner, size)
    o = orc.Oracle(s, abi.params(time_step=1e-6, iterations=1, gravity=(0, 0, 0)))
    o.step(1)
    c = o.contacts()
    # detection runs on the positions at the start of the step
    expect = [i for i in range(len(pts)) if inside(pts[i], corner, size)]
    assert list(c["vertex"]) == expect == [1, 2, 3, 4, 5]
    for k, i in enumerate(expect):
        ax, sg, _ = box_side(pts[i], corner, size)
        n = np.zeros(3)
        n[ax] = sg
        assert np.array_equal(c["normal"][k], n), (i, c["normal"][k], n)
    assert np.array_equal(c["normal"][expect.index(3)], [0.0, 1.0, 0.0])
    assert np.array_equal(c["normal"][expect.index(4)], [1.0, 0.0, 0.0])


def test_box_json_reader(tmp_path):
    obj = tmp_path / "cloth.obj"
    obj.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3\nf 1 3 4\n")
    js = tmp_path / "scene.json"
    js.write_text("""{
 "Parameters": {"Frame number": 1, "LocalGlobal": 5, "Timestep": 1e-3, "Type": "friction",
   "Steps per frame": 1, "Self-collision": false, "Self-collision tolerance": 1.0e-2,
   "Gravity": [0.0, 0.0, -9.81]},
 "Friction coefficients": [[0.25]],
 "Meshes": [{"Obj filename": "cloth.obj", "Area Density": 1.0, "Bending": 1e-3,
             "Stretching": 1e2, "Material Identifier": 0}],
 "Obstacles": [{"Type": "Axis Aligned Box", "Position": [-1.0, -2.0, -3.0],
                "Material Identifier": 0, "Size": [2.0, 4.0, 3.001]}]
}""")
    sc = native.getSceneFromJSONFileName(str(js))
    d = sc.desc()
    assert d.n_obstacles == 1
    ob = d.obstacles[0]
    assert ob.type == abi.PDF_OBSTACLE_BOX
    assert list(ob.center) == [-1.0, -2.0, -3.0]
    assert list(ob.size) == [2.0, 4.0, 3.001]


def test_box_json_requires_size(tmp_path):
    obj = tmp_path / "cloth.obj"
    obj.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nf 1 2 3\n")
    js = tmp_path / "scene.json"
    js.write_text("""{
 "Parameters": {"Frame number": 1, "LocalGlobal": 5, "Timestep": 1e-3, "Type": "friction",
   "Steps per frame": 1, "Self-collision": false, "Self-collision tolerance": 1.0e-2,
   "Gravity": [0.0, 0.0, -9.81]},
 "Friction coefficients": [[0.25]],
 "Meshes": [{"Obj filename": "cloth.obj", "Area Density": 1.0, "Bending": 1e-3,
             "Stretching": 1e2, "Material Identifier": 0}],
 "Obstacles": [{"Type": "Axis Aligned Box", "Position": [0.0, 0.0, 0.0],
                "Material Identifier": 0}]
}""")
    with pytest.raises(native.PdfError):
        native.getSceneFromJSONFileName(str(js))


def cloth_on_box(n=24, mu=0.4):
    """A cloth dropped across the +z face of a box narrower than the cloth: the
    middle rests on the face, the overhang drapes past the edges."""
    pos, tri = scenes.grid_mesh(n, 1.0, z=0.001)
    s = scenes.Scene(friction=((mu,),))
    s.add_mesh(pos, tri, area_density=0.1, bending=1e-2, stretching=1e3)
    s.add_box((-0.3, -0.3, -0.5), (0.6, 0.6, 0.5 + 0.003))
    return s


@pytest.mark.gpu
def test_box_steps_match_oracle():
    s = cloth_on_box()
    p = abi.params(time_step=2e-3, iterations=20)
    g = native.Simulation(s, p)
    o = orc.Oracle(s, p)
    for _ in range(8):
        rg = g.step(1)
        ro = o.step(1)
        assert rg.n_contacts == ro.n_contacts
    assert rg.n_contacts > 0
    cg, co = g.contacts(), o.contacts()
    assert np.array_equal(cg["vertex"], co["vertex"])
    assert np.array_equal(cg["normal"], co["normal"])
    qg, vg = g.state()
    qo, vo = o.state()
    rel = np.abs(qg - qo).max() / np.abs(qo).max()
    assert rel < 1e-6, rel
    assert np.abs(vg - vo).max() <= 1e-5 * max(np.abs(vo).max(), 1e-12)
