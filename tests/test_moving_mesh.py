"""Key-framed moving-mesh obstacle (src/physics/MovingMesh.cpp:28-264, JSON
reader src/scene_building.cpp:248-276).

The obstacle holds key frames f = 0..F-1 reached at times f * interval.  Its
clock starts at 0 with key frames 0 and 1 around it; each step, after the
solve, the clock advances by the time step, the pair of key frames moves on by
at most one, and while the clock lies between the pair the current mesh is
their linear interpolation.  A contact on it moves with the barycentric point
of the two key frames: speed = (next - previous) / interval while the clock is
between them, zero otherwise.  Expected values are derived here from those
rules, not from the oracle."""
import numpy as np
import pytest

from climatenet_b200 import abi, native, scenes
from oracle import oracle as orc


def expected_clocks(n_steps, dt, interval, n_frames):
    """Per step: (index of the next key frame, in movement) at detection time,
    restating MovingMesh::update / isInMovement (MovingMesh.cpp:43-57, 253-257)."""
    clock, nxt, out = 0.0, 1, []
    for _ in range(n_steps):
        moving = (nxt - 1) * interval <= clock <= nxt * interval
        out.append((nxt, moving))
        clock += dt
        if nxt * interval < clock and nxt + 1 < n_frames:
            nxt += 1
    return out


def floor_frames(heights, shift=(0.0, 0.0), side=2.0):
    """A square floor of two triangles, normal +z, one key frame per height
    (and per horizontal shift, applied proportionally to the frame index)."""
    base = np.array([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], dtype=float) * [side / 2, side / 2, 1]
    frames = []
    for f, h in enumerate(heights):
        fr = base.copy()
        fr[:, 2] = h
        fr[:, 0] += shift[0] * f
        fr[:, 1] += shift[1] * f
        frames.append(fr)
    return np.array(frames), np.array([[0, 1, 2], [0, 2, 3]], dtype=np.int32)


def triangle_on_floor(heights, interval, tol=0.05, mu=0.5, shift=(0.0, 0.0)):
    pos = np.array([[0.0, 0.0, 0.001], [0.1, 0.0, 0.001], [0.0, 0.1, 0.001]])
    s = scenes.Scene(friction=((mu,),))
    s.add_mesh(pos, np.array([[0, 1, 2]]), area_density=2.0, bending=1e-3, stretching=100.0)
    frames, tris = floor_frames(heights, shift)
    s.add_moving_mesh(frames, tris, interval, tol)
    return s


def test_rising_floor_lifts_a_resting_triangle():
    # floor rising at 0.1 m/s: a resting vertex in contact sticks to it
    dt, interval, rate = 1e-3, 0.01, 0.1
    heights = [rate * interval * f for f in range(6)]
    o = orc.Oracle(triangle_on_floor(heights, interval), abi.params(time_step=dt, iterations=20))
    o.step(1)
    c = o.contacts()
    assert list(c["vertex"]) == [0, 1, 2]
    assert np.array_equal(c["normal"], [[0.0, 0.0, 1.0]] * 3)
    assert np.allclose(c["speed"], [[0.0, 0.0, rate]] * 3, rtol=1e-12, atol=0)
    _, v = o.state()
    assert np.allclose(v, [[0.0, 0.0, rate]] * 3, rtol=0, atol=1e-10)


def test_sliding_floor_drags_with_friction_limit():
    # floor moving sideways at 1 m/s with mu = 0.5: slip, the vertex gains
    # mu g dt of tangential speed in one step
    dt, interval, g, mu = 1e-3, 0.01, 9.81, 0.5
    heights = [0.0] * 4
    o = orc.Oracle(triangle_on_floor(heights, interval, mu=mu, shift=(interval * 1.0, 0.0)),
                   abi.params(time_step=dt, iterations=20))
    o.step(1)
    c = o.contacts()
    assert np.allclose(c["speed"], [[1.0, 0.0, 0.0]] * 3, rtol=1e-12, atol=1e-15)
    _, v = o.state()
    assert np.allclose(v[:, 0], mu * g * dt, rtol=1e-9)
    assert np.abs(v[:, 1:]).max() < 1e-10


@pytest.mark.parametrize("dt,interval", [(1e-3, 2.5e-3), (2.5e-3, 1e-3), (1e-3, 1e-3)])
def test_clock_and_key_frame_advance(dt, interval):
    # distinct speed per key-frame pair: pair (f-1, f) moves the floor up by
    # f * 1e-4, so the speed names the pair; no gravity, a generous tolerance
    n_frames, steps = 5, 14
    heights = np.cumsum([0.0] + [f * 1e-4 for f in range(1, n_frames)])
    s = triangle_on_floor(heights, interval, tol=0.5)
    o = orc.Oracle(s, abi.params(time_step=dt, iterations=3, gravity=(0, 0, 0)))
    for k, (nxt, moving) in enumerate(expected_clocks(steps, dt, interval, n_frames)):
        o.step(1)
        c = o.contacts()
        assert c["vertex"].shape[0] == 3
        want = (nxt * 1e-4) / interval if moving else 0.0
        assert np.allclose(c["speed"][:, 2], want, rtol=1e-9, atol=0), (k, nxt, moving, c["speed"][:, 2])
        assert np.abs(c["speed"][:, :2]).max() == 0.0


def test_interpolated_mesh_sets_the_contact_set():
    # the floor drops away faster than gravity once the clock passes 5 ms:
    # the vertices leave the tolerance band and the contact set empties
    dt, interval = 1e-3, 5e-3
    heights = [0.0, 0.0, -1.0]
    o = orc.Oracle(triangle_on_floor(heights, interval, tol=0.01), abi.params(time_step=dt, iterations=5))
    seen = []
    for _ in range(8):
        seen.append(o.step(1).n_contacts)
    assert seen[0] == 3 and seen[-1] == 0


def write_frames(tmp_path, heights, prefix="floor_", suffix=3):
    for f, h in enumerate(heights):
        name = f"{prefix}{f:0{suffix}d}.obj" if suffix else f"{prefix}{f}.obj"
        (tmp_path / name).write_text(
            f"v -1 -1 {h}\nv 1 -1 {h}\nv 1 1 {h}\nv -1 1 {h}\nf 1 2 3\nf 1 3 4\n")


def moving_scene_json(tmp_path, extra=""):
    (tmp_path / "cloth.obj").write_text("v 0 0 0.001\nv 0.1 0 0.001\nv 0 0.1 0.001\nf 1 2 3\n")
    js = tmp_path / "scene.json"
    js.write_text("""{
 "Parameters": {"Frame number": 1, "LocalGlobal": 5, "Timestep": 1e-3, "Type": "friction",
   "Steps per frame": 1, "Self-collision": false, "Self-collision tolerance": 1.0e-2,
   "Gravity": [0.0, 0.0, -9.81]},
 "Friction coefficients": [[0.25]],
 "Meshes": [{"Obj filename": "cloth.obj", "Area Density": 1.0, "Bending": 1e-3,
             "Stretching": 1e2, "Material Identifier": 0}],
 "Obstacles": [{"Type": "Moving Mesh", "Obj Prefix": "floor_", "Suffix Size": 3,
                "Number Frame": 3, "Material Identifier": 0, "Time Between Frame": 0.01,
                "Collision tolerance": 0.02 %s}]
}""" % extra)
    return js


def test_moving_mesh_json_reader(tmp_path):
    write_frames(tmp_path, [0.0, 0.1, 0.3])
    sc = native.getSceneFromJSONFileName(str(moving_scene_json(tmp_path)))
    d = sc.desc()
    ob = d.obstacles[0]
    assert ob.type == abi.PDF_OBSTACLE_MOVING_MESH
    assert (ob.n_frames, ob.n_vertices, ob.n_triangles) == (3, 4, 2)
    assert ob.frame_interval == 0.01 and ob.threshold == 0.02
    z = [ob.vertices[3 * (f * 4 + i) + 2] for f in range(3) for i in range(4)]
    # OBJ coordinates are rounded through float, like the reference's reader
    want = [float(np.float32(h)) for h in (0.0, 0.1, 0.3) for _ in range(4)]
    assert z == want
    assert [ob.triangles[k] for k in range(6)] == [0, 1, 2, 0, 2, 3]


def test_moving_mesh_json_missing_frame(tmp_path):
    write_frames(tmp_path, [0.0, 0.1])  # the scene asks for three
    with pytest.raises(native.PdfError):
        native.getSceneFromJSONFileName(str(moving_scene_json(tmp_path)))


def test_moving_mesh_json_unpadded_names(tmp_path):
    write_frames(tmp_path, [0.0, 0.1, 0.3], suffix=0)
    js = moving_scene_json(tmp_path)
    js.write_text(js.read_text().replace('"Suffix Size": 3', '"Suffix Size": 0'))
    d = native.getSceneFromJSONFileName(str(js)).desc()
    assert d.obstacles[0].n_frames == 3


def cloth_on_moving_floor(n=24):
    """A cloth resting on a floor that rises, pauses, then slides sideways."""
    pos, tri = scenes.grid_mesh(n, 1.0, z=0.002)
    s = scenes.Scene(friction=((0.4,),))
    s.add_mesh(pos, tri, area_density=0.1, bending=1e-2, stretching=1e3)
    interval = 4e-3
    heights = [0.0, 0.0004, 0.0008, 0.0008, 0.0008, 0.0006]
    frames, tris = floor_frames(heights)
    frames[4:, :, 0] += 0.003
    frames[5:, :, 1] -= 0.002
    s.add_moving_mesh(frames, tris, interval, 0.01)
    return s


@pytest.mark.gpu
def test_moving_mesh_steps_match_oracle():
    s = cloth_on_moving_floor()
    p = abi.params(time_step=2e-3, iterations=20)
    g = native.Simulation(s, p)
    o = orc.Oracle(s, p)
    moved = False
    for _ in range(14):
        rg = g.step(1)
        ro = o.step(1)
        assert rg.n_contacts == ro.n_contacts
        cg, co = g.contacts(), o.contacts()
        assert np.array_equal(cg["vertex"], co["vertex"])
        assert np.array_equal(cg["normal"], co["normal"])
        # the speed is (next - previous key-frame point) / interval: positions
        # that agree to rounding give barycentric weights that agree to
        # rounding, and the frame difference amplifies that by |p| / interval
        assert np.allclose(cg["speed"], co["speed"], rtol=0, atol=1e-12)
        moved |= bool(np.abs(co["speed"]).max() > 0)
    assert moved and rg.n_contacts > 0
    qg, vg = g.state()
    qo, vo = o.state()
    assert np.abs(qg - qo).max() / np.abs(qo).max() < 1e-6
    # the cloth ends at rest on the floor: velocities near zero, compared
    # against the run's velocity scale (the floor moved at up to 0.75 m/s)
    assert np.abs(vg - vo).max() <= 1e-5 * max(np.abs(vo).max(), 1e-3)
