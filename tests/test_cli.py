"""The command-line driver (climatenet_b200/_build/pdf_run, src/main.cpp:40-124
equivalent), the "log" reader (src/log_building.cpp:28-129), frame capture,
per-sample statistics (exportStats) and the Alart-Curnier trace
(PRINT_ALART_CURNIER_ERROR, SFE:720-752)."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

from climatenet_b200 import abi, native, scenes
from conftest import ROOT, incline_closed_form

PDF_RUN = os.path.join(ROOT, "climatenet_b200", "_build", "pdf_run")


def write_obj(path, v, t):
    with open(path, "w") as f:
        for x in v:
            f.write("v %r %r %r\n" % tuple(float(c) for c in x))
        for tri in t:
            f.write("f %d %d %d\n" % tuple(int(k) + 1 for k in tri))


def grid_scene_json(tmp_path, frames=3, spf=2, log=None, sphere=True, n=6):
    pos, tri = scenes.grid_mesh(n, 1.0, z=-0.2455)
    write_obj(tmp_path / "cloth.obj", pos, tri)
    doc = {
        "Parameters": {"Frame number": frames, "LocalGlobal": 8, "Timestep": 5e-3, "Type": "friction",
                       "Steps per frame": spf, "Self-collision": False, "Self-collision tolerance": 1e-2,
                       "Gravity": [0.0, 0.0, -9.81]},
        "Friction coefficients": [[0.3]],
        "Meshes": [{"Obj filename": "cloth.obj", "Area Density": 0.1, "Bending": 1e-2, "Stretching": 1e3,
                    "Material Identifier": 0}],
        "Obstacles": ([{"Type": "Sphere", "Position": [0.0, 0.0, -0.5], "Radius": 0.25,
                        "Material Identifier": 0}] if sphere else []),
    }
    if log is not None:
        doc["log"] = log
    js = tmp_path / "scene.json"
    js.write_text(json.dumps(doc))
    return js


# ---------------------------------------------------------------- CPU


def test_log_reader(tmp_path):
    js = grid_scene_json(tmp_path, log=[{"type": "position", "vertices": [0, 2]},
                                        {"type": "velocity", "vertices": [1]}])
    assert native.load_log(str(js)) == [("position", [0, 2]), ("velocity", [1])]
    assert native.load_log(str(grid_scene_json(tmp_path))) == []


@pytest.mark.parametrize("entry,needle", [
    ({"type": "speed", "vertices": [0]}, 'Log type "speed" is unsupported'),
    ({"type": "position"}, "vertices"),
    ({"type": "position", "vertices": [-1]}, "vertices"),
    ({"type": "position", "vertices": [0.5]}, "vertices"),
])
def test_log_reader_errors(tmp_path, entry, needle):
    js = grid_scene_json(tmp_path, log=[entry])
    with pytest.raises(native.PdfError) as e:
        native.load_log(str(js))
    assert needle in str(e.value)


def test_cli_usage_and_output_directories(tmp_path):
    r = subprocess.run([PDF_RUN], capture_output=True, text=True)
    assert r.returncode != 0 and "1 argument expected" in r.stderr
    js = grid_scene_json(tmp_path)
    (tmp_path / "data0").mkdir()
    # without a GPU the run stops at pdf_create, after preparing data1
    r = subprocess.run([PDF_RUN, str(js)], capture_output=True, text=True, cwd=tmp_path)
    if r.returncode == 0:
        pytest.skip("a GPU is present: the full run is covered by the GPU tests")
    assert "simulation" in r.stderr
    assert (tmp_path / "data1" / "scene.json").read_text() == js.read_text()
    assert (tmp_path / "data1" / "output").is_dir()


# ---------------------------------------------------------------- GPU

STATS_SECTIONS = ["LHS computation time (µs)", "Cholesky computation time (µs)", "Iteration time (µs)",
                  "Collision detection time (µs)", "Number of self collisions", "Solver time (µs)",
                  "Full RHS computation time (µs)", "Step time (µs)", "RHS base computation time (µs)",
                  "RHS friction overhead (µs)"]
STATS_SELF = ["LHS computation time (µs)", "Cholesky computation time (µs)", "Iteration time (µs)",
              "Collision detection time (µs)", "Number of collisions", "Self collision detection time (µs)",
              "Number of self collisions", "Solver time (µs)", "Full RHS computation time (µs)",
              "Step time (µs)", "RHS base computation time (µs)", "RHS friction overhead (µs)",
              "Self collision time (µs)", "Self collision ordering time (µs)"]


def parse_stats(text):
    """{section: {"Number": n, "Min value": x, ...} or {"Value": x} or {}}, in file order."""
    out = {}
    for block in text.split("-------------------"):
        lines = [ln for ln in block.strip("\n").split("\n") if ln.strip()]
        if not lines:
            continue
        vals = {}
        for ln in lines[1:]:
            if "(No data)" in ln:
                continue
            k, v = ln.split(":")
            vals[k.strip()] = float(v)
        out[lines[0]] = vals
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("self_collision", [False, True])
def test_stats_sections_and_sample_counts(tmp_path, self_collision):
    s = scenes.cloth_on_sphere(n=16, side=1.0, z=-0.2455, mu=0.3, layers=2 if self_collision else 1,
                               sphere_center=(0, 0, -0.5), sphere_radius=0.25)
    K, steps = 6, 5
    p = abi.params(time_step=5e-3, iterations=K, self_collision=self_collision, self_tol=1e-2)
    g = native.Simulation(s, p)
    contacts = []
    for _ in range(steps):
        r = g.step(1)
        contacts.append((r.n_contacts, r.n_self_contacts))
    g.export_stats(str(tmp_path / "stats.txt"))
    st = parse_stats((tmp_path / "stats.txt").read_text())
    assert list(st) == (STATS_SELF if self_collision else STATS_SECTIONS)
    assert st["LHS computation time (µs)"]["Value"] > 0
    assert st["Cholesky computation time (µs)"]["Value"] > 0
    for name in ["Iteration time (µs)", "Solver time (µs)", "Full RHS computation time (µs)",
                 "RHS base computation time (µs)"]:
        assert st[name]["Number"] == steps * K, name
    assert st["RHS friction overhead (µs)"]["Number"] == K * sum(1 for c, s_ in contacts if c + s_ > 0)
    for name in ["Collision detection time (µs)", "Step time (µs)"]:
        assert st[name]["Number"] == steps, name
    for name, v in st.items():
        if "Number" in v:
            assert v["Min value"] <= v["Mean value"] <= v["Max value"], name
    assert 0 < st["Solver time (µs)"]["Mean value"] < st["Iteration time (µs)"]["Mean value"]
    assert st["Iteration time (µs)"]["Mean value"] * K <= st["Step time (µs)"]["Max value"] * 1.05
    if self_collision:
        ns = [s_ for _, s_ in contacts if s_ > 0]
        assert ns, "the two layers should touch"
        assert st["Number of self collisions"]["Number"] == len(ns)
        assert st["Number of self collisions"]["Max value"] == max(ns)
        assert st["Self collision time (µs)"]["Number"] == K * len(ns)
    else:
        assert st["Number of self collisions"] == {}


@pytest.mark.gpu
def test_frame_capture_overlaps_next_steps():
    s = scenes.cloth_on_sphere(n=20, side=1.0, z=-0.2455, mu=0.3, sphere_center=(0, 0, -0.5),
                               sphere_radius=0.25)
    g = native.Simulation(s, abi.params(time_step=5e-3, iterations=10))
    g.step(2)
    q_ref, _ = g.state()
    g.frame_capture(0)
    g.step(3)  # the copy must have read q before these steps overwrote it
    q1, _ = g.state()
    g.frame_capture(1)
    assert np.array_equal(g.frame_wait(0), q_ref)
    assert np.array_equal(g.frame_wait(1), q1)
    assert not np.array_equal(q_ref, q1)


@pytest.mark.gpu
def test_vertices_gather_and_ac_trace():
    s = scenes.cloth_on_sphere(n=16, side=1.0, z=-0.2455, mu=0.3, layers=2, sphere_center=(0, 0, -0.5),
                               sphere_radius=0.25)
    K = 7
    g = native.Simulation(s, abi.params(time_step=5e-3, iterations=K, self_collision=True, self_tol=1e-2,
                                        trace_alart_curnier=1))
    for _ in range(4):
        r = g.step(1)
    q, v = g.state()
    idx = np.array([0, 5, 17, len(q) - 1])
    qg, vg = g.vertices(idx)
    assert np.array_equal(qg, q[idx]) and np.array_equal(vg, v[idx])
    tr, nc = g.alart_curnier_trace()
    assert tr.shape == (K, r.n_contacts + r.n_self_contacts, 2)
    assert nc == r.n_contacts > 0 and r.n_self_contacts > 0
    # the last iteration's norms are the contacts' AC norms: |AC|^2 = t^2 + n^2
    ac = np.concatenate([g.contacts()["ac"], g.self_contacts()["ac"]])
    assert np.allclose(np.hypot(tr[-1, :, 0], tr[-1, :, 1]), ac, rtol=1e-12, atol=1e-300)
    # and their mean is the step's residual
    assert abs(np.hypot(tr[-1, :, 0], tr[-1, :, 1]).mean() - r.residual) <= 1e-12 * max(r.residual, 1e-300)


def read_log_blocks(text):
    """Velocity / position blocks of the log callbacks, parsed the way the
    reference's post-processing reads them (a "<Kind> <n>" line, then per
    vertex a "v<i>" line and three coordinate lines)."""
    lines = text.split("\n")
    out = {"Velocity": [], "Position": []}
    k = 0
    while k < len(lines):
        ln = lines[k]
        if ln.startswith("Velocity") or ln.startswith("Position"):
            kind, n = ln.split()
            pts = []
            k += 1
            for _ in range(int(n)):
                assert lines[k].startswith("v")
                pts.append([float(lines[k + 1]), float(lines[k + 2]), float(lines[k + 3])])
                k += 4
            out[kind].append(pts)
        else:
            k += 1
    return out


@pytest.mark.gpu
def test_cli_grid_run_frames_logs_trace(tmp_path):
    frames, spf = 3, 2
    # odd grid: the centre vertex starts within the sphere's 1 cm margin
    js = grid_scene_json(tmp_path, frames=frames, spf=spf, n=7,
                         log=[{"type": "position", "vertices": [0, 7]}, {"type": "velocity", "vertices": [3]}])
    r = subprocess.run([PDF_RUN, str(js), "--print-alart-curnier"], capture_output=True, text=True, cwd=tmp_path,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    out = r.stdout
    steps = frames * spf
    assert [int(x) for x in re.findall(r"^Time Step: (\d+)$", out, re.M)] == list(range(steps))
    assert out.count("Saving Mesh") == frames
    # progress: at most one 5 % milestone per step, as in the reference's loop
    todo, want = list(range(5, 101, 5)), []
    for i in range(steps):
        if todo and i >= todo[0] * (steps - 1) / 100.0:
            want.append("%d%% done" % todo.pop(0))
    assert r.stderr.strip().split("\n") == want
    # same scene through the Python mirror: frames are steps 0, spf, 2 spf
    sc = native.getSceneFromJSONFileName(str(js))
    p, _, _ = native.load_params(str(js))
    g = native.Simulation(sc, p)
    states = []
    for i in range(steps):
        g.step(1)
        states.append(g.state())
    for f in range(frames):
        obj = (tmp_path / "data0" / "output" / ("out_%06d.obj" % f)).read_text().split("\n")
        vs = np.array([[float(x) for x in ln.split()[1:]] for ln in obj if ln.startswith("v ")])
        fs = [ln for ln in obj if ln.startswith("f ")]
        assert len(fs) == 2 * 6 * 6 and fs[0] == "f 1 2 9"
        # default stream formatting keeps 6 significant digits
        assert np.allclose(vs, states[f * spf][0], rtol=1e-5, atol=1e-6)
    logs = read_log_blocks(out)
    assert len(logs["Position"]) == steps and len(logs["Velocity"]) == steps
    for i in range(steps):
        q, v = states[i]
        assert np.allclose(logs["Position"][i], q[[0, 7]], rtol=1e-5, atol=1e-6)
        assert np.allclose(logs["Velocity"][i], v[[3]], rtol=1e-5, atol=1e-6)
    # every iteration of every step prints one tangential and one normal line
    tang = [ln for ln in out.split("\n") if ln.startswith("TangentialAlartCurnier ")]
    norm = [ln for ln in out.split("\n") if ln.startswith("NormalAlartCurnier ")]
    assert len(tang) == len(norm) == steps * p.local_global_iterations
    vals = [list(map(float, ln.split(" ")[1:-1])) for ln in norm]
    assert all(len(x) > 0 and min(x) >= 0 for x in vals)
    assert not any(ln.startswith("SelfTangentialAlartCurnier") for ln in out.split("\n"))
    st = parse_stats((tmp_path / "data0" / "stats.txt").read_text())
    assert st["Step time (µs)"]["Number"] == steps
    assert (tmp_path / "data0" / "scene.json").exists()


@pytest.mark.gpu
def test_cli_analytic_incline_known_answer(tmp_path):
    """The reference's Figure-5 scene with its "log" section, run through the
    driver; the logged velocities and heights follow the closed form."""
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "analytic_incline.json")))
    write_obj(tmp_path / "cloth.obj", g["cloth_vertices"], g["cloth_triangles"])
    write_obj(tmp_path / "support.obj", g["support_vertices"], g["support_triangles"])
    doc = {"Parameters": g["parameters"], "Friction coefficients": g["friction"],
           "Meshes": [dict(g["mesh"], **{"Obj filename": "cloth.obj"})],
           "Obstacles": [dict(g["obstacle"], **{"Path": "support.obj"})],
           "log": [{"type": "velocity", "vertices": [0, 1, 2, 3]},
                   {"type": "position", "vertices": [0, 1, 2, 3]}]}
    js = tmp_path / "analytic.json"
    js.write_text(json.dumps(doc, indent=1))
    r = subprocess.run([PDF_RUN, str(js)], capture_output=True, text=True, cwd=tmp_path, timeout=600)
    assert r.returncode == 0, r.stderr
    logs = read_log_blocks(r.stdout)
    P = g["parameters"]
    steps = P["Frame number"] * P["Steps per frame"]
    assert len(logs["Velocity"]) == steps
    dt = P["Timestep"]
    for i in range(steps):
        speed, height = incline_closed_form((i + 1) * dt)
        vel = np.array(logs["Velocity"][i])
        pos = np.array(logs["Position"][i])
        # printed with 6 significant digits; the scheme itself matches the
        # closed-form speed to round-off and the height to first order in dt
        assert abs(np.linalg.norm(vel.mean(0)) - speed) < 1e-5 * max(speed, 0.1), (i, speed)
        assert abs(pos[:, 2].mean() - height) < 2e-3 + 1e-5, (i, height)
