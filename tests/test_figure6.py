"""Alart-Curnier convergence trace on the GPU against the CPU oracle, on an
analogue of the reference's Figure-6 scene.

The reference demonstrates the convergence of its contact iteration with
replicability/scenes/Square1/iterations_300.json (figure_6.sh): a drape with
area density 3, stretching 2e2, bending 5e-4, falling on a sphere of radius
0.5 centred at (0, 0, -0.52) that turns about z by 0.1 rad per key frame
(200 key frames, 35 ms apart, collision tolerance 1.5 cm), above a plane at
z = -1; mu 0.1, dt 5e-3, 300 PD iterations per step.  Its key frames are
rigid rotations of one UV sphere, so they are generated here; the drape is a
regular grid of the same extent (the reference's drape mesh is not shipped
with this repository).  The oracle's run of the reference's own scene is in
tests/golden/figure6_oracle_ac.json (tests/golden/make_figure6.py).

The GPU and the oracle step side by side (the GPU state is reset to the
oracle's after every step, so that both detect contacts on identical
positions); at steps 50 and 100 every contact's per-iteration tangential and
normal AC norms, printed by PRINT_ALART_CURNIER_ERROR builds (SFE:720-752),
must agree to 1e-6 relative.
"""
import json
import os

import numpy as np
import pytest

from climatenet_b200 import abi, native, scenes
from oracle.oracle import Oracle

HERE = os.path.dirname(os.path.abspath(__file__))


def uv_sphere(radius, center, segments, rings):
    """Vertices (poles + rings x segments) and outward triangles of a UV sphere."""
    cz = np.asarray(center, dtype=float)
    V = [cz + [0, 0, radius]]
    for r in range(1, rings):
        th = np.pi * r / rings
        for s in range(segments):
            ph = 2 * np.pi * s / segments
            V.append(cz + radius * np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)]))
    V.append(cz + [0, 0, -radius])
    V = np.array(V)
    south = len(V) - 1

    def idx(r, s):
        return 1 + (r - 1) * segments + (s % segments)

    T = []
    for s in range(segments):
        T.append([0, idx(1, s), idx(1, s + 1)])
        T.append([south, idx(rings - 1, s + 1), idx(rings - 1, s)])
    for r in range(1, rings - 1):
        for s in range(segments):
            a, b, c, d = idx(r, s), idx(r, s + 1), idx(r + 1, s), idx(r + 1, s + 1)
            T.append([a, c, d])
            T.append([a, d, b])
    return V, np.array(T, dtype=np.int32)


def figure6_analogue(n=40, frames=200):
    s = scenes.Scene(friction=((0.1,),))
    p, t = scenes.grid_mesh(n, 2.4, z=0.09314)
    s.add_mesh(p, t, area_density=3.0, bending=5e-4, stretching=2e2)
    center = np.array([0.0, 0.0, -0.52])
    V0, T = uv_sphere(0.5, center, 24, 24)
    keys = []
    for k in range(frames):
        a = 0.1 * k
        R = np.array([[np.cos(a), -np.sin(a), 0.0], [np.sin(a), np.cos(a), 0.0], [0.0, 0.0, 1.0]])
        keys.append((V0 - center) @ R.T + center)
    s.add_moving_mesh(np.array(keys), T, 35e-3, 1.5e-2)
    s.add_plane((0.0, 0.0, -1.0), (0.0, 0.0, 1.0))
    return s


def test_reference_scene_fixture_shows_convergence():
    """The oracle's run of the reference's own Figure-6 scene: the normal AC
    falls by orders of magnitude over the 300 iterations at every read step,
    the tangential one decreases, and what remains of the mean after
    100 iterations comes from contacts that took off (their stale local force
    enters the reference's AC norm)."""
    g = json.load(open(os.path.join(HERE, "golden", "figure6_oracle_ac.json")))
    for step in ("50", "100", "200", "300"):
        d = g["steps"][step]
        assert d["contacts"] > 0 and d["iterations"] == 300
        N, T = np.array(d["mean_normal"]), np.array(d["mean_tangential"])
        assert N[-1] < 0.25 * N[0], step
        assert T[-1] < T[0], step
        assert N[99] < 0.5 * N[9] or N[99] < 1e-4, step


@pytest.mark.gpu
def test_ac_trace_matches_oracle_on_figure6_analogue():
    s = figure6_analogue()
    p = abi.params(time_step=5e-3, iterations=300, trace_alart_curnier=1)
    g = native.Simulation(s, p)
    o = Oracle(s, abi.params(time_step=5e-3, iterations=300))
    o.trace_alart_curnier(True)
    checked = 0
    for k in range(101):
        g.step(1)
        o.step(1)
        if k in (50, 100):
            tg, ncg = g.alart_curnier_trace()
            to, nco = o.alart_curnier_trace()
            assert ncg == nco and tg.shape == to.shape, k
            assert ncg > 0, k
            scale = max(np.abs(to).max(), 1e-12)
            err = np.abs(tg - to).max() / scale
            mean_n = to[:, :nco, 1].mean(axis=1)
            print("step %d: %d contacts, trace rel. diff %.2e, mean normal AC %.2e -> %.2e"
                  % (k, nco, err, mean_n[0], mean_n[-1]))
            assert err < 1e-6, (k, err)
            checked += 1
        qo, vo = o.state()
        g.set_state(qo, vo)
    assert checked == 2
