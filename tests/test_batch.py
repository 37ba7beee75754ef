"""Batching: many cloth instances stepped as one block-diagonal scene.

CPU: the batched scene (oracle) equals the instances stepped one by one, so
the per-mesh obstacle restriction and the shared global matrix change
nothing.  GPU: the batched scene on the device equals the oracle's.
"""
import numpy as np
import pytest

from climatenet_b200 import abi, native, scenes
from oracle.oracle import Oracle


def _split(q, scene):
    return [q[m["vertex_offset"]:m["vertex_offset"] + m["n_vertices"]] for m in scene.meshes]


def test_batched_scene_equals_independent_instances():
    s, insts, pk = scenes.batch_scene(n_instances=3, seed=4)
    p = abi.params(**pk)
    ob = Oracle(s, p)
    ob.step(4)
    qb, _ = ob.state()
    parts = _split(qb, s)
    for k, inst in enumerate(insts):
        si = scenes.instance_scene(inst)
        oi = Oracle(si, p)
        oi.step(4)
        qi, _ = oi.state()
        side = int(np.ceil(np.sqrt(len(insts))))
        off = np.array([3.0 * (k % side), 3.0 * (k // side), 0.0])
        assert np.abs(parts[k] - off - qi).max() < 1e-9 * max(1.0, np.abs(qi).max())


@pytest.mark.gpu
def test_gpu_batch_matches_oracle():
    s, insts, pk = scenes.batch_scene(n_instances=6, seed=4)
    p = abi.params(**pk)
    g = native.Simulation(s, p)
    o = Oracle(s, p)
    for _ in range(6):
        rg = g.step(1)
        ro = o.step(1)
        assert rg.n_contacts == ro.n_contacts
    qg, _ = g.state()
    qo, _ = o.state()
    assert np.abs(qg - qo).max() / np.abs(qo).max() < 1e-6
    st = g.stats()
    assert st.sweep_chunk in (32, 64, 128)


@pytest.mark.gpu
@pytest.mark.parametrize("use_graph", [1, 0])  # conditional WHILE graph / host-driven loop
def test_tolerance_mode_matches_oracle(use_graph):
    s = scenes.cloth_on_sphere(n=30, side=1.0, z=-0.2455, mu=0.3, sphere_center=(0, 0, -0.5),
                               sphere_radius=0.25, pins=True)
    p = abi.params(time_step=5e-3, iterations=60, residual_tolerance=0.05, use_graph=use_graph)
    g = native.Simulation(s, p)
    o = Oracle(s, p)
    total = 0
    for _ in range(5):
        rg = g.step(1)
        ro = o.step(1)
        assert rg.iterations == ro.iterations
        assert 1 <= rg.iterations <= 60
        total += rg.iterations
    assert g.stats().iterations == total  # counted on the device
    qg, _ = g.state()
    qo, _ = o.state()
    assert np.abs(qg - qo).max() / np.abs(qo).max() < 1e-6
