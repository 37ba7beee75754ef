"""GPU step loop against the FP64 CPU oracle, through the C ABI.

Tolerances: FP64 path 1e-6 relative on vertex positions over a 10-step
horizon, contact sets identical, Alart-Curnier residual
within 1e-6 relative; detection candidate and pairing sets bit-exact.
"""
import numpy as np
import pytest

from climatenet_b200 import abi, native, scenes
from conftest import incline_closed_form, load_incline
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

REL = 1e-6


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def draped_cloth(n=30, z=-0.2455, mu=0.3, pins=True):
    """A cloth starting right on top of the sphere so that contacts exist from step 0."""
    s = scenes.cloth_on_sphere(n=n, side=1.0, z=z, mu=mu, sphere_center=(0, 0, -0.5),
                               sphere_radius=0.25, pins=pins)
    return s


def run_pair(scene, params, steps):
    g = native.Simulation(scene, params)
    o = Oracle(scene, params)
    for _ in range(steps):
        rg = g.step(1)
        ro = o.step(1)
        assert rg.n_contacts == ro.n_contacts and rg.n_self_contacts == ro.n_self_contacts
    return g, o, rg, ro


def test_fp64_one_step_matches_oracle():
    s = draped_cloth()
    p = abi.params(time_step=5e-3, iterations=30)
    g, o, rg, ro = run_pair(s, p, 1)
    cg, co = g.contacts(), o.contacts()
    assert rg.n_contacts > 0
    assert np.array_equal(cg["vertex"], co["vertex"])
    assert np.allclose(cg["normal"], co["normal"], rtol=0, atol=1e-15)
    qg, vg = g.state()
    qo, vo = o.state()
    assert rel_err(qg, qo) < REL and rel_err(vg, vo) < REL
    assert abs(rg.residual - ro.residual) <= REL * max(ro.residual, 1e-12) + 1e-14


@pytest.mark.parametrize("use_graph", [0, 1])
def test_fp64_ten_steps_match_oracle(use_graph):
    s = draped_cloth()
    p = abi.params(time_step=5e-3, iterations=30, use_graph=use_graph)
    g, o, rg, ro = run_pair(s, p, 10)
    qg, vg = g.state()
    qo, vo = o.state()
    assert rel_err(qg, qo) < REL, rel_err(qg, qo)
    assert rel_err(vg, vo) < 1e-5
    assert np.allclose(g.contacts()["force"], o.contacts()["force"], rtol=1e-5, atol=1e-12)


def test_rotating_sphere_contact_speed():
    s = scenes.cloth_on_sphere(n=24, side=1.0, z=0.001, mu=0.5, sphere_center=(0, 0, -0.5),
                               sphere_radius=0.5, rotating=1.0)
    p = abi.params(time_step=2e-3, iterations=20)
    g, o, rg, ro = run_pair(s, p, 3)
    cg, co = g.contacts(), o.contacts()
    assert np.abs(cg["speed"]).max() > 0  # rotation started after the first step
    assert np.allclose(cg["speed"], co["speed"], rtol=0, atol=1e-15)
    qg, _ = g.state()
    qo, _ = o.state()
    assert rel_err(qg, qo) < REL


def test_incline_known_answer_on_gpu():
    s, p, P = load_incline()
    g = native.Simulation(s, p)
    o = Oracle(s, p)
    worst = 0.0
    for k in range(400):
        g.step(1)
        o.step(1)
        qg, vg = g.state()
        sp, _ = incline_closed_form((k + 1) * P["Timestep"])
        worst = max(worst, abs(np.linalg.norm(vg.mean(0)) - sp))
    qo, vo = o.state()
    assert worst < 1e-8
    assert rel_err(qg, qo) < REL


def layered(n=16, layers=3, gap=0.0009, side=0.4, seed=5):
    rng = np.random.default_rng(seed)
    P, T = [], []
    for k in range(layers):
        p, t = scenes.grid_mesh(n, side, z=k * gap)
        p[:, :2] += 0.002 * rng.standard_normal((len(p), 2))
        p[:, 2] += 0.0003 * rng.standard_normal(len(p))
        P.append(p)
        T.append(t + k * n * n)
    return np.concatenate(P), np.concatenate(T)


def test_candidate_sets_bit_exact():
    from oracle import oracle as orc
    pos, tris = layered()
    for tol in (1e-3, 2.5e-3):
        got = native.detect_candidates(pos, tris, tol)
        exp = orc.self_candidates(pos, tris, tol)
        assert np.array_equal(got, exp), tol


def test_self_pairing_bit_exact():
    from oracle import oracle as orc
    pos, tris = layered()
    g = native.detect_self_collisions(pos, tris, 1.5e-3)
    o = orc.self_collisions(pos, tris, 1.5e-3)
    assert g["vertex"].shape[0] > 0
    for k in ("vertex", "partner", "face"):
        assert np.array_equal(g[k], o[k]), k
    assert np.array_equal(g["normal"], o["normal"])


def test_self_collision_step_matches_oracle():
    pos, tris = layered(n=14, layers=3, gap=0.0009)
    s = scenes.Scene(friction=((0.4,),))
    s.add_mesh(pos, tris, area_density=0.1, bending=1e-2, stretching=1e3)
    s.add_sphere((0, 0, -0.3), 0.3)
    p = abi.params(time_step=2.5e-3, iterations=20, self_collision=True, self_tol=1e-3)
    g, o, rg, ro = run_pair(s, p, 5)
    assert rg.n_self_contacts > 0
    sg, so = g.self_contacts(), o.self_contacts()
    for k in ("vertex", "partner", "face"):
        assert np.array_equal(sg[k], so[k]), k
    lg, og = g.self_levels()
    lo, oo = o.self_levels()
    assert np.array_equal(lg, lo)
    for l in range(len(lg) - 1):  # same contacts on every level (order inside a level is free)
        assert sorted(og[lg[l]:lg[l + 1]]) == sorted(oo[lo[l]:lo[l + 1]])
    qg, _ = g.state()
    qo, _ = o.state()
    assert rel_err(qg, qo) < REL, rel_err(qg, qo)


def test_fp32_refine_matches_fp64_oracle():
    s = draped_cloth()
    p = abi.params(time_step=5e-3, iterations=30, precision=abi.PDF_FP32_REFINE)
    g = native.Simulation(s, p)
    o = Oracle(s, abi.params(time_step=5e-3, iterations=30))
    for _ in range(10):
        g.step(1)
        o.step(1)
    qg, _ = g.state()
    qo, _ = o.state()
    assert rel_err(qg, qo) < REL, rel_err(qg, qo)


def test_nan_state_is_rejected():
    s = draped_cloth(n=8)
    g = native.Simulation(s, abi.params())
    q, v = g.state()
    q[3, 1] = np.nan
    with pytest.raises(native.PdfError) as e:
        g.set_state(q=q)
    assert e.value.status == abi.PDF_NAN_DETECTED


def test_indefinite_matrix_is_reported():
    s = scenes.cloth_on_sphere(n=8, stretching=-1e3)
    with pytest.raises(native.PdfError) as e:
        native.Simulation(s, abi.params())
    assert e.value.status == abi.PDF_NOT_SPD
