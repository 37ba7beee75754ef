"""Hand-computed cases for the oracle: constraint projections, the three
contact regimes (stick, slip, take-off), obstacle margins, closest point and
the candidate set.  Each expected value is derived in the test from the
reference's formulas, not from the oracle."""
import numpy as np
import pytest

from climatenet_b200 import abi, scenes
from oracle import oracle as orc


def one_triangle(z=0.0, density=1.0, stretch=10.0):
    pos = np.array([[0.0, 0.0, z], [0.1, 0.0, z], [0.0, 0.1, z]])
    tri = np.array([[0, 1, 2]])
    return pos, tri


def test_spring_projection_matches_formula():
    # SpringConstraint::addConstraintProjection: sqrt(k) * L * normalize(x_i - x_j)
    pos, tri = one_triangle()
    s = scenes.Scene(friction=((0.3,),))
    s.add_mesh(pos, tri, area_density=1.0, bending=1e-3, stretching=16.0)
    o = orc.Oracle(s, abi.params(time_step=1e-3, iterations=5))
    rng = np.random.default_rng(0)
    q = pos + 0.01 * rng.standard_normal(pos.shape)
    p = o.projections(q)
    assert p.shape == (3, 3)  # three springs, no interior vertex
    rest = {frozenset(e): np.linalg.norm(pos[e[0]] - pos[e[1]]) for e in [(0, 1), (1, 2), (2, 0)]}
    for row in p:
        # each row is 4 * L * unit vector along one edge (either orientation)
        matched = False
        for e, L in rest.items():
            a, b = tuple(e)
            d = q[a] - q[b]
            u = d / np.linalg.norm(d)
            if np.allclose(row, 4.0 * L * u, rtol=0, atol=1e-14) or np.allclose(row, -4.0 * L * u, atol=1e-14):
                matched = True
        assert matched, row


def mean_value_coeffs(mid, ring):
    """getLaplaceBeltramiDiscretisationMeanValueCoefficients (geometry_util.cpp:673-710)
    with getMeanValue (:766-775): angle at the 2nd argument."""
    def mv(v1, v2, v3):
        e1, e2 = v1 - v2, v3 - v2
        l = np.linalg.norm(e1) * np.linalg.norm(e2)
        c = e1 @ e2 / l
        if 1 - c == 0:
            return 0.0
        return (1 - c) / (np.linalg.norm(np.cross(e1, e2)) / l)
    n = len(ring)
    out = []
    for i in range(n):
        v, cw, ccw = ring[i], ring[(i + 1) % n], ring[(i - 1) % n]
        out.append((mv(v, mid, cw) + mv(v, ccw, mid)) / np.linalg.norm(v - mid))
    return np.array(out)


def test_bending_projection_matches_formula():
    # a fan of 6 triangles around vertex 0; ring listed counter-clockwise
    ang = np.linspace(0, 2 * np.pi, 7)[:-1] + np.array([0, .1, -.05, .2, 0, -.1])
    rad = np.array([1.0, 0.9, 1.1, 1.0, 0.95, 1.05])
    ring = np.stack([rad * np.cos(ang), rad * np.sin(ang), 0.05 * np.sin(3 * ang)], 1)
    pos = np.concatenate([[[0.0, 0.0, 0.02]], ring])
    tri = np.array([[0, 1 + i, 1 + (i + 1) % 6] for i in range(6)])
    s = scenes.Scene(friction=((0.3,),))
    s.add_mesh(pos, tri, area_density=1.0, bending=4.0, stretching=1.0)
    o = orc.Oracle(s, abi.params(time_step=1e-3, iterations=5))
    # CGAL circulates the 1-ring clockwise (opposite(next(h))): reverse the CCW list
    cw_ring = [1, 6, 5, 4, 3, 2]
    c = mean_value_coeffs(pos[0], pos[cw_ring])
    coef = np.concatenate([[c.sum()], -c])
    idx = [0] + cw_ring
    rest_norm = np.linalg.norm(coef @ pos[idx])
    rng = np.random.default_rng(1)
    q = pos + 0.05 * rng.standard_normal(pos.shape)
    lap = coef @ q[idx]
    expect = 2.0 * (rest_norm / np.linalg.norm(lap)) * lap
    p = o.projections(q)
    assert np.allclose(p[-1], expect, rtol=1e-12, atol=1e-15)


def _plane_triangle(v0, mu=0.3):
    pos, tri = one_triangle(z=0.0)
    s = scenes.Scene(friction=((mu,),))
    s.add_mesh(pos, tri, area_density=2.0, bending=1e-3, stretching=100.0)
    s.add_plane((0.0, 0.0, 0.0), (0.0, 0.0, 1.0))
    s.vel = np.tile(np.asarray(v0, dtype=float), (3, 1))
    return s


def test_stick_contact_cancels_gravity():
    dt, g = 1e-3, 9.81
    o = orc.Oracle(_plane_triangle((0, 0, 0)), abi.params(time_step=dt, iterations=10))
    o.step(1)
    q, v = o.state()
    assert np.abs(v).max() < 1e-12
    c = o.contacts()
    m = o.masses()
    # r = (m dt g, 0, 0) in the local frame (normal first)
    assert np.allclose(c["force"][:, 0], m * dt * g, rtol=1e-10)
    assert np.abs(c["force"][:, 1:]).max() < 1e-14
    assert c["ac"].max() < 1e-12


def test_slip_contact_decelerates_by_mu_g_dt():
    dt, g, mu, u = 1e-3, 9.81, 0.3, 0.5
    o = orc.Oracle(_plane_triangle((u, 0, 0), mu=mu), abi.params(time_step=dt, iterations=10))
    o.step(1)
    q, v = o.state()
    assert np.allclose(v[:, 0], u - mu * g * dt, rtol=0, atol=1e-12)
    assert np.abs(v[:, 1:]).max() < 1e-12
    c = o.contacts()
    r = c["force"]
    assert np.allclose(np.hypot(r[:, 1], r[:, 2]), mu * r[:, 0], rtol=1e-12)


def test_take_off_keeps_free_flight():
    dt, g = 1e-3, 9.81
    o = orc.Oracle(_plane_triangle((0, 0, 1.0)), abi.params(time_step=dt, iterations=10))
    o.step(1)
    q, v = o.state()
    assert np.allclose(v[:, 2], 1.0 - g * dt, atol=1e-12)
    assert o.contacts()["vertex"].shape[0] == 3  # detected, then released


def test_sphere_margin_is_one_centimetre():
    pos = np.array([[0.0, 0.0, 0.5 + 0.0099], [1.0, 0.0, 0.5 + 0.0101 + 0.0], [0.0, 1.0, 3.0]])
    s = scenes.Scene(friction=((0.3,),))
    s.add_mesh(pos, np.array([[0, 1, 2]]), area_density=1.0, bending=1e-3, stretching=1.0)
    s.add_sphere((0.0, 0.0, 0.0), 0.5)
    s.add_sphere((1.0, 0.0, 0.0), 0.5)
    o = orc.Oracle(s, abi.params(time_step=1e-4, iterations=2, gravity=(0, 0, 0)))
    o.step(1)
    c = o.contacts()
    # vertex 0 is 0.0099 outside sphere 0 -> contact; vertex 1 is 0.0101 outside sphere 1 -> none
    assert list(c["vertex"]) == [0]


def test_closest_point_regions():
    a, b, c = np.array([0., 0, 0]), np.array([1., 0, 0]), np.array([0., 1, 0])
    cases = [
        ((0.25, 0.25, 0.3), (0.25, 0.25, 0), (0.5, 0.25, 0.25)),   # face
        ((-1, -1, 0), (0, 0, 0), (1, 0, 0)),                        # vertex a
        ((2, -0.5, 0), (1, 0, 0), (0, 1, 0)),                       # vertex b
        ((0.5, -1, 0), (0.5, 0, 0), (0.5, 0.5, 0)),                 # edge ab
        ((1, 1, 0), (0.5, 0.5, 0), (0, 0.5, 0.5)),                  # edge bc
    ]
    for p, cp_exp, bary_exp in cases:
        cp, bary = orc.closest_point(np.array(p, float), a, b, c, 10.0)
        assert np.allclose(cp, cp_exp) and np.allclose(bary, bary_exp), (p, cp, bary)
    # the reference's early exit: |ap|^2 - |ab|^2 - |ac|^2 > tol2 returns vertex a
    cp, bary = orc.closest_point(np.array([5., 5, 0]), a, b, c, 1e-3)
    assert np.allclose(bary, (1, 0, 0)) and np.allclose(cp, a)


def brute_candidates(pos, tris, tol):
    t = 1.1 * tol
    lo = pos[tris].min(1)
    hi = pos[tris].max(1)
    out = []
    for v in range(len(pos)):
        ok = np.all((lo <= pos[v] + t) & (pos[v] - t <= hi), axis=1)
        out += [(v, k) for k in np.nonzero(ok)[0]]
    return np.array(out, dtype=np.int64).reshape(-1, 2)


def layered_mesh(n=12, layers=2, gap=0.002, seed=3):
    rng = np.random.default_rng(seed)
    P, T = [], []
    for k in range(layers):
        p, t = scenes.grid_mesh(n, 0.3, z=k * gap)
        p[:, 2] += 0.0015 * rng.standard_normal(len(p))
        P.append(p)
        T.append(t + k * n * n)
    return np.concatenate(P), np.concatenate(T)


def test_candidate_set_equals_brute_force():
    pos, tris = layered_mesh()
    tol = 2e-3
    got = orc.self_candidates(pos, tris, tol)
    exp = brute_candidates(pos, tris, tol)
    assert np.array_equal(got, exp)


def test_self_collision_pairs_are_node_node():
    pos, tris = layered_mesh()
    sc = orc.self_collisions(pos, tris, 2e-3)
    assert sc["vertex"].shape[0] > 0
    for v, p, f in zip(sc["vertex"], sc["partner"], sc["face"]):
        assert p in f and v not in f
