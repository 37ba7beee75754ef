"""Mesh obstacles with many triangles, where the device walks an LBVH over the
obstacle instead of scanning every triangle: the contact sets, normals and
states must still equal the oracle's triangle-order scan
(StaticMesh.cpp:33-56, MovingMesh.cpp:164-249, checkMeshCollision
geometry_util.cpp:32-92)."""
import numpy as np
import pytest

from climatenet_b200 import abi, native, scenes
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def uv_sphere(radius, n_lat=24, n_lon=48, center=(0.0, 0.0, 0.0)):
    """Closed UV sphere, triangles counter-clockwise seen from outside."""
    verts = [(0.0, 0.0, radius)]
    for i in range(1, n_lat):
        th = np.pi * i / n_lat
        for j in range(n_lon):
            ph = 2 * np.pi * j / n_lon
            verts.append((radius * np.sin(th) * np.cos(ph), radius * np.sin(th) * np.sin(ph), radius * np.cos(th)))
    verts.append((0.0, 0.0, -radius))
    v = np.array(verts) + np.asarray(center)
    tris = []
    ring = lambda i, j: 1 + (i - 1) * n_lon + (j % n_lon)
    for j in range(n_lon):
        tris.append((0, ring(1, j), ring(1, j + 1)))
    for i in range(1, n_lat - 1):
        for j in range(n_lon):
            a, b, c, d = ring(i, j), ring(i, j + 1), ring(i + 1, j), ring(i + 1, j + 1)
            tris.append((a, c, d))
            tris.append((a, d, b))
    south = len(verts) - 1
    for j in range(n_lon):
        tris.append((south, ring(n_lat - 1, j + 1), ring(n_lat - 1, j)))
    return v, np.array(tris, dtype=np.int32)


def cloth_over_mesh_sphere(moving=False):
    # the grid is shifted off the sphere's meridian planes: a vertex right
    # above an edge between two facets is at equal distance from both, and
    # which one wins then hangs on the last bit of its position
    pos, tri = scenes.grid_mesh(24, 1.0, z=0.003, center=(0.01234, 0.00567))
    s = scenes.Scene(friction=((0.3,),))
    s.add_mesh(pos, tri, area_density=0.1, bending=1e-2, stretching=1e3)
    v, t = uv_sphere(0.5, center=(0.0, 0.0, -0.5))
    if moving:
        frames = np.stack([v + np.array([0.002 * f, 0.0, 0.001 * f]) for f in range(4)])
        s.add_moving_mesh(frames, t, 4e-3, 0.01)
    else:
        s.add_mesh_obstacle(v, t, 0.01)
    return s, len(t)


def closest_point(p, a, b, c):
    """Closest point of triangle abc to p (Ericson's region test)."""
    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = ab @ ap, ac @ ap
    if d1 <= 0 and d2 <= 0:
        return a
    bp = p - b
    d3, d4 = ab @ bp, ac @ bp
    if d3 >= 0 and d4 <= d3:
        return b
    vc = d1 * d4 - d3 * d2
    if vc <= 0 and d1 >= 0 and d3 <= 0:
        return a + d1 / (d1 - d3) * ab
    cp = p - c
    d5, d6 = ab @ cp, ac @ cp
    if d6 >= 0 and d5 <= d6:
        return c
    vb = d5 * d2 - d1 * d6
    if vb <= 0 and d2 >= 0 and d6 <= 0:
        return a + d2 / (d2 - d6) * ac
    va = d3 * d6 - d5 * d4
    if va <= 0 and (d4 - d3) >= 0 and (d5 - d6) >= 0:
        return b + (d4 - d3) / ((d4 - d3) + (d5 - d6)) * (c - b)
    den = 1 / (va + vb + vc)
    return a + ab * (vb * den) + ac * (vc * den)


def facet_distance(x, normal, verts, tris):
    """Smallest squared distance from x to the facets with this normal."""
    best = np.inf
    for tr in tris:
        a, b, c = verts[tr]
        n = np.cross(b - a, c - a)
        n /= np.linalg.norm(n)
        if np.allclose(n, normal, rtol=0, atol=1e-12):
            cp = closest_point(x, a, b, c)
            best = min(best, (cp - x) @ (cp - x))
    return best


@pytest.mark.parametrize("moving", [False, True])
def test_mesh_sphere_obstacle_matches_oracle(moving):
    """Contact sets, facet normals and contact speeds equal the oracle's at
    every one of 10 steps, and each step's positions agree to 1e-6.  After
    every step the GPU is reset to the oracle's state, so that both detect on
    identical positions: over a convex facet mesh a vertex above an edge is
    at equal distance from two facets, and which one wins hangs on the last
    bit of its position (the GPU's atomic sums and the oracle do not share
    those bits); on identical positions the choice must be identical, also
    for the key-framed mesh, whose interpolation both sides round alike."""
    s, nt = cloth_over_mesh_sphere(moving)
    assert nt > 2000
    p = abi.params(time_step=2e-3, iterations=15)
    g = native.Simulation(s, p)
    o = orc.Oracle(s, p)
    moved = False
    for step in range(10):
        rg = g.step(1)
        ro = o.step(1)
        assert rg.n_contacts == ro.n_contacts, step
        cg, co = g.contacts(), o.contacts()
        assert np.array_equal(cg["vertex"], co["vertex"]), step
        assert np.array_equal(cg["normal"], co["normal"]), step
        assert np.allclose(cg["speed"], co["speed"], rtol=0, atol=1e-12), step
        moved |= bool(np.abs(co["speed"]).max() > 0)
        qg, vg = g.state()
        qo, vo = o.state()
        assert np.abs(qg - qo).max() / np.abs(qo).max() < 1e-6, step
        g.set_state(qo, vo)
    assert rg.n_contacts >= 5 and moved == moving


def test_facet_distance_helper_sees_ties():
    """The tie geometry the reset guards against: a point above the edge
    shared by two facets of the UV sphere is at equal distance from both."""
    v, t = uv_sphere(0.5)
    a, b, c = v[t[100]]
    n = np.cross(b - a, c - a)
    n /= np.linalg.norm(n)
    assert np.isfinite(facet_distance(a + 0.001 * n, n, v, t))
