"""Obstacle detection cost per step for each obstacle kind under the
500 x 500 cloth of the benchmark workload (250k vertices): the device time
from the step's start to the end of obstacle detection (CUDA events, mean
over the steps), and the contacts found.

  python -m climatenet_b200.profile_detect [--n 500] [--steps 8]
"""
import argparse

import numpy as np

from . import abi, native, scenes


def uv_sphere(radius, n_lat, n_lon, center):
    """Closed UV sphere, triangles counter-clockwise seen from outside."""
    verts = [(0.0, 0.0, radius)]
    for i in range(1, n_lat):
        th = np.pi * i / n_lat
        for j in range(n_lon):
            ph = 2 * np.pi * j / n_lon
            verts.append((radius * np.sin(th) * np.cos(ph), radius * np.sin(th) * np.sin(ph), radius * np.cos(th)))
    verts.append((0.0, 0.0, -radius))
    v = np.array(verts) + np.asarray(center)

    def ring(i, j):
        return 1 + (i - 1) * n_lon + (j % n_lon)
    tris = [(0, ring(1, j), ring(1, j + 1)) for j in range(n_lon)]
    for i in range(1, n_lat - 1):
        for j in range(n_lon):
            a, b, c, d = ring(i, j), ring(i, j + 1), ring(i + 1, j), ring(i + 1, j + 1)
            tris += [(a, c, d), (a, d, b)]
    south = len(verts) - 1
    tris += [(south, ring(n_lat - 1, j + 1), ring(n_lat - 1, j)) for j in range(n_lon)]
    return v, np.array(tris, dtype=np.int32)


def scene(kind, n):
    pos, tri = scenes.grid_mesh(n, 2.0, z=0.005)
    s = scenes.Scene(friction=((0.5,),))
    s.add_mesh(pos, tri, area_density=0.1, bending=1e-2, stretching=1e3)
    c = (0.0, 0.0, -0.5)
    if kind == "sphere":
        s.add_sphere(c, 0.5)
    elif kind == "plane":
        s.add_plane((0.0, 0.0, -0.2), (0.0, 0.0, 1.0))
    elif kind == "box":
        s.add_box((-0.5, -0.5, -1.0), (1.0, 1.0, 1.0 + 0.004))
    else:
        # about the size of the reference's key-framed sphere (2,452 vertices, 4,900 faces)
        v, t = uv_sphere(0.5, 50, 49, c)
        if kind == "mesh":
            s.add_mesh_obstacle(v, t, 0.01)
        else:
            # key frames of a sphere turning about z at 1 rad/s, every 10 ms
            frames = []
            for f in range(40):
                a = 0.01 * f
                R = np.array([[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]])
                frames.append((v - c) @ R.T + c)
            s.add_moving_mesh(np.array(frames), t, 0.01, 0.01)
    return s


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=500)
    ap.add_argument("--steps", type=int, default=8)
    args = ap.parse_args()
    for kind in ("sphere", "plane", "box", "mesh", "moving-mesh"):
        s = scene(kind, args.n)
        g = native.Simulation(s, abi.params(time_step=2e-3, iterations=5))
        g.step(2)
        s0 = g.stats()
        for _ in range(args.steps):
            r = g.step(1)
        s1 = g.stats()
        ms = (s1.detection_ms - s0.detection_ms) / args.steps
        print("%-12s detection %.3f ms per step, %d contacts, %d obstacle triangles"
              % (kind, ms, r.n_contacts, s.obstacles[0].get("triangles", np.zeros((0, 3))).shape[0]), flush=True)
        g.close()


if __name__ == "__main__":
    main()
