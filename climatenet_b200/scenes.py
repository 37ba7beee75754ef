"""In-memory scene building: square cloth grids, spheres and the benchmark
workloads (all synthetic, seeded).

A scene here is the in-memory equivalent of the reference's scene JSON
(src/scene_building.cpp:49-202): one or more dynamic meshes with area density,
bending and stretching weights and a material id, obstacles, an optional list of
attachment pins and the friction table.  ``Scene.desc()`` returns the
``pdf_scene_desc`` of include/pdf.h; the numpy arrays it points into are kept
alive by the Scene object.
"""
import ctypes as C

import numpy as np

from . import abi


def grid_mesh(n, side, z=0.0, center=(0.0, 0.0)):
    """Square n x n vertex grid of the given side length at height z.

    Vertex (i, j) -> index j * n + i, x along i, y along j.  One diagonal per
    quad; both triangles counter-clockwise seen from +z (normal +z).
    Returns (positions (n*n, 3) float64, triangles (2 (n-1)^2, 3) int32).
    """
    xs = np.linspace(-0.5 * side, 0.5 * side, n) + center[0]
    ys = np.linspace(-0.5 * side, 0.5 * side, n) + center[1]
    X, Y = np.meshgrid(xs, ys)  # [j, i]
    pos = np.stack([X.ravel(), Y.ravel(), np.full(n * n, float(z))], axis=1)
    i, j = np.meshgrid(np.arange(n - 1), np.arange(n - 1))
    v00 = (j * n + i).ravel()
    v10 = v00 + 1
    v01 = v00 + n
    v11 = v01 + 1
    t1 = np.stack([v00, v10, v11], axis=1)
    t2 = np.stack([v00, v11, v01], axis=1)
    tris = np.empty((2 * len(v00), 3), dtype=np.int32)
    tris[0::2] = t1
    tris[1::2] = t2
    return pos.astype(np.float64), tris


class Scene:
    """Mutable scene description; call desc() to get the C struct."""

    def __init__(self, friction=((0.3,),)):
        self.rest = np.zeros((0, 3))
        self.pos = None
        self.vel = None
        self.tris = np.zeros((0, 3), dtype=np.int32)
        self.meshes = []  # dicts
        self.pins = []    # (vertex, weight, position)
        self.obstacles = []
        self.friction = np.array(friction, dtype=np.float64)
        self._keep = []

    # -- meshes --------------------------------------------------------
    def add_mesh(self, positions, triangles, area_density=0.1, bending=1e-2,
                 stretching=1e3, material=0, current=None):
        """Append one dynamic mesh (triangles given mesh-local)."""
        v0 = len(self.rest)
        t0 = len(self.tris)
        positions = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
        triangles = np.asarray(triangles, dtype=np.int32).reshape(-1, 3)
        self.rest = np.concatenate([self.rest, positions])
        self.tris = np.concatenate([self.tris, triangles + v0]).astype(np.int32)
        cur = positions if current is None else np.asarray(current, dtype=np.float64).reshape(-1, 3)
        self.pos = cur.copy() if self.pos is None else np.concatenate([self.pos, cur])
        self.meshes.append(dict(vertex_offset=v0, n_vertices=len(positions),
                                triangle_offset=t0, n_triangles=len(triangles),
                                area_density=area_density, bending=bending,
                                stretching=stretching, material=material))
        return v0

    def add_pin(self, vertex, weight, position=None):
        if position is None:
            position = self.pos[vertex]
        self.pins.append((int(vertex), float(weight), np.asarray(position, dtype=np.float64)))

    # -- obstacles -----------------------------------------------------
    def add_sphere(self, center, radius, material=0):
        self.obstacles.append(dict(type=abi.PDF_OBSTACLE_SPHERE, center=center,
                                   radius=radius, material=material))

    def add_rotating_sphere(self, center, radius, axis, angular_speed, start_time=0.0, material=0):
        self.obstacles.append(dict(type=abi.PDF_OBSTACLE_ROTATING_SPHERE, center=center,
                                   radius=radius, axis=axis, angular_speed=angular_speed,
                                   rotation_start_time=start_time, material=material))

    def add_plane(self, point, normal, material=0):
        self.obstacles.append(dict(type=abi.PDF_OBSTACLE_PLANE, point=point, normal=normal,
                                   material=material))

    def add_box(self, position, size, material=0):
        """Axis-aligned box; `position` is its corner with the smallest coordinates."""
        self.obstacles.append(dict(type=abi.PDF_OBSTACLE_BOX, center=position, size=size, material=material))

    def add_mesh_obstacle(self, vertices, triangles, threshold, material=0):
        self.obstacles.append(dict(type=abi.PDF_OBSTACLE_MESH,
                                   vertices=np.ascontiguousarray(vertices, dtype=np.float64),
                                   triangles=np.ascontiguousarray(triangles, dtype=np.int32),
                                   threshold=threshold, material=material))

    def add_moving_mesh(self, frames, triangles, frame_interval, tolerance, material=0):
        """Key-framed moving mesh: `frames` (F, V, 3), key frame f reached at
        time f * frame_interval, linear interpolation in between."""
        frames = np.ascontiguousarray(frames, dtype=np.float64)
        if frames.ndim != 3 or frames.shape[0] < 2 or frames.shape[2] != 3:
            raise ValueError("frames must be (F >= 2, V, 3)")
        self.obstacles.append(dict(type=abi.PDF_OBSTACLE_MOVING_MESH, frames=frames,
                                   triangles=np.ascontiguousarray(triangles, dtype=np.int32),
                                   frame_interval=frame_interval, threshold=tolerance,
                                   material=material))

    @property
    def n_vertices(self):
        return len(self.rest)

    # -- C view --------------------------------------------------------
    def desc(self):
        """Build a pdf_scene_desc pointing into this object's arrays."""
        self._keep = []

        def dptr(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            self._keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_double))

        def iptr(a):
            a = np.ascontiguousarray(a, dtype=np.int32)
            self._keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_int32))

        d = abi.pdf_scene_desc()
        d.n_vertices = len(self.rest)
        d.rest_positions = dptr(self.rest)
        d.positions = dptr(self.pos) if self.pos is not None else None
        d.velocities = dptr(self.vel) if self.vel is not None else None
        d.n_triangles = len(self.tris)
        d.triangles = iptr(self.tris)
        meshes = (abi.pdf_mesh_desc * len(self.meshes))()
        for k, m in enumerate(self.meshes):
            for key, val in m.items():
                setattr(meshes[k], key, val)
        self._keep.append(meshes)
        d.n_meshes = len(self.meshes)
        d.meshes = meshes
        d.n_pins = len(self.pins)
        if self.pins:
            d.pin_vertices = iptr(np.array([p[0] for p in self.pins]))
            d.pin_weights = dptr(np.array([p[1] for p in self.pins]))
            d.pin_positions = dptr(np.array([p[2] for p in self.pins]))
        obs = (abi.pdf_obstacle * max(1, len(self.obstacles)))()
        for k, o in enumerate(self.obstacles):
            ob = obs[k]
            ob.type = o["type"]
            ob.material = o.get("material", 0)
            ob.mesh = o.get("mesh", -1)
            for key in ("center", "axis", "point", "normal", "size"):
                if key in o:
                    for c in range(3):
                        getattr(ob, key)[c] = float(o[key][c])
            for key in ("radius", "angular_speed", "rotation_start_time", "threshold", "frame_interval"):
                if key in o:
                    setattr(ob, key, float(o[key]))
            if o["type"] == abi.PDF_OBSTACLE_MESH:
                ob.n_vertices = len(o["vertices"])
                ob.n_triangles = len(o["triangles"])
                ob.vertices = dptr(o["vertices"])
                ob.triangles = iptr(o["triangles"])
            elif o["type"] == abi.PDF_OBSTACLE_MOVING_MESH:
                ob.n_frames = o["frames"].shape[0]
                ob.n_vertices = o["frames"].shape[1]
                ob.n_triangles = len(o["triangles"])
                ob.vertices = dptr(o["frames"])
                ob.triangles = iptr(o["triangles"])
        self._keep.append(obs)
        d.n_obstacles = len(self.obstacles)
        d.obstacles = obs
        d.n_materials = self.friction.shape[0]
        d.friction = dptr(self.friction)
        return d


# ---------------------------------------------------------------------------
# The benchmark workloads (synthetic, seeded).  Each returns (Scene, params
# kwargs, number of steps).

def cloth_on_sphere(n=30, side=1.0, z=0.0, layers=1, spacing=0.005, area_density=0.1,
                    stretching=1e3, bending=1e-2, mu=0.3, sphere_center=(0.0, 0.0, -0.5),
                    sphere_radius=0.25, pins=False, pin_weight=1e6, rotating=None):
    """Square cloth layers (one mesh, ``layers`` connected components) over a sphere."""
    s = Scene(friction=((mu,),))
    allp, allt = [], []
    for k in range(layers):
        p, t = grid_mesh(n, side, z + k * spacing)
        allt.append(t + k * n * n)
        allp.append(p)
    s.add_mesh(np.concatenate(allp), np.concatenate(allt), area_density=area_density,
               bending=bending, stretching=stretching)
    if pins:
        s.add_pin((n - 1) * n, pin_weight)
        s.add_pin((n - 1) * n + n - 1, pin_weight)
    if rotating is None:
        s.add_sphere(sphere_center, sphere_radius)
    else:
        s.add_rotating_sphere(sphere_center, sphere_radius, (0.0, 0.0, 1.0), rotating, 0.0)
    return s


def workload(cfg, n_override=None):
    """The benchmark shapes: (scene, step parameters, step count) of the 30 x 30
    pinned cloth (1), three stacked 128 x 128 layers (2), the 500 x 500 cloth on
    the rotating sphere (3) and two 256 x 256 layers on a rotating sphere (5)."""
    if cfg == 1:
        n = n_override or 30
        s = cloth_on_sphere(n=n, side=1.0, z=0.0, mu=0.3, sphere_center=(0, 0, -0.5),
                            sphere_radius=0.25, pins=True)
        return s, dict(time_step=5e-3, iterations=30), 200
    if cfg == 2:
        n = n_override or 128
        s = cloth_on_sphere(n=n, side=1.0, z=0.0, layers=3, spacing=0.005, mu=0.4,
                            sphere_center=(0, 0, -0.35), sphere_radius=0.3)
        return s, dict(time_step=2.5e-3, iterations=20, self_collision=True, self_tol=1e-3), 400
    if cfg == 3:
        n = n_override or 500
        # 5 mm above the sphere top: inside the 1 cm contact margin from step 0
        s = cloth_on_sphere(n=n, side=2.0, z=0.005, mu=0.5, sphere_center=(0, 0, -0.5),
                            sphere_radius=0.5, rotating=1.0)
        return s, dict(time_step=2e-3, iterations=20, self_collision=True, self_tol=2e-3), 300
    if cfg == 5:
        n = n_override or 256
        s = cloth_on_sphere(n=n, side=1.2, z=0.05, layers=2, spacing=0.001, mu=0.6,
                            sphere_center=(0, 0, -0.4), sphere_radius=0.4, rotating=1.0)
        return s, dict(time_step=2e-3, iterations=20, self_collision=True, self_tol=1e-3), 500
    raise ValueError("unknown workload %r" % (cfg,))


def batch_instances(n_instances=64, seed=4):
    """Batching shape: instances with n ~ U{20..150}, R ~ U[0.2, 0.5],
    mu ~ U[0.1, 0.8], height above the sphere top ~ U[0.1, 0.5] (numpy PCG64,
    seed 4).  Returns a list of dicts (n, R, mu, h)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n_instances):
        out.append(dict(n=int(rng.integers(20, 151)), R=float(rng.uniform(0.2, 0.5)),
                        mu=float(rng.uniform(0.1, 0.8)), h=float(rng.uniform(0.1, 0.5))))
    return out


def instance_scene(inst):
    """One instance of the batch as a scene of its own (for parity checks)."""
    s = cloth_on_sphere(n=inst["n"], side=1.0, z=inst["h"], mu=inst["mu"],
                        sphere_center=(0, 0, -inst["R"]), sphere_radius=inst["R"])
    return s


def batch_scene(n_instances=64, seed=4, spacing=3.0, subset=None):
    """All instances of the batch as ONE scene: instance k is mesh k (material
    k) translated by a grid offset, with its own sphere restricted to mesh k
    (material n_instances + k, friction table entry [k][n_instances + k] =
    mu_k).  The global matrix is block diagonal, so one factorisation and one
    set of launches per PD iteration step every instance together.
    `subset` (instance indices) builds the scene of those instances only, each
    at the offset it has in the whole batch (one rank's shard)."""
    insts = batch_instances(n_instances, seed)
    keep = list(range(len(insts))) if subset is None else sorted(subset)
    m = len(keep)
    fr = np.zeros((2 * m, 2 * m))
    for j, k in enumerate(keep):
        fr[j, m + j] = insts[k]["mu"]
    s = Scene(friction=fr)
    side = int(np.ceil(np.sqrt(len(insts))))
    for j, k in enumerate(keep):
        it = insts[k]
        ox, oy = spacing * (k % side), spacing * (k // side)
        p, t = grid_mesh(it["n"], 1.0, z=it["h"], center=(ox, oy))
        s.add_mesh(p, t, area_density=0.1, bending=1e-2, stretching=1e3, material=j)
        s.obstacles.append(dict(type=abi.PDF_OBSTACLE_SPHERE, center=(ox, oy, -it["R"]), radius=it["R"],
                                material=m + j, mesh=j))
    return s, [insts[k] for k in keep], dict(time_step=2.5e-3, iterations=20)


def instance_cost(inst):
    """Estimated per-iteration work of one n x n instance: nnz(A) of its
    springs and bending rows plus nnz(L) of a nested-dissection factor of
    the grid (31/4 N log2 N, George's bound for 2D grids)."""
    n = inst["n"]
    N = n * n
    E = 2 * n * (n - 1) + (n - 1) ** 2
    B = max(0, n - 2) ** 2
    return 2 * E + 7 * B + 7.75 * N * np.log2(N)


def shard_instances(insts, world):
    """Instances of a batch onto `world` ranks: greedy bin packing by
    estimated cost (largest first, each onto the least-loaded rank, ties to
    the lower rank).  Returns per rank the sorted instance indices.  The
    instances are independent, so the ranks step their shards without any
    collective."""
    order = sorted(range(len(insts)), key=lambda k: (-instance_cost(insts[k]), k))
    load = [0.0] * world
    shards = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda j: (load[j], j))
        shards[r].append(k)
        load[r] += instance_cost(insts[k])
    return [sorted(sh) for sh in shards]
