"""ctypes binding of the B200 step-loop library (climatenet_b200/_build/libpdf_b200.so).

There is no fallback: if the library is missing or no CUDA device is usable,
every call raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libpdf_b200.so")
_lib = None


class PdfError(RuntimeError):
    """A pdf_* call returned a non-zero status."""

    def __init__(self, status, msg):
        super().__init__("%s: %s" % (abi.STATUS_NAMES.get(status, status), msg))
        self.status = status


def lib():
    """Load (once) and return the native library; raise if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("climatenet_b200 native library not built: %s (run __graft_entry__.build())"
                          % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    i32 = C.c_int32
    L.pdf_params_default.argtypes = [C.POINTER(abi.pdf_params)]
    L.pdf_global_error.restype = C.c_char_p
    L.pdf_last_error.argtypes = [vp]
    L.pdf_last_error.restype = C.c_char_p
    L.pdf_scene_load_json.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.pdf_scene_view.argtypes = [vp, C.POINTER(abi.pdf_scene_desc)]
    L.pdf_scene_free.argtypes = [vp]
    L.pdf_params_load_json.argtypes = [C.c_char_p, C.POINTER(abi.pdf_params), C.POINTER(i32), C.POINTER(i32)]
    L.pdf_create.argtypes = [C.POINTER(abi.pdf_scene_desc), C.POINTER(abi.pdf_params), C.POINTER(vp)]
    L.pdf_step.argtypes = [vp, i32, C.POINTER(abi.pdf_step_report)]
    L.pdf_get_state.argtypes = [vp, vp, vp]
    L.pdf_set_state.argtypes = [vp, vp, vp]
    L.pdf_device_state.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]
    L.pdf_get_contacts.argtypes = [vp, vp, i32, C.POINTER(i32)]
    L.pdf_get_self_contacts.argtypes = [vp, vp, i32, C.POINTER(i32)]
    L.pdf_get_self_levels.argtypes = [vp, vp, i32, vp, i32, C.POINTER(i32)]
    L.pdf_get_stats.argtypes = [vp, C.POINTER(abi.pdf_stats)]
    L.pdf_export_stats.argtypes = [vp, C.c_char_p]
    L.pdf_get_residual_history.argtypes = [vp, vp, i32, C.POINTER(i32)]
    L.pdf_time_phase.argtypes = [vp, i32, i32, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.pdf_check_wait_timeout.argtypes = [vp, i32]
    L.pdf_set_sweep_schedule.argtypes = [vp, i32, i32, i32, i32]
    L.pdf_time_solve_parts.argtypes = [vp, i32, C.POINTER(C.c_double)]
    L.pdf_factor_check.argtypes = [C.POINTER(abi.pdf_scene_desc), C.POINTER(abi.pdf_params), vp, vp]
    L.pdf_detect_candidates_noalloc.argtypes = [vp, i32, vp, i32, C.c_double, vp, i32, C.POINTER(i32), vp]
    L.pdf_destroy.argtypes = [vp]
    L.pdf_detect_candidates.argtypes = [vp, i32, vp, i32, C.c_double, vp, i32, C.POINTER(i32), i32]
    L.pdf_detect_self_collisions.argtypes = [vp, i32, vp, i32, C.c_double, vp, i32, C.POINTER(i32), i32]
    L.pdf_mlp_param_count.restype = i32
    L.pdf_mlp_init.argtypes = [vp, C.c_uint64]
    L.pdf_mlp_save.argtypes = [C.c_char_p, vp]
    L.pdf_mlp_load.argtypes = [C.c_char_p, vp]
    L.pdf_mlp_forward.argtypes = [vp, vp, i32, vp, i32]
    L.pdf_mlp_gradient.argtypes = [vp, vp, vp, i32, vp, C.POINTER(C.c_double), i32]
    L.pdf_mlp_fit.argtypes = [vp, vp, vp, i32, i32, i32, C.c_double, C.c_uint64, i32, C.POINTER(C.c_double),
                              C.POINTER(C.c_double)]
    L.pdf_mlp_set_weights.argtypes = [vp, vp, i32]
    L.pdf_mlp_get_weights.argtypes = [vp, vp, i32]
    L.pdf_mlp_log.argtypes = [vp, i32]
    L.pdf_mlp_samples.argtypes = [vp, vp, vp, i32, C.POINTER(i32)]
    L.pdf_mlp_train.argtypes = [vp, i32, i32, C.c_double, C.c_uint64, C.POINTER(C.c_double),
                                C.POINTER(C.c_double)]
    L.pdf_frame_capture.argtypes = [vp, i32]
    L.pdf_frame_wait.argtypes = [vp, i32, C.POINTER(C.POINTER(C.c_double))]
    L.pdf_get_vertices.argtypes = [vp, vp, i32, vp, vp]
    L.pdf_get_alart_curnier_trace.argtypes = [vp, vp, C.c_int64, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]
    L.pdf_log_load_json.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.pdf_log_view.argtypes = [vp, C.POINTER(i32), C.POINTER(C.POINTER(abi.pdf_log_entry))]
    L.pdf_log_free.argtypes = [vp]
    _lib = L
    return L


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _check(status, handle=None):
    if status != 0:
        L = lib()
        msg = L.pdf_last_error(handle) if handle else L.pdf_global_error()
        raise PdfError(status, (msg or b"").decode())


class LoadedScene:
    """A scene read from the reference's JSON format (getSceneFromJSONDocument)."""

    def __init__(self, path):
        h = C.c_void_p()
        _check(lib().pdf_scene_load_json(os.fsencode(path), C.byref(h)))
        self.h = h
        self._desc = abi.pdf_scene_desc()
        _check(lib().pdf_scene_view(self.h, C.byref(self._desc)))

    def desc(self):
        return self._desc

    @property
    def n_vertices(self):
        return self._desc.n_vertices

    def __del__(self):
        if getattr(self, "h", None):
            lib().pdf_scene_free(self.h)
            self.h = None


def load_params(path):
    """getSimulationParametersFromJSONDocument: (pdf_params, frames, steps per frame)."""
    p = abi.pdf_params()
    fr = C.c_int32()
    spf = C.c_int32()
    _check(lib().pdf_params_load_json(os.fsencode(path), C.byref(p), C.byref(fr), C.byref(spf)))
    return p, fr.value, spf.value


class Simulation:
    """One simulation handle; the drop-in for SimulationBase (step, exportStats)."""

    def __init__(self, scene, params):
        L = lib()
        self._scene = scene
        self._desc = scene.desc()
        self.params = params
        h = C.c_void_p()
        _check(L.pdf_create(C.byref(self._desc), C.byref(params), C.byref(h)))
        self.h = h
        self.n = self._desc.n_vertices

    def close(self):
        if getattr(self, "h", None):
            lib().pdf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except TypeError:
            pass  # interpreter shutdown: the module's globals are already gone

    def step(self, n=1):
        rep = abi.pdf_step_report()
        _check(lib().pdf_step(self.h, n, C.byref(rep)), self.h)
        return rep

    def state(self):
        q = np.empty((self.n, 3))
        v = np.empty((self.n, 3))
        _check(lib().pdf_get_state(self.h, _ptr(q), _ptr(v)), self.h)
        return q, v

    def set_state(self, q=None, v=None):
        qa = None if q is None else np.ascontiguousarray(q, dtype=np.float64)
        va = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        _check(lib().pdf_set_state(self.h, None if qa is None else _ptr(qa),
                                   None if va is None else _ptr(va)), self.h)

    def device_state(self):
        q = C.c_void_p()
        v = C.c_void_p()
        s = C.c_void_p()
        _check(lib().pdf_device_state(self.h, C.byref(q), C.byref(v), C.byref(s)), self.h)
        return q.value, v.value, s.value

    def _contacts(self, fn):
        n = C.c_int32()
        _check(fn(self.h, None, 0, C.byref(n)), self.h)
        arr = (abi.pdf_contact * max(1, n.value))()
        _check(fn(self.h, arr, n.value, C.byref(n)), self.h)
        return abi.contacts_to_numpy(arr, n.value)

    def contacts(self):
        return self._contacts(lib().pdf_get_contacts)

    def self_contacts(self):
        return self._contacts(lib().pdf_get_self_contacts)

    def self_levels(self):
        nl = C.c_int32()
        _check(lib().pdf_get_self_levels(self.h, None, 0, None, 0, C.byref(nl)), self.h)
        ns = self.self_contacts()["vertex"].shape[0]
        ptr = np.zeros(nl.value + 1, dtype=np.int32)
        order = np.zeros(max(1, ns), dtype=np.int32)
        _check(lib().pdf_get_self_levels(self.h, _ptr(ptr), nl.value + 1, _ptr(order), ns, C.byref(nl)),
               self.h)
        return ptr, order[:ns]

    def stats(self):
        s = abi.pdf_stats()
        _check(lib().pdf_get_stats(self.h, C.byref(s)), self.h)
        return s

    def export_stats(self, path):
        _check(lib().pdf_export_stats(self.h, os.fsencode(path)), self.h)

    exportStats = export_stats

    def set_sweep_schedule(self, chunk, cut_level, upper_mode, block_shape=1):
        """Pin the solve schedule (work-item width, subtree-block cut level,
        upper mode 0 = dependency-driven items / 1 = level launches, block
        kernel launch shape 0-4)."""
        _check(lib().pdf_set_sweep_schedule(self.h, chunk, cut_level, upper_mode, block_shape), self.h)

    def time_solve_parts(self, reps=10):
        """Device ms of the five launches of one solve: block forward, upper
        forward, upper backward, block backward, upper write-back."""
        out = (C.c_double * 5)()
        _check(lib().pdf_time_solve_parts(self.h, reps, out), self.h)
        return list(out)

    def time_phase(self, phase, reps=10):
        """(ms per repetition, algorithmic bytes) of one phase run in isolation."""
        ms = C.c_double()
        by = C.c_double()
        _check(lib().pdf_time_phase(self.h, phase, reps, C.byref(ms), C.byref(by)), self.h)
        return ms.value, by.value

    def frame_capture(self, slot):
        """Start an asynchronous copy of q into pinned frame buffer `slot`."""
        _check(lib().pdf_frame_capture(self.h, slot), self.h)

    def frame_wait(self, slot):
        """Positions (N, 3) of the copy started by frame_capture(slot)."""
        p = C.POINTER(C.c_double)()
        _check(lib().pdf_frame_wait(self.h, slot, C.byref(p)), self.h)
        return np.ctypeslib.as_array(p, shape=(self.n, 3)).copy()

    def vertices(self, idx):
        """(q, v) of the listed vertices, gathered on the device."""
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        q = np.empty((len(idx), 3))
        v = np.empty((len(idx), 3))
        _check(lib().pdf_get_vertices(self.h, _ptr(idx), len(idx), _ptr(q), _ptr(v)), self.h)
        return q, v

    def alart_curnier_trace(self):
        """Per-iteration (tangential, |normal|) AC norms of the last step's
        contacts: array (iterations, contacts + self contacts, 2), and the
        obstacle-contact count."""
        it, nc, ns = C.c_int32(), C.c_int32(), C.c_int32()
        _check(lib().pdf_get_alart_curnier_trace(self.h, None, 0, C.byref(it), C.byref(nc), C.byref(ns)), self.h)
        out = np.zeros((it.value, nc.value + ns.value, 2))
        _check(lib().pdf_get_alart_curnier_trace(self.h, _ptr(out), out.size, C.byref(it), C.byref(nc),
                                                 C.byref(ns)), self.h)
        return out, nc.value

    def residual_history(self):
        n = C.c_int32()
        lib().pdf_get_residual_history(self.h, None, 0, C.byref(n))
        out = np.zeros(max(1, n.value))
        lib().pdf_get_residual_history(self.h, _ptr(out), n.value, C.byref(n))
        return out[:n.value]


    # ---- learned warm start ------------------------------------------------
    def mlp_set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(lib().pdf_mlp_set_weights(self.h, _ptr(w), w.size), self.h)

    def mlp_get_weights(self):
        w = np.zeros(abi.MLP_PARAMS, dtype=np.float32)
        _check(lib().pdf_mlp_get_weights(self.h, _ptr(w), w.size), self.h)
        return w

    def mlp_log(self, capacity):
        """Start (or restart, empty) the per-contact sample log; 0 stops it."""
        _check(lib().pdf_mlp_log(self.h, capacity), self.h)

    def mlp_samples(self):
        n = C.c_int32()
        _check(lib().pdf_mlp_samples(self.h, None, None, 0, C.byref(n)), self.h)
        X = np.zeros((max(1, n.value), abi.MLP_IN), dtype=np.float32)
        T = np.zeros((max(1, n.value), abi.MLP_OUT), dtype=np.float32)
        _check(lib().pdf_mlp_samples(self.h, _ptr(X), _ptr(T), n.value, C.byref(n)), self.h)
        return X[:n.value], T[:n.value]

    def mlp_train(self, epochs=20, batch=4096, lr=1e-3, seed=0):
        """Train the handle's weights on its logged samples on the GPU; (train, held-out) loss."""
        tl, vl = C.c_double(), C.c_double()
        _check(lib().pdf_mlp_train(self.h, epochs, batch, lr, seed, C.byref(tl), C.byref(vl)), self.h)
        return tl.value, vl.value


def mlp_init(seed=0):
    w = np.zeros(abi.MLP_PARAMS, dtype=np.float32)
    _check(lib().pdf_mlp_init(_ptr(w), seed))
    return w


def mlp_save(path, w):
    w = np.ascontiguousarray(w, dtype=np.float32)
    _check(lib().pdf_mlp_save(str(path).encode(), _ptr(w)))


def mlp_load(path):
    w = np.zeros(abi.MLP_PARAMS, dtype=np.float32)
    _check(lib().pdf_mlp_load(str(path).encode(), _ptr(w)))
    return w


def mlp_forward(w, X, device=0):
    """BF16 tensor-core forward of the warm-start MLP on the GPU."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    Y = np.zeros((X.shape[0], abi.MLP_OUT), dtype=np.float32)
    _check(lib().pdf_mlp_forward(_ptr(w), _ptr(X), X.shape[0], _ptr(Y), device))
    return Y


def mlp_gradient(w, X, T, device=0):
    """(loss, gradient) of the mean squared error, GPU backward kernels."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    T = np.ascontiguousarray(T, dtype=np.float32)
    g = np.zeros(abi.MLP_PARAMS, dtype=np.float32)
    loss = C.c_double()
    _check(lib().pdf_mlp_gradient(_ptr(w), _ptr(X), _ptr(T), X.shape[0], _ptr(g), C.byref(loss), device))
    return loss.value, g


def mlp_fit(w, X, T, epochs=20, batch=4096, lr=1e-3, seed=0, device=0):
    """Adam training on the GPU; returns (weights, train loss, held-out loss)."""
    w = np.array(w, dtype=np.float32, copy=True)
    X = np.ascontiguousarray(X, dtype=np.float32)
    T = np.ascontiguousarray(T, dtype=np.float32)
    tl, vl = C.c_double(), C.c_double()
    _check(lib().pdf_mlp_fit(_ptr(w), _ptr(X), _ptr(T), X.shape[0], epochs, batch, lr, seed, device,
                             C.byref(tl), C.byref(vl)))
    return w, tl.value, vl.value


def load_log(path):
    """The scene JSON's "log" entries: [(kind, vertex indices)] with kind
    "position" or "velocity" (getLogCallBacksFromJSONDocument)."""
    h = C.c_void_p()
    _check(lib().pdf_log_load_json(os.fsencode(path), C.byref(h)))
    try:
        n = C.c_int32()
        ent = C.POINTER(abi.pdf_log_entry)()
        _check(lib().pdf_log_view(h, C.byref(n), C.byref(ent)))
        names = {abi.PDF_LOG_POSITION: "position", abi.PDF_LOG_VELOCITY: "velocity"}
        return [(names[ent[k].kind], [ent[k].vertices[i] for i in range(ent[k].n_vertices)])
                for k in range(n.value)]
    finally:
        lib().pdf_log_free(h)


def getSceneFromJSONFileName(path):
    """Mirror of getSceneFromJSONFileName (src/scene_building.cpp:41-47)."""
    return LoadedScene(path)


def getSimulationParametersFromJSONFileName(path):
    """Mirror of getSimulationParametersFromJSONFileName (src/simulation_building.cpp:29-35)."""
    return load_params(path)[0]


def getSimulation(scene, params):
    """Mirror of getSimulation (src/simulation_building.cpp:80-98)."""
    return Simulation(scene, params)


def factor_check(scene, params, b):
    """Host emulation of the device solve on the tiled factor layout (no GPU)."""
    d = scene.desc()
    bb = np.ascontiguousarray(b, dtype=np.float64)
    x = np.empty_like(bb)
    _check(lib().pdf_factor_check(C.byref(d), C.byref(params), _ptr(bb), _ptr(x)))
    return x


def detect_candidates(positions, triangles, tolerance, device=0, cap=None):
    """Vertex-triangle box candidates of one mesh, sorted (vertex, triangle)."""
    pos = np.ascontiguousarray(positions, dtype=np.float64)
    tris = np.ascontiguousarray(triangles, dtype=np.int32)
    n = C.c_int32()
    if cap is None:
        cap = 64 * len(pos) + 1024
    out = np.zeros((cap, 2), dtype=np.int32)
    _check(lib().pdf_detect_candidates(_ptr(pos), len(pos), _ptr(tris), len(tris), tolerance,
                                       _ptr(out), cap, C.byref(n), device))
    return out[:n.value]


def detect_self_collisions(positions, triangles, tolerance, device=0):
    """Self collisions (greedy node-node pairing) of one mesh."""
    pos = np.ascontiguousarray(positions, dtype=np.float64)
    tris = np.ascontiguousarray(triangles, dtype=np.int32)
    n = C.c_int32()
    cap = 2 * len(pos) + 16
    arr = (abi.pdf_contact * cap)()
    _check(lib().pdf_detect_self_collisions(_ptr(pos), len(pos), _ptr(tris), len(tris), tolerance,
                                            arr, cap, C.byref(n), device))
    return abi.contacts_to_numpy(arr, n.value)
