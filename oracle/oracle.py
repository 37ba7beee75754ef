"""ctypes wrapper of the FP64 CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from climatenet_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build():
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(abi.pdf_scene_desc), C.POINTER(abi.pdf_params), C.POINTER(vp)]
        L.orc_step.argtypes = [vp, C.c_int32, C.POINTER(abi.pdf_step_report)]
        L.orc_get_state.argtypes = [vp, C.c_void_p, C.c_void_p]
        L.orc_set_state.argtypes = [vp, C.c_void_p, C.c_void_p]
        L.orc_get_contacts.argtypes = [vp, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]
        L.orc_get_self_contacts.argtypes = [vp, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]
        L.orc_get_self_levels.argtypes = [vp, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32,
                                          C.POINTER(C.c_int32)]
        L.orc_get_residual_history.argtypes = [vp, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]
        L.orc_trace_alart_curnier.argtypes = [vp, C.c_int32]
        L.orc_get_residual_applied_history.argtypes = [vp, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]
        L.orc_get_alart_curnier_trace.argtypes = [vp, C.c_void_p, C.c_int64, C.POINTER(C.c_int32),
                                                  C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.orc_get_sizes.argtypes = [vp, C.c_void_p]
        L.orc_projections.argtypes = [vp, C.c_void_p, C.c_void_p]
        L.orc_rhs_base.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_last_rhs.argtypes = [vp, C.c_void_p]
        L.orc_solve.argtypes = [vp, C.c_void_p]
        L.orc_lhs_csr.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]
        L.orc_masses.argtypes = [vp, C.c_void_p]
        L.orc_time.argtypes = [vp]
        L.orc_time.restype = C.c_double
        L.orc_last_error.restype = C.c_char_p
        L.orc_destroy.argtypes = [vp]
        L.orc_self_candidates.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_double,
                                          C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]
        L.orc_self_collisions.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_double,
                                          C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]
        L.orc_closest_point.argtypes = [C.c_void_p] * 4 + [C.c_double, C.c_void_p, C.c_void_p]
        L.orc_mlp_set_weights.argtypes = [vp, C.c_void_p, C.c_int32]
        L.orc_mlp_log.argtypes = [vp, C.c_int32]
        L.orc_mlp_samples.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]
        L.orc_mlp_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class OracleError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (abi.STATUS_NAMES.get(status, status), msg))
        self.status = status


class Oracle:
    """FP64 CPU simulation with the reference's step semantics."""

    def __init__(self, scene, params):
        L = lib()
        self._scene = scene
        self._desc = scene.desc()
        self._params = params
        h = C.c_void_p()
        st = L.orc_create(C.byref(self._desc), C.byref(params), C.byref(h))
        if st != 0:
            raise OracleError(st, L.orc_last_error().decode())
        self.h = h
        self.n = scene.n_vertices

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def step(self, n=1):
        rep = abi.pdf_step_report()
        st = lib().orc_step(self.h, n, C.byref(rep))
        if st != 0:
            raise OracleError(st, "step")
        return rep

    def state(self):
        q = np.empty((self.n, 3))
        v = np.empty((self.n, 3))
        lib().orc_get_state(self.h, _ptr(q), _ptr(v))
        return q, v

    def set_state(self, q=None, v=None):
        qa = None if q is None else np.ascontiguousarray(q, dtype=np.float64)
        va = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        lib().orc_set_state(self.h, None if qa is None else _ptr(qa), None if va is None else _ptr(va))

    def residual_applied_history(self):
        """Per iteration of the last step: mean AC norm with the force each
        contact applied (zero after a take-off)."""
        n = C.c_int32()
        lib().orc_get_residual_applied_history(self.h, None, 0, C.byref(n))
        out = np.zeros(max(1, n.value))
        lib().orc_get_residual_applied_history(self.h, _ptr(out), n.value, C.byref(n))
        return out[:n.value]

    def trace_alart_curnier(self, enable=True):
        lib().orc_trace_alart_curnier(self.h, 1 if enable else 0)

    def alart_curnier_trace(self):
        """Per-iteration (tangential, |normal|) AC norms of the last step's
        contacts: array (iterations, contacts + self contacts, 2), and the
        obstacle-contact count (the layout of the product's trace)."""
        it, nc, ns = C.c_int32(), C.c_int32(), C.c_int32()
        lib().orc_get_alart_curnier_trace(self.h, None, 0, C.byref(it), C.byref(nc), C.byref(ns))
        out = np.zeros((it.value, nc.value + ns.value, 2))
        lib().orc_get_alart_curnier_trace(self.h, _ptr(out), out.size, C.byref(it), C.byref(nc),
                                          C.byref(ns))
        return out, nc.value

    def contacts(self):
        n = C.c_int32()
        lib().orc_get_contacts(self.h, None, 0, C.byref(n))
        arr = (abi.pdf_contact * max(1, n.value))()
        lib().orc_get_contacts(self.h, arr, n.value, C.byref(n))
        return abi.contacts_to_numpy(arr, n.value)

    def self_contacts(self):
        n = C.c_int32()
        lib().orc_get_self_contacts(self.h, None, 0, C.byref(n))
        arr = (abi.pdf_contact * max(1, n.value))()
        lib().orc_get_self_contacts(self.h, arr, n.value, C.byref(n))
        return abi.contacts_to_numpy(arr, n.value)

    def self_levels(self):
        nl = C.c_int32()
        lib().orc_get_self_levels(self.h, None, 0, None, 0, C.byref(nl))
        ns = self.self_contacts()["vertex"].shape[0]
        ptr = np.zeros(nl.value + 1, dtype=np.int32)
        order = np.zeros(max(1, ns), dtype=np.int32)
        lib().orc_get_self_levels(self.h, _ptr(ptr), nl.value + 1, _ptr(order), ns, C.byref(nl))
        return ptr, order[:ns]

    def mlp_set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        st = lib().orc_mlp_set_weights(self.h, _ptr(w), w.size)
        if st != 0:
            raise OracleError(st, "weights")

    def mlp_log(self, capacity):
        lib().orc_mlp_log(self.h, capacity)

    def mlp_samples(self):
        n = C.c_int32()
        lib().orc_mlp_samples(self.h, None, None, 0, C.byref(n))
        X = np.zeros((max(1, n.value), abi.MLP_IN), dtype=np.float32)
        T = np.zeros((max(1, n.value), abi.MLP_OUT), dtype=np.float32)
        lib().orc_mlp_samples(self.h, _ptr(X), _ptr(T), n.value, C.byref(n))
        return X[:n.value], T[:n.value]

    def residual_history(self):
        n = C.c_int32()
        lib().orc_get_residual_history(self.h, None, 0, C.byref(n))
        out = np.zeros(max(1, n.value))
        lib().orc_get_residual_history(self.h, _ptr(out), n.value, C.byref(n))
        return out[:n.value]

    def sizes(self):
        s = np.zeros(4, dtype=np.int64)
        lib().orc_get_sizes(self.h, _ptr(s))
        return dict(rows=int(s[0]), nnz_a=int(s[1]), nnz_lhs=int(s[2]), nnz_l=int(s[3]))

    def projections(self, q):
        rows = self.sizes()["rows"]
        p = np.empty((rows, 3))
        q = np.ascontiguousarray(q, dtype=np.float64)
        lib().orc_projections(self.h, _ptr(q), _ptr(p))
        return p

    def rhs_base(self, qn, tn, vk):
        out = np.empty((self.n, 3))
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (qn, tn, vk)]
        lib().orc_rhs_base(self.h, _ptr(a[0]), _ptr(a[1]), _ptr(a[2]), _ptr(out))
        return out

    def last_rhs(self):
        out = np.empty((self.n, 3))
        lib().orc_last_rhs(self.h, _ptr(out))
        return out

    def solve(self, b):
        x = np.ascontiguousarray(b, dtype=np.float64).copy()
        lib().orc_solve(self.h, _ptr(x))
        return x

    def lhs(self):
        import scipy.sparse as sp
        nnz = C.c_int64()
        lib().orc_lhs_csr(self.h, None, None, None, C.byref(nnz))
        rp = np.zeros(self.n + 1, dtype=np.int32)
        col = np.zeros(nnz.value, dtype=np.int32)
        val = np.zeros(nnz.value)
        lib().orc_lhs_csr(self.h, _ptr(rp), _ptr(col), _ptr(val), C.byref(nnz))
        return sp.csr_matrix((val, col, rp), shape=(self.n, self.n))

    def masses(self):
        m = np.empty(self.n)
        lib().orc_masses(self.h, _ptr(m))
        return m

    @property
    def time(self):
        return lib().orc_time(self.h)


def self_candidates(pos, tris, tol):
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    tris = np.ascontiguousarray(tris, dtype=np.int32)
    n = C.c_int32()
    lib().orc_self_candidates(_ptr(pos), len(pos), _ptr(tris), len(tris), tol, None, 0, C.byref(n))
    out = np.zeros((max(1, n.value), 2), dtype=np.int32)
    lib().orc_self_candidates(_ptr(pos), len(pos), _ptr(tris), len(tris), tol, _ptr(out), n.value,
                              C.byref(n))
    return out[:n.value]


def self_collisions(pos, tris, tol):
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    tris = np.ascontiguousarray(tris, dtype=np.int32)
    n = C.c_int32()
    lib().orc_self_collisions(_ptr(pos), len(pos), _ptr(tris), len(tris), tol, None, 0, C.byref(n))
    arr = (abi.pdf_contact * max(1, n.value))()
    lib().orc_self_collisions(_ptr(pos), len(pos), _ptr(tris), len(tris), tol, arr, n.value,
                              C.byref(n))
    return abi.contacts_to_numpy(arr, n.value)


def closest_point(p, a, b, c, tol2):
    arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (p, a, b, c)]
    cp = np.zeros(3)
    bary = np.zeros(3)
    lib().orc_closest_point(*[_ptr(x) for x in arrs], tol2, _ptr(cp), _ptr(bary))
    return cp, bary


def mlp_forward_bf16(w, X):
    """The warm-start MLP with the tensor cores' bfloat16 rounding emulated."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    Y = np.zeros((X.shape[0], abi.MLP_OUT), dtype=np.float32)
    lib().orc_mlp_forward(_ptr(w), _ptr(X), X.shape[0], _ptr(Y))
    return Y
