"""The allocation-free candidate detection entry point.

pdf_detect_candidates_noalloc exists for callers that cannot allocate device
memory when they need candidate pairs (a host framework's memory pool, a
real-time loop with a fixed memory budget, an allocator that is not the CUDA
runtime's): its workspace is one fixed device array inside the library.  These
tests call it through the C ABI on device buffers.  The first one makes two
calls in a row (the second reuses the array the first left behind) and checks
both results against the allocating entry point pdf_detect_candidates and
against the CPU oracle's candidate set.  Candidate pairs are integers, so every
comparison is exact.  The others check the documented limits: more triangles
than the array holds, and more pairs than the caller's capacity, both return
PDF_CAPACITY_EXCEEDED and leave the output untouched.
"""
import ctypes as C

import numpy as np
import pytest

from climatenet_b200 import abi, native, scenes
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

MAX_TRIANGLES = 65536   # the entry point's documented triangle limit


def _layered(n=40, layers=3, gap=0.0009, side=0.5, seed=11):
    rng = np.random.default_rng(seed)
    P, T = [], []
    for k in range(layers):
        p, t = scenes.grid_mesh(n, side, z=k * gap)
        p[:, :2] += 0.002 * rng.standard_normal((len(p), 2))
        p[:, 2] += 0.0003 * rng.standard_normal(len(p))
        P.append(p)
        T.append(t + k * n * n)
    return np.concatenate(P), np.concatenate(T).astype(np.int32)


def _call(pos, tris, tol, cap):
    """One call on device copies of pos / tris; returns (status, n, pairs)."""
    import torch
    dev = torch.device("cuda:0")
    torch.cuda.set_device(0)
    dpos = torch.from_numpy(np.ascontiguousarray(pos)).to(dev)
    dtri = torch.from_numpy(np.ascontiguousarray(tris)).to(dev)
    out = torch.full((max(cap, 1), 2), -1, dtype=torch.int32, device=dev)
    n = C.c_int32(-1)
    torch.cuda.synchronize()
    st = native.lib().pdf_detect_candidates_noalloc(C.c_void_p(dpos.data_ptr()), len(pos),
                                                    C.c_void_p(dtri.data_ptr()), len(tris), tol,
                                                    C.c_void_p(out.data_ptr()), cap, C.byref(n), None)
    return st, n.value, out.cpu().numpy()


def test_noalloc_candidates_match_allocating_entry_point_and_oracle():
    pos, tris = _layered()
    tol = 1.5e-3
    expected = native.detect_candidates(pos, tris, tol)
    oracle_set = orc.self_candidates(pos, tris, tol)
    assert expected.shape[0] > 0
    assert np.array_equal(expected, oracle_set)
    cap = expected.shape[0] + 64
    for call in range(2):
        st, n, out = _call(pos, tris, tol, cap)
        assert st == 0, native.lib().pdf_global_error()
        assert n == expected.shape[0], (call, n)
        assert np.array_equal(out[:n], expected), call
        assert np.array_equal(out[:n], oracle_set), call
        assert (out[n:] == -1).all(), call


def test_noalloc_rejects_more_triangles_than_the_array_holds():
    pos, tris = scenes.grid_mesh(183, 1.0)          # 66,248 triangles
    tris = tris[:MAX_TRIANGLES + 1].astype(np.int32)
    st, n, out = _call(pos, tris, 1e-3, 1024)
    assert st == abi.PDF_CAPACITY_EXCEEDED
    assert (out == -1).all()
    # the limit itself is accepted
    st, n, out = _call(pos, tris[:MAX_TRIANGLES], 1e-3, 64 * len(pos))
    assert st == 0, native.lib().pdf_global_error()
    assert n == native.detect_candidates(pos, tris[:MAX_TRIANGLES], 1e-3).shape[0]


def test_noalloc_reports_the_count_when_the_output_is_too_small():
    pos, tris = _layered(n=24)
    tol = 1.5e-3
    expected = native.detect_candidates(pos, tris, tol)
    assert expected.shape[0] > 10
    st, n, out = _call(pos, tris, tol, expected.shape[0] - 1)
    assert st == abi.PDF_CAPACITY_EXCEEDED
    assert n == expected.shape[0]
    assert (out == -1).all()
