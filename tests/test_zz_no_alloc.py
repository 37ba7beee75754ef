"""The allocation-free candidate detection entry point.

pdf_detect_candidates_noalloc exists for callers that cannot allocate device
memory when they need candidate pairs (a host framework's memory pool, a
real-time loop with a fixed memory budget, an allocator that is not the CUDA
runtime's): its workspace is one fixed device array inside the library.  This
test calls it through the C ABI on device buffers, twice in a row (the second
call reuses the array the first one left behind), and checks both results
against the allocating entry point pdf_detect_candidates.  Candidate pairs are
integers, so the comparison is exact.
"""
import ctypes as C

import numpy as np
import pytest

from climatenet_b200 import native, scenes

pytestmark = pytest.mark.gpu


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


def test_noalloc_candidates_match_allocating_entry_point():
    import torch
    pos, tris = _layered()
    tol = 1.5e-3
    expected = native.detect_candidates(pos, tris, tol)
    assert expected.shape[0] > 0
    dev = torch.device("cuda:0")
    torch.cuda.set_device(0)
    dpos = torch.from_numpy(pos).to(dev)
    dtri = torch.from_numpy(tris).to(dev)
    cap = expected.shape[0] + 64
    L = native.lib()
    for call in range(2):
        out = torch.full((cap, 2), -1, dtype=torch.int32, device=dev)
        n = C.c_int32(-1)
        torch.cuda.synchronize()
        st = L.pdf_detect_candidates_noalloc(C.c_void_p(dpos.data_ptr()), len(pos), C.c_void_p(dtri.data_ptr()),
                                             len(tris), tol, C.c_void_p(out.data_ptr()), cap, C.byref(n), None)
        assert st == 0, native.lib().pdf_global_error()
        assert n.value == expected.shape[0], (call, n.value)
        got = out[:n.value].cpu().numpy()
        assert np.array_equal(got, expected), call
