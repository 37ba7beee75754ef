"""The product's factorisation and tiled sweep layout, checked on the CPU:
a host emulation of the two device sweeps (same work items and index
arithmetic, every index bounds-checked) solves the global-step system, and
the result is compared with the oracle's independent sparse Cholesky."""
import numpy as np
import pytest

from climatenet_b200 import abi, native, scenes
from oracle.oracle import Oracle


@pytest.mark.parametrize("n,layers", [(12, 1), (30, 1), (40, 3), (90, 1), (160, 1)])
def test_tiled_solve_matches_oracle(n, layers):
    s = scenes.cloth_on_sphere(n=n, layers=layers, pins=(layers == 1))
    p = abi.params(time_step=2e-3, iterations=5)
    rng = np.random.default_rng(n)
    b = rng.standard_normal((s.n_vertices, 3))
    x = native.factor_check(s, p, b)
    o = Oracle(s, p)
    xo = o.solve(b)
    assert np.abs(x - xo).max() <= 1e-9 * np.abs(xo).max()
    # and it really solves the system
    A = o.lhs()
    r = A @ x - b
    assert np.abs(r).max() <= 1e-9 * np.abs(b).max()
