"""Fixed capacities of the step path are reported, not silently truncated.

Self-collision detection keeps at most 32 candidate triangles per vertex
before the closest-point filter.  Twelve flat layers 0.2 mm apart under a
self-collision tolerance of 1 mm put every interior vertex's query box
(half-width 1.1 mm) over the triangles of about ten other layers, far more
than 32 candidates: pdf_step must return PDF_CAPACITY_EXCEEDED with the
candidate message, and the stand-alone detection (no per-vertex limit) must
see those candidates.
"""
import numpy as np
import pytest

from climatenet_b200 import abi, native, scenes

pytestmark = pytest.mark.gpu


def stacked(layers=12, gap=2e-4, n=10, side=0.1):
    P, T = [], []
    for k in range(layers):
        p, t = scenes.grid_mesh(n, side, z=k * gap)
        P.append(p)
        T.append(t + k * n * n)
    return np.concatenate(P), np.concatenate(T).astype(np.int32)


def test_more_than_32_candidates_per_vertex_is_reported():
    pos, tris = stacked()
    cand = native.detect_candidates(pos, tris, 1e-3)
    per_vertex = np.bincount(cand[:, 0], minlength=len(pos))
    assert per_vertex.max() > 32
    s = scenes.Scene(friction=((0.3,),))
    s.add_mesh(pos, tris, area_density=0.1, bending=1e-2, stretching=1e3)
    g = native.Simulation(s, abi.params(time_step=1e-3, iterations=5, self_collision=True, self_tol=1e-3))
    with pytest.raises(native.PdfError) as e:
        g.step(1)
    assert e.value.status == abi.PDF_CAPACITY_EXCEEDED
    assert "32 self-collision candidates" in str(e.value)
