"""GPU against the FP64 CPU oracle at the benchmark's own shapes.

* 30 x 30 pinned cloth falling from z = 0 onto a sphere of radius 0.25
  (mu 0.3, dt 5e-3, 30 PD iterations), run as specified for its 200 steps:
  positions within 1e-6 relative at every one of the first 10 steps, and the
  drift over the whole run bounded and reported.
* Three stacked 128 x 128 layers (5 mm apart) on a sphere of radius 0.3
  (mu 0.4, self-collision tolerance 1 mm, dt 2.5e-3, 20 PD iterations): over
  the steps where the layers land, the self-contact candidate set, the
  closest-point hits and the greedy pairing of the GPU step are compared bit
  for bit with the oracle's detection on the same start-of-step positions;
  positions within 1e-6 relative over the first 10 steps.
* The 500 x 500 cloth on the rotating sphere (mu 0.5, self-collision 2 mm,
  dt 2e-3, 20 PD iterations): FP64 GPU within 1e-6 of the oracle over 4
  steps, and FP32 + FP64-residual refinement within 1e-6 of both, errors
  reported.
"""
import numpy as np
import pytest

from climatenet_b200 import abi, native, scenes
from oracle import oracle as orc
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_pinned_cloth_30_as_specified():
    s, kw, steps = scenes.workload(1)
    assert steps == 200
    p = abi.params(**kw)
    g = native.Simulation(s, p)
    o = Oracle(s, p)
    worst_first10, worst, contacts_seen = 0.0, 0.0, 0
    for k in range(steps):
        rg = g.step(1)
        ro = o.step(1)
        assert rg.n_contacts == ro.n_contacts, k
        contacts_seen = max(contacts_seen, rg.n_contacts)
        qg, _ = g.state()
        qo, _ = o.state()
        e = rel_err(qg, qo)
        worst = max(worst, e)
        if k < 10:
            worst_first10 = max(worst_first10, e)
    print("30x30 pinned cloth: max rel. position error %.2e over steps 1-10, %.2e over %d steps; "
          "up to %d contacts" % (worst_first10, worst, steps, contacts_seen))
    assert contacts_seen > 0
    assert worst_first10 < 1e-6
    assert worst < 1e-4


def test_three_layers_128_sets_bit_exact():
    s, kw, _ = scenes.workload(2)
    p = abi.params(**kw)
    tris = np.ascontiguousarray(s.tris, dtype=np.int32)
    tol = p.self_collision_tolerance
    g = native.Simulation(s, p)
    o = Oracle(s, p)
    compared, with_self = 0, 0
    for k in range(70):
        q_start, _ = g.state()          # detection runs on start-of-step positions
        rg = g.step(1)
        o.step(1)
        if k < 10:
            qg, _ = g.state()
            qo, _ = o.state()
            assert rel_err(qg, qo) < 1e-6, (k, rel_err(qg, qo))
        if k >= 40 and k % 5 == 0:
            # the step's pairing against the oracle's detection on the same positions
            exp = orc.self_collisions(q_start, tris, tol)
            got = g.self_contacts()
            for key in ("vertex", "partner", "face"):
                assert np.array_equal(got[key], exp[key]), (k, key)
            # candidate boxes and closest-point hits of the stand-alone GPU detection
            assert np.array_equal(native.detect_candidates(q_start, tris, tol),
                                  orc.self_candidates(q_start, tris, tol)), k
            hits = native.detect_self_collisions(q_start, tris, tol)
            for key in ("vertex", "partner", "face"):
                assert np.array_equal(hits[key], exp[key]), (k, key)
            compared += 1
            with_self += rg.n_self_contacts > 0
    print("3 x 128^2 layers: %d steps compared, %d with self contacts" % (compared, with_self))
    assert compared >= 6 and with_self >= 1


def test_cloth_500_fp64_and_fp32_refine_against_oracle():
    s, kw, _ = scenes.workload(3)
    p64 = abi.params(**kw)
    p32 = abi.params(**dict(kw, precision=abi.PDF_FP32_REFINE))
    g64 = native.Simulation(s, p64)
    g32 = native.Simulation(s, p32)
    o = Oracle(s, p64)
    for k in range(4):
        r64 = g64.step(1)
        g32.step(1)
        ro = o.step(1)
        assert r64.n_contacts == ro.n_contacts and r64.n_self_contacts == ro.n_self_contacts, k
        q64, _ = g64.state()
        q32, _ = g32.state()
        qo, _ = o.state()
        e64, e32, e3264 = rel_err(q64, qo), rel_err(q32, qo), rel_err(q32, q64)
        print("500x500 step %d: FP64 vs oracle %.2e, FP32+refine vs oracle %.2e, vs FP64 GPU %.2e"
              % (k + 1, e64, e32, e3264))
        assert e64 < 1e-6
        assert e32 < 1e-6 and e3264 < 1e-6
    assert abs(r64.residual - ro.residual) <= 1e-6 * ro.residual + 1e-14
