"""Bounded device waits: a dependency that is never satisfied ends in a clean
error, not a hang.

The supernodal sweeps wait (bounded polls of a completion counter) for the
supernodes an item depends on.  pdf_check_wait_timeout runs one solve whose
targets lie one solve ahead of the counters, so that no wait can be
satisfied, with a short poll limit.  Every wait must give up, the call must
return PDF_DEVICE_TIMEOUT, and the GPU context must stay usable: a fresh
handle on the same device then steps exactly like the CPU oracle.
"""
import numpy as np
import pytest

from climatenet_b200 import abi, native, scenes
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def _scene():
    return scenes.cloth_on_sphere(n=40, side=1.0, z=-0.2455, mu=0.3, sphere_center=(0, 0, -0.5),
                                  sphere_radius=0.25, pins=True)


def test_unsatisfiable_dependency_times_out_then_a_fresh_handle_steps():
    import torch
    p = abi.params(time_step=5e-3, iterations=10)
    g = native.Simulation(_scene(), p)
    st = native.lib().pdf_check_wait_timeout(g.h, 200)
    assert st == abi.PDF_DEVICE_TIMEOUT, native.lib().pdf_last_error(g.h)
    g.close()
    torch.cuda.synchronize()   # the context still answers
    s = _scene()
    g2 = native.Simulation(s, p)
    o = Oracle(s, p)
    rep = g2.step(3)
    o.step(3)
    qg, vg = g2.state()
    qo, vo = o.state()
    assert rep.n_contacts > 0
    assert np.abs(qg - qo).max() <= 1e-6 * np.abs(qo).max()
    assert np.abs(vg - vo).max() <= 1e-6 * max(np.abs(vo).max(), 1e-12)
