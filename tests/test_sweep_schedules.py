"""Every solve schedule against the FP64 CPU oracle, through the C ABI.

The global solve (SimulationSpeed::solve, the reference's sparse Cholesky
back-substitution) runs on the device under a schedule the autotuner picks at
create: work-item width, subtree-block cut level, and the mode of the
supernodes above the blocks (dependency-driven work items in one launch, or
one launch per elimination-tree level), and the launch shape of the block
kernels (warps per CTA, CTAs per SM, bulk-copy ring depth).  Every schedule
must give the oracle's trajectory: 1e-6 relative on positions and speeds
over 4 steps with contacts (the schedules differ only in
the order of FP64 additions), and identical contact counts.  Pinning a schedule after steps
were taken under a captured CUDA graph must replace the graph's launches.
"""
import numpy as np
import pytest

from climatenet_b200 import abi, native, scenes
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

REL = 1e-6


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def draped(n=60):
    return scenes.cloth_on_sphere(n=n, side=1.0, z=-0.2455, mu=0.3, sphere_center=(0, 0, -0.5),
                                  sphere_radius=0.25, pins=True)


@pytest.fixture(scope="module")
def oracle_run():
    s = draped()
    o = Oracle(s, abi.params(time_step=5e-3, iterations=20))
    traj, counts = [], []
    for _ in range(4):
        r = o.step(1)
        traj.append(o.state())
        counts.append(r.n_contacts)
    assert counts[-1] > 0
    return s, traj, counts


@pytest.mark.parametrize("precision", [abi.PDF_FP64, abi.PDF_FP32_REFINE])
@pytest.mark.parametrize("chunk,cut,mode,shape", [(64, 0, 0, 1), (64, 0, 1, 3), (32, 3, 0, 2), (32, 3, 1, 1),
                                                  (128, 5, 1, 0), (64, 7, 0, 1), (64, 7, 1, 0), (64, 2, 1, 3),
                                                  (64, 3, 1, 4)])
def test_schedule_matches_oracle(oracle_run, chunk, cut, mode, shape, precision):
    s, traj, counts = oracle_run
    g = native.Simulation(s, abi.params(time_step=5e-3, iterations=20, precision=precision))
    g.set_sweep_schedule(chunk, cut, mode, shape)
    st = g.stats()
    assert (st.sweep_chunk, st.sweep_cut_level, st.sweep_upper_mode, st.sweep_block_shape) == (chunk, cut, mode, shape)
    for k in range(4):
        r = g.step(1)
        assert r.n_contacts == counts[k]
        q, v = g.state()
        assert rel_err(q, traj[k][0]) < REL and rel_err(v, traj[k][1]) < REL
    g.close()


def test_schedule_change_replaces_captured_graph(oracle_run):
    s, traj, counts = oracle_run
    g = native.Simulation(s, abi.params(time_step=5e-3, iterations=20, use_graph=1))
    g.set_sweep_schedule(64, 2, 0, 0)
    g.step(2)
    g.set_sweep_schedule(32, 2, 1, 3)
    g.step(2)
    q, v = g.state()
    assert rel_err(q, traj[3][0]) < REL and rel_err(v, traj[3][1]) < REL
    g.close()


def test_schedule_rejects_values_outside_the_tuned_sets(oracle_run):
    s, _, _ = oracle_run
    g = native.Simulation(s, abi.params(time_step=5e-3, iterations=20))
    for args in ((48, 0, 0, 1), (64, 8, 0, 1), (64, -1, 0, 1), (64, 0, 2, 1), (64, 0, 0, 5), (64, 0, 0, -1)):
        with pytest.raises(native.PdfError):
            g.set_sweep_schedule(*args)
    g.close()


def test_schedule_that_does_not_fit_is_rejected():
    """The 500 x 500 cloth's blocks at cut level 7 hold up to 976 columns and
    258 rows outside (FP64: 29.6 KB of vector and 23.4 KB of y slice per
    block besides the slab ring): four CTAs of them do not fit one SM's
    shared memory.  The handle keeps a working schedule (the same cut level,
    dependency-driven upper items, one CTA of 8 warps per SM)."""
    s, pk, _ = scenes.workload(3)
    g = native.Simulation(s, abi.params(**pk))
    with pytest.raises(native.PdfError, match="do not fit"):
        g.set_sweep_schedule(64, 7, 1, 3)
    st = g.stats()
    assert (st.sweep_cut_level, st.sweep_upper_mode, st.sweep_block_shape) == (7, 0, 0)
    r = g.step(1)
    q, _ = g.state()
    assert np.isfinite(q).all() and r.iterations == pk["iterations"]
    g.close()


def test_handles_with_different_schedules_coexist(oracle_run):
    """A kernel's shared-memory limit is process-wide: configuring a second
    handle with a small plan must not break the first handle's larger one
    (its direct launches and its captured graph)."""
    s, traj, counts = oracle_run
    p = abi.params(time_step=5e-3, iterations=20)
    a = native.Simulation(s, p)
    a.set_sweep_schedule(64, 7, 1, 0)  # one CTA of the largest blocks per SM
    a.step(1)
    b = native.Simulation(s, p)
    b.set_sweep_schedule(64, 0, 1, 3)  # four CTAs of the smallest blocks per SM
    b.step(1)
    a.step(3)
    q, v = a.state()
    assert rel_err(q, traj[3][0]) < REL and rel_err(v, traj[3][1]) < REL
    a.close()
    b.close()
