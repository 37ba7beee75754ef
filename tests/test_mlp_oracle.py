"""Learned warm start, CPU side: the FP64 MLP oracle, the bfloat16 emulation
of the tensor-core forward, the contact features and the warm-started first
iteration of the CPU oracle (known answers on a cloth resting on a plane).
"""
import numpy as np
import pytest

from climatenet_b200 import abi, native, scenes
from oracle import mlp_oracle as M
from oracle.oracle import Oracle, OracleError, mlp_forward_bf16

G = 9.81


def plane_scene(n=8, mu=0.2, z=0.005):
    """A flat n x n cloth 5 mm above the plane z = 0 (inside its 1.5 cm margin)."""
    s = scenes.Scene(friction=((mu,),))
    p, t = scenes.grid_mesh(n, 0.5, z=z)
    s.add_mesh(p, t)
    s.add_plane((0.0, 0.0, 0.0), (0.0, 0.0, 1.0))
    return s


def constant_weights(y):
    """A network whose output is the constant y (all weights 0, b3 = y)."""
    w = np.zeros(abi.MLP_PARAMS, dtype=np.float32)
    w[-3:] = y
    return w


def test_param_count():
    assert M.N_PARAMS == abi.MLP_PARAMS == native.lib().pdf_mlp_param_count() == 5059


def test_fp64_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    w = rng.normal(0, 0.3, M.N_PARAMS)
    X = rng.normal(0, 1, (40, M.IN))
    T = rng.normal(0, 1, (40, M.OUT))
    _, g = M.loss_and_grad(w, X, T)
    eps = 1e-6
    for i in rng.choice(M.N_PARAMS, 40, replace=False):
        e = np.zeros(M.N_PARAMS)
        e[i] = eps
        fd = (M.loss_and_grad(w + e, X, T)[0] - M.loss_and_grad(w - e, X, T)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i]))


def test_bf16_emulation_close_to_fp64():
    rng = np.random.default_rng(2)
    w = native.mlp_init(seed=3)
    X = rng.normal(0, 1, (500, M.IN)).astype(np.float32)
    Y = mlp_forward_bf16(w, X)
    Y64 = M.forward(w, X)
    # three layers of bfloat16 rounding (2^-9 relative each)
    assert np.abs(Y - Y64).max() <= 2e-2 * np.abs(Y64).max()
    assert np.abs(Y - Y64).max() > 0  # the rounding is really emulated


def test_init_is_seeded_and_he_scaled():
    a, b, c = native.mlp_init(5), native.mlp_init(5), native.mlp_init(6)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    W1 = M.unpack(a)["W1"]
    assert 0.5 < W1.std() / np.sqrt(2.0 / M.IN) < 1.5


def test_weights_file_round_trip(tmp_path):
    w = native.mlp_init(7)
    native.mlp_save(tmp_path / "w.bin", w)
    assert np.array_equal(native.mlp_load(tmp_path / "w.bin"), w)
    (tmp_path / "bad.bin").write_bytes(b"not a weights file")
    with pytest.raises(native.PdfError):
        native.mlp_load(tmp_path / "bad.bin")


def test_features_and_targets_known_answer():
    """Cloth at rest 5 mm above a plane: the predictor velocity is g dt straight
    into the plane and the converged force stops it, r = m |g| dt n."""
    mu, dt = 0.2, 2e-3
    s = plane_scene(mu=mu)
    o = Oracle(s, abi.params(time_step=dt, iterations=5))
    o.mlp_log(10000)
    o.step(2)
    X, T = o.mlp_samples()
    n = s.n_vertices
    assert X.shape == (2 * n, 10)
    first, second = X[:n], X[n:]
    np.testing.assert_allclose(first[:, 0], -1.0, rtol=1e-6)
    np.testing.assert_allclose(first[:, 1:3], 0.0, atol=1e-6)
    np.testing.assert_allclose(first[:, 3], 0.5, rtol=1e-6)
    np.testing.assert_allclose(first[:, 4:7], 0.0, atol=0)  # no previous step
    np.testing.assert_allclose(first[:, 7], mu, rtol=1e-7)
    np.testing.assert_allclose(first[:, 8], -1.0, rtol=1e-7)
    np.testing.assert_allclose(first[:, 9], 1.0)
    np.testing.assert_allclose(T[:n, 0], 1.0, rtol=1e-6)
    np.testing.assert_allclose(T[:n, 1:], 0.0, atol=1e-6)
    # second step: the previous impulse, in the contact frame, is (1, 0, 0)
    np.testing.assert_allclose(second[:, 4], 1.0, rtol=1e-6)
    np.testing.assert_allclose(second[:, 5:7], 0.0, atol=1e-6)


# contact frame on the plane: n = +z, t = n x e_x = +y, b = n x t = -x
@pytest.mark.parametrize("y,v_over_gdt", [
    ((0.5, 0.0, 0.0), (0.0, 0.0, -0.5)),
    ((0.5, 0.3, 0.0), (0.0, 0.1, -0.5)),   # tangential part clamped to mu r_N = 0.1
    ((0.5, 0.0, -0.05), (0.05, 0.0, -0.5)),  # inside the cone: kept
    ((-1.0, 0.0, 0.0), (0.0, 0.0, -1.0)),  # predicted separation: no force
])
def test_warm_start_first_iteration_known_answer(y, v_over_gdt):
    """One PD iteration with a constant prediction y: the cloth translates
    rigidly with v = t_n + B cone(y) |g| dt (mu = 0.2)."""
    dt = 2e-3
    s = plane_scene(mu=0.2)
    o = Oracle(s, abi.params(time_step=dt, iterations=1, warm_start=abi.PDF_WARM_MLP))
    o.mlp_set_weights(constant_weights(y))
    o.step(1)
    _, v = o.state()
    want = np.array(v_over_gdt) * G * dt
    np.testing.assert_allclose(v, np.broadcast_to(want, v.shape), atol=1e-12)


def test_warm_start_requires_weights():
    o = Oracle(plane_scene(), abi.params(time_step=2e-3, iterations=2, warm_start=abi.PDF_WARM_MLP))
    with pytest.raises(OracleError):
        o.step(1)


def test_standardisation_folds_into_the_weights():
    """Weights trained on standardised data, folded back, give the same
    network on raw features (FP64 oracle forward)."""
    from climatenet_b200 import warmstart
    rng = np.random.default_rng(3)
    X = rng.normal(0, 1, (400, 10)) * np.array([20, 5, 3, 0.1, 300, 80, 80, 0.2, 0.2, 0]) + \
        np.array([-3, 0, 0, 0.9, 100, 0, 0, 0.5, -0.9, 1])
    T = rng.normal(0, 1, (400, 3)) * np.array([300, 100, 90]) + np.array([120, 0, 0])
    mu, sigma, nu, tau = warmstart.normalisation(X, T)
    assert sigma[9] == 1.0 and mu[9] == 0.0  # the bias feature is left alone
    w = native.mlp_init(4).astype(np.float64)
    wf = warmstart.fold(w, mu, sigma, nu, tau)
    y_std = M.forward(w, (X - mu) / sigma) * tau + nu
    y_raw = M.forward(wf.astype(np.float64), X)
    np.testing.assert_allclose(y_raw, y_std, rtol=1e-4, atol=1e-4 * np.abs(y_std).max())
