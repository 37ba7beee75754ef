"""Training pipeline of the learned contact warm start.

The step loop logs one (features, converged local force) sample per obstacle
contact (``Simulation.mlp_log``); this module turns such samples into network
weights with the library's GPU training kernels:

* inputs and targets are standardised (per feature mean / standard deviation,
  the constant bias feature left alone) so that Adam sees unit-scale data;
* the network is trained on the standardised data (``native.mlp_fit``: BF16
  tensor-core forward / backward, Adam, seeded shuffle, 90/10 split);
* the standardisation is folded back into the first and last layers, so the
  step loop evaluates the network on the raw features it computes.

It has no counterpart in the reference, whose contact solver has no learned
component.
"""
import numpy as np

from . import abi, native

_SHAPES = [("W1", (abi.MLP_HIDDEN, abi.MLP_IN)), ("b1", (abi.MLP_HIDDEN,)),
           ("W2", (abi.MLP_HIDDEN, abi.MLP_HIDDEN)), ("b2", (abi.MLP_HIDDEN,)),
           ("W3", (abi.MLP_OUT, abi.MLP_HIDDEN)), ("b3", (abi.MLP_OUT,))]


def unpack(w):
    out, o = {}, 0
    for name, shp in _SHAPES:
        k = int(np.prod(shp))
        out[name] = np.asarray(w[o:o + k], dtype=np.float64).reshape(shp)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in _SHAPES]).astype(np.float32)


def normalisation(X, T):
    """Per-feature (mu, sigma) of the inputs and (nu, tau) of the targets."""
    X = np.asarray(X, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    mu, sigma = X.mean(0), X.std(0)
    const = sigma < 1e-12          # constant features (the bias input)
    mu[const] = 0.0
    sigma[const] = 1.0
    nu, tau = T.mean(0), T.std(0)
    tau[tau < 1e-12] = 1.0
    return mu, sigma, nu, tau


def fold(w, mu, sigma, nu, tau):
    """Weights for raw inputs / outputs from weights trained on
    (x - mu) / sigma -> (t - nu) / tau."""
    p = unpack(w)
    W1 = p["W1"] / sigma[None, :]
    b1 = p["b1"] - (p["W1"] * (mu / sigma)[None, :]).sum(1)
    W3 = tau[:, None] * p["W3"]
    b3 = tau * p["b3"] + nu
    return pack({"W1": W1, "b1": b1, "W2": p["W2"], "b2": p["b2"], "W3": W3, "b3": b3})


def collect(scene, params, steps, capacity=None, return_state=False):
    """Cold-start run of `steps` steps logging every obstacle contact; with
    return_state, also the state (q, v) the run ends in."""
    sim = native.Simulation(scene, params)
    sim.mlp_log(capacity or 4_000_000)
    for _ in range(steps):
        sim.step(1)
    X, T = sim.mlp_samples()
    state = sim.state() if return_state else None
    sim.close()
    return (X, T, state) if return_state else (X, T)


def select(scene, params, candidates, tolerance, start, steps=10, cap=60):
    """Picks among trained weight sets on a validation stretch: each candidate
    drives `steps` iterate-to-tolerance steps from the state `start` (q, v)
    of `scene`, a stretch its training data did not contain.  Returns (index
    of the candidate with the fewest mean PD iterations, lower mean residual
    on ties; per-candidate stats)."""
    p = dict(params)
    p.update(iterations=cap, residual_tolerance=tolerance, warm_start=abi.PDF_WARM_MLP)
    sim = native.Simulation(scene, abi.params(**p))
    stats = []
    for w in candidates:
        sim.mlp_set_weights(w)
        sim.set_state(*start)  # also drops the impulse memory of the previous candidate
        its, res = [], []
        for _ in range(steps):
            r = sim.step(1)
            its.append(r.iterations)
            if r.n_contacts + r.n_self_contacts > 0:
                res.append(r.residual)
        stats.append({"mean_pd_iterations": float(np.mean(its)),
                      "mean_residual": float(np.mean(res)) if res else 0.0})
    sim.close()
    best = min(range(len(candidates)),
               key=lambda k: (stats[k]["mean_pd_iterations"], stats[k]["mean_residual"]))
    return best, stats


def cold_stretch(scene, params, tolerance, start, steps=10, cap=60):
    """The cold-start solver on the stretch `select` uses: mean PD iterations
    and mean residual over `steps` iterate-to-tolerance steps from `start`."""
    p = dict(params)
    p.update(iterations=cap, residual_tolerance=tolerance, warm_start=abi.PDF_WARM_NONE)
    sim = native.Simulation(scene, abi.params(**p))
    sim.set_state(*start)
    its, res = [], []
    for _ in range(steps):
        r = sim.step(1)
        its.append(r.iterations)
        if r.n_contacts + r.n_self_contacts > 0:
            res.append(r.residual)
    sim.close()
    return {"mean_pd_iterations": float(np.mean(its)), "mean_residual": float(np.mean(res)) if res else 0.0}


def train(X, T, epochs=30, batch=4096, lr=2e-3, seed=0, device=0):
    """Weights (raw features in, raw forces out) and the losses, trained on the GPU.

    Returns (weights, info) with info = dict(train_loss, val_loss, samples,
    dropped_nonfinite): the losses are those of the standardised problem (1.0
    = predicting the mean); samples with a non-finite feature or target are
    not trained on and are counted in dropped_nonfinite."""
    X = np.asarray(X)
    T = np.asarray(T)
    # samples with a non-finite feature or target are left out (and counted)
    keep = np.isfinite(X).all(1) & np.isfinite(T).all(1)
    dropped = int(len(X) - keep.sum())
    if dropped:
        X, T = X[keep], T[keep]
    mu, sigma, nu, tau = normalisation(X, T)
    Xn = ((np.asarray(X, dtype=np.float64) - mu) / sigma).astype(np.float32)
    Tn = ((np.asarray(T, dtype=np.float64) - nu) / tau).astype(np.float32)
    w0 = native.mlp_init(seed)
    w, tl, vl = native.mlp_fit(w0, Xn, Tn, epochs=epochs, batch=batch, lr=lr, seed=seed, device=device)
    return fold(w, mu, sigma, nu, tau), dict(train_loss=tl, val_loss=vl, samples=len(X), dropped_nonfinite=dropped)


def judge(scene, params, weights, tolerance, steps=10, warmup=3, cap=60, start=None):
    """The cold-start solver as judge of the learned warm start.

    Runs the scene twice from the same state in iterate-to-tolerance mode
    (`tolerance` on the mean Alart-Curnier residual, at most `cap` PD
    iterations): cold, and with the warm start.  Returns a dict with the mean
    iterations and residuals of both runs and `use`: whether the warm start
    needed fewer iterations (ties go to the cold start, the fallback).
    `params` are abi.params keyword arguments; `start` (q, v), when given, is
    the state both runs restart from after their `warmup` steps."""
    out = {}
    for name, w in (("cold", None), ("warm", weights)):
        p = dict(params)
        p.update(iterations=cap, residual_tolerance=tolerance,
                 warm_start=abi.PDF_WARM_MLP if w is not None else abi.PDF_WARM_NONE)
        sim = native.Simulation(scene, abi.params(**p))
        if w is not None:
            sim.mlp_set_weights(w)
        sim.step(warmup)
        if start is not None:
            sim.set_state(*start)
        its, res = [], []
        for _ in range(steps):
            r = sim.step(1)
            its.append(r.iterations)
            if r.n_contacts + r.n_self_contacts > 0:
                res.append(r.residual)
        sim.close()
        out[name] = {"mean_pd_iterations": float(np.mean(its)),
                     "mean_residual": float(np.mean(res)) if res else 0.0}
    out["use"] = out["warm"]["mean_pd_iterations"] < out["cold"]["mean_pd_iterations"]
    return out
