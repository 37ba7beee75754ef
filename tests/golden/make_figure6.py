"""Generate tests/golden/figure6_oracle_ac.json: the Alart-Curnier convergence
of the reference's Figure-6 scene, computed by the FP64 CPU oracle.

The scene is the reference's own convergence demonstration:
replicability/scenes/Square1/iterations_300.json (run by
replicability/figure_6.sh:5), a 5,988-vertex drape on a key-framed rotating
sphere ("Moving Mesh", 200 OBJ key frames) above a plane, 300 PD iterations
per step, mu 0.1.  replicability/alart_curnier_data_processing.py:9-95 reads
the per-contact tangential and normal Alart-Curnier norms that the
PRINT_ALART_CURNIER_ERROR build prints every iteration (SFE:720-752), keeps
the steps 50, 100, 200 and 300 ("Time Step: i" lines, i from 0,
src/main.cpp:86-90) and plots, per iteration, the mean over the step's
contacts.  This script computes the same means with the oracle and stores
them with the contact counts.

Usage (reads the reference's scene and meshes, so it runs where the reference
tree exists; the output fixture travels with the repository):

    python tests/golden/make_figure6.py <reference root> [--steps 300]
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from climatenet_b200 import native  # noqa: E402  (JSON front end: host code only)
from oracle import oracle as orc  # noqa: E402

READ_STEPS = (50, 100, 200, 300)   # alart_curnier_data_processing.py:14


def run(reference_root, last_step, read_steps):
    cwd = os.getcwd()
    os.chdir(os.path.join(reference_root, "replicability"))   # figure_6.sh runs from there
    try:
        js = "scenes/Square1/iterations_300.json"
        scene = native.LoadedScene(js)
        params, frames, spf = native.load_params(js)
        sim = orc.Oracle(scene, params)
    finally:
        os.chdir(cwd)
    sim.trace_alart_curnier(True)
    out = {}
    t0 = time.time()
    for i in range(last_step + 1):
        rep = sim.step(1)
        if i in read_steps:
            tr, nc = sim.alart_curnier_trace()
            obst = tr[:, :nc, :]
            out[str(i)] = {
                "contacts": int(nc),
                "iterations": int(tr.shape[0]),
                "mean_tangential": obst[:, :, 0].mean(axis=1).tolist() if nc else [],
                "mean_normal": obst[:, :, 1].mean(axis=1).tolist() if nc else [],
                "max_tangential": obst[:, :, 0].max(axis=1).tolist() if nc else [],
                "max_normal": obst[:, :, 1].max(axis=1).tolist() if nc else [],
            }
            print("step %d: %d contacts, mean T %.3e -> %.3e, mean N %.3e -> %.3e (%.0f s)" % (
                i, nc, out[str(i)]["mean_tangential"][0], out[str(i)]["mean_tangential"][-1],
                out[str(i)]["mean_normal"][0], out[str(i)]["mean_normal"][-1], time.time() - t0),
                flush=True)
        elif rep.n_contacts and i % 25 == 0:
            print("step %d: %d contacts (%.0f s)" % (i, rep.n_contacts, time.time() - t0), flush=True)
    meta = {"scene": "replicability/scenes/Square1/iterations_300.json",
            "vertices": int(scene.n_vertices), "pd_iterations": int(params.local_global_iterations),
            "time_step": params.time_step, "steps_run": last_step + 1,
            "generator": "tests/golden/make_figure6.py (FP64 CPU oracle)"}
    return {"meta": meta, "steps": out}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("reference_root", help="root of the reference source tree")
    ap.add_argument("--steps", type=int, default=max(READ_STEPS))
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden", "figure6_oracle_ac.json"))
    a = ap.parse_args()
    res = run(a.reference_root, a.steps, set(s for s in READ_STEPS if s <= a.steps))
    with open(a.out, "w") as f:
        json.dump(res, f)
    print("wrote", a.out)


if __name__ == "__main__":
    main()
