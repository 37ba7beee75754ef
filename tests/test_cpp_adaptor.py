"""The C++ front with the reference's simulation-building interface
(include/pdf_simulation.hpp: getSceneFromJSONFileName,
getSimulationParametersFromJSONFileName, getSimulation, step, exportStats),
compiled into a small driver (tests/cpp/adaptor_main.cpp) the way the
reference's main loop uses SimulationBase (src/main.cpp:40-124)."""
import os
import subprocess

import numpy as np
import pytest

from climatenet_b200 import native
from conftest import ROOT
from oracle.oracle import Oracle
from test_cli import grid_scene_json

LIB_DIR = os.path.join(ROOT, "climatenet_b200", "_build")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = tmp_path_factory.mktemp("adaptor") / "adaptor_main"
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "adaptor_main.cpp"), "-o", str(out), "-L", LIB_DIR,
                    "-lpdf_b200", "-Wl,-rpath," + LIB_DIR], check=True)
    return str(out)


def _run(driver, tmp_path, steps):
    js = grid_scene_json(tmp_path, n=9)
    return subprocess.run([driver, str(js), str(steps), str(tmp_path / "q.bin"), str(tmp_path / "stats.txt")],
                          cwd=tmp_path, capture_output=True, text=True, timeout=300), js


def test_adaptor_loads_the_scene_and_reports_a_missing_device(driver, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present: the GPU test drives the adaptor")
    r, _ = _run(driver, tmp_path, 3)
    assert "scene: 81 vertices, 3 frames of 2 steps, 8 PD iterations" in r.stdout, r.stdout + r.stderr
    assert r.returncode == 3, r.stdout + r.stderr
    assert "pdf error 8" in r.stdout


@pytest.mark.gpu
def test_adaptor_steps_like_the_oracle(driver, tmp_path):
    r, js = _run(driver, tmp_path, 6)
    assert r.returncode == 0, r.stdout + r.stderr
    q = np.fromfile(tmp_path / "q.bin", dtype=np.float64).reshape(-1, 3)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        scene = native.LoadedScene(str(js))
        params, _, _ = native.load_params(str(js))
        o = Oracle(scene, params)
    finally:
        os.chdir(cwd)
    o.step(6)
    qo, _ = o.state()
    assert np.abs(q - qo).max() <= 1e-6 * np.abs(qo).max()
    stats = (tmp_path / "stats.txt").read_text()
    for section in ("Cholesky computation time", "Iteration time", "Solver time", "Step time",
                    "RHS friction overhead"):
        assert section in stats
