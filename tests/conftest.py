import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle and the product library once per session."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "climatenet_b200")], check=True)


def load_incline():
    """The reference's Figure-5 known-answer scene (committed fixture)."""
    from climatenet_b200 import abi, scenes
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "analytic_incline.json")))
    s = scenes.Scene(friction=g["friction"])
    m = g["mesh"]
    s.add_mesh(np.array(g["cloth_vertices"]), np.array(g["cloth_triangles"]),
               area_density=m["Area Density"], bending=m["Bending"], stretching=m["Stretching"])
    s.add_mesh_obstacle(np.array(g["support_vertices"]), np.array(g["support_triangles"]),
                        g["obstacle"]["Threshold"])
    P = g["parameters"]
    p = abi.params(time_step=P["Timestep"], iterations=P["LocalGlobal"], gravity=P["Gravity"])
    return s, p, P


def incline_closed_form(t, g=9.81, angle=np.pi / 4, h0=0.2, mu=0.1, support=0.0):
    """Closed-form sliding motion of replicability/analytic_example_data_processing.py:53-147
    (free fall, inelastic impact with friction, then constant acceleration along
    the incline).  Returns (speed, height)."""
    ti = np.sqrt(2 * (h0 - support) / g)
    if t < ti:
        return g * t, h0 - 0.5 * g * t * t
    va = g * ti * (np.cos(angle) - np.sin(angle) * mu)
    a = g * (np.sin(angle) - np.cos(angle) * mu)
    return va + a * (t - ti), support - np.sin(angle) * (va * (t - ti) + 0.5 * a * (t - ti) ** 2)
