"""Regenerates the committed golden fixtures from the reference checkout.

Run where the reference source tree exists, with its root as the only
argument; the fixtures it writes are small JSON files that the tests read on
any machine.

  analytic_incline.json: the two OBJ meshes of the reference's Figure-5
  known-answer scene (mesh/analytic/cloth.obj and support.obj, coordinates
  rounded through float as the reference's OBJ reader does) and the scene
  parameters of scenes/analytic.json.  The closed-form motion it is checked
  against is restated in tests/test_oracle_kat.py.
"""
import json
import os
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_fixtures.py <reference root>")
REF = sys.argv[1]
HERE = os.path.dirname(os.path.abspath(__file__))


def read_obj(path):
    V, F = [], []
    for line in open(path):
        t = line.split()
        if not t:
            continue
        if t[0] == "v":
            V.append([float(np.float32(float(x))) for x in t[1:4]])
        elif t[0] == "f":
            F.append([int(x.split("/")[0]) - 1 for x in t[1:4]])
    return V, F


def main():
    cv, cf = read_obj(os.path.join(REF, "mesh/analytic/cloth.obj"))
    sv, sf = read_obj(os.path.join(REF, "mesh/analytic/support.obj"))
    scene = json.load(open(os.path.join(REF, "scenes/analytic.json")))
    out = {
        "source": "mesh/analytic/{cloth,support}.obj and scenes/analytic.json of the reference",
        "cloth_vertices": cv, "cloth_triangles": cf,
        "support_vertices": sv, "support_triangles": sf,
        "parameters": scene["Parameters"],
        "mesh": {k: v for k, v in scene["Meshes"][0].items() if k != "Obj filename"},
        "obstacle": {k: v for k, v in scene["Obstacles"][0].items() if k != "Path"},
        "friction": scene["Friction coefficients"],
    }
    with open(os.path.join(HERE, "analytic_incline.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote analytic_incline.json")


if __name__ == "__main__":
    main()
