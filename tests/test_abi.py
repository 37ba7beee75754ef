"""The C ABI without a GPU: every symbol declared in include/pdf.h is exported,
the ctypes mirror has the C layout, and the JSON / OBJ front end (host code)
follows the reference's key spellings, typing rules and errors."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from climatenet_b200 import abi, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pdf.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(pdf_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", native.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (pdf_[a-z0-9_]+)", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    assert len(declared_functions()) >= 20


def test_struct_layout_matches_c(tmp_path):
    structs = ["pdf_obstacle", "pdf_mesh_desc", "pdf_scene_desc", "pdf_params", "pdf_step_report",
               "pdf_stats", "pdf_contact", "pdf_log_entry"]
    prog = ['#include <stdio.h>', '#include "%s"' % HEADER, "int main(void){"]
    for s in structs:
        prog.append('printf("%%s %%zu\\n", "%s", sizeof(%s));' % (s, s))
    prog.append("return 0;}")
    src = tmp_path / "sz.c"
    src.write_text("\n".join(prog))
    exe = tmp_path / "sz"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    sizes = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split("\n")
                 if line)
    for s in structs:
        assert int(sizes[s]) == C.sizeof(getattr(abi, s)), s


def write_scene(tmp_path, params_extra="", mesh_extra="", density="1.0"):
    obj = tmp_path / "cloth.obj"
    obj.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3\nf 1 3 4\n")
    js = tmp_path / "scene.json"
    js.write_text("""{
 "Parameters": {"Frame number": 3, "LocalGlobal": 7, "Timestep": 2e-3, "Type": "friction",
   "Steps per frame": 2, "Self-collision": false, "Self-collision tolerance": 1.0e-2,
   "Gravity": [0.0, 0.0, -9.81] %s},
 "Friction coefficients": [[0.25]],
 "Meshes": [{"Obj filename": "cloth.obj", "Area Density": %s, "Bending": 1e-3,
             "Stretching": 1e2, "Material Identifier": 0 %s}],
 "Obstacles": [{"Type": "Sphere", "Position": [0.0, 0.0, -1.0], "Radius": 0.5,
                "Material Identifier": 0},
               {"Type": "Rotating Sphere", "Position": [0.0, 0.0, -1.0], "Radius": 0.5,
                "Rotation Axe": [0.0, 0.0, 2.0], "Radial Speed": 1.0,
                "Rotation Start Time": 0.0, "Material Identifier": 0}]
}""" % (params_extra, density, mesh_extra))
    return js


def test_json_scene_and_parameters(tmp_path):
    js = write_scene(tmp_path, params_extra=', "Air damping": 0.5')
    sc = native.getSceneFromJSONFileName(str(js))
    d = sc.desc()
    assert d.n_vertices == 4 and d.n_triangles == 2 and d.n_meshes == 1 and d.n_obstacles == 2
    assert d.obstacles[1].type == abi.PDF_OBSTACLE_ROTATING_SPHERE
    assert d.friction[0] == 0.25
    p, frames, spf = native.load_params(str(js))
    assert (p.local_global_iterations, frames, spf) == (7, 3, 2)
    assert p.time_step == 2e-3 and p.air_damping == 0.5 and p.self_collision == 0


def test_air_damping_is_optional(tmp_path):
    p, _, _ = native.load_params(str(write_scene(tmp_path)))
    assert p.air_damping == 0.0


def test_attachment_extension_key(tmp_path):
    js = write_scene(tmp_path, mesh_extra=', "Attachments": [{"Vertex": 3, "Weight": 1e4}]')
    sc = native.getSceneFromJSONFileName(str(js))
    d = sc.desc()
    assert d.n_pins == 1 and d.pin_vertices[0] == 3 and d.pin_weights[0] == 1e4


def test_integer_where_double_required_is_rejected(tmp_path):
    # rapidjson IsDouble() is false for "1": jsonRequireDouble throws
    js = write_scene(tmp_path, density="1")
    with pytest.raises(native.PdfError) as e:
        native.getSceneFromJSONFileName(str(js))
    assert e.value.status == abi.PDF_INVALID_ARG and "type error with key Area Density" in str(e.value)


def test_missing_key_and_malformed_json(tmp_path):
    js = tmp_path / "bad.json"
    js.write_text('{"Meshes": [], "Obstacles": []}')
    with pytest.raises(native.PdfError) as e:
        native.getSceneFromJSONFileName(str(js))
    assert "cannot found key Friction coefficients" in str(e.value)
    js.write_text('{"Friction coefficients": [[0.1]], ')
    with pytest.raises(native.PdfError) as e:
        native.getSceneFromJSONFileName(str(js))
    assert e.value.status == abi.PDF_INVALID_ARG


def test_missing_obj_is_io_error(tmp_path):
    js = write_scene(tmp_path)
    os.remove(tmp_path / "cloth.obj")
    with pytest.raises(native.PdfError) as e:
        native.getSceneFromJSONFileName(str(js))
    assert e.value.status == abi.PDF_IO_ERROR


def test_obj_coordinates_pass_through_float(tmp_path):
    js = write_scene(tmp_path)
    (tmp_path / "cloth.obj").write_text("v 0.1 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3\nf 1 3 4\n")
    sc = native.getSceneFromJSONFileName(str(js))
    d = sc.desc()
    assert d.rest_positions[0] == float(np.float32(0.1)) != 0.1


def test_create_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from climatenet_b200 import scenes
    s = scenes.cloth_on_sphere(n=6)
    with pytest.raises(native.PdfError) as e:
        native.Simulation(s, abi.params())
    assert e.value.status == abi.PDF_NO_DEVICE
