"""The C ABI from plain C (CPU): tests/c_harness.c compiles as C99 against
include/topgpu.h, links libtopgpu.so and reports the same mesh, BC and model
file results as the Python bindings."""
import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from top_gpu_on_matlab_b200.fea import Mesh
from top_gpu_on_matlab_b200.topvoxel import node_index, write_topvoxel

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c_harness_matches_python(tmp_path):
    lib_dir = ROOT / "top_gpu_on_matlab_b200"
    exe = tmp_path / "harness"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "c_harness.c"), "-L", str(lib_dir), "-ltopgpu",
                    "-Wl,-rpath," + str(lib_dir), "-o", str(exe)], check=True)
    shape = (6, 10, 5)
    ys, zs = np.meshgrid(np.arange(7), np.arange(6), indexing="ij")
    fix = np.column_stack([node_index(ys.ravel(), 0, zs.ravel(), shape), np.ones((ys.size, 3), int)])
    load = np.array([[node_index(3, 10, 0, shape), 0.0, 0.0, -1.0]])
    path = tmp_path / "m.TopVoxel"
    write_topvoxel(path, np.ones(shape, bool), fix, [load], passive=[1, 2, 7])
    out = subprocess.run([str(exe), str(path)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    d = json.loads(out.stdout)

    m = Mesh(np.ones((8, 16, 8), bool))
    m.apply_optcase(1)
    info = m.info()
    assert d["version"] == 1 and d["levels"] == len(info)
    assert d["Ne"] == info[0]["numElements"] and d["Nn"] == info[0]["numNodes"]
    assert d["nFix"] == m.get(0, "fixingCond").size and d["nF"] == m.get(0, "F").size
    assert d["nEleMapBack"] == m.get(0, "eleMapBack").size
    assert d["Fsum"] == pytest.approx(float(m.get(0, "F").sum()), abs=1e-12)
    assert d["smallBufferRefused"] == 1 and d["unknownName"] != 0
    f = Mesh.from_topvoxel(path)
    assert d["file"]["nPassive"] == f.passive_elements.size == 3
    assert tuple(d["file"]["resolution"]) == f.shape == shape
