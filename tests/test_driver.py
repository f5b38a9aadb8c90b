"""The TOP_GPU driver's host logic on the CPU (TOP_GPU.m:1-327): folder names
and their _tN suffixes, InitialSettings passed to the solver, the loop's stop
rule, the per-iteration lines, RunLog.log and the result files.  The device
solver is replaced by a stand-in that plays a fixed history."""
import math
import os

import numpy as np
import pytest

from top_gpu_on_matlab_b200 import driver as D
from top_gpu_on_matlab_b200.topvoxel import node_index, write_topvoxel


class ScriptedSolver:
    """fea.Solver's loop interface with a scripted history: change 0.2/k,
    sharpness 0.5/k after iteration k"""

    made = []

    def __init__(self, mesh, **kw):
        self.mesh, self.kw, self.k = mesh, kw, 0
        self.ne = mesh.info()[0]["numElements"] * (64 if mesh.super_element else 1)
        ScriptedSolver.made.append(self)

    def set_passive(self, ids):
        self.passive = np.asarray(ids)

    def opt_begin(self, V0, rMin, nLoop, ft):
        self.prm = (V0, rMin, nLoop, ft)
        return 123.5

    def opt_step(self):
        self.k += 1
        k = self.k
        return dict(c=100.0 / k, vol=0.12, sharp=0.5 / k, cons=1e-9, change=0.2 / k, pcgIts=10 + k,
                    msAssemble=1.0, msSolve=2.0, msOpt=0.5, msFilter=0.25, msTotal=4.0)

    def opt_state(self):
        return self.k, 0.2 / self.k, 0.5 / self.k

    def opt_case_its(self):                      # two load cases splitting the record's count
        return [5, 5 + self.k]

    def design(self):
        x = np.linspace(0.0, 1.0, self.ne)
        return x, x


def test_folder_names():
    assert D.folder_name(np.ones((6, 12, 6), bool), 2, 0.2, math.sqrt(3), 1, 8, 1, 0) == \
        "case2_12x6x6_V0.2_r1.732_ft1_n8_mp1_se0"
    assert D.folder_name("./data/femur.TopVoxel", 1, 0.4, math.sqrt(3), 2, 50, 0, 0) == \
        "femur_V0.4_r1.732_ft2_n50_mp0_se0"


def test_output_path_suffixes(tmp_path):
    a = D.output_path(str(tmp_path), "run")
    b = D.output_path(str(tmp_path), "run")
    c = D.output_path(str(tmp_path), "run")
    assert [os.path.basename(p) for p in (a, b, c)] == ["run", "run_t1", "run_t2"]


def test_iteration_lines():
    rec = dict(c=1234.5, vol=0.125, sharp=0.5, cons=-0.25, change=0.0625,
               msTotal=1500.0, msAssemble=250.0, msSolve=1000.0, msOpt=125.0, msFilter=62.5)
    a, b = D.iteration_lines(7, rec)
    assert a == " It.:   7 Obj.:  1.23450000e+03 Vol.:1.2500e-01 Sharp.:5.0000e-01 Cons.:-2.50e-01 Ch.:6.25e-02"
    assert b == (" It.: 7 (Time)... Total per-It.: 1.50e+00s; Assemb.: 2.50e-01s; CG: 1.00e+00s;"
                 " Opti.: 1.25e-01s; Filtering: 6.25e-02s.")


def test_run_writes_the_reference_files(tmp_path):
    ScriptedSolver.made.clear()
    out = D.TOP_GPU(np.ones((6, 12, 6), bool), optCase=1, V0=0.12, nLoop=8, ft=1, mixed_Precision=1,
                    out_root=str(tmp_path), solver_class=ScriptedSolver, log=lambda s: None)
    s = ScriptedSolver.made[-1]
    assert s.kw == dict(E0=1.0, Emin=1e-6, penal=3.0, tol=1e-3, maxIT=800, omega=0.6, mixed=True, outer_fp32=False)
    assert s.prm == (0.12, math.sqrt(3), 8, 1) and len(out["history"]) == 8 and out["cSolid"] == 123.5
    assert os.path.basename(out["path"]) == "case1_12x6x6_V0.12_r1.732_ft1_n8_mp1_se0"
    names = sorted(os.listdir(out["path"]))
    assert names == ["DesignVolume.nii", "RunLog.log", "c_Target.dat", "history.json", "iters_Target.dat",
                     "sharp_Target.dat", "solvetiming_Target.dat", "timing_Target.dat"]
    log = open(os.path.join(out["path"], "RunLog.log")).read().splitlines()
    assert log[1] == "Compliance of Fully Solid Domain:     1.235000e+02"
    assert sum(l.startswith(" It.:") for l in log) == 2 * 8
    iters = open(os.path.join(out["path"], "iters_Target.dat")).read().split()
    assert iters == [str(v) for k in range(1, 9) for v in (5, 5 + k)]      # per load case, per iteration


def test_loop_stops_on_sharpness(tmp_path):
    out = D.TOP_GPU(np.ones((6, 12, 6), bool), nLoop=500, out_root=str(tmp_path), solver_class=ScriptedSolver,
                    log=lambda s: None)
    assert len(out["history"]) == 50          # sharpness 0.5/k reaches 0.01 at k = 50 (TOP_GPU.m:177)


def test_super_element_run(tmp_path):
    out = D.TOP_GPU(np.ones((4, 8, 4), bool), optCase=2, V0=0.2, nLoop=2, ft=2, super_element=1,
                    out_root=str(tmp_path), solver_class=ScriptedSolver, log=lambda s: None)
    assert "xPhys_sorted.dat" in os.listdir(out["path"])


def test_argument_errors(tmp_path):
    with pytest.raises(ValueError, match="ft = 2"):
        D.TOP_GPU(np.ones((4, 8, 4), bool), ft=1, super_element=1, out_root=str(tmp_path), solver_class=ScriptedSolver)
    with pytest.raises(ValueError, match="Inappropriate"):
        D.TOP_GPU(np.ones((2, 8, 4), bool), out_root=str(tmp_path), solver_class=ScriptedSolver)
    shape = (6, 8, 6)
    ys, zs = np.meshgrid(np.arange(7), np.arange(7), indexing="ij")
    fix = np.column_stack([node_index(ys.ravel(), 0, zs.ravel(), shape), np.ones((ys.size, 3), int)])
    load = np.array([[node_index(3, 8, 0, shape), 0.0, 0.0, -1.0]])
    path = tmp_path / "p.TopVoxel"
    write_topvoxel(path, np.ones(shape, bool), fix, [load], passive=[1, 2])
    D.TOP_GPU(str(path), nLoop=1, out_root=str(tmp_path), solver_class=ScriptedSolver, log=lambda s: None)
    assert list(ScriptedSolver.made[-1].passive) == [1, 2]        # the file's passive list reaches the solver
    write_topvoxel(path, np.ones(shape, bool), fix, [load])
    out = D.TOP_GPU(str(path), nLoop=3, out_root=str(tmp_path), solver_class=ScriptedSolver, log=lambda s: None)
    assert os.path.basename(out["path"]) == "p_V0.12_r1.732_ft1_n3_mp0_se0" and len(out["history"]) == 3
