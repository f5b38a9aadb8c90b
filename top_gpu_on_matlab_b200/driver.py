"""TOP_GPU(inputModel, name, value, ...) -- the reference's driver
(TOP_GPU.m:1-327) on the library: model, boundary conditions, the
optimisation loop on the device, the per-iteration log lines and the result
files, in the reference's output folder.

    TOP_GPU(np.ones((24, 48, 24), bool), optCase=1, V0=0.12)
    TOP_GPU("./data/model.TopVoxel", V0=0.4, ft=2)

Settings not exposed as parameters are InitialSettings' (TOP_GPU.m:386-402):
E0 = 1, Emin = 1e-6, nu = 0.3, p = 3, tol = 1e-3, maxIT = 800, omega = 0.6,
coarsestResolutionControl = 20000; cell size 1/nelx for logical arrays, 1
for files.  mixed_Precision = 1 runs the V-cycle in FP32 with the outer PCG
in FP64 (outer_fp32=True also runs the outer product in FP32, as the
reference's mixed mode does, TOP_GPU.m:683-684).
"""
import math
import os
import time

import numpy as np

from . import results

SETTINGS = dict(E0=1.0, Emin=1.0e-6, nu=0.3, penal=3.0, tol=1.0e-3, maxIT=800, omega=0.6, control=20000)


def folder_name(input_model, optCase, V0, rMin, ft, nLoop, mixed_Precision, super_element):
    """The run's folder name (TOP_GPU.m:57-67)."""
    if isinstance(input_model, np.ndarray):
        nely, nelx, nelz = input_model.shape
        return "case%d_%dx%dx%d_V%.4g_r%.4g_ft%d_n%d_mp%d_se%d" % (
            optCase, nelx, nely, nelz, V0, rMin, ft, nLoop, mixed_Precision, super_element)
    model = os.path.splitext(os.path.basename(str(input_model)))[0]
    return "%s_V%.4g_r%.4g_ft%d_n%d_mp%d_se%d" % (model, V0, rMin, ft, nLoop, mixed_Precision, super_element)


def output_path(root, name):
    """./out/<name>/, or <name>_t1, _t2, ... when it exists (TOP_GPU.m:68-76); created."""
    path = os.path.join(root, name)
    if os.path.isdir(path):
        k = 1
        while os.path.isdir(os.path.join(root, "%s_t%d" % (name, k))):
            k += 1
        path = os.path.join(root, "%s_t%d" % (name, k))
    os.makedirs(path)
    return path


def iteration_lines(loop, rec):
    """The two lines printed per iteration (TOP_GPU.m:287-291); times in seconds."""
    a = " It.:%4i Obj.:%16.8e Vol.:%6.4e Sharp.:%6.4e Cons.:%4.2e Ch.:%4.2e" % (
        loop, rec["c"], rec["vol"], rec["sharp"], rec["cons"], rec["change"])
    b = (" It.: %i (Time)... Total per-It.: %8.2es; Assemb.: %8.2es; CG: %8.2es; Opti.: %8.2es; Filtering: %8.2es."
         % (loop, rec["msTotal"] / 1e3, rec["msAssemble"] / 1e3, rec["msSolve"] / 1e3, rec["msOpt"] / 1e3,
            rec["msFilter"] / 1e3))
    return a, b


def _model(input_model, optCase, super_element):
    from .fea import Mesh
    if isinstance(input_model, np.ndarray):
        mask = np.asarray(input_model, dtype=bool)
        if mask.ndim != 3 or min(mask.shape) < 3:
            raise ValueError("Inappropriate Input Model! (a 3-D logical array, at least 3 voxels per axis)")
        m = Mesh(mask, control=SETTINGS["control"], nu=SETTINGS["nu"], super_element=super_element)
        m.apply_optcase(optCase)
        return m
    if super_element:
        raise ValueError("super_element = 1 needs a box domain given as a logical array")
    return Mesh.from_topvoxel(input_model, control=SETTINGS["control"], nu=SETTINGS["nu"])


def TOP_GPU(input_model, optCase=1, V0=0.12, rMin=math.sqrt(3), nLoop=50, ft=1, mixed_Precision=0,
            super_element=0, out_root="./out", outer_fp32=False, solver_class=None, log=print):
    """Run the optimisation; returns dict(xPhys, history, cSolid, path)."""
    if super_element and ft != 2:
        raise ValueError("super_element = 1 needs ft = 2 (the PDE density filter)")
    if ft not in (0, 1, 2):
        raise ValueError("ft must be 0, 1 or 2")
    if solver_class is None:
        from .fea import Solver as solver_class
    if not isinstance(input_model, np.ndarray) and not isinstance(input_model, (str, os.PathLike)):
        input_model = np.asarray(input_model, dtype=bool)
    path = output_path(out_root, folder_name(input_model, optCase, V0, rMin, ft, nLoop, mixed_Precision,
                                             super_element))
    lines = []

    def say(text):
        lines.append(text)
        log(text)

    t0 = time.perf_counter()
    mesh = _model(input_model, optCase, super_element)
    say("Preparing Voxel-based FEA Model Costs %10.1fs" % (time.perf_counter() - t0))
    s = solver_class(mesh, E0=SETTINGS["E0"], Emin=SETTINGS["Emin"], penal=SETTINGS["penal"], tol=SETTINGS["tol"],
                     maxIT=SETTINGS["maxIT"], omega=SETTINGS["omega"], mixed=bool(mixed_Precision),
                     outer_fp32=bool(outer_fp32))
    passive = getattr(mesh, "passive_elements", None)
    if passive is not None and passive.size:
        s.set_passive(passive)                                     # TOP_GPU.m:123-125
    t_start = time.perf_counter()
    c_solid = s.opt_begin(V0=V0, rMin=rMin, nLoop=nLoop, ft=ft)
    say("Compliance of Fully Solid Domain: %16.6e" % c_solid)
    history, iters = [], []
    loop, change, sharp = 0, 1.0, 1.0
    while loop < nLoop and change > 0.0001 and sharp > 0.01:       # TOP_GPU.m:177
        rec = s.opt_step()
        loop, change, sharp = s.opt_state()
        history.append(rec)
        iters.extend(s.opt_case_its())                             # lssIts, one per load case
        for text in iteration_lines(loop, rec):
            say(text)
    xphys, _ = s.design()          # [Ne], or [64 x Ne] column-major for super elements
    t = lambda key: sum(r[key] for r in history) / 1e3
    say("..........Solving FEA Costs: %10.4es." % (t("msAssemble") + t("msSolve")))
    say("..........Optimization (inc. sentivity analysis, update) Costs: %10.4es." % t("msOpt"))
    say("..........Performing PDE Filtering Costs: %10.4es." % t("msFilter"))
    say("..........Performing Topology Optimization Costs (in total): %10.4es." % (time.perf_counter() - t_start))
    results.write_results(path, mesh, xphys, history, iters)
    with open(os.path.join(path, "RunLog.log"), "w") as f:
        f.write("\n".join(lines) + "\n")
    return dict(xPhys=xphys, history=history, cSolid=c_solid, path=path)
