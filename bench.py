"""Benchmark: PCG ms per optimisation iteration on the 96x192x96 cantilever.

Workload (the metric's configuration): true(96,192,96) voxels (1,769,472
elements, 5,447,811 DOFs), cantilever BCs (optCase 1), E0 = 1, Emin = 1e-9,
nu = 0.3, SIMP p = 3, V0 = 0.12, rMin = sqrt(3), ft = 1 sensitivity filter,
five multigrid levels (coarsestResolutionControl 400; 192x96x96 ->
48x24x24 -> 24x12x12 -> 12x6x6 -> 6x3x3), damped Jacobi omega = 0.6,
relative residual 1e-6.  One step = one optimisation iteration of
TOP_GPU.m:176-292 on the device: SIMP moduli, Galerkin assembly of every
coarse level + coarsest Cholesky, the PCG state solve warm-started from the
previous iteration, element energies, sensitivity filter and OC update.
W warm-up iterations run first (iterations 1..W after the fully solid
solve), then K timed iterations (W+1..W+K).

value = mean PCG ms of the timed iterations on the mixed-precision path
(FP32 V-cycle, FP64 outer recurrence / matvec / coarsest Cholesky), device
time from CUDA events with inputs resident in HBM.  The same iterations run
on the plain FP64 path for the ratio; the compliance error is the largest
relative difference of any iteration's compliance between the two paths,
the density error the max-abs difference of xPhys after the last one.  e2e
runs the same iterations through the C ABI with the design held on the host
(pinned): the design goes up before and comes back after every iteration.

After the timed region the mixed path's last design is solved once more on
the device and by the FP64 oracle (cold start, same tolerance): the line
reports the compliance and displacement-field errors against the oracle.

--impl reference times the FP64 CPU restatement of the reference (oracle/,
the MATLAB driver cannot run here) on the host cores: each step times two
oracle PCG iterations on the workload's first design, and the PCG ms per
optimisation iteration is projected with the FP64 PCG iteration count of the
same optimisation iterations, recorded from this benchmark's FP64 device path
(bench_fp64_its.json; the device FP64 path and the oracle take the same
iteration counts to +-1, tests/test_gpu_solver.py).  The line says
"projected" and gives the multiplier and its source.
"""
import argparse
import atexit
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SHAPE = (96, 192, 96)
CONTROL = 400
V0 = 0.12
E0, EMIN, PENAL, NU = 1.0, 1e-9, 3.0, 0.3
TOL, MAXIT, OMEGA = 1e-6, 800, 0.6
RMIN, FT = 3 ** 0.5, 1
WORKLOAD = "cantilever_96x192x96_ft1_optimisation_iterations"
# DRAM bytes (read + write) per launch of a level-0 stiffness product on this
# workload, from one-launch ncu captures (dram__bytes_read.sum +
# dram__bytes_write.sum), keyed by precision and the kernel configuration
# (kind, tile y, tile x, CTAs); a configuration without a capture reports null
NCU_TRAFFIC = {
    ("fp64", 3, 16, 8, 1184): 74.58e6,
    ("fp64", 3, 16, 8, 1776): 74.51e6,
    ("fp32", 3, 16, 16, 888): 32.89e6,
    ("fp32", 3, 16, 8, 888): 38.16e6,
    ("fp32", 3, 16, 8, 1776): 31.75e6,
    ("fp32", 3, 16, 8, 2368): 31.68e6,
}
ITS_RECORD = ROOT / "bench_fp64_its.json"


def _env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons.  Started before
    the solid solve and the warm-up steps so that the sampler is running when
    the timed region begins; mark() at the start of the timed region, stop()
    at its end reports the samples taken in between (the warm-up ones only if
    the timed region was shorter than one sampling interval)."""

    def __init__(self, index, interval_ms=50, exe="nvidia-smi"):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.start_row = 0
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen([exe, "-i", str(index), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                       "-lms", str(interval_ms)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        if self.p is not None:
            atexit.register(self._end)                  # also when the bench fails before stop()

    def _end(self):
        if self.p is not None and self.p.poll() is None:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()

    def _rows(self):
        rows = []
        try:
            text = Path(self.f.name).read_text()
        except OSError:
            return rows
        for line in text.splitlines(keepends=True):
            if not line.endswith("\n"):
                break                                   # a line still being written
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        return rows

    def mark(self):
        if self.p is not None:
            self.start_row = len(self._rows())

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if self.p is None:
            return out
        self._end()
        self.f.flush()
        rows = self._rows()
        timed = rows[self.start_row:]
        use = timed if timed else rows
        if use:
            sm = [float(r[1]) for r in use if r[1].replace(".", "").isdigit()]
            mx = [float(r[2]) for r in use if r[2].replace(".", "").isdigit()]
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            reasons = sorted({names[i] for r in use for i in range(4) if r[5 + i] == "Active"})
            out = {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                   "reasons": reasons, "samples": len(use),
                   "window": ("warm-up and timed (no sample visible at the start of the timed region)"
                              if self.start_row == 0 else
                              "timed" if timed else "warm-up (timed region shorter than the sampling interval)")}
        try:
            os.unlink(self.f.name)
        except OSError:
            pass
        return out


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _cpu_cores():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


class OracleWorkload:
    """The workload on the FP64 oracle (C + OpenMP, all host cores): model,
    hierarchy and BCs built once; the design set and assembled on demand."""

    def __init__(self):
        from oracle import oracle as O
        self.cores = _cpu_cores()
        os.environ.setdefault("OMP_NUM_THREADS", str(self.cores))
        self.o = O.Model(np.ones(SHAPE, bool), control=CONTROL)
        self.o.apply_optcase(1)
        self.o.set_material(E0, EMIN, PENAL)
        self.o.set_solver(TOL, MAXIT, OMEGA)
        self.ne = self.o.level(0).numElements
        self.b = self.o.F()[:, 0]

    def set_design(self, xPhys):
        self.o.set_density(np.ascontiguousarray(xPhys, dtype=np.float64))
        t0 = time.perf_counter()
        self.o.assemble()
        return 1e3 * (time.perf_counter() - t0)

    def pcg_ms_per_iter(self, iters=2):
        """ms per PCG iteration over `iters` iterations from a zero start."""
        t0 = time.perf_counter()
        _, its, _ = self.o.pcg(self.b, maxIT=iters, tol=1e-300)
        return 1e3 * (time.perf_counter() - t0) / its

    def solve(self):
        """Solving_PCG at the workload's tolerance from a zero start: (U, its, relres, ms)."""
        t0 = time.perf_counter()
        U, its, res = self.o.pcg(self.b)
        return U, its, res, 1e3 * (time.perf_counter() - t0)


def workload_config(levels, world):
    ny, nx, nz = SHAPE
    return {"workload": WORKLOAD, "shape": list(SHAPE), "elements": ny * nx * nz,
            "dofs": 3 * (ny + 1) * (nx + 1) * (nz + 1), "levels": levels,
            "control": CONTROL, "tol": TOL, "V0": V0, "rMin": RMIN, "ft": FT,
            "precision": "mixed (FP32 V-cycle, FP64 outer)",
            "l2": "working set > L2 per PCG iteration; kernel timings flush L2",
            "parallelism": "replicas" if world > 1 else "single"}


def recorded_fp64_its(warmup, steps):
    """Mean FP64 PCG iterations of optimisation iterations warmup+1 ..
    warmup+steps from the record of this benchmark's FP64 device path, or
    None when the record does not reach that far."""
    if not ITS_RECORD.exists():
        return None, None
    rec = json.loads(ITS_RECORD.read_text())
    its = rec["fp64_pcg_its_per_opt_iter"]
    if warmup + steps > len(its):
        return None, rec
    return float(np.mean(its[warmup:warmup + steps])), rec


def max_over_ranks(values, device, world):
    """Per-rank timings -> the job's: the maximum over ranks of each value (one
    all-reduce; every rank calls it at the same point).  One rank: unchanged."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def run_reference(args):
    rank, world, _ = _env_rank()
    if rank != 0:
        return
    its, rec = recorded_fp64_its(args.warmup, args.steps)
    if its is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "no FP64 PCG iteration record for optimisation iterations %d-%d in %s"
                          % (args.warmup + 1, args.warmup + args.steps, ITS_RECORD.name)}), flush=True)
        return
    ow = OracleWorkload()
    asm_ms = ow.set_design(np.full(ow.ne, V0))
    samples = []
    for k in range(args.warmup + args.steps):
        ms_it = ow.pcg_ms_per_iter(2)
        if k >= args.warmup:
            samples.append(ms_it)
    ms_it = float(np.mean(samples))
    value = ms_it * its
    cfg = workload_config(ow.o.numLevels, world)
    cfg["opt_iters_timed"] = "%d-%d" % (args.warmup + 1, args.warmup + args.steps)
    cfg["precision"] = "fp64 (oracle)"
    line = {
        "impl": "reference", "metric": "PCG ms/opt-iter", "value": value, "unit": "ms",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": value,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": cfg,
        "projected": True,
        "projection": {"ms_per_pcg_iter": ms_it, "multiplier": its,
                       "multiplier_source": "mean FP64 PCG iterations of optimisation iterations %d-%d measured by "
                                            "this benchmark's FP64 device path (%s, %s)"
                                            % (args.warmup + 1, args.warmup + args.steps, ITS_RECORD.name,
                                               rec.get("source", "")),
                       "timed_pcg_iterations": 2 * args.steps},
        "cpu_baseline": {"value": value, "unit": "ms", "cores": ow.cores, "kind": "port",
                         "sample": "2 FP64 PCG iterations of the oracle per step (%d steps timed), ms/iteration "
                                   "x %.2f PCG iterations per optimisation iteration" % (args.steps, its),
                         "assemble_ms": asm_ms},
        "e2e": {"value": value, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    from top_gpu_on_matlab_b200._lib import check, lib
    import ctypes as C

    rank, world, local = _env_rank()
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    mask = np.ones(SHAPE, bool)
    mesh = Mesh(mask, control=CONTROL)
    mesh.apply_optcase(1)
    info = mesh.info()
    ne, nn = info[0]["numElements"], info[0]["numNodes"]
    stream = torch.cuda.current_stream()

    tuned = {}      # per solver: {"fp64": (ms, config), "fp32": (ms, config)}

    def make(mixed):
        s = Solver(mesh, E0=E0, Emin=EMIN, penal=PENAL, tol=TOL, maxIT=MAXIT, omega=OMEGA, mixed=mixed)
        c_solid = s.opt_begin(V0=V0, rMin=RMIN, nLoop=1 << 20, ft=FT)
        # level-0 kernel autotuner (kind, tile shape, CTA count) on the
        # products this solver's PCG makes, epilogues included; it leaves the
        # fastest configuration of each precision set
        tuned["mixed" if mixed else "fp64"] = s.autotune(nrep=5)
        return s, c_solid

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    results = {}
    for name, mixed in (("fp64", False), ("mixed", True)):
        # the sampler starts ahead of the solid solve and the warm-up steps, so
        # that it is sampling when the timed region begins
        clk = Clocks(local) if name == "mixed" else None
        s, c_solid = make(mixed)
        recs = [s.opt_step() for _ in range(args.warmup)]
        barrier()
        if clk:
            clk.mark()
        n0 = s.launches
        t0 = torch.cuda.Event(enable_timing=True); t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        timed = [s.opt_step() for _ in range(args.steps)]
        t1.record(stream)
        barrier()
        launches = s.launches - n0
        clocks = clk.stop() if clk else None
        total = t0.elapsed_time(t1)
        vals = max_over_ranks([float(np.mean([r["msSolve"] for r in timed])), total / args.steps,
                               float(np.mean([r["msAssemble"] for r in timed]))], dev, world)
        xp, _ = s.design()
        results[name] = dict(solver=s, pcg_ms=float(vals[0]), step_ms=float(vals[1]), asm_ms=float(vals[2]),
                             its=[r["pcgIts"] for r in timed], c=[r["c"] for r in recs + timed],
                             its_all=[r["pcgIts"] for r in recs + timed],
                             rows=timed, launches=launches, clocks=clocks, xPhys=xp, c_solid=c_solid)
    mixed, fp64 = results["mixed"], results["fp64"]
    comp_err = max(abs(a - b) / abs(b) for a, b in zip(mixed["c"], fp64["c"]))
    dens_err = float((mixed["xPhys"] - fp64["xPhys"]).abs().max())
    del fp64["solver"]

    # ---- e2e: the same optimisation iterations through the C ABI with the
    # design on the host (pinned): H2D of (xPhys, x) before each iteration,
    # D2H of the new design after it (the compliance comes back in the record)
    s, _ = make(True)
    xp_h = torch.full((ne,), V0, dtype=torch.float64).pin_memory()
    x_h = torch.full((ne,), V0, dtype=torch.float64).pin_memory()
    e2e = []
    for k in range(args.warmup + args.steps):
        barrier()
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.set_design(xp_h, x_h)
        s.opt_step()
        s.get_design_into(xp_h, x_h)
        e1.record(stream)
        torch.cuda.synchronize()
        if k >= args.warmup:
            e2e.append(e0.elapsed_time(e1))
    e2e_ms = max_over_ranks([float(np.mean(e2e))], dev, world)[0]
    del s

    # ---- kernel roofline: level-0 stiffness products, L2 flushed ----
    s = mixed["solver"]
    peak, peak_kind = _peaks()
    flush = 512 << 20
    tk = {}
    for which, key in ((0, "l0_f64"), (1, "l0_f32"), (2, "vcycle_f32"), (3, "l1_f32"), (4, "restrict01_f32"),
                       (5, "prolong10_f32")):
        ms = C.c_double(0)
        check(lib().top_solver_time_kernel(s._h, which, 20, flush, C.byref(ms)), "time_kernel")
        tk[key] = ms.value
    bytes64 = 6 * nn * 8 + ne * 8
    bytes32 = 6 * nn * 4 + ne * 4
    flops = 1152 * ne
    # mixed PCG iteration: 1 FP64 outer product + 2 FP32 level-0 smoother products
    share64, share32 = tk["l0_f64"], 2 * tk["l0_f32"]
    if share64 >= share32:
        prec, dom, t_dom, byt = "fp64", "level-0 K*u FP64 (outer K*p)", tk["l0_f64"], bytes64
    else:
        prec, dom, t_dom, byt = "fp32", "level-0 K*u FP32 (V-cycle)", tk["l0_f32"], bytes32
    cfg_dom = tuple(int(v) for v in tuned["mixed"][prec][1])
    dom += ", kind %d, %dx%d tiles, %d CTAs" % cfg_dom
    traffic = NCU_TRAFFIC.get((prec,) + cfg_dom)
    achieved = byt / (t_dom * 1e-3) / 1e9
    its_m = float(np.mean(mixed["its"]))
    its_d = float(np.mean(fp64["its"]))
    cfg = workload_config(len(info), world)
    assert cfg["elements"] == ne and cfg["dofs"] == 3 * nn
    cfg["opt_iters_timed"] = "%d-%d" % (args.warmup + 1, args.warmup + args.steps)
    line = {
        "metric": "PCG ms/opt-iter", "value": mixed["pcg_ms"], "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": mixed["step_ms"],
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic",
        "config": cfg,
        "pcg_its": its_m, "fp64_pcg_ms": fp64["pcg_ms"], "fp64_pcg_its": its_d,
        "fp64_pcg_its_per_opt_iter": fp64["its_all"], "mixed_pcg_its_per_opt_iter": mixed["its_all"],
        "mixed_vs_fp64_speedup": fp64["pcg_ms"] / mixed["pcg_ms"],
        "opt_iter_ms": {"mixed": mixed["step_ms"], "fp64": fp64["step_ms"]},
        "compliance_rel_err_mixed_vs_fp64": comp_err,
        "density_maxabs_err_mixed_vs_fp64": dens_err,
        "assembly_ms": mixed["asm_ms"], "fp64_assembly_ms": fp64["asm_ms"],
        "kernel_ms": tk,
        "l0_autotune": {solver: {k: {"ms_per_pcg_iteration": v[0], "kind_ty_tx_ctas": list(v[1])} for k, v in t.items()}
                        for solver, t in tuned.items()},
        "matvec_gbs": {"fp64": bytes64 / (tk["l0_f64"] * 1e-3) / 1e9, "fp32": bytes32 / (tk["l0_f32"] * 1e-3) / 1e9},
        "matvec_tflops": {"fp64": flops / (tk["l0_f64"] * 1e-3) / 1e12, "fp32": flops / (tk["l0_f32"] * 1e-3) / 1e12},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
                     "algorithmic_bytes": byt, "traffic": traffic,
                     "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch of this "
                                        "kernel configuration" if traffic is not None else
                                        "no ncu capture of this kernel configuration")},
        "gpu_launches": mixed["launches"],
        "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": 2 * ne * 8, "d2h_bytes_per_step": 2 * ne * 8,
                "includes": "whole optimisation iteration through the C ABI: H2D design, SIMP, assembly, "
                            "PCG, sensitivities, filter, OC, D2H design and compliance"},
        "clocks": mixed["clocks"],
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        # oracle leg (outside every timed region): the bounded CPU sample, then
        # the mixed path's last design solved by the device and by the oracle
        ow = OracleWorkload()
        asm_ms = ow.set_design(np.full(ow.ne, V0))
        ms_it = float(np.mean([ow.pcg_ms_per_iter(2) for _ in range(3)]))
        line["cpu_baseline"] = {"value": ms_it * its_d, "unit": "ms", "cores": ow.cores, "kind": "port",
                                "sample": "3 x 2 FP64 PCG iterations of the oracle (C + OpenMP) on this problem, "
                                          "ms/iteration x the mean FP64 iteration count of the timed "
                                          "optimisation iterations (%.2f)" % its_d,
                                "assemble_ms": asm_ms}
        if not args.no_oracle_check:
            line["vs_oracle"] = oracle_check(ow, mixed["solver"], mixed["xPhys"])
    if rank == 0 and args.record_its:
        ITS_RECORD.write_text(json.dumps({
            "fp64_pcg_its_per_opt_iter": fp64["its_all"],
            "source": "bench.py --steps %d --warmup %d --record-its on one %s, %s; level-0 kernels %s" % (
                args.steps, args.warmup, torch.cuda.get_device_name(dev), time.strftime("%Y-%m-%d"),
                json.dumps({k: list(v[1]) for k, v in tuned["fp64"].items()})),
        }, indent=1) + "\n")
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def oracle_check(ow, s, xPhys):
    """The mixed path's last design, solved from a zero start by the mixed
    device solver and by the FP64 oracle at the same tolerance: compliance
    F'U and the displacement field compared (TOP_GPU.m:186-191)."""
    import torch
    xp = xPhys.detach().cpu().numpy()
    s.set_density(xPhys)
    s.assemble()
    U, its, res = s.pcg(0)
    Ud = U.cpu().numpy()
    ow.set_design(xp)
    Uo, its_o, res_o, ms_o = ow.solve()
    c_d, c_o = float(ow.b @ Ud), float(ow.b @ Uo)
    return {"design": "xPhys after the last timed mixed-precision iteration",
            "compliance_rel_err": abs(c_d - c_o) / abs(c_o),
            "displacement_rel_err_max": float(np.abs(Ud - Uo).max() / np.abs(Uo).max()),
            "displacement_rel_err_l2": float(np.linalg.norm(Ud - Uo) / np.linalg.norm(Uo)),
            "pcg_its": {"device_mixed": its, "oracle_fp64": its_o},
            "relres": {"device_mixed": res, "oracle_fp64": res_o},
            "oracle_solve_ms": ms_o, "oracle_cores": ow.cores}


def run_kernels_only(args):
    """Build the workload's mixed solver, assemble, and time --steps launches
    each of the level-0 stiffness products (FP64 outer, FP32 smoother), of
    one V-cycle and of the level-1 FP32 product, L2 not flushed.  Few launches: the command the ncu captures
    of those kernels run.  --l0 fp64=K,TY,TX,CTAS / fp32=... selects the
    level-0 kernel configurations (default: the solver's)."""
    import ctypes as C
    import torch
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    from top_gpu_on_matlab_b200._lib import check, lib
    mesh = Mesh(np.ones(SHAPE, bool), control=CONTROL)
    mesh.apply_optcase(1)
    s = Solver(mesh, E0=E0, Emin=EMIN, penal=PENAL, tol=TOL, maxIT=MAXIT, omega=OMEGA, mixed=True)
    ne = mesh.info()[0]["numElements"]
    s.set_density(torch.full((ne,), V0, dtype=torch.float64, device="cuda"))
    s.assemble()
    for spec in args.l0 or []:
        prec, vals = spec.split("=")
        s.set_l0_kernel(prec == "fp32", *[int(v) for v in vals.split(",")])
    out = {}
    for which, key in ((0, "l0_f64"), (1, "l0_f32"), (2, "vcycle_f32"), (3, "l1_f32")):
        ms = C.c_double(0)
        check(lib().top_solver_time_kernel(s._h, which, args.steps, 0, C.byref(ms)), "time_kernel")
        out[key] = ms.value
    print(json.dumps({"kernels_only": out, "workload": WORKLOAD,
                      "l0": {"fp64": s.l0_kernel(False), "fp32": s.l0_kernel(True)}}), flush=True)


def run_probe(args):
    """Small, fixed workloads for profiler captures (no timing printed that
    the benchmark uses): 'pcg' runs one warm-up and one measured mixed PCG
    solve of the workload at its first design with the launches made one by
    one, the measured one inside the NVTX range "probe"; 'assembly' runs the
    Galerkin assembly of every coarse level five times after two warm-ups."""
    import torch
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    mesh = Mesh(np.ones(SHAPE, bool), control=CONTROL)
    mesh.apply_optcase(1)
    ne = mesh.info()[0]["numElements"]
    s = Solver(mesh, E0=E0, Emin=EMIN, penal=PENAL, tol=TOL, maxIT=MAXIT, omega=OMEGA, mixed=True)
    for spec in args.l0 or []:
        prec, vals = spec.split("=")
        s.set_l0_kernel(prec == "fp32", *[int(v) for v in vals.split(",")])
    s.set_density(torch.full((ne,), V0, dtype=torch.float64, device="cuda"))
    s.assemble()
    out = {"probe": args.probe, "workload": WORKLOAD, "l0": {"fp64": s.l0_kernel(False), "fp32": s.l0_kernel(True)}}
    if args.probe == "pcg":
        s.set_graphs(False)
        s.pcg(0)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("probe")
        _, its, _ = s.pcg(0)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        out["pcg_its"] = its
    else:
        for _ in range(2):
            s.assemble()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("probe")
        for _ in range(5):
            s.assemble()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample and the oracle check")
    ap.add_argument("--no-oracle-check", action="store_true",
                    help="skip the oracle solve of the last design (the CPU baseline sample still runs)")
    ap.add_argument("--record-its", action="store_true",
                    help="write the FP64 PCG iterations per optimisation iteration to %s" % ITS_RECORD.name)
    ap.add_argument("--kernels-only", action="store_true", help="time a few launches of the level-0 kernels (profiling)")
    ap.add_argument("--l0", action="append", help="with --kernels-only / --probe: fp64=KIND,TY,TX,CTAS or fp32=...")
    ap.add_argument("--probe", choices=["pcg", "assembly"], help="a small fixed workload for profiler captures")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "RANK" not in os.environ:
        # one replica per GPU: relaunch under torch.distributed.run
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(args.gpus),
               "--master-addr", "127.0.0.1", "--master-port", os.environ.get("MASTER_PORT", "29517"),
               str(Path(__file__).resolve())] + sys.argv[1:]
        sys.exit(subprocess.call(cmd))
    if args.probe:
        run_probe(args)
    elif args.kernels_only:
        run_kernels_only(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
