"""Host-side mirror of TOP_GPU's FEA model and solver over libtopgpu.so.

``Mesh`` is CreateVoxelFEAmodel / FEA_VoxelBasedDiscretization /
Solving_BuildingMeshHierarchy / FEA_ApplyBoundaryCondition /
Solving_SetupKeWithFixedDOFs (TOP_GPU.m:403-536, 1276-1442, 1505-1727), built
on the host by the library (no GPU needed).  ``Solver`` holds one model on the
GPU and provides Solving_AssembleFEAstencil, Solving_KbyU_MatrixFree,
Solving_Vcycle and Solving_PCG (TOP_GPU.m:602-878, 1033-1267).
"""
import ctypes as C
import os

import numpy as np
import torch

from ._lib import (OptParams, OptRecord, SolverParams, TOP_ERR_NOT_CONVERGED, TOP_OK, TOP_PREC_FP64,
                   TOP_PREC_MIXED, TopGpuError, check, last_error, lib)

_INT_ARRAYS = {"passiveElements", "resolution", "eleMapBack", "eleMapForward", "eNodMat", "nodMapBack", "nodMapForward", "nodesOnBoundary",
               "elementsOnBoundary", "elementUpwardMap", "transferMat", "solidNodeMapCoarser2Finer",
               "mapUniqueKes", "eleWithFixedDOFs", "fixingCond"}


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Mesh:
    """Voxel FEA model: mesh hierarchy, element matrices, boundary conditions."""

    def __init__(self, mask, control=20000, nu=0.3, cell=None, super_element=0):
        mask = np.asarray(mask, dtype=bool)
        if mask.ndim != 3:
            raise ValueError("mask must be a 3-D logical array (nely x nelx x nelz)")
        ny, nx, nz = mask.shape
        self.shape = (ny, nx, nz)
        if cell is None:
            cell = 1.0 / nx      # logical-array models: cellSize_ = 1/nelx (TOP_GPU.m:61, 392)
        self._mask = np.asfortranarray(mask.astype(np.uint8))
        h = C.c_void_p()
        check(lib().top_mesh_create(_p(self._mask), ny, nx, nz, control, nu, cell, super_element, C.byref(h)),
              "top_mesh_create")
        self._h = h
        self.super_element = super_element

    @classmethod
    def from_topvoxel(cls, path, control=20000, nu=0.3):
        """A .TopVoxel model file (CreateVoxelFEAmodel, TOP_GPU.m:416-496), its
        fixations and load cases applied; cellSize 1 as for file models.
        .passive_elements (compact, 1-based) and .density_layout (the file's
        per-voxel densities, may be empty) come with it."""
        self = cls.__new__(cls)
        h = C.c_void_p()
        check(lib().top_mesh_create_from_topvoxel(os.fsencode(str(path)), control, nu, C.byref(h)),
              "top_mesh_create_from_topvoxel")
        self._h = h
        self.super_element = 0
        self.shape = tuple(int(v) for v in self.get(0, "resolution"))
        self.passive_elements = self.get(0, "passiveElements")
        self.density_layout = self.get(0, "densityLayout")
        return self

    def close(self):
        if getattr(self, "_h", None):
            lib().top_mesh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def info(self):
        out = np.zeros(1 + 8 * 16, dtype=np.int64)
        check(lib().top_mesh_info(self._h, _p(out), out.size), "top_mesh_info")
        nl = int(out[0])
        levels = []
        for l in range(nl):
            v = out[1 + 8 * l: 9 + 8 * l]
            levels.append(dict(resX=int(v[0]), resY=int(v[1]), resZ=int(v[2]), spanWidth=int(v[3]),
                               numElements=int(v[4]), numNodes=int(v[5]), intermediateNumNodes=int(v[6]),
                               nUnique=int(v[7])))
        return levels

    @property
    def numLevels(self):
        return len(self.info())

    def get(self, level, name):
        n = C.c_int64()
        check(lib().top_mesh_get(self._h, level, name.encode(), None, 0, C.byref(n)), "top_mesh_get")
        dt = np.int32 if name in _INT_ARRAYS else np.float64
        a = np.zeros(n.value, dtype=dt)
        check(lib().top_mesh_get(self._h, level, name.encode(), _p(a), a.size, None), "top_mesh_get")
        return a

    def apply_optcase(self, opt):
        check(lib().top_mesh_apply_optcase(self._h, opt), "top_mesh_apply_optcase")

    def apply_bc(self, fixing, loads, weights=None):
        fixing = np.ascontiguousarray(fixing, dtype=np.float64)
        loads = [np.ascontiguousarray(l, dtype=np.float64) for l in loads]
        n = np.array([len(l) for l in loads], dtype=np.int64)
        ptrs = (C.c_void_p * len(loads))(*[l.ctypes.data for l in loads])
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        check(lib().top_mesh_apply_bc(self._h, len(fixing), _p(fixing), len(loads), _p(n), ptrs,
                                      None if w is None else _p(w)), "top_mesh_apply_bc")


class Solver:
    """One voxel model resident on the GPU (current CUDA device)."""

    def __init__(self, mesh: Mesh, E0=1.0, Emin=1e-6, penal=3.0, tol=1e-3, maxIT=800, omega=0.6,
                 mixed=False, outer_fp32=False):
        self.mesh = mesh
        p = SolverParams(E0=E0, Emin=Emin, penal=penal, tol=tol, maxIT=maxIT, omega=omega,
                         precision=TOP_PREC_MIXED if mixed else TOP_PREC_FP64, outerFP32=int(bool(outer_fp32)))
        self.params = p
        torch.cuda.init()
        h = C.c_void_p()
        check(lib().top_solver_create(mesh.handle, C.byref(p), C.byref(h)), "top_solver_create")
        self._h = h
        sz = np.zeros(3, dtype=np.int64)
        check(lib().top_solver_sizes(self._h, _p(sz)), "top_solver_sizes")
        self.numLevels, self.nLoads, self.numDOFs = (int(v) for v in sz)
        self.levels = mesh.info()
        self.set_stream(torch.cuda.current_stream())

    def close(self):
        if getattr(self, "_h", None):
            lib().top_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        check(lib().top_solver_set_stream(self._h, C.c_void_p(stream.cuda_stream)), "top_solver_set_stream")

    @staticmethod
    def _dev(t, n=None, dtype=torch.float64):
        if not isinstance(t, torch.Tensor):
            t = torch.as_tensor(np.asarray(t), dtype=dtype)
        t = t.to(device="cuda", dtype=dtype).contiguous()
        if n is not None and t.numel() != n:
            raise ValueError("expected %d entries, got %d" % (n, t.numel()))
        return t

    @property
    def num_design(self):
        """Design variables: one per element, 64 per super-element (sub-voxels)."""
        return self.levels[0]["numElements"] * (64 if self.mesh.super_element else 1)

    def set_modulus(self, E):
        E = self._dev(E, self.num_design)
        check(lib().top_solver_set_modulus(self._h, E.data_ptr(), 1), "top_solver_set_modulus")

    def set_density(self, x):
        x = self._dev(x, self.num_design)
        check(lib().top_solver_set_density(self._h, x.data_ptr(), 1), "top_solver_set_density")

    def assemble(self):
        check(lib().top_solver_assemble(self._h), "top_solver_assemble")

    def matvec(self, level, u, fp32=False):
        n = 3 * self.levels[level]["numNodes"]
        u = self._dev(u, n)
        y = torch.zeros(n, dtype=torch.float64, device="cuda")
        check(lib().top_solver_matvec(self._h, level, u.data_ptr(), y.data_ptr(), int(fp32)), "top_solver_matvec")
        return y

    def vcycle(self, r):
        r = self._dev(r, self.numDOFs)
        z = torch.zeros_like(r)
        check(lib().top_solver_vcycle(self._h, r.data_ptr(), z.data_ptr()), "top_solver_vcycle")
        return z

    def restrict(self, ii, r):
        r = self._dev(r, 3 * self.levels[ii - 1]["numNodes"])
        out = torch.zeros(3 * self.levels[ii]["numNodes"], dtype=torch.float64, device="cuda")
        check(lib().top_solver_restrict(self._h, ii, r.data_ptr(), out.data_ptr()), "top_solver_restrict")
        return out

    def interpolate(self, ii, x):
        x = self._dev(x, 3 * self.levels[ii]["numNodes"])
        out = torch.zeros(3 * self.levels[ii - 1]["numNodes"], dtype=torch.float64, device="cuda")
        check(lib().top_solver_interpolate(self._h, ii, x.data_ptr(), out.data_ptr()), "top_solver_interpolate")
        return out

    def diag(self, level):
        out = torch.zeros(3 * self.levels[level]["numNodes"], dtype=torch.float64, device="cuda")
        check(lib().top_solver_get_diag(self._h, level, out.data_ptr()), "top_solver_get_diag")
        return out

    def Ks(self, level):
        ne = self.levels[level]["numElements"]
        out = torch.zeros(576 * ne, dtype=torch.float64, device="cuda")
        check(lib().top_solver_get_ks(self._h, level, out.data_ptr()), "top_solver_get_ks")
        return out

    def pcg_all(self, U=None):
        """All load cases as one batched PCG; returns (U [3Nn x nLoads] as a
        column-major flat tensor, its list, relres list)."""
        nd = 3 * self.levels[0]["numNodes"]
        out = torch.zeros(nd * self.nLoads, dtype=torch.float64, device="cuda")
        warm = 0
        if U is not None:
            out.copy_(self._dev(U, nd * self.nLoads))
            warm = 1
        its = (C.c_int * self.nLoads)()
        res = (C.c_double * self.nLoads)()
        st = lib().top_solver_pcg_all(self._h, out.data_ptr(), warm, its, res)
        if st not in (TOP_OK, TOP_ERR_NOT_CONVERGED):
            check(st, "top_solver_pcg_all")
        return out, list(its), list(res)

    def pcg(self, load_case=0, U=None, b=None, raise_on_maxit=False):
        """Solving_PCG on load case k (or an explicit rhs b); U is the warm start.

        Returns (U, its, relres).  Reaching maxIT prints the reference's warning
        (TOP_GPU.m:656-659) unless raise_on_maxit is set.
        """
        warm = U is not None
        U = torch.zeros(self.numDOFs, dtype=torch.float64, device="cuda") if U is None else self._dev(U, self.numDOFs).clone()
        its, res = C.c_int(0), C.c_double(0)
        if b is None:
            st = lib().top_solver_pcg(self._h, load_case, U.data_ptr(), int(warm), C.byref(its), C.byref(res))
        else:
            b = self._dev(b, self.numDOFs)
            st = lib().top_solver_pcg_rhs(self._h, b.data_ptr(), U.data_ptr(), int(warm), C.byref(its), C.byref(res))
        if st == TOP_ERR_NOT_CONVERGED and not raise_on_maxit:
            print("Warning: Exceed the maximum iterate numbers")
            print("The iterative process stops at residual = %10.4f" % res.value)
        elif st != TOP_OK:
            raise TopGpuError(st, "Solving_PCG", last_error())
        return U, its.value, res.value

    def unit_compliance(self, U):
        U = self._dev(U, self.numDOFs)
        ce = torch.zeros(self.levels[0]["numElements"], dtype=torch.float64, device="cuda")
        check(lib().top_solver_unit_compliance(self._h, U.data_ptr(), ce.data_ptr()), "top_solver_unit_compliance")
        return ce

    # -- optimisation steps (TOP_GPU.m:141-292) --------------------------------
    def filter_setup(self, rMin):
        check(lib().top_solver_filter_setup(self._h, float(rMin)), "top_solver_filter_setup")

    def filter(self, src):
        src = self._dev(src, self.levels[0]["numElements"])
        out = torch.zeros_like(src)
        its = C.c_int(0)
        check(lib().top_solver_filter(self._h, src.data_ptr(), out.data_ptr(), C.byref(its)), "top_solver_filter")
        return out, its.value

    def set_passive(self, ids):
        """Passive elements (compact 1-based ids, e.g. Mesh.passive_elements):
        design 1 in the OC update and after the filter (TOP_GPU.m:239, 270)."""
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        check(lib().top_solver_set_passive(self._h, _p(ids) if ids.size else None, ids.size), "top_solver_set_passive")

    def opt_begin(self, V0=0.12, rMin=np.sqrt(3), nLoop=50, ft=1):
        self._opt = OptParams(V0=V0, rMin=rMin, nLoop=nLoop, ft=ft)
        cs = C.c_double(0)
        check(lib().top_solver_opt_begin(self._h, C.byref(self._opt), C.byref(cs)), "top_solver_opt_begin")
        return cs.value

    def opt_step(self):
        rec = OptRecord()
        check(lib().top_solver_opt_step(self._h, C.byref(rec)), "top_solver_opt_step")
        return {k: getattr(rec, k) for k, _ in OptRecord._fields_}

    def opt_case_its(self):
        """PCG iterations per load case in the last opt_step's state solves."""
        its = (C.c_int * max(1, self.nLoads))()
        n = C.c_int(0)
        check(lib().top_solver_opt_case_its(self._h, its, len(its), C.byref(n)), "top_solver_opt_case_its")
        return [its[k] for k in range(n.value)]

    def opt_state(self):
        loop, ch, sh = C.c_int(0), C.c_double(0), C.c_double(0)
        check(lib().top_solver_opt_state(self._h, C.byref(loop), C.byref(ch), C.byref(sh)), "top_solver_opt_state")
        return loop.value, ch.value, sh.value

    def design(self):
        ne = self.num_design
        xp = torch.zeros(ne, dtype=torch.float64, device="cuda")
        x = torch.zeros(ne, dtype=torch.float64, device="cuda")
        check(lib().top_solver_get_design(self._h, xp.data_ptr(), x.data_ptr()), "top_solver_get_design")
        return xp, x

    def set_design(self, xPhys=None, x=None):
        """Replace the design the next opt_step starts from (device or pinned/pageable host tensors)."""
        ne = self.num_design
        ptrs = []
        for v in (xPhys, x):
            if v is None:
                ptrs.append(None)
                continue
            if v.dtype != torch.float64 or v.numel() != ne or not v.is_contiguous():
                raise ValueError("set_design: contiguous float64 vectors of numElements expected")
            ptrs.append(v.data_ptr())
        check(lib().top_solver_set_design(self._h, ptrs[0], ptrs[1]), "top_solver_set_design")

    def get_design_into(self, xPhys=None, x=None):
        """Copy the current design into given tensors (device or host); blocks until done."""
        check(lib().top_solver_get_design(self._h, None if xPhys is None else xPhys.data_ptr(),
                                          None if x is None else x.data_ptr()), "top_solver_get_design")

    def set_l0_kernel(self, fp32, kind, ty=16, tx=16, ctas=0):
        """Level-0 product kernel for one precision: kind 0 dense node-centric, 1 Walsh-basis
        tiles of ty x tx element columns on ctas CTAs (0: as many as fit at once)."""
        check(lib().top_solver_set_l0_kernel(self._h, int(bool(fp32)), kind, ty, tx, ctas),
              "top_solver_set_l0_kernel")

    def l0_kernel(self, fp32):
        out = (C.c_int * 4)()
        check(lib().top_solver_get_l0_kernel(self._h, int(bool(fp32)), out), "top_solver_get_l0_kernel")
        return tuple(out)

    def sensitivity(self, xPhys, objective="compliance", dof=None, load_case=0, ft=0, x=None, tol=0.0):
        """Adjoint sensitivity dJ/dx at design xPhys (CUDA float64 [Ne]).  objective
        "compliance" (self-adjoint) or "displacement" (J = U[dof], adjoint solve);
        ft 0/1/2 chains through no filter / the sensitivity filter / the PDE
        density filter (filter_setup first).  Returns (dJdx, J, pcg_its)."""
        from ._lib import SensParams
        obj = {"compliance": 0, "displacement": 1}[objective]
        prm = SensParams(objective=obj, loadCase=load_case, dof=-1 if dof is None else int(dof), ft=ft, tol=tol)
        ne = self.levels[0]["numElements"]
        if xPhys.dtype != torch.float64 or xPhys.numel() != ne or not xPhys.is_cuda:
            raise ValueError("sensitivity: CUDA float64 xPhys of numElements expected")
        out = torch.empty(ne, dtype=torch.float64, device=xPhys.device)
        J, its = C.c_double(0), C.c_int(0)
        check(lib().top_solver_sensitivity(self._h, C.byref(prm), xPhys.data_ptr(),
                                           None if x is None else x.data_ptr(), out.data_ptr(),
                                           C.byref(J), C.byref(its)), "top_solver_sensitivity")
        return out, J.value, its.value

    def super_filter_setup(self, rMin):
        check(lib().top_solver_super_filter_setup(self._h, rMin), "top_solver_super_filter_setup")

    def super_filter(self, src, mode):
        """Super-element density filter on [64 x Ne] vectors: mode 0 = imfilter(src./Hs, h),
        1 = imfilter(src, h)./Hs."""
        src = self._dev(src, self.num_design)
        out = torch.empty_like(src)
        check(lib().top_solver_super_filter(self._h, src.data_ptr(), out.data_ptr(), mode), "top_solver_super_filter")
        return out

    def set_coarse_persistent(self, on):
        """V-cycle levels from 1 (on = 1 / True) or from 2 (on = 2) down in one cooperative
        launch, or one launch per step (0 / False)."""
        check(lib().top_solver_set_coarse_persistent(self._h, int(on)), "top_solver_set_coarse_persistent")

    def set_pcg_beta(self, flexible):
        """False: the reference's beta = rho/rhoOld; True: flexible (Polak-Ribiere) beta."""
        check(lib().top_solver_set_pcg_beta(self._h, int(bool(flexible))), "top_solver_set_pcg_beta")

    def set_tail_operator(self, on):
        """The V-cycle from its highest level with at most 2500 DOFs down as one
        operator formed at assembly: True / False / None (the default: in mixed
        precision only).  Returns the level it starts at (0: not in use)."""
        level = C.c_int(0)
        mode = -1 if on is None else int(bool(on))
        check(lib().top_solver_set_tail_operator(self._h, mode, C.byref(level)), "top_solver_set_tail_operator")
        return level.value

    def test_withhold_tile(self):
        """Arm the coarse product's failure-path test: the next two-pass
        coarse product withholds one tile copy and the call reports it."""
        check(lib().top_solver_test_withhold_tile(self._h), "top_solver_test_withhold_tile")

    def set_graphs(self, on):
        """Run PCG iterations as captured CUDA graphs (default) or launch by launch."""
        check(lib().top_solver_set_graphs(self._h, int(bool(on))), "top_solver_set_graphs")

    def autotune(self, nrep=5, flush_bytes=512 << 20):
        """Pick the fastest level-0 kernel per precision on the products this
        solver's PCG iteration makes (epilogues included); returns
        {"fp64": (ms per iteration, (kind, ty, tx, ctas)), "fp32": (...)}."""
        ms = (C.c_double * 2)()
        cfg = (C.c_int * 8)()
        check(lib().top_solver_autotune(self._h, nrep, flush_bytes, ms, cfg), "top_solver_autotune")
        return {"fp64": (ms[0], tuple(cfg[0:4])), "fp32": (ms[1], tuple(cfg[4:8]))}

    @property
    def launches(self):
        """Kernels launched by this solver since creation."""
        n = C.c_int64(0)
        check(lib().top_solver_launch_count(self._h, C.byref(n)), "top_solver_launch_count")
        return n.value

    def optimize(self, V0=0.12, rMin=np.sqrt(3), nLoop=50, ft=1):
        """TOP_GPU's optimisation loop on the device; returns (xPhys, history, cSolid)."""
        prm = OptParams(V0=V0, rMin=rMin, nLoop=nLoop, ft=ft)
        hist = (OptRecord * max(1, nLoop))()
        n, cs = C.c_int(0), C.c_double(0)
        xp = torch.zeros(self.num_design, dtype=torch.float64, device="cuda")
        check(lib().top_solver_optimize(self._h, C.byref(prm), xp.data_ptr(), hist, C.byref(n), C.byref(cs)),
              "top_solver_optimize")
        rows = [{k: getattr(hist[i], k) for k, _ in OptRecord._fields_} for i in range(n.value)]
        return xp, rows, cs.value
