"""ctypes binding of the FP64 CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py as the checker.  The product package never imports it.
Arrays returned by the accessors are numpy copies in MATLAB layout
(column-major, 1-based int32 indices).
"""
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB = None

i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
f64p = C.POINTER(C.c_double)


class OLevel(C.Structure):
    _fields_ = [
        ("resX", C.c_int), ("resY", C.c_int), ("resZ", C.c_int), ("spanWidth", C.c_int),
        ("numElements", C.c_int64), ("numNodes", C.c_int64), ("numDOFs", C.c_int64),
        ("eleMapBack", i32p), ("eleMapForward", i32p), ("eNodMat", i32p),
        ("nodMapBack", i32p), ("nodMapForward", i32p),
        ("nNodesOnBoundary", C.c_int64), ("nodesOnBoundary", i32p),
        ("nElementsOnBoundary", C.c_int64), ("elementsOnBoundary", i32p),
        ("numNod2Eles", i32p),
        ("elementUpwardMap", i32p), ("intermediateNumNodes", C.c_int64),
        ("transferMat", i32p), ("transferMatCoeffi", f64p),
        ("solidNodeMapCoarser2Finer", i32p), ("RI", f64p),
        ("Ke", C.c_double * 576), ("Ks", f64p), ("diagK", f64p),
        ("incPtr", i64p), ("incIdx", i32p),
    ]


class OModel(C.Structure):
    _fields_ = [
        ("nely", C.c_int), ("nelx", C.c_int), ("nelz", C.c_int),
        ("E0", C.c_double), ("Emin", C.c_double), ("nu", C.c_double),
        ("penal", C.c_double), ("cellSize", C.c_double),
        ("tol", C.c_double), ("omega", C.c_double), ("maxIT", C.c_int),
        ("control", C.c_int), ("superElement", C.c_int),
        ("numLevels", C.c_int), ("L", C.POINTER(OLevel)),
        ("nFix", C.c_int64), ("fixingCond", i32p),
        ("nLoads", C.c_int), ("F", f64p), ("objWeights", f64p),
        ("mapUniqueKes", i32p), ("nUnique", C.c_int64), ("eleWithFixedDOFs", i32p),
        ("uniqueKesFree", f64p), ("uniqueKesFixed", f64p),
        ("eleModulus", f64p), ("I_mat", f64p), ("K_mat", f64p),
        ("nCoarseDOF", C.c_int64), ("cholBW", C.c_int64), ("cholL", f64p),
        ("KEF", C.c_double * 64), ("diagPrecondF", f64p), ("nFilterNodes", C.c_int64),
        ("filterENod", i32p), ("nFilterEles", C.c_int64),
        ("fincPtr", i64p), ("fincIdx", i32p),
        ("lastPcgIts", C.c_int),
        ("passive", C.POINTER(C.c_uint8)),
    ]


def build():
    """Compile liboracle.so from its C source (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)


def lib():
    global _LIB
    if _LIB is None:
        so = _HERE / "liboracle.so"
        if not so.exists():
            build()
        L = C.CDLL(str(so))
        L.orc_create.restype = C.POINTER(OModel)
        L.orc_create.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int]
        L.orc_destroy.argtypes = [C.POINTER(OModel)]
        L.orc_apply_optcase.argtypes = [C.POINTER(OModel), C.c_int]
        L.orc_apply_bc.argtypes = [C.POINTER(OModel), C.c_int64, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_set_material.argtypes = [C.POINTER(OModel), C.c_double, C.c_double, C.c_double]
        L.orc_set_solver.argtypes = [C.POINTER(OModel), C.c_double, C.c_int, C.c_double]
        L.orc_element_stiffness.argtypes = [C.c_double, C.c_double, C.c_void_p]
        L.orc_super_Imat.argtypes = [C.c_double, C.c_void_p]
        L.orc_RI_table.restype = f64p
        L.orc_RI_table.argtypes = [C.c_int]
        L.orc_subele_nodmat.restype = i32p
        L.orc_subele_nodmat.argtypes = [C.c_int]
        L.orc_gather.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64]
        L.orc_scatter.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64]
        L.orc_scatter_accum3.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64]
        L.orc_assemble_ks_level2.argtypes = [C.c_void_p] * 8 + [C.c_int64, C.c_int, C.c_int64]
        L.orc_assemble_ks_higher.argtypes = [C.c_void_p] * 4 + [C.c_int64, C.c_int]
        L.orc_assemble_ks_level2_super.argtypes = [C.c_void_p] * 8 + [C.c_int64, C.c_int, C.c_int64]
        L.orc_set_density.argtypes = [C.POINTER(OModel), C.c_void_p]
        L.orc_set_modulus.argtypes = [C.POINTER(OModel), C.c_void_p]
        L.orc_assemble.argtypes = [C.POINTER(OModel)]
        L.orc_matvec.argtypes = [C.POINTER(OModel), C.c_int, C.c_void_p, C.c_void_p]
        L.orc_vcycle.argtypes = [C.POINTER(OModel), C.c_void_p, C.c_void_p]
        L.orc_restrict.argtypes = [C.POINTER(OModel), C.c_int, C.c_void_p, C.c_void_p]
        L.orc_interpolate.argtypes = [C.POINTER(OModel), C.c_int, C.c_void_p, C.c_void_p]
        L.orc_coarsest_solve.argtypes = [C.POINTER(OModel), C.c_void_p, C.c_void_p]
        L.orc_pcg.argtypes = [C.POINTER(OModel), C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_void_p]
        L.orc_unit_compliance.argtypes = [C.POINTER(OModel), C.c_void_p, C.c_void_p]
        L.orc_unit_compliance_super.argtypes = [C.POINTER(OModel), C.c_void_p, C.c_void_p]
        L.orc_pre_compute_der.argtypes = [C.POINTER(OModel), C.c_void_p, C.c_void_p]
        L.orc_pde_filter_setup.argtypes = [C.POINTER(OModel), C.c_double]
        L.orc_pde_filter.argtypes = [C.POINTER(OModel), C.c_void_p, C.c_void_p]
        L.orc_top_opt.argtypes = [C.POINTER(OModel), C.c_double, C.c_double, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_solve_state.argtypes = [C.POINTER(OModel), C.c_void_p, C.c_int]
        L.orc_set_passive.argtypes = [C.POINTER(OModel), C.c_void_p, C.c_int64]
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _arr(ptr, n, dtype):
    if not ptr or n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(int(n),)).astype(dtype, copy=True)


def element_stiffness(nu=0.3, cell=1.0):
    Ke = np.zeros(576)
    lib().orc_element_stiffness(nu, cell, _p(Ke))
    return Ke.reshape(24, 24, order="F")


def super_imat(cell=1.0):
    I = np.zeros(576 * 64)
    lib().orc_super_Imat(cell, _p(I))
    return I.reshape(576, 64, order="F")


def ri_table(span):
    n = (span + 1) ** 3
    return _arr(lib().orc_RI_table(span), n * 8, np.float64).reshape(n, 8, order="F")


def subele_nodmat(span):
    return _arr(lib().orc_subele_nodmat(span), span ** 3 * 8, np.int32).reshape(span ** 3, 8)


class Level:
    """numpy view (copies) of one oracle mesh level, MATLAB layout."""

    def __init__(self, L: OLevel, ii: int):
        self.index = ii
        self.resX, self.resY, self.resZ, self.spanWidth = L.resX, L.resY, L.resZ, L.spanWidth
        self.numElements, self.numNodes, self.numDOFs = L.numElements, L.numNodes, L.numDOFs
        ng = L.resX * L.resY * L.resZ
        nn = (L.resX + 1) * (L.resY + 1) * (L.resZ + 1)
        self.eleMapBack = _arr(L.eleMapBack, L.numElements, np.int32)
        self.eleMapForward = _arr(L.eleMapForward, ng, np.int32)
        self.eNodMat = _arr(L.eNodMat, L.numElements * 8, np.int32).reshape(L.numElements, 8, order="F")
        self.nodMapBack = _arr(L.nodMapBack, L.numNodes, np.int32)
        self.nodMapForward = _arr(L.nodMapForward, nn, np.int32)
        self.nodesOnBoundary = _arr(L.nodesOnBoundary, L.nNodesOnBoundary, np.int32)
        self.elementsOnBoundary = _arr(L.elementsOnBoundary, L.nElementsOnBoundary, np.int32)
        self.Ke = np.ctypeslib.as_array(L.Ke).copy().reshape(24, 24, order="F")
        if ii > 0:
            s = L.spanWidth
            self.elementUpwardMap = _arr(L.elementUpwardMap, L.numElements * s ** 3, np.int32).reshape(L.numElements, s ** 3, order="F")
            self.intermediateNumNodes = L.intermediateNumNodes
            nI = (s + 1) ** 3
            self.transferMat = _arr(L.transferMat, nI * L.numElements, np.int32).reshape(nI, L.numElements, order="F")
            self.transferMatCoeffi = _arr(L.transferMatCoeffi, L.intermediateNumNodes, np.float64)
            self.RI = _arr(L.RI, nI * 8, np.float64).reshape(nI, 8, order="F")
        self._L = L

    def Ks(self):
        return _arr(self._L.Ks, 576 * self.numElements, np.float64).reshape(24, 24, self.numElements, order="F")

    def diagK(self):
        return _arr(self._L.diagK, self.numDOFs, np.float64)


class Model:
    """Oracle model: voxel mask -> mesh hierarchy, BCs, solver, optimiser."""

    def __init__(self, mask, control=20000, nu=0.3, cell=None, super_element=0):
        mask = np.asarray(mask, dtype=bool)
        ny, nx, nz = mask.shape
        self.mask = np.asfortranarray(mask.astype(np.uint8))
        if cell is None:
            cell = 1.0 / nx      # logical input: cellSize_ = 1/nelx (TOP_GPU.m:61, 392)
        self._m = lib().orc_create(_p(self.mask), ny, nx, nz, control, nu, cell, super_element)
        if not self._m:
            raise ValueError("oracle: inappropriate input model")
        self.super_element = super_element

    def close(self):
        if self._m:
            lib().orc_destroy(self._m)
            self._m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def m(self) -> OModel:
        return self._m.contents

    @property
    def numLevels(self):
        return self.m.numLevels

    def level(self, ii) -> Level:
        return Level(self.m.L[ii], ii)

    # -- BCs / parameters --------------------------------------------------
    def apply_optcase(self, opt):
        if lib().orc_apply_optcase(self._m, opt):
            raise ValueError("oracle: BC generation failed")

    def apply_bc(self, fixing, loads, weights=None):
        fixing = np.ascontiguousarray(fixing, dtype=np.float64)
        loads = [np.ascontiguousarray(l, dtype=np.float64) for l in loads]
        n = np.array([len(l) for l in loads], dtype=np.int64)
        ptrs = (C.c_void_p * len(loads))(*[l.ctypes.data for l in loads])
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        rc = lib().orc_apply_bc(self._m, len(fixing), _p(fixing), len(loads), _p(n), ptrs,
                                None if w is None else _p(w))
        if rc:
            raise ValueError("oracle: BC application failed")

    def set_material(self, E0=1.0, Emin=1e-6, penal=3.0):
        lib().orc_set_material(self._m, E0, Emin, penal)

    def set_solver(self, tol=1e-3, maxIT=800, omega=0.6):
        lib().orc_set_solver(self._m, tol, maxIT, omega)

    # -- accessors ----------------------------------------------------------
    def F(self):
        m = self.m
        n = m.L[0].numDOFs
        return _arr(m.F, n * m.nLoads, np.float64).reshape(n, m.nLoads, order="F")

    def fixingCond(self):
        m = self.m
        return _arr(m.fixingCond, m.nFix * 4, np.int32).reshape(m.nFix, 4, order="F")

    def mapUniqueKes(self):
        return _arr(self.m.mapUniqueKes, self.m.L[0].numElements, np.int32)

    def uniqueKes(self):
        m = self.m
        sl = 64 if m.superElement else 1
        fr = _arr(m.uniqueKesFree, 576 * sl * m.nUnique, np.float64)
        fx = _arr(m.uniqueKesFixed, 576 * m.nUnique, np.float64)
        return fr.reshape(576 * sl, m.nUnique, order="F"), fx.reshape(576, m.nUnique, order="F")

    def eleWithFixedDOFs(self):
        return _arr(self.m.eleWithFixedDOFs, self.m.nUnique, np.int32)

    def objWeights(self):
        return _arr(self.m.objWeights, self.m.nLoads, np.float64)

    def I_mat(self):
        return _arr(self.m.I_mat, 576 * 64, np.float64).reshape(576, 64, order="F")

    def K_mat(self):
        return _arr(self.m.K_mat, 576 * self.m.L[0].numElements, np.float64).reshape(576, -1, order="F")

    # -- solver -------------------------------------------------------------
    def set_density(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64).ravel(order="F")
        lib().orc_set_density(self._m, _p(x))

    def set_modulus(self, E):
        E = np.ascontiguousarray(np.asarray(E, dtype=np.float64).ravel(order="F"))
        lib().orc_set_modulus(self._m, _p(E))

    def assemble(self):
        if lib().orc_assemble(self._m):
            raise RuntimeError("oracle: coarsest matrix not positive definite")

    def matvec(self, level, u):
        n = self.m.L[level].numDOFs
        u = np.ascontiguousarray(u, dtype=np.float64)
        y = np.zeros(n)
        lib().orc_matvec(self._m, level, _p(u), _p(y))
        return y

    def vcycle(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        x = np.zeros(self.m.L[0].numDOFs)
        lib().orc_vcycle(self._m, _p(r), _p(x))
        return x

    def restrict(self, ii, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        out = np.zeros(self.m.L[ii].numDOFs)
        lib().orc_restrict(self._m, ii, _p(r), _p(out))
        return out

    def interpolate(self, ii, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros(self.m.L[ii - 1].numDOFs)
        lib().orc_interpolate(self._m, ii, _p(x), _p(out))
        return out

    def coarsest_solve(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        x = np.zeros_like(r)
        lib().orc_coarsest_solve(self._m, _p(r), _p(x))
        return x

    def pcg(self, b, x0=None, tol=None, maxIT=None):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
        res = C.c_double(0)
        its = lib().orc_pcg(self._m, _p(b), _p(x), 0 if x0 is None else 1,
                            self.m.tol if tol is None else tol,
                            self.m.maxIT if maxIT is None else maxIT, C.byref(res))
        return x, its, res.value

    def solve_state(self, U=None):
        n = self.m.L[0].numDOFs
        warm = U is not None
        U = np.zeros((n, self.m.nLoads), order="F") if U is None else np.array(U, dtype=np.float64, order="F", copy=True)
        its = lib().orc_solve_state(self._m, _p(U), 1 if warm else 0)
        return U, its

    def unit_compliance(self, U):
        U = np.asfortranarray(U, dtype=np.float64)
        ce = np.zeros(self.m.L[0].numElements)
        fn = lib().orc_unit_compliance_super if self.super_element else lib().orc_unit_compliance
        fn(self._m, _p(U), _p(ce))
        return ce

    def pre_compute_der(self, U):
        U = np.asfortranarray(U, dtype=np.float64)
        dc = np.zeros((64, self.m.L[0].numElements), order="F")
        lib().orc_pre_compute_der(self._m, _p(U), _p(dc))
        return dc

    def pde_filter_setup(self, rMin):
        lib().orc_pde_filter_setup(self._m, rMin)

    def pde_filter(self, src):
        src = np.ascontiguousarray(src, dtype=np.float64)
        out = np.zeros(self.m.L[0].numElements)
        lib().orc_pde_filter(self._m, _p(src), _p(out))
        return out

    def set_passive(self, ids):
        """passive elements (1-based compact ids; empty clears): design 1 inside
        the OC bisection and after the filter (TOP_GPU.m:239/247, 270/273)"""
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        if lib().orc_set_passive(self._m, _p(ids), ids.size):
            raise ValueError("oracle: passive element id out of range")

    def top_opt(self, V0=0.12, rMin=np.sqrt(3), nLoop=50, ft=1):
        ne = self.m.L[0].numElements * (64 if self.super_element else 1)
        xp = np.zeros(ne)
        hist = np.zeros((max(nLoop, 1), 6))
        cs = C.c_double(0)
        n = lib().orc_top_opt(self._m, V0, rMin, nLoop, ft, _p(xp), _p(hist), C.byref(cs))
        if n < 0:
            raise RuntimeError("oracle: optimisation failed (%d)" % n)
        return xp, hist[:n], cs.value


# -- the six MEX kernels ---------------------------------------------------
def gather(u_nx3, eNod):
    u = np.asfortranarray(u_nx3, dtype=np.float64)
    e = np.asfortranarray(eNod, dtype=np.int32)
    ne = e.shape[0]
    out = np.zeros((ne, 24), order="F")
    lib().orc_gather(_p(out), _p(u), _p(e), ne, u.shape[0])
    return out


def scatter(Y_nx3, eNod, uMat):
    Y = np.array(Y_nx3, dtype=np.float64, order="F", copy=True)
    e = np.asfortranarray(eNod, dtype=np.int32)
    U = np.asfortranarray(uMat, dtype=np.float64)
    lib().orc_scatter(_p(Y), _p(e), _p(U), e.shape[0], Y.shape[0])
    return Y


def scatter_accum3(keys, Tmp, xF):
    k = np.ascontiguousarray(keys, dtype=np.int32).ravel(order="F")
    T = np.asfortranarray(Tmp, dtype=np.float64)
    X = np.array(xF, dtype=np.float64, order="F", copy=True)
    lib().orc_scatter_accum3(_p(k), _p(T), T.shape[0], _p(X), X.shape[0])
    return X


def assemble_ks_level2(upMap, eleModulus, K0, Pch, mapUnique, uFree, uFixed):
    up = np.asfortranarray(upMap, dtype=np.int32)
    nE, nCh = up.shape
    Ks = np.zeros((24, 24, nE), order="F")
    em = np.ascontiguousarray(eleModulus, dtype=np.float64).ravel(order="F")
    k0 = np.asfortranarray(K0, dtype=np.float64)
    P = np.asfortranarray(Pch, dtype=np.float64)
    mu = np.ascontiguousarray(mapUnique, dtype=np.int32)
    nU = 0 if uFree is None or np.size(uFree) == 0 else np.shape(uFree)[-1]
    fr = None if nU == 0 else np.asfortranarray(uFree, dtype=np.float64)
    fx = None if nU == 0 else np.asfortranarray(uFixed, dtype=np.float64)
    lib().orc_assemble_ks_level2(_p(Ks), _p(up), _p(em), _p(k0), _p(P), _p(mu),
                                 None if fr is None else _p(fr), None if fx is None else _p(fx), nE, nCh, nU)
    return Ks


def assemble_ks_higher(upMap, KsPrev, Psub):
    up = np.asfortranarray(upMap, dtype=np.int32)
    nE, nS = up.shape
    Ks = np.zeros((24, 24, nE), order="F")
    kp = np.asfortranarray(KsPrev, dtype=np.float64)
    P = np.asfortranarray(Psub, dtype=np.float64)
    lib().orc_assemble_ks_higher(_p(Ks), _p(up), _p(kp), _p(P), nE, nS)
    return Ks


def assemble_ks_level2_super(upMap, Ks0, Psub, mapUnique, eleModulus, uFree, uFixed):
    up = np.asfortranarray(upMap, dtype=np.int32)
    nE, nS = up.shape
    Ks = np.zeros((24, 24, nE), order="F")
    k0 = np.asfortranarray(Ks0, dtype=np.float64)
    P = np.asfortranarray(Psub, dtype=np.float64)
    mu = np.ascontiguousarray(mapUnique, dtype=np.int32)
    em = np.asfortranarray(eleModulus, dtype=np.float64)
    nU = 0 if uFree is None or np.size(uFree) == 0 else np.shape(uFixed)[-1]
    fr = None if nU == 0 else np.asfortranarray(uFree, dtype=np.float64)
    fx = None if nU == 0 else np.asfortranarray(uFixed, dtype=np.float64)
    lib().orc_assemble_ks_level2_super(_p(Ks), _p(up), _p(k0), _p(P), _p(mu), _p(em),
                                       None if fr is None else _p(fr), None if fx is None else _p(fx), nE, nS, nU)
    return Ks
