"""The allocation-free level-2 assembly entry point against the regular one.

top_assemble_ks_level2_noalloc serves callers that cannot let the library
allocate device memory inside a call (a MEX gateway living under MATLAB's
gpuArray memory pool, or an application that reserves its memory once and
must avoid cudaMalloc/cudaFree synchronisation).  The test calls it through
the C ABI three times in a row and compares each result with
top_assemble_ks_level2:
  1. a 64-child level-2 assembly with fixed-DOF children;
  2. the same with a NaN in the element matrix, which fills every row of the
     fixed scratch with NaN (both entry points return NaN there);
  3. an 8-child assembly on the next level, whose GEMM still loads scratch
     rows 8..63: it is finite only if the call clears what call 2 left.
It also checks, through the device's default memory pool, that a call of the
allocation-free entry point takes no pool memory while the regular one does.
It lives in a file of its own so that it runs last.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _pch(span):
    RI, SUB = O.ri_table(span), O.subele_nodmat(span)
    P = np.zeros((24, 24, span ** 3))
    for s in range(span ** 3):
        for i in range(8):
            for c in range(3):
                P[3 * i + c, c::3, s] = RI[SUB[s, i] - 1, :]
    return P


def _col(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a).ravel(order="F"))).to("cuda", dtype)


def _both(upMap, E, K0, P, mu, fr, fx):
    from top_gpu_on_matlab_b200._lib import TOP_F64, check, lib
    nE, nCh = upMap.shape
    nU = fr.shape[1] if fr is not None else 0
    args = [_col(upMap, torch.int32), _col(E), _col(K0), _col(P), _col(mu, torch.int32)]
    fr_t = _col(fr) if nU else None
    fx_t = _col(fx) if nU else None
    out = []
    for name in ("top_assemble_ks_level2", "top_assemble_ks_level2_noalloc"):
        Ks = torch.full((576 * nE,), float("nan"), dtype=torch.float64, device="cuda")
        fn = getattr(lib(), name)
        check(fn(Ks.data_ptr(), args[0].data_ptr(), args[1].data_ptr(), args[2].data_ptr(), args[3].data_ptr(),
                 args[4].data_ptr(), fr_t.data_ptr() if nU else None, fx_t.data_ptr() if nU else None,
                 nE, nCh, E.size, nU, TOP_F64, None), name)
        out.append(Ks.cpu().numpy())
    return out


def test_noalloc_matches_regular_entry_point_three_calls():
    # call 1: level-2 Galerkin assembly, 64 children, with fixed-DOF children
    m = O.Model(np.ones((8, 16, 8), bool))
    m.apply_optcase(1)
    L0, L1, L2 = m.level(0), m.level(1), m.level(2)
    E = 0.05 + np.random.default_rng(21).random(L0.numElements)
    fr, fx = m.uniqueKes()
    ref, new = _both(L1.elementUpwardMap, E, L0.Ke, _pch(4), m.mapUniqueKes(), fr, fx)
    assert np.isfinite(new).all()
    assert np.abs(new - ref).max() <= 1e-13 * np.abs(ref).max()
    # call 2: a NaN in K0 makes every child matrix Q_s = P_s' K0 P_s NaN, so
    # all 64 scratch rows hold NaN afterwards; both entry points agree on it
    K0nan = np.array(L0.Ke, copy=True)
    K0nan[0, 0] = np.nan
    ref_n, new_n = _both(L1.elementUpwardMap, E, K0nan, _pch(4), m.mapUniqueKes(), fr, fx)
    assert np.array_equal(np.isnan(new_n), np.isnan(ref_n)) and np.isnan(new_n).any()
    # call 3: 8 children on the next level (different sizes, no boundary lists);
    # its GEMM multiplies scratch rows 8..63 by zero, so a result that is
    # finite and equal to the regular one shows those rows were cleared
    E2 = 0.2 + np.random.default_rng(22).random(L1.numElements)
    ref2, new2 = _both(L2.elementUpwardMap, E2, L1.Ke, _pch(2), np.zeros(L1.numElements, np.int32), None, None)
    assert np.isfinite(new2).all()
    assert np.abs(new2 - ref2).max() <= 1e-13 * np.abs(ref2).max()


def _pool_used_high():
    """(reset, read) of the high-water mark of memory in use from the current
    device's default memory pool (the pool cudaMallocAsync draws on), through
    the driver API."""
    import ctypes as C
    cu = C.CDLL("libcuda.so.1")
    dev = C.c_int(0)
    assert cu.cuCtxGetDevice(C.byref(dev)) == 0
    pool = C.c_void_p()
    assert cu.cuDeviceGetDefaultMemPool(C.byref(pool), dev) == 0
    USED_MEM_HIGH = 8                                   # CU_MEMPOOL_ATTR_USED_MEM_HIGH

    def reset():
        zero = C.c_uint64(0)
        assert cu.cuMemPoolSetAttribute(pool, USED_MEM_HIGH, C.byref(zero)) == 0

    def read():
        v = C.c_uint64(0)
        assert cu.cuMemPoolGetAttribute(pool, USED_MEM_HIGH, C.byref(v)) == 0
        return v.value
    return reset, read


def test_noalloc_takes_no_pool_memory():
    from top_gpu_on_matlab_b200._lib import TOP_F64, check, lib
    m = O.Model(np.ones((8, 16, 8), bool))
    m.apply_optcase(1)
    L0, L1 = m.level(0), m.level(1)
    E = 0.05 + np.random.default_rng(23).random(L0.numElements)
    fr, fx = m.uniqueKes()
    up, nE, nCh = L1.elementUpwardMap, L1.elementUpwardMap.shape[0], L1.elementUpwardMap.shape[1]
    args = [_col(up, torch.int32), _col(E), _col(L0.Ke), _col(_pch(4)), _col(m.mapUniqueKes(), torch.int32),
            _col(fr), _col(fx)]
    Ks = torch.zeros(576 * nE, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    reset, read = _pool_used_high()
    used = {}
    for name in ("top_assemble_ks_level2_noalloc", "top_assemble_ks_level2"):
        fn = getattr(lib(), name)
        fn(Ks.data_ptr(), *[a.data_ptr() for a in args[:5]], None, None, nE, nCh, E.size, 0, TOP_F64, None)
        torch.cuda.synchronize()
        reset()
        check(fn(Ks.data_ptr(), *[a.data_ptr() for a in args], nE, nCh, E.size, fr.shape[1], TOP_F64, None), name)
        torch.cuda.synchronize()
        used[name] = read()
    assert used["top_assemble_ks_level2_noalloc"] == 0, used
    assert used["top_assemble_ks_level2"] >= 576 * 64 * 8, used


def test_noalloc_rejects_more_than_64_children():
    from top_gpu_on_matlab_b200._lib import TOP_ERR_SHAPE, TOP_F64, lib
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    st = lib().top_assemble_ks_level2_noalloc(dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
                                              dummy.data_ptr(), dummy.data_ptr(), None, None, 1, 65, 1, 0, TOP_F64, None)
    assert st == TOP_ERR_SHAPE
