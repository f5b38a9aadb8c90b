"""The allocation-free level-2 assembly entry point against the regular one.

top_assemble_ks_level2_noalloc serves callers that cannot let the library
allocate device memory inside a call (a MEX gateway living under MATLAB's
gpuArray memory pool, or an application that reserves its memory once and
must avoid cudaMalloc/cudaFree synchronisation).  This test calls it through
the C ABI twice in a row -- a 64-child level-2 assembly, then an 8-child one
that only works if the fixed scratch left behind by the first call is
cleared -- and compares each result with top_assemble_ks_level2.  It lives in
a file of its own so that it runs last.
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


def test_noalloc_matches_regular_entry_point_twice():
    # call 1: level-2 Galerkin assembly, 64 children, with fixed-DOF children
    m = O.Model(np.ones((8, 16, 8), bool))
    m.apply_optcase(1)
    L0, L1, L2 = m.level(0), m.level(1), m.level(2)
    E = 0.05 + np.random.default_rng(21).random(L0.numElements)
    fr, fx = m.uniqueKes()
    ref, new = _both(L1.elementUpwardMap, E, L0.Ke, _pch(4), m.mapUniqueKes(), fr, fx)
    assert np.isfinite(new).all()
    assert np.abs(new - ref).max() <= 1e-13 * np.abs(ref).max()
    # call 2: 8 children on the next level (different sizes, no boundary lists);
    # the scratch rows 8..63 written by call 1 must not leak into the result
    E2 = 0.2 + np.random.default_rng(22).random(L1.numElements)
    ref2, new2 = _both(L2.elementUpwardMap, E2, L1.Ke, _pch(2), np.zeros(L1.numElements, np.int32), None, None)
    assert np.isfinite(new2).all()
    assert np.abs(new2 - ref2).max() <= 1e-13 * np.abs(ref2).max()


def test_noalloc_rejects_more_than_64_children():
    from top_gpu_on_matlab_b200._lib import TOP_ERR_SHAPE, TOP_F64, lib
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    st = lib().top_assemble_ks_level2_noalloc(dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
                                              dummy.data_ptr(), dummy.data_ptr(), None, None, 1, 65, 1, 0, TOP_F64, None)
    assert st == TOP_ERR_SHAPE
