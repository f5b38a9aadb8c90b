"""The six MEX drop-ins on the GPU vs the oracle's restatement of the reference kernels."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mx():
    from top_gpu_on_matlab_b200 import mex
    return mex


@pytest.fixture(scope="module")
def model():
    m = O.Model(np.ones((8, 16, 8), bool))
    m.apply_optcase(1)
    return m


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("u32", [False, True])
def test_gathering_inplace_bit_exact(mx, model, dt, u32):
    L = model.level(0)
    u = np.random.default_rng(0).standard_normal((L.numNodes, 3)).astype(dt)
    eN = L.eNodMat.astype(np.uint32 if u32 else np.int32)
    gU = mx.gpu_array(u)
    gE = mx.gpu_array(eN)
    gUMat = mx.zeros((L.numElements, 24), dtype=torch.float64 if dt == np.float64 else torch.float32)
    mx.Gathering_inplace(gUMat, gU, gE)
    torch.cuda.synchronize()
    ref = O.gather(u.astype(np.float64), L.eNodMat)
    assert np.array_equal(mx.gather(gUMat).astype(np.float64), ref)


@pytest.mark.parametrize("dt,tol", [(np.float64, 1e-14), (np.float32, 1e-5)])
def test_scattering_inplace(mx, model, dt, tol):
    L = model.level(0)
    rng = np.random.default_rng(1)
    uMat = rng.standard_normal((L.numElements, 24)).astype(dt)
    Y0 = rng.standard_normal((L.numNodes, 3)).astype(dt)
    eN = L.eNodMat.copy()
    eN[3, 2] = 0                    # skipped: outside [1, numNodes]
    eN[7, 5] = L.numNodes + 5
    Y = mx.gpu_array(Y0)
    mx.Scattering_inplace(Y, mx.gpu_array(eN.astype(np.int32)), mx.gpu_array(uMat))
    ref = O.scatter(Y0.astype(np.float64), eN, uMat.astype(np.float64))
    assert _rel(mx.gather(Y).astype(np.float64), ref) < tol


@pytest.mark.parametrize("dt,tol", [(np.float64, 1e-14), (np.float32, 1e-5)])
def test_scatter_accum3_inplace(mx, dt, tol):
    rng = np.random.default_rng(2)
    N, M = 20000, 3000
    keys = rng.integers(-3, M + 4, N).astype(np.int32)
    Tmp = rng.standard_normal((N, 3)).astype(dt)
    X0 = rng.standard_normal((M, 3)).astype(dt)
    X = mx.gpu_array(X0)
    mx.scatter_accum3_inplace(mx.gpu_array(keys), mx.gpu_array(Tmp), X)
    torch.cuda.synchronize()
    ref = O.scatter_accum3(keys, Tmp.astype(np.float64), X0.astype(np.float64))
    assert _rel(mx.gather(X).astype(np.float64), ref) < tol


def _pch(span):
    RI, SUB = O.ri_table(span), O.subele_nodmat(span)
    nch = span ** 3
    P = np.zeros((24, 24, nch))
    for s in range(nch):
        for i in range(8):
            for c in range(3):
                P[3 * i + c, c::3, s] = RI[SUB[s, i] - 1, :]
    return P


@pytest.mark.parametrize("with_bc", [True, False])
def test_assembleKs_level2_inplace(mx, model, with_bc):
    L0, L1 = model.level(0), model.level(1)
    E = 0.05 + np.random.default_rng(3).random(L0.numElements)
    P = _pch(4)
    mu = model.mapUniqueKes()
    fr, fx = model.uniqueKes()
    if not with_bc:
        fr = fx = np.zeros((576, 0))
    ref = O.assemble_ks_level2(L1.elementUpwardMap, E, L0.Ke, P, mu, fr if with_bc else None, fx if with_bc else None)
    Ks = mx.zeros((24, 24, L1.numElements))
    mx.assembleKs_level2_inplace(Ks, mx.gpu_array(L1.elementUpwardMap.astype(np.int32)), mx.gpu_array(E),
                                 mx.gpu_array(L0.Ke.ravel(order="F")), mx.gpu_array(P), mx.gpu_array(mu.astype(np.int32)),
                                 mx.gpu_array(fr), mx.gpu_array(fx))
    assert _rel(mx.gather(Ks), ref) < 1e-13


def test_assembleKs_level2_inplace_single(mx, model):
    L0, L1 = model.level(0), model.level(1)
    E = (0.05 + np.random.default_rng(4).random(L0.numElements)).astype(np.float32)
    P = _pch(4).astype(np.float32)
    mu = model.mapUniqueKes()
    fr, fx = (a.astype(np.float32) for a in model.uniqueKes())
    ref = O.assemble_ks_level2(L1.elementUpwardMap, E.astype(float), L0.Ke, P.astype(float), mu, fr.astype(float), fx.astype(float))
    Ks = mx.zeros((24, 24, L1.numElements), dtype=torch.float32)
    mx.assembleKs_level2_inplace(Ks, mx.gpu_array(L1.elementUpwardMap.astype(np.int32)), mx.gpu_array(E),
                                 mx.gpu_array(L0.Ke.ravel(order="F").astype(np.float32)), mx.gpu_array(P),
                                 mx.gpu_array(mu.astype(np.int32)), mx.gpu_array(fr), mx.gpu_array(fx))
    assert _rel(mx.gather(Ks).astype(float), ref) < 1e-5


def test_assembleKs_higherLevel_inplace(mx, model):
    L1, L2 = model.level(1), model.level(2)
    rng = np.random.default_rng(5)
    A = rng.standard_normal((24, 24, L1.numElements))
    KsPrev = np.einsum("ijk,ljk->ilk", A, A)
    P = _pch(2)
    ref = O.assemble_ks_higher(L2.elementUpwardMap, KsPrev, P)
    Ks = mx.zeros((24, 24, L2.numElements))
    mx.assembleKs_higherLevel_inplace(Ks, mx.gpu_array(L2.elementUpwardMap.astype(np.int32)), mx.gpu_array(KsPrev), mx.gpu_array(P))
    assert _rel(mx.gather(Ks), ref) < 1e-13


def test_assembleKs_level2_superEle_inplace(mx):
    m = O.Model(np.ones((6, 12, 6), bool), super_element=1)
    m.apply_optcase(1)
    L0, L1 = m.level(0), m.level(1)
    rng = np.random.default_rng(6)
    Esub = 0.05 + rng.random((64, L0.numElements))
    I = m.I_mat()
    Ks0 = I @ Esub
    P = _pch(4)
    mu = m.mapUniqueKes()
    fr, fx = m.uniqueKes()
    ref = O.assemble_ks_level2_super(L1.elementUpwardMap, Ks0, P, mu, Esub, fr.reshape(576, 64, -1, order="F"), fx)
    Ks = mx.zeros((24, 24, L1.numElements))
    mx.assembleKs_level2_superEle_inplace(Ks, mx.gpu_array(L1.elementUpwardMap.astype(np.int32)), mx.gpu_array(Ks0),
                                          mx.gpu_array(P), mx.gpu_array(mu.astype(np.int32)), mx.gpu_array(Esub),
                                          mx.gpu_array(fr.reshape(576, 64, -1, order="F")), mx.gpu_array(fx))
    assert _rel(mx.gather(Ks), ref) < 1e-13


def test_error_identifiers(mx, model):
    from top_gpu_on_matlab_b200 import TopGpuError
    L = model.level(0)
    gU = mx.gpu_array(np.zeros((L.numNodes, 3)))
    gE = mx.gpu_array(L.eNodMat.astype(np.int32))
    with pytest.raises(TopGpuError) as ei:
        mx.Gathering_inplace(mx.zeros((L.numElements, 24), dtype=torch.float32), gU, gE)
    assert ei.value.identifier == "Gathering_inplace:Type"
    with pytest.raises(TopGpuError) as ei:
        mx.Gathering_inplace(mx.zeros((L.numElements, 23)), gU, gE)
    assert ei.value.identifier == "Gathering_inplace:Shape"
    with pytest.raises(TopGpuError) as ei:
        mx.scatter_accum3_inplace(mx.gpu_array(np.ones(4, np.int32)), mx.gpu_array(np.zeros((4, 3))),
                                  mx.gpu_array(np.zeros((4, 3), np.float32)))
    assert ei.value.identifier == "scatter_accum3:Type"
    with pytest.raises(TopGpuError) as ei:
        mx.assembleKs_level2_inplace(mx.zeros((24, 24, 3)), mx.gpu_array(np.ones((2, 8), np.int32)), mx.gpu_array(np.ones(4)),
                                     mx.gpu_array(np.ones(576)), mx.gpu_array(np.ones((24, 24, 8))),
                                     mx.gpu_array(np.zeros(4, np.int32)), None, None)
    assert ei.value.identifier == "assembleKs_level2_inplace:Shape"


def test_empty_inputs(mx):
    gU = mx.gpu_array(np.zeros((5, 3)))
    mx.Gathering_inplace(mx.zeros((0, 24)), gU, mx.zeros((0, 8), dtype=torch.int32))
    Y = mx.gpu_array(np.ones((5, 3)))
    mx.Scattering_inplace(Y, mx.zeros((0, 8), dtype=torch.int32), mx.zeros((0, 24)))
    assert np.array_equal(mx.gather(Y), np.ones((5, 3)))
