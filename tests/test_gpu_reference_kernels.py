"""Drop-ins and oracle vs the reference's own CUDA kernels, compiled unmodified
for sm_100a (oracle/_ref, built by oracle/ref_build.sh)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import refkernels as R

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="reference kernels not built")]


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


def _pch(span):
    RI, SUB = O.ri_table(span), O.subele_nodmat(span)
    P = np.zeros((24, 24, span ** 3))
    for s in range(span ** 3):
        for i in range(8):
            for c in range(3):
                P[3 * i + c, c::3, s] = RI[SUB[s, i] - 1, :]
    return P


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_gather_bit_exact_vs_reference(mx, model, dt):
    L = model.level(0)
    u = np.random.default_rng(0).standard_normal((L.numNodes, 3)).astype(dt)
    tdt = torch.float64 if dt == np.float64 else torch.float32
    ref, ours = mx.zeros((L.numElements, 24), dtype=tdt), mx.zeros((L.numElements, 24), dtype=tdt)
    gU, gE = mx.gpu_array(u), mx.gpu_array(L.eNodMat.astype(np.int32))
    R.call("Gathering_inplace", ref, gU, gE)
    mx.Gathering_inplace(ours, gU, gE)
    torch.cuda.synchronize()
    assert np.array_equal(mx.gather(ref), mx.gather(ours))
    assert np.array_equal(mx.gather(ref).astype(float), O.gather(u.astype(float), L.eNodMat))


def test_scatter_vs_reference(mx, model):
    L = model.level(0)
    rng = np.random.default_rng(1)
    uMat = rng.standard_normal((L.numElements, 24))
    Yr, Yo = mx.gpu_array(np.zeros((L.numNodes, 3))), mx.gpu_array(np.zeros((L.numNodes, 3)))
    eN, gU = mx.gpu_array(L.eNodMat.astype(np.int32)), mx.gpu_array(uMat)
    R.call("Scattering_inplace", Yr, eN, gU)
    mx.Scattering_inplace(Yo, eN, gU)
    ref = mx.gather(Yr)
    assert _rel(mx.gather(Yo), ref) < 1e-14
    assert _rel(O.scatter(np.zeros((L.numNodes, 3)), L.eNodMat, uMat), ref) < 1e-14


def test_scatter_accum3_vs_reference(mx):
    rng = np.random.default_rng(2)
    N, M = 5000, 800
    keys = rng.integers(-2, M + 3, N).astype(np.int32)
    Tmp = rng.standard_normal((N, 3))
    Xr, Xo = mx.gpu_array(np.zeros((M, 3))), mx.gpu_array(np.zeros((M, 3)))
    R.call("scatter_accum3_inplace", mx.gpu_array(keys), mx.gpu_array(Tmp), Xr)
    mx.scatter_accum3_inplace(mx.gpu_array(keys), mx.gpu_array(Tmp), Xo)
    torch.cuda.synchronize()
    ref = mx.gather(Xr)
    assert _rel(mx.gather(Xo), ref) < 1e-14
    assert _rel(O.scatter_accum3(keys, Tmp, np.zeros((M, 3))), ref) < 1e-14


def test_assemble_level2_vs_reference(mx, model):
    L0, L1 = model.level(0), model.level(1)
    E = 0.05 + np.random.default_rng(3).random(L0.numElements)
    P = _pch(4)
    mu = model.mapUniqueKes()
    fr, fx = model.uniqueKes()
    args = lambda: (mx.gpu_array(L1.elementUpwardMap.astype(np.int32)), mx.gpu_array(E), mx.gpu_array(L0.Ke.ravel(order="F")),
                    mx.gpu_array(P), mx.gpu_array(mu.astype(np.int32)), mx.gpu_array(fr), mx.gpu_array(fx))
    Kr, Ko = mx.zeros((24, 24, L1.numElements)), mx.zeros((24, 24, L1.numElements))
    R.call("assembleKs_level2_inplace", Kr, *args())
    mx.assembleKs_level2_inplace(Ko, *args())
    ref = mx.gather(Kr)
    assert _rel(mx.gather(Ko), ref) < 1e-13
    assert _rel(O.assemble_ks_level2(L1.elementUpwardMap, E, L0.Ke, P, mu, fr, fx), ref) < 1e-14


def test_assemble_higher_vs_reference(mx, model):
    L1, L2 = model.level(1), model.level(2)
    A = np.random.default_rng(5).standard_normal((24, 24, L1.numElements))
    KsPrev = np.einsum("ijk,ljk->ilk", A, A)
    P = _pch(2)
    Kr, Ko = mx.zeros((24, 24, L2.numElements)), mx.zeros((24, 24, L2.numElements))
    up = mx.gpu_array(L2.elementUpwardMap.astype(np.int32))
    R.call("assembleKs_higherLevel_inplace", Kr, up, mx.gpu_array(KsPrev), mx.gpu_array(P))
    mx.assembleKs_higherLevel_inplace(Ko, up, mx.gpu_array(KsPrev), mx.gpu_array(P))
    ref = mx.gather(Kr)
    assert _rel(mx.gather(Ko), ref) < 1e-13
    assert _rel(O.assemble_ks_higher(L2.elementUpwardMap, KsPrev, P), ref) < 1e-14


def test_assemble_super_vs_reference(mx):
    m = O.Model(np.ones((6, 12, 6), bool), super_element=1)
    m.apply_optcase(1)
    L0, L1 = m.level(0), m.level(1)
    Esub = 0.05 + np.random.default_rng(6).random((64, L0.numElements))
    Ks0 = m.I_mat() @ Esub
    P = _pch(4)
    mu = m.mapUniqueKes()
    fr, fx = m.uniqueKes()
    fr3 = fr.reshape(576, 64, -1, order="F")
    args = lambda: (mx.gpu_array(L1.elementUpwardMap.astype(np.int32)), mx.gpu_array(Ks0), mx.gpu_array(P),
                    mx.gpu_array(mu.astype(np.int32)), mx.gpu_array(Esub), mx.gpu_array(fr3), mx.gpu_array(fx))
    Kr, Ko = mx.zeros((24, 24, L1.numElements)), mx.zeros((24, 24, L1.numElements))
    R.call("assembleKs_level2_superEle_inplace", Kr, *args())
    mx.assembleKs_level2_superEle_inplace(Ko, *args())
    ref = mx.gather(Kr)
    assert _rel(mx.gather(Ko), ref) < 1e-13
    assert _rel(O.assemble_ks_level2_super(L1.elementUpwardMap, Ks0, P, mu, Esub, fr3, fx), ref) < 1e-14


def test_reference_error_ids_match_ours(mx, model):
    from top_gpu_on_matlab_b200 import TopGpuError
    L = model.level(0)
    gU = mx.gpu_array(np.zeros((L.numNodes, 3)))
    gE = mx.gpu_array(L.eNodMat.astype(np.int32))
    bad = mx.zeros((L.numElements, 23))
    with pytest.raises(R.RefError) as er:
        R.call("Gathering_inplace", bad, gU, gE)
    with pytest.raises(TopGpuError) as eo:
        mx.Gathering_inplace(bad, gU, gE)
    assert er.value.identifier == eo.value.identifier == "Gathering_inplace:Shape"
