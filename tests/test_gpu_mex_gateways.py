"""The six MEX gateway sources (top_gpu_on_matlab_b200/mex/*.cpp, built
against the MEX stand-in by tests/mex_build.sh) next to the reference's own
gateways (its .cu files compiled unmodified against the same stand-in): the
same mxArrays in, the same in-place results out, and the same error
identifiers for a wrong class and a wrong shape."""
import subprocess
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import refkernels as R

ROOT = Path(__file__).resolve().parents[1]
GW = ROOT / "tests" / "_mexgw"

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="reference kernels not built")]


@pytest.fixture(scope="module")
def mx():
    subprocess.run(["bash", str(ROOT / "tests" / "mex_build.sh")], check=True)
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


def _both(name, out_ref, out_ours, *args):
    R.call(name, out_ref, *args)
    R.call(name, out_ours, *args, libdir=GW)


def _ids(name, *args):
    """error identifiers of the reference's gateway and ours on the same call"""
    ids = []
    for d in (None, GW):
        with pytest.raises(R.RefError) as e:
            R.call(name, *args, libdir=d)
        ids.append(e.value.identifier)
    return ids


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_gathering(mx, model, dt):
    L = model.level(0)
    tdt = torch.float64 if dt == np.float64 else torch.float32
    u = np.random.default_rng(0).standard_normal((L.numNodes, 3)).astype(dt)
    ref, ours = mx.zeros((L.numElements, 24), dtype=tdt), mx.zeros((L.numElements, 24), dtype=tdt)
    gU, gE = mx.gpu_array(u), mx.gpu_array(L.eNodMat.astype(np.int32))
    _both("Gathering_inplace", ref, ours, gU, gE)
    assert np.array_equal(mx.gather(ref), mx.gather(ours))
    # class: int64 nodes; shape: a 23-column output
    assert _ids("Gathering_inplace", ours, gU, mx.gpu_array(L.eNodMat.astype(np.float64))) == ["Gathering_inplace:Type"] * 2
    assert _ids("Gathering_inplace", mx.zeros((L.numElements, 23), dtype=tdt), gU, gE) == ["Gathering_inplace:Shape"] * 2


def test_scattering(mx, model):
    L = model.level(0)
    uMat = np.random.default_rng(1).standard_normal((L.numElements, 24))
    Yr, Yo = mx.gpu_array(np.zeros((L.numNodes, 3))), mx.gpu_array(np.zeros((L.numNodes, 3)))
    eN, gU = mx.gpu_array(L.eNodMat.astype(np.int32)), mx.gpu_array(uMat)
    _both("Scattering_inplace", Yr, Yo, eN, gU)
    assert _rel(mx.gather(Yo), mx.gather(Yr)) < 1e-14
    assert _ids("Scattering_inplace", Yo, mx.gpu_array(L.eNodMat.astype(np.float64)), gU) == ["Scattering_inplace:type"] * 2
    assert _ids("Scattering_inplace", mx.gpu_array(np.zeros((L.numNodes, 4))), eN, gU) == ["Scattering_inplace:shape"] * 2


def test_scatter_accum3(mx):
    rng = np.random.default_rng(2)
    N, M = 5000, 800
    keys = mx.gpu_array(rng.integers(-2, M + 3, N).astype(np.int32))
    Tmp = mx.gpu_array(rng.standard_normal((N, 3)))
    Xr, Xo = mx.gpu_array(np.zeros((M, 3))), mx.gpu_array(np.zeros((M, 3)))
    R.call("scatter_accum3_inplace", keys, Tmp, Xr)
    R.call("scatter_accum3_inplace", keys, Tmp, Xo, libdir=GW)
    assert _rel(mx.gather(Xo), mx.gather(Xr)) < 1e-14
    assert _ids("scatter_accum3_inplace", keys, mx.gpu_array(np.zeros((N, 3), np.float32)), Xo) == ["scatter_accum3:type"] * 2
    assert _ids("scatter_accum3_inplace", keys, mx.gpu_array(np.zeros((N, 2))), Xo) == ["scatter_accum3:shape"] * 2


def test_assemble_level2(mx, model):
    L0, L1 = model.level(0), model.level(1)
    E = 0.05 + np.random.default_rng(3).random(L0.numElements)
    mu = model.mapUniqueKes()
    fr, fx = model.uniqueKes()
    args = (mx.gpu_array(L1.elementUpwardMap.astype(np.int32)), mx.gpu_array(E), mx.gpu_array(L0.Ke),
            mx.gpu_array(_pch(4)), mx.gpu_array(mu.astype(np.int32)), mx.gpu_array(fr), mx.gpu_array(fx))
    Kr, Ko = mx.zeros((24, 24, L1.numElements)), mx.zeros((24, 24, L1.numElements))
    _both("assembleKs_level2_inplace", Kr, Ko, *args)
    assert _rel(mx.gather(Ko), mx.gather(Kr)) < 1e-13
    bad = list(args)
    bad[0] = mx.gpu_array(L1.elementUpwardMap.astype(np.float64))
    assert _ids("assembleKs_level2_inplace", Ko, *bad) == ["assembleKs_level2_inplace:Type"] * 2
    bad = list(args)
    bad[3] = mx.gpu_array(_pch(2))
    assert _ids("assembleKs_level2_inplace", Ko, *bad) == ["assembleKs_level2_inplace:Shape"] * 2


def test_assemble_higher(mx, model):
    L1, L2 = model.level(1), model.level(2)
    A = np.random.default_rng(5).standard_normal((24, 24, L1.numElements))
    KsPrev = mx.gpu_array(np.einsum("ijk,ljk->ilk", A, A))
    up, P = mx.gpu_array(L2.elementUpwardMap.astype(np.int32)), mx.gpu_array(_pch(2))
    Kr, Ko = mx.zeros((24, 24, L2.numElements)), mx.zeros((24, 24, L2.numElements))
    _both("assembleKs_higherLevel_inplace", Kr, Ko, up, KsPrev, P)
    assert _rel(mx.gather(Ko), mx.gather(Kr)) < 1e-13
    assert _ids("assembleKs_higherLevel_inplace", Ko, up, KsPrev, mx.gpu_array(_pch(2).astype(np.float32))) == \
        ["assembleKs_higherLevel_inplace:Type"] * 2
    assert _ids("assembleKs_higherLevel_inplace", Ko, up, KsPrev, mx.gpu_array(_pch(4))) == \
        ["assembleKs_higherLevel_inplace:Shape"] * 2


def test_assemble_super(mx):
    m = O.Model(np.ones((6, 12, 6), bool), super_element=1)
    m.apply_optcase(1)
    L0, L1 = m.level(0), m.level(1)
    Esub = 0.05 + np.random.default_rng(6).random((64, L0.numElements))
    fr, fx = m.uniqueKes()
    args = (mx.gpu_array(L1.elementUpwardMap.astype(np.int32)), mx.gpu_array(m.I_mat() @ Esub), mx.gpu_array(_pch(4)),
            mx.gpu_array(m.mapUniqueKes().astype(np.int32)), mx.gpu_array(Esub),
            mx.gpu_array(fr.reshape(576, 64, -1, order="F")), mx.gpu_array(fx))
    Kr, Ko = mx.zeros((24, 24, L1.numElements)), mx.zeros((24, 24, L1.numElements))
    _both("assembleKs_level2_superEle_inplace", Kr, Ko, *args)
    assert _rel(mx.gather(Ko), mx.gather(Kr)) < 1e-13
    bad = list(args)
    bad[4] = mx.gpu_array(Esub.astype(np.float32))
    assert _ids("assembleKs_level2_superEle_inplace", Ko, *bad) == ["assembleKs_level2_superEle_inplace:Type"] * 2
    bad = list(args)
    bad[4] = mx.gpu_array(Esub[:63])
    assert _ids("assembleKs_level2_superEle_inplace", Ko, *bad) == ["assembleKs_level2_superEle_inplace:Shape"] * 2
