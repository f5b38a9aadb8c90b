"""Result files (CPU): the history .dat formats of TOP_GPU.m:307-321 against
hand-written lines, the NIfTI-1 volume read back field by field, and the
super-element spatial order (gen_index_mapping, TOP_GPU.m:2673-2697) against
the block placement of IO_ExportDesignInVolume_nii (TOP_GPU.m:548-567)."""
import struct

import numpy as np
import pytest

from top_gpu_on_matlab_b200 import results as R
from top_gpu_on_matlab_b200.fea import Mesh


def test_fprintf_formats():
    assert R._fmt_e(1234.5, 30, 16) == "        1.2345000000000000e+03"
    assert R._fmt_e(0.0, 30, 16) == "        0.0000000000000000e+00"
    assert R._fmt_e(-2.0 ** -30, 30, 16) == "       -9.3132257461547852e-10"
    assert R._fmt_e(-0.375, 30, 16) == "       -3.7500000000000000e-01"
    assert R._fmt_e(1e100, 30, 16) == "       1.0000000000000000e+100"
    assert R._fmt_e(0.0123, 16, 6) == "    1.230000e-02"
    assert R._fmt_e(float("nan"), 16, 6) == "             NaN"
    assert R._fmt_e(float("-inf"), 16, 6) == "            -Inf"


def _records(n, rng):
    return [dict(c=float(rng.random() * 100), sharp=float(rng.random()), msTotal=float(rng.random() * 50),
                 msSolve=float(rng.random() * 20), pcgIts=int(rng.integers(5, 60))) for _ in range(n)]


def test_history_files(tmp_path):
    recs = _records(7, np.random.default_rng(0))
    R.write_history(tmp_path, recs)
    read = lambda name: (tmp_path / name).read_text().splitlines()
    assert read("c_Target.dat") == ["%30.16e" % r["c"] for r in recs]
    assert read("sharp_Target.dat") == ["%30.16e" % r["sharp"] for r in recs]
    assert read("timing_Target.dat") == ["%16.6e" % (r["msTotal"] / 1e3) for r in recs]
    assert read("solvetiming_Target.dat") == ["%16.6e" % (r["msSolve"] / 1e3) for r in recs]
    assert read("iters_Target.dat") == [str(r["pcgIts"]) for r in recs]
    assert all(len(l) == 30 for l in read("c_Target.dat"))
    import json
    h = json.loads((tmp_path / "history.json").read_text())
    assert [r["iteration"] for r in h] == list(range(1, 8))
    assert all(r["c"] == q["c"] and r["total_s"] == q["msTotal"] / 1e3 and r["cg_s"] == q["msSolve"] / 1e3
               for r, q in zip(h, recs))
    R.write_history(tmp_path, recs, iters=[3, 4, 5])          # per-solve counts (several load cases)
    assert read("iters_Target.dat") == ["3", "4", "5"]


def _read_nifti(path):
    b = path.read_bytes()
    h = {"sizeof_hdr": struct.unpack_from("<i", b, 0)[0], "dim": struct.unpack_from("<8h", b, 40),
         "datatype": struct.unpack_from("<h", b, 70)[0], "bitpix": struct.unpack_from("<h", b, 72)[0],
         "pixdim": struct.unpack_from("<8f", b, 76), "vox_offset": struct.unpack_from("<f", b, 108)[0],
         "sform_code": struct.unpack_from("<h", b, 254)[0], "srow": struct.unpack_from("<12f", b, 280),
         "magic": b[344:348]}
    dt = {64: "<f8", 16: "<f4"}[h["datatype"]]
    n = int(np.prod(h["dim"][1:1 + h["dim"][0]]))
    data = np.frombuffer(b, dtype=dt, count=n, offset=int(h["vox_offset"]))
    return h, data.reshape(h["dim"][1:4], order="F")


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_nifti_volume(tmp_path, dtype):
    v = np.random.default_rng(1).random((3, 4, 5)).astype(dtype)
    p = tmp_path / "v.nii"
    R.write_nifti(p, v)
    h, back = _read_nifti(p)
    assert h["sizeof_hdr"] == 348 and h["magic"] == b"n+1\x00" and h["vox_offset"] == 352.0
    assert h["dim"] == (3, 3, 4, 5, 1, 1, 1, 1)
    assert (h["datatype"], h["bitpix"]) == ((64, 64) if dtype == np.float64 else (16, 32))
    assert h["pixdim"][1:4] == (1.0, 1.0, 1.0) and h["sform_code"] == 1
    assert h["srow"] == (1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0)
    assert p.stat().st_size == 352 + v.nbytes
    assert np.array_equal(back, v)


def test_design_volume_places_compact_elements():
    mask = np.ones((5, 6, 4), bool)
    mask[1:3, 2:4, :] = False
    m = Mesh(mask)
    info = m.info()[0]
    res = (info["resY"], info["resX"], info["resZ"])
    emb = m.get(0, "eleMapBack")
    x = np.random.default_rng(2).random(emb.size)
    V = R.design_volume(emb, res, x)
    assert V.shape == res
    assert np.array_equal(V.ravel(order="F")[emb - 1], x)
    assert V[1:3, 2:4, :].sum() == 0 and V[5:, :, :].sum() == 0     # void and padding


def test_super_spatial_order_matches_block_volume():
    ny, nx, nz = 3, 2, 2
    ne = ny * nx * nz
    x = np.random.default_rng(3).random((64, ne))
    order = R.super_spatial_order(nx, ny, nz)
    assert np.array_equal(np.sort(order), np.arange(64 * ne))
    V = R.design_volume(np.arange(1, ne + 1), (ny, nx, nz), x, super_element=True)
    assert V.dtype == np.float32 and V.shape == (4 * ny, 4 * nx, 4 * nz)
    assert np.array_equal(V.ravel(order="F"), x.ravel(order="F")[order].astype(np.float32))


def test_write_results_files(tmp_path):
    m = Mesh(np.ones((4, 8, 4), bool))
    ne = m.info()[0]["numElements"]
    x = np.random.default_rng(4).random(ne)
    recs = _records(3, np.random.default_rng(5))
    R.write_results(tmp_path, m, x, recs)
    names = sorted(p.name for p in tmp_path.iterdir())
    assert names == ["DesignVolume.nii", "c_Target.dat", "history.json", "iters_Target.dat", "sharp_Target.dat",
                     "solvetiming_Target.dat", "timing_Target.dat"]
    _, V = _read_nifti(tmp_path / "DesignVolume.nii")
    assert np.array_equal(V.ravel(order="F")[m.get(0, "eleMapBack") - 1], x)
    ms = Mesh(np.ones((4, 8, 4), bool), super_element=1)
    xs = np.random.default_rng(6).random((64, ms.info()[0]["numElements"]))
    out = tmp_path / "super"
    R.write_results(out, ms, xs, recs)
    lines = (out / "xPhys_sorted.dat").read_text().splitlines()
    assert len(lines) == xs.size
    ref = xs.ravel(order="F")[R.super_spatial_order(8, 4, 4)]
    assert np.array_equal(np.array([float(l) for l in lines]), ref)
