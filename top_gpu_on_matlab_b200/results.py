"""Result files of an optimisation run, as TOP_GPU writes them at the end
(TOP_GPU.m:293-326, IO_ExportDesignInVolume_nii 539-571):

    c_Target.dat            objective per iteration          %30.16e
    sharp_Target.dat        sharpness per iteration          %30.16e
    timing_Target.dat       total time per iteration (s)     %16.6e
    solvetiming_Target.dat  CG time per iteration (s)        %16.6e
    iters_Target.dat        PCG iterations per solve         %d
    xPhys_sorted.dat        super-element designs in spatial order   %30.16e
    DesignVolume.nii        the design on the padded voxel grid (NIfTI-1)
    history.json            one object per iteration: objective, volume,
                            sharpness, constraint, change, PCG iterations and
                            the tHist columns (TOP_GPU.m:283) in seconds

Histories come from the solver's per-iteration records (keys c, sharp,
msSolve, msTotal, pcgIts as returned by Solver.opt_step / Solver.optimize);
times there are milliseconds and are written in seconds, like the
reference's tic/toc.  The reference lists PCG iterations once per load case
and iteration; a record holds their sum over the load cases, so
iters_Target.dat takes the per-case counts when given (`iters`, from
Solver.opt_case_its, as the driver passes them) and the record's count
otherwise (the same for one load case).
"""
import json
import math
import os
import struct

import numpy as np


def _fmt_e(v, width, prec):
    """C / MATLAB fprintf('%<width>.<prec>e'); non-finite values as MATLAB prints them."""
    v = float(v)
    if math.isnan(v):
        return "NaN".rjust(width)
    if math.isinf(v):
        return ("Inf" if v > 0 else "-Inf").rjust(width)
    return "%*.*e" % (width, prec, v)


def _write_column(path, values, fmt):
    with open(path, "w") as f:
        for v in values:
            f.write(fmt(v) + "\n")


def write_history(out_dir, records, iters=None):
    """c_Target, sharp_Target, timing_Target, solvetiming_Target and
    iters_Target (TOP_GPU.m:307-321)."""
    os.makedirs(out_dir, exist_ok=True)
    j = lambda name: os.path.join(out_dir, name)
    _write_column(j("iters_Target.dat"), iters if iters is not None else [r["pcgIts"] for r in records],
                  lambda v: "%d" % int(v))
    _write_column(j("c_Target.dat"), [r["c"] for r in records], lambda v: _fmt_e(v, 30, 16))
    _write_column(j("sharp_Target.dat"), [r["sharp"] for r in records], lambda v: _fmt_e(v, 30, 16))
    _write_column(j("timing_Target.dat"), [r["msTotal"] / 1e3 for r in records], lambda v: _fmt_e(v, 16, 6))
    _write_column(j("solvetiming_Target.dat"), [r["msSolve"] / 1e3 for r in records], lambda v: _fmt_e(v, 16, 6))
    rows = []
    for k, r in enumerate(records, start=1):
        row = {"iteration": k}
        for key in ("c", "vol", "sharp", "cons", "change", "pcgIts"):
            if key in r:
                row[key] = r[key]
        for name, key in (("assembling_s", "msAssemble"), ("cg_s", "msSolve"), ("optimisation_s", "msOpt"),
                          ("filtering_s", "msFilter"), ("total_s", "msTotal")):
            if key in r:
                row[name] = r[key] / 1e3
        rows.append(row)
    with open(j("history.json"), "w") as f:
        json.dump(rows, f, indent=1)


def super_spatial_order(nelx, nely, nelz, n=4):
    """gen_index_mapping (TOP_GPU.m:2673-2697): map_old2new, 0-based -- entry i
    of the spatial (n nely) x (n nelx) x (n nelz) grid (y fastest) is entry
    map[i] of a super-element design [n^3 x Ne] in column-major order."""
    nY, nX, nZ = n * nely, n * nelx, n * nelz
    i = np.arange(nX * nY * nZ, dtype=np.int64)
    iy, ix, iz = i % nY, (i // nY) % nX, i // (nY * nX)
    big = iy // n + nely * (ix // n + nelx * (iz // n))
    local = iy % n + n * (ix % n + n * (iz % n))
    return local + n ** 3 * big


def write_xphys_sorted(path, xphys, nelx, nely, nelz):
    """xPhys_sorted.dat (TOP_GPU.m:297-303): a super-element design [64 x Ne]
    (box domain) in spatial order."""
    x = np.asarray(xphys, dtype=np.float64).reshape(-1, order="F") if np.ndim(xphys) == 2 else np.asarray(xphys, dtype=np.float64)
    _write_column(path, x[super_spatial_order(nelx, nely, nelz)], lambda v: _fmt_e(v, 30, 16))


def design_volume(ele_map_back, res, xphys, super_element=False, n=4):
    """The array IO_ExportDesignInVolume_nii writes (TOP_GPU.m:544-567): the
    design on the padded voxel grid res = (resY, resX, resZ), zero on void
    voxels; super-element designs [n^3 x Ne] expand each element into its
    n x n x n sub-voxels (single precision, as the reference allocates)."""
    ry, rx, rz = res
    emb = np.asarray(ele_map_back, dtype=np.int64) - 1
    if not super_element:
        v = np.zeros(ry * rx * rz)
        v[emb] = np.asarray(xphys, dtype=np.float64).ravel()
        return v.reshape((ry, rx, rz), order="F")
    blocks = np.asarray(xphys, dtype=np.float64).reshape(n ** 3, -1, order="F")
    out = np.zeros((ry * n, rx * n, rz * n), dtype=np.float32)
    iy, ix, iz = emb % ry, (emb // ry) % rx, emb // (ry * rx)
    for t in range(emb.size):
        out[iy[t] * n:(iy[t] + 1) * n, ix[t] * n:(ix[t] + 1) * n, iz[t] * n:(iz[t] + 1) * n] = \
            blocks[:, t].reshape((n, n, n), order="F")
    return out


_NIFTI_TYPES = {np.dtype(np.float64): (64, 64), np.dtype(np.float32): (16, 32)}   # datatype code, bitpix


def write_nifti(path, volume):
    """A single-file NIfTI-1 image (.nii) of a 3-D array, column-major (the
    first axis fastest, as MATLAB stores it): 348-byte header, 4 zero bytes
    (no extension), the data from byte 352.  Unit voxel spacing, identity
    sform (code 1), no qform, float64 or float32 data."""
    v = np.asarray(volume)
    if v.ndim != 3:
        raise ValueError("a 3-D volume")
    if v.dtype not in _NIFTI_TYPES:
        v = v.astype(np.float64)
    code, bitpix = _NIFTI_TYPES[v.dtype]
    hdr = bytearray(348)
    struct.pack_into("<i", hdr, 0, 348)                                  # sizeof_hdr
    hdr[38] = ord("r")                                                   # regular
    struct.pack_into("<8h", hdr, 40, 3, *v.shape, 1, 1, 1, 1)            # dim
    struct.pack_into("<hh", hdr, 70, code, bitpix)                       # datatype, bitpix
    struct.pack_into("<8f", hdr, 76, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0)   # pixdim (qfac = 1)
    struct.pack_into("<f", hdr, 108, 352.0)                              # vox_offset
    struct.pack_into("<ff", hdr, 112, 1.0, 0.0)                          # scl_slope, scl_inter
    hdr[123] = 0                                                         # xyzt_units: unknown
    struct.pack_into("<hh", hdr, 252, 0, 1)                              # qform_code, sform_code
    struct.pack_into("<12f", hdr, 280, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0)    # srow_x, srow_y, srow_z
    hdr[344:348] = b"n+1\x00"                                            # magic
    with open(path, "wb") as f:
        f.write(bytes(hdr))
        f.write(b"\x00\x00\x00\x00")
        f.write(np.asarray(v, dtype=v.dtype.newbyteorder("<")).tobytes(order="F"))


def write_results(out_dir, mesh, xphys, records, iters=None):
    """All of the above for a finished run: mesh = the fea.Mesh the solver
    was built on, xphys = its final physical design (compact element order;
    [64 x Ne] in super-element mode), records = the per-iteration records."""
    os.makedirs(out_dir, exist_ok=True)
    xphys = xphys.detach().cpu().numpy() if hasattr(xphys, "detach") else np.asarray(xphys)
    info = mesh.info()[0]
    res = (info["resY"], info["resX"], info["resZ"])
    sup = bool(getattr(mesh, "super_element", 0))
    if sup:
        ny, nx, nz = mesh.shape
        write_xphys_sorted(os.path.join(out_dir, "xPhys_sorted.dat"), xphys.reshape(64, -1, order="F"), nx, ny, nz)
    write_nifti(os.path.join(out_dir, "DesignVolume.nii"),
                design_volume(mesh.get(0, "eleMapBack"), res, xphys, super_element=sup))
    write_history(out_dir, records, iters)
