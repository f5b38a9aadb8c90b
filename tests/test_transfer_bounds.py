"""Index and alignment checks, on the CPU, for the span-4 transfer kernels that
read and write four fine y slots as one vector (restrict_y_kernel and
prolong4_kernel with V4, csrc/topgpu_grid.cuh).

The grid geometry is restated from make_geom (csrc/topgpu_solver.cu): node
counts N = res + 1, pitch PY = roundup(NY + 1, 4), PX = NX + 2, PZ = NZ + 2,
plane = PY PX, component stride cs = plane PZ + 2 kMargin, origin = PY + plane.
Vectors are allocated as ncomp * cs values starting kMargin before index 0 of
component 0; the flag bytes as cs bytes starting at index 0.  Every access
of the vector paths must start on a multiple of 4 values and stay inside those
allocations, for the hierarchies the solver builds and for ragged sizes."""
import math

import numpy as np
import pytest

from oracle import oracle as O

K_MARGIN = 64


def geom(res_y, res_x, res_z):
    NY, NX, NZ = res_y + 1, res_x + 1, res_z + 1
    PY = (NY + 1 + 3) // 4 * 4
    plane = PY * (NX + 2)
    cs = plane * (NZ + 2) + 2 * K_MARGIN
    return dict(NY=NY, NX=NX, NZ=NZ, PY=PY, plane=plane, cs=cs, origin=PY + plane)


def check_restrict_y_v4(gf, NYc, ncomp=3):
    """restrict_y_kernel<T, 4, true>: component c reads slots base + 4 QY - 4 ..
    base + 4 QY + 3, base = origin + PY X + plane Z, for QY < NYc, X < NXf, Z < NZf."""
    lo = gf["origin"] - 4
    hi = gf["origin"] + gf["PY"] * (gf["NX"] - 1) + gf["plane"] * (gf["NZ"] - 1) + 4 * (NYc - 1) + 3
    assert lo % 4 == 0 and (gf["PY"] % 4, gf["plane"] % 4, gf["cs"] % 4) == (0, 0, 0)
    assert lo >= -K_MARGIN                                        # component 0 from its margin on
    assert (ncomp - 1) * gf["cs"] + hi < ncomp * gf["cs"] - K_MARGIN   # last component within the allocation
    # the taps that are used (4 QY - 3 .. 4 QY + 3 clipped to the grid) lie in column X
    assert min(4 * (NYc - 1) + 3, gf["NY"] - 1) < gf["PY"]


def check_prolong4_v4(gf, ncomp=3):
    """prolong4_kernel<T, TR, XB, true>: slots i0 .. i0 + 3, i0 = origin + 4 qy +
    PY X + plane Z, qy < ceil(NY / 4); vectors of ncomp components and the flag bytes."""
    nqy = math.ceil(gf["NY"] / 4)
    assert 4 * (nqy - 1) + 3 < gf["PY"]                         # the four slots stay in their column
    i0_min = gf["origin"]
    i0_max = gf["origin"] + 4 * (nqy - 1) + gf["PY"] * (gf["NX"] - 1) + gf["plane"] * (gf["NZ"] - 1)
    assert i0_min % 4 == 0 and i0_max % 4 == 0
    assert i0_max + 3 < gf["cs"]                                   # flag bytes (cs of them)
    assert (ncomp - 1) * gf["cs"] + i0_max + 3 < ncomp * gf["cs"] - K_MARGIN


MODELS = [
    ((24, 48, 24), 20000), ((24, 48, 24), 50), ((20, 30, 14), 20000), ((10, 60, 10), 20000),
    ((96, 192, 96), 400), ((8, 16, 8), 20000),
]


@pytest.mark.parametrize("shape,control", MODELS)
def test_vector_transfer_accesses_in_bounds_for_built_hierarchies(shape, control):
    o = O.Model(np.ones(shape, bool), control=control)
    for l in range(1, o.numLevels):
        f, c = o.level(l - 1), o.level(l)
        if c.spanWidth != 4:
            continue
        gf = geom(f.resY, f.resX, f.resZ)
        check_restrict_y_v4(gf, c.resY + 1)
        check_prolong4_v4(gf)
        # a batch of right-hand sides sits at stride 3 cs: also a multiple of 4
        assert (3 * gf["cs"]) % 4 == 0


@pytest.mark.parametrize("res_y", list(range(1, 41)))
def test_vector_transfer_accesses_in_bounds_for_ragged_sizes(res_y):
    """fine y sizes that are not multiples of the span (coarse size rounded up)"""
    for res_x, res_z in ((1, 1), (3, 5), (8, 4)):
        gf = geom(res_y, res_x, res_z)
        check_restrict_y_v4(gf, math.ceil(res_y / 4) + 1)
        check_prolong4_v4(gf)
