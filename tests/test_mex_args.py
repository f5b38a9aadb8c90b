"""The MEX-named mirror's host-side checks (CPU): every gateway refuses host
arrays with its own <Name>:Args identifier before any device call, as the
reference's gateways refuse non-gpuArray inputs, and the MATLAB dimension
rules used by the shape checks."""
import numpy as np
import pytest
import torch

from top_gpu_on_matlab_b200 import mex
from top_gpu_on_matlab_b200._lib import TOP_ERR_ARGS, TopGpuError

# gateway, arguments, the identifier prefix the reference's gateway uses
# (scatter_accum3_inplace.cu:11-79 reports as "scatter_accum3:")
GATEWAYS = [
    ("Gathering_inplace", 3, "Gathering_inplace"), ("Scattering_inplace", 3, "Scattering_inplace"),
    ("scatter_accum3_inplace", 3, "scatter_accum3"),
    ("assembleKs_level2_inplace", 8, "assembleKs_level2_inplace"),
    ("assembleKs_higherLevel_inplace", 4, "assembleKs_higherLevel_inplace"),
    ("assembleKs_level2_superEle_inplace", 8, "assembleKs_level2_superEle_inplace"),
]


@pytest.mark.parametrize("name,nargs,prefix", GATEWAYS)
def test_host_arrays_are_refused(name, nargs, prefix):
    args = [torch.zeros((4, 3), dtype=torch.float64) for _ in range(nargs)]
    with pytest.raises(TopGpuError) as e:
        getattr(mex, name)(*args)
    assert e.value.status == TOP_ERR_ARGS
    assert e.value.identifier == prefix + ":Args"
    assert "gpuArray" in str(e.value)


def test_matlab_dims():
    assert mex._dims(torch.zeros(5)) == [5, 1]
    assert mex._dims(torch.zeros(3, 4, 1, 1)) == [3, 4]
    assert mex._dims(torch.zeros(576, 7)) == [576, 7]
    assert mex._dims(torch.zeros(24, 24, 9)) == [24, 24, 9]


def test_column_major_strides():
    assert mex._fortran_strides((3, 4, 5)) == (1, 3, 12)
    t = torch.zeros(12).as_strided((3, 4), (1, 3))
    assert mex._is_fortran(t) and not mex._is_fortran(torch.zeros(3, 4))
    a = np.arange(12.0).reshape(3, 4, order="F")
    assert np.array_equal(mex.gather(torch.from_numpy(a.ravel(order="F")).as_strided((3, 4), (1, 3))), a)
