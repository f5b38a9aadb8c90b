"""The six MEX gateway sources (top_gpu_on_matlab_b200/mex/*.cpp) compile
against the MEX stand-in with -Werror (tests/mex_build.sh), export
mexFunction, and refuse a wrong number of arguments with the reference
gateway's own identifier -- checked on the host, before any device call,
next to the reference's gateway compiled from its own source."""
import subprocess
from pathlib import Path

import pytest
import torch

from oracle import refkernels as R

ROOT = Path(__file__).resolve().parents[1]
GW = ROOT / "tests" / "_mexgw"

# gateway, a wrong argument count, the identifier the reference raises
ARITY = [
    ("Gathering_inplace", 2, "Gathering_inplace:Args"),
    ("Scattering_inplace", 4, "Scattering_inplace:arity"),
    ("scatter_accum3_inplace", 2, "scatter_accum3:args"),
    ("assembleKs_level2_inplace", 7, "assembleKs_level2_inplace:Input"),
    ("assembleKs_higherLevel_inplace", 3, "assembleKs_higherLevel_inplace:Input"),
    ("assembleKs_level2_superEle_inplace", 9, "assembleKs_level2_superEle_inplace:Input"),
]


@pytest.fixture(scope="module")
def built():
    subprocess.run(["bash", str(ROOT / "tests" / "mex_build.sh")], check=True)
    return GW


def test_gateways_export_mexfunction(built):
    for name in R.NAMES:
        out = subprocess.run(["nm", "-D", str(built / ("lib%s.so" % name))], capture_output=True, text=True, check=True).stdout
        assert " T mexFunction" in out and " T shim_call" in out, name


@pytest.mark.parametrize("name,nargs,ident", ARITY)
def test_arity_identifier_matches_reference(built, name, nargs, ident):
    args = [torch.zeros(3, dtype=torch.float64) for _ in range(nargs)]
    with pytest.raises(R.RefError) as ours:
        R.call(name, *args, libdir=built, sync=False)
    assert ours.value.identifier == ident
    if R.available():
        with pytest.raises(R.RefError) as ref:
            R.call(name, *args, sync=False)
        assert ref.value.identifier == ident


def test_outputs_refused_where_the_reference_refuses_them(built):
    for name, ident in (("Gathering_inplace", "Gathering_inplace:Args"), ("scatter_accum3_inplace", "scatter_accum3:nlhs")):
        args = [torch.zeros(3, dtype=torch.float64) for _ in range(3)]
        with pytest.raises(R.RefError) as ours:
            R.call(name, *args, nlhs=1, libdir=built, sync=False)
        assert ours.value.identifier == ident
