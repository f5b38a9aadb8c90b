"""B200 (sm_100a) implementation of the TOP_GPU FEA hot path.

Drop-in MEX entry points live in :mod:`top_gpu_on_matlab_b200.mex`, the
voxel model and the fused GPU solver in :mod:`top_gpu_on_matlab_b200.fea`,
the TOP_GPU driver in :mod:`top_gpu_on_matlab_b200.driver`, model files in
:mod:`top_gpu_on_matlab_b200.topvoxel` and result files in
:mod:`top_gpu_on_matlab_b200.results`.  All compute runs in libtopgpu.so;
importing without it raises ImportError.
"""
from ._lib import TopGpuError, lib

lib()   # the CUDA library is required: no CPU fallback

from .driver import TOP_GPU  # noqa: E402

__all__ = ["TOP_GPU", "TopGpuError", "lib"]
