"""Call the reference's CUDA MEX kernels (compiled by oracle/ref_build.sh).

TEST INFRASTRUCTURE ONLY.  Each library in oracle/_ref is one reference .cu
file compiled unmodified against the MEX stand-in in oracle/mexshim; this
module wraps CUDA tensors (MATLAB column-major layout) as the stand-in's
mxArray and calls the library's mexFunction.  The reference launches on the
legacy default stream; calls are synchronised on both sides.
"""
import ctypes as C
from pathlib import Path

import torch

_DIR = Path(__file__).resolve().parent / "_ref"
NAMES = ["Gathering_inplace", "Scattering_inplace", "scatter_accum3_inplace", "assembleKs_level2_inplace",
         "assembleKs_higherLevel_inplace", "assembleKs_level2_superEle_inplace"]
_CLS = {torch.float64: 6, torch.float32: 7, torch.int32: 12, torch.uint32: 13}


class MxArray(C.Structure):
    _fields_ = [("cls", C.c_int), ("ndim", C.c_size_t), ("dims", C.c_size_t * 8),
                ("data", C.c_void_p), ("on_gpu", C.c_int)]


class RefError(RuntimeError):
    def __init__(self, ident, msg):
        self.identifier = ident
        super().__init__("%s: %s" % (ident, msg))


_LIBS = {}


def available(libdir=None):
    d = Path(libdir) if libdir is not None else _DIR
    return all((d / ("lib%s.so" % n)).exists() for n in NAMES)


def _lib(name, libdir=None):
    d = Path(libdir) if libdir is not None else _DIR
    key = (str(d), name)
    if key not in _LIBS:
        so = C.CDLL(str(d / ("lib%s.so" % name)))
        so.shim_call.restype = C.c_int
        so.shim_call.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_char_p, C.c_int]
        _LIBS[key] = so
    return _LIBS[key]


def _mx(t, dims=None):
    a = MxArray()
    if t is None or t.numel() == 0:
        a.cls = _CLS.get(t.dtype, 6) if t is not None else 6
        a.ndim = 2
        a.dims[0] = 0
        a.dims[1] = 0
        a.data = None
    else:
        a.cls = _CLS[t.dtype]
        d = list(dims if dims is not None else t.shape)
        while len(d) < 2:
            d.append(1)
        a.ndim = len(d)
        for i, v in enumerate(d):
            a.dims[i] = int(v)
        a.data = t.data_ptr()
    a.on_gpu = 1
    return a


def call(name, *args, nlhs=0, libdir=None, sync=True):
    """args: CUDA tensors (column-major) or (tensor, dims) pairs.  libdir: a
    directory of other gateway libraries built against the same stand-in
    (default: the reference's, oracle/_ref).  sync=False skips the device
    synchronisation (for calls that fail their argument checks on the host)."""
    arrs = []
    for x in args:
        if isinstance(x, tuple):
            arrs.append(_mx(x[0], x[1]))
        else:
            arrs.append(_mx(x))
    prhs = (C.POINTER(MxArray) * len(arrs))(*[C.pointer(a) for a in arrs])
    plhs = (C.POINTER(MxArray) * max(1, nlhs))()
    err = C.create_string_buffer(600)
    if sync:
        torch.cuda.synchronize()
    rc = _lib(name, libdir).shim_call(nlhs, C.cast(plhs, C.c_void_p), len(arrs), C.cast(prhs, C.c_void_p), err, 600)
    if sync:
        torch.cuda.synchronize()
    if rc:
        ident, _, msg = err.value.decode().partition("|")
        raise RefError(ident, msg)
