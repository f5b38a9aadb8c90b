"""The six MEX entry points of TOP_GPU, on CUDA tensors, over libtopgpu.so.

Each function keeps the reference gateway's name, argument order, in-place
semantics, argument checks and error identifiers:

    Gathering_inplace(gUMat, gU, gE)                     Gathering_inplace.cu:75-171
    Scattering_inplace(Y, eNodMat, uMat)                 Scattering_inplace.cu:81-146
    scatter_accum3_inplace(keys, Tmp, xF)                scatter_accum3_inplace.cu:115-145
    assembleKs_level2_inplace(d_Ks, d_upMap, d_eleModulus, d_K_0, d_Pch,
                              d_mapUnique, d_uniqueFree, d_uniqueFixed)
                                                         assembleKs_level2_inplace.cu:165-284
    assembleKs_higherLevel_inplace(d_Ks, d_upMap, d_KsPrev, d_Psub)
                                                         assembleKs_higherLevel_inplace.cu:134-217
    assembleKs_level2_superEle_inplace(d_Ks, d_upMap, d_Ks0, d_Psub, d_mapUnique,
                                       d_eleModulus, d_uniqueFree, d_uniqueFixed)
                                                         assembleKs_level2_superEle_inplace.cu:178-325

A MATLAB gpuArray is represented by a CUDA tensor with MATLAB's shape and
column-major (Fortran) strides; ``gpu_array`` and ``gather`` convert from and
to numpy the way gpuArray() and gather() do.
"""
import numpy as np
import torch

from ._lib import TOP_F32, TOP_F64, TopGpuError, TOP_ERR_ARGS, TOP_ERR_SHAPE, TOP_ERR_TYPE, check, lib


def gpu_array(a, dtype=None, device="cuda"):
    """numpy array -> column-major CUDA tensor with MATLAB's shape."""
    a = np.asarray(a)
    if dtype is not None:
        a = a.astype(dtype)
    shape = a.shape
    flat = torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).to(device)
    if len(shape) <= 1:
        return flat
    return flat.as_strided(shape, _fortran_strides(shape))


def zeros(shape, dtype=torch.float64, device="cuda"):
    """gpuArray.zeros(shape) in column-major layout."""
    n = int(np.prod(shape)) if len(shape) else 1
    flat = torch.zeros(n, dtype=dtype, device=device)
    return flat if len(shape) <= 1 else flat.as_strided(tuple(shape), _fortran_strides(shape))


def gather(t):
    """CUDA tensor (column-major) -> numpy array with the same shape."""
    t = t.detach()
    shape = tuple(t.shape)
    if t.dim() <= 1:
        return t.cpu().numpy()
    flat = t.as_strided((t.numel(),), (1,)).cpu().numpy() if _is_fortran(t) else t.cpu().numpy().ravel(order="F")
    return flat.reshape(shape, order="F")


def _fortran_strides(shape):
    st, acc = [], 1
    for n in shape:
        st.append(acc)
        acc *= int(n)
    return tuple(st)


def _is_fortran(t):
    if t.dim() <= 1:
        return t.dim() == 0 or t.stride(0) == 1 or t.numel() <= 1
    exp = _fortran_strides(t.shape)
    return all(s == e or n == 1 for s, e, n in zip(t.stride(), exp, t.shape))


def _err(name, status, msg):
    raise TopGpuError(status, name, msg)


def _need(name, t, what):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        _err(name, TOP_ERR_ARGS, "%s must be a gpuArray (CUDA tensor)." % what)
    if not _is_fortran(t):
        _err(name, TOP_ERR_ARGS, "%s must be stored column-major (as a gpuArray is)." % what)
    return t


def _need_all(name, **tensors):
    """_need on every given tensor (None: an optional argument left out)."""
    for what, t in tensors.items():
        if t is not None:
            _need(name, t, what)


def _dtype_code(name, t, what):
    if t.dtype == torch.float64:
        return TOP_F64
    if t.dtype == torch.float32:
        return TOP_F32
    _err(name, TOP_ERR_TYPE, "%s must be single or double gpuArray." % what)


def _dims(t):
    """MATLAB dims: trailing singleton dimensions dropped, at least 2."""
    d = list(t.shape)
    while len(d) > 2 and d[-1] == 1:
        d.pop()
    while len(d) < 2:
        d.append(1)
    return d


def _stream():
    return torch.cuda.current_stream().cuda_stream


def Gathering_inplace(gUMat, gU, gE):
    n = "Gathering_inplace"
    for t, w in ((gUMat, "gUMat"), (gU, "gU"), (gE, "gE")):
        _need(n, t, w)
    cls = _dtype_code(n, gU, "gU")
    if gUMat.dtype != gU.dtype:
        _err(n, TOP_ERR_TYPE, "gUMat precision must match gU.")
    if gE.dtype not in (torch.int32, torch.uint32):
        _err(n, TOP_ERR_TYPE, "gE must be int32 or uint32 gpuArray.")
    du, de, do = _dims(gU), _dims(gE), _dims(gUMat)
    if len(du) != 2 or du[1] != 3:
        _err(n, TOP_ERR_SHAPE, "gU must be (numNodes x 3).")
    if len(de) != 2 or de[1] != 8:
        _err(n, TOP_ERR_SHAPE, "gE must be (nElem x 8).")
    if len(do) != 2 or do[0] != de[0] or do[1] != 24:
        _err(n, TOP_ERR_SHAPE, "gUMat must be (nElem x 24).")
    check(lib().top_gather(gUMat.data_ptr(), gU.data_ptr(), gE.data_ptr(), int(gE.dtype == torch.uint32),
                           de[0], du[0], cls, _stream()), n)


def Scattering_inplace(Y, eNodMat, uMat):
    n = "Scattering_inplace"
    for t, w in ((Y, "Y"), (eNodMat, "eNodMat"), (uMat, "uMat")):
        _need(n, t, w)
    dy = _dims(Y)
    if len(dy) != 2 or dy[1] != 3:
        _err(n, TOP_ERR_SHAPE, "Y must be [numNodes x 3].")
    if eNodMat.dtype != torch.int32:
        _err(n, TOP_ERR_TYPE, "eNodMat must be gpuArray(int32).")
    de = _dims(eNodMat)
    if len(de) != 2 or de[1] != 8:
        _err(n, TOP_ERR_SHAPE, "eNodMat must be [Ne x 8] int32 (1-based).")
    du = _dims(uMat)
    if len(du) != 2 or du[0] != de[0] or du[1] != 24:
        _err(n, TOP_ERR_SHAPE, "uMat must be [Ne x 24] double.")
    cls = _dtype_code(n, Y, "Y")
    if uMat.dtype != Y.dtype:
        # the reference reinterprets uMat with Y's class (Scattering_inplace.cu:114-122);
        # a mismatch there reads garbage, here it is rejected
        _err(n, TOP_ERR_TYPE, "uMat class must match Y.")
    check(lib().top_scatter(Y.data_ptr(), eNodMat.data_ptr(), uMat.data_ptr(), de[0], dy[0], cls, _stream()), n)


def scatter_accum3_inplace(keys, Tmp, xF):
    n = "scatter_accum3"
    for t in (keys, Tmp, xF):
        if not isinstance(t, torch.Tensor) or not t.is_cuda:
            _err(n, TOP_ERR_ARGS, "All inputs must be gpuArray.")
    for t, w in ((keys, "transferMat"), (Tmp, "Tmp"), (xF, "xFiner")):
        _need(n, t, w)
    dt, dx = _dims(Tmp), _dims(xF)
    if len(dt) != 2 or dt[1] != 3:
        _err(n, TOP_ERR_SHAPE, "`Tmp` must be [N x 3] gpuArray.")
    if len(dx) != 2 or dx[1] != 3:
        _err(n, TOP_ERR_SHAPE, "`xFiner` must be [M x 3] gpuArray.")
    if keys.dtype != torch.int32:
        _err(n, TOP_ERR_TYPE, "`transferMat` must be int32 gpuArray.")
    if Tmp.dtype != xF.dtype:
        _err(n, TOP_ERR_TYPE, "`Tmp` and `xFiner` must have the same class (single/double).")
    cls = _dtype_code(n, Tmp, "Tmp")
    check(lib().top_scatter_accum3(keys.data_ptr(), Tmp.data_ptr(), dt[0], xF.data_ptr(), dx[0], cls, _stream()), n)


def _opt(t):
    return None if t is None or t.numel() == 0 else t.data_ptr()


def assembleKs_level2_inplace(d_Ks, d_upMap, d_eleModulus, d_K_0, d_Pch, d_mapUnique, d_uniqueFree, d_uniqueFixed):
    n = "assembleKs_level2_inplace"
    _need_all(n, d_Ks=d_Ks, d_upMap=d_upMap, d_eleModulus=d_eleModulus, d_K_0=d_K_0, d_Pch=d_Pch,
              d_mapUnique=d_mapUnique, d_uniqueFree=d_uniqueFree, d_uniqueFixed=d_uniqueFixed)
    cls = _dtype_code(n, d_Ks, "d_Ks")
    if d_upMap.dtype != torch.int32 or d_mapUnique.dtype != torch.int32:
        _err(n, TOP_ERR_TYPE, "d_upMap and d_mapUnique must be int32 gpuArray.")
    dk = list(d_Ks.shape)
    if d_Ks.dim() == 2 and dk == [24, 24]:
        dk = [24, 24, 1]
    if len(dk) != 3 or dk[0] != 24 or dk[1] != 24:
        _err(n, TOP_ERR_SHAPE, "d_Ks must be [24 x 24 x nElem].")
    nElem = dk[2]
    du = _dims(d_upMap)
    if len(du) != 2 or du[0] != nElem:
        _err(n, TOP_ERR_SHAPE, "d_upMap must be [nElem x nCh].")
    nCh = du[1]
    dp = list(d_Pch.shape) + [1] * (3 - d_Pch.dim())
    if dp[0] != 24 or dp[1] != 24 or dp[2] != nCh:
        _err(n, TOP_ERR_SHAPE, "d_Pch must be [24 x 24 x nCh].")
    if d_K_0.numel() != 576:
        _err(n, TOP_ERR_SHAPE, "d_K_0 must contain 576 elements.")
    nUnique = 0
    if d_uniqueFree is not None and d_uniqueFree.numel() > 0:
        df = _dims(d_uniqueFree)
        if len(df) != 2 or df[0] != 576:
            _err(n, TOP_ERR_SHAPE, "d_uniqueFree must be [576 x nUnique] or empty.")
        nUnique = df[1]
    if d_uniqueFixed is not None and d_uniqueFixed.numel() > 0:
        dx = _dims(d_uniqueFixed)
        if len(dx) != 2 or dx[0] != 576 or dx[1] != nUnique:
            _err(n, TOP_ERR_SHAPE, "d_uniqueFixed must be [576 x nUnique] matching d_uniqueFree.")
    for t in (d_eleModulus, d_K_0, d_Pch):
        if t.dtype != d_Ks.dtype:
            _err(n, TOP_ERR_TYPE, "d_eleModulus/d_K_0/d_Pch must match d_Ks class.")
    for t, w in ((d_uniqueFree, "d_uniqueFree"), (d_uniqueFixed, "d_uniqueFixed")):
        if t is not None and t.numel() > 0 and t.dtype != d_Ks.dtype:
            _err(n, TOP_ERR_TYPE, "%s class must match d_Ks." % w)
    check(lib().top_assemble_ks_level2(d_Ks.data_ptr(), d_upMap.data_ptr(), d_eleModulus.data_ptr(), d_K_0.data_ptr(),
                                       d_Pch.data_ptr(), d_mapUnique.data_ptr(), _opt(d_uniqueFree), _opt(d_uniqueFixed),
                                       nElem, nCh, d_eleModulus.numel(), nUnique, cls, _stream()), n)
    return d_Ks


def assembleKs_higherLevel_inplace(d_Ks, d_upMap, d_KsPrev, d_Psub):
    n = "assembleKs_higherLevel_inplace"
    _need_all(n, d_Ks=d_Ks, d_upMap=d_upMap, d_KsPrev=d_KsPrev, d_Psub=d_Psub)
    cls = _dtype_code(n, d_Ks, "d_Ks")
    if d_upMap.dtype != torch.int32:
        _err(n, TOP_ERR_TYPE, "d_upMap must be int32 gpuArray.")
    if d_KsPrev.dtype != d_Ks.dtype or d_Psub.dtype != d_Ks.dtype:
        _err(n, TOP_ERR_TYPE, "d_KsPrev and d_Psub must match d_Ks class.")
    dk = list(d_Ks.shape) + [1] * (3 - d_Ks.dim())
    if dk[0] != 24 or dk[1] != 24:
        _err(n, TOP_ERR_SHAPE, "d_Ks must be [24 x 24 x nElem].")
    nElem = dk[2]
    du = _dims(d_upMap)
    if len(du) != 2 or du[0] != nElem:
        _err(n, TOP_ERR_SHAPE, "d_upMap must be [nElem x nSub].")
    nSub = du[1]
    dpv = list(d_KsPrev.shape) + [1] * (3 - d_KsPrev.dim())
    if dpv[0] != 24 or dpv[1] != 24:
        _err(n, TOP_ERR_SHAPE, "d_KsPrev must be [24 x 24 x nFinElem].")
    dp = list(d_Psub.shape) + [1] * (3 - d_Psub.dim())
    if dp[0] != 24 or dp[1] != 24 or dp[2] != nSub:
        _err(n, TOP_ERR_SHAPE, "d_Psub must be [24 x 24 x nSub].")
    check(lib().top_assemble_ks_higher(d_Ks.data_ptr(), d_upMap.data_ptr(), d_KsPrev.data_ptr(), d_Psub.data_ptr(),
                                       nElem, nSub, dpv[2], cls, _stream()), n)
    return d_Ks


def assembleKs_level2_superEle_inplace(d_Ks, d_upMap, d_Ks0, d_Psub, d_mapUnique, d_eleModulus, d_uniqueFree, d_uniqueFixed):
    n = "assembleKs_level2_superEle_inplace"
    _need_all(n, d_Ks=d_Ks, d_upMap=d_upMap, d_Ks0=d_Ks0, d_Psub=d_Psub, d_mapUnique=d_mapUnique,
              d_eleModulus=d_eleModulus, d_uniqueFree=d_uniqueFree, d_uniqueFixed=d_uniqueFixed)
    cls = _dtype_code(n, d_Ks, "d_Ks")
    if d_upMap.dtype != torch.int32 or d_mapUnique.dtype != torch.int32:
        _err(n, TOP_ERR_TYPE, "d_upMap and d_mapUnique must be int32 gpuArray.")
    for t in (d_Ks0, d_Psub, d_eleModulus):
        if t.dtype != d_Ks.dtype:
            _err(n, TOP_ERR_TYPE, "d_Ks0, d_Psub, d_eleModulus must match d_Ks class.")
    dk = list(d_Ks.shape) + [1] * (3 - d_Ks.dim())
    if dk[0] != 24 or dk[1] != 24:
        _err(n, TOP_ERR_SHAPE, "d_Ks must be [24 x 24 x nElem].")
    nElem = dk[2]
    du = _dims(d_upMap)
    if len(du) != 2 or du[0] != nElem:
        _err(n, TOP_ERR_SHAPE, "d_upMap must be [nElem x nSub].")
    nSub = du[1]
    if d_Ks0.numel() % 576:
        _err(n, TOP_ERR_SHAPE, "d_Ks0 total elements must be a multiple of 576.")
    dp = list(d_Psub.shape) + [1] * (3 - d_Psub.dim())
    if dp[0] != 24 or dp[1] != 24 or dp[2] != nSub:
        _err(n, TOP_ERR_SHAPE, "d_Psub must be [24 x 24 x nSub].")
    if d_eleModulus.numel() % 64:
        _err(n, TOP_ERR_SHAPE, "d_eleModulus total elements must be a multiple of 64.")
    nUnique = 0
    if d_uniqueFree is not None and d_uniqueFree.numel() > 0:
        df = list(d_uniqueFree.shape)
        if len(df) == 3:
            if df[0] != 576 or df[1] != 64:
                _err(n, TOP_ERR_SHAPE, "d_uniqueFree must be [576 x 64 x nUnique].")
            nUnique = df[2]
        elif len(df) == 2:
            if df[0] != 576 * 64:
                _err(n, TOP_ERR_SHAPE, "d_uniqueFree must be [576*64 x nUnique] or [576 x 64 x nUnique].")
            nUnique = df[1]
        else:
            _err(n, TOP_ERR_SHAPE, "d_uniqueFree must be 2-D or 3-D.")
    if d_uniqueFixed is not None and d_uniqueFixed.numel() > 0:
        dx = _dims(d_uniqueFixed)
        if len(dx) != 2 or dx[0] != 576 or dx[1] != nUnique:
            _err(n, TOP_ERR_SHAPE, "d_uniqueFixed must be [576 x nUnique] matching d_uniqueFree.")
    check(lib().top_assemble_ks_level2_super(d_Ks.data_ptr(), d_upMap.data_ptr(), d_Ks0.data_ptr(), d_Psub.data_ptr(),
                                             d_mapUnique.data_ptr(), d_eleModulus.data_ptr(), _opt(d_uniqueFree),
                                             _opt(d_uniqueFixed), nElem, nSub, d_Ks0.numel() // 576, nUnique, cls,
                                             _stream()), n)
    return d_Ks
