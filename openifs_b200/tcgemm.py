"""ctypes binding of the surrogate network's tcgen05 GEMM (cs_conv_gemm,
include/cloudsc_surrogate.h).  Tensors are CUDA tensors; the call is
asynchronous on the current torch stream."""
import ctypes

from . import cloudsc

EPI_SILU, EPI_LINEAR_F32, EPI_BWD = 0, 1, 2


class GemmDesc(ctypes.Structure):
    _fields_ = [("a", ctypes.c_void_p), ("w", ctypes.c_void_p), ("rows", ctypes.c_int32),
                ("k", ctypes.c_int32), ("n", ctypes.c_int32), ("taps", ctypes.c_int32),
                ("lp", ctypes.c_int32), ("klev", ctypes.c_int32), ("epi", ctypes.c_int32),
                ("bias", ctypes.c_void_p), ("out", ctypes.c_void_p), ("out_pre", ctypes.c_void_p),
                ("resid", ctypes.c_void_p), ("zprev", ctypes.c_void_p), ("gout", ctypes.c_void_p),
                ("outf", ctypes.c_void_p), ("err", ctypes.c_void_p)]


_fn = None


def _lib_fn():
    global _fn
    if _fn is None:
        L = cloudsc.lib()
        L.cs_conv_gemm.argtypes = [ctypes.POINTER(GemmDesc), ctypes.c_void_p]
        L.cs_conv_gemm.restype = ctypes.c_int
        _fn = L.cs_conv_gemm
    return _fn


def set_impl(impl):
    """0: warp-specialised kernel (default); 1: the single-thread pipeline."""
    L = cloudsc.lib()
    L.cs_set_gemm_impl.argtypes = [ctypes.c_int32]
    L.cs_set_gemm_impl.restype = ctypes.c_int
    if L.cs_set_gemm_impl(int(impl)) != 0:
        raise ValueError(impl)


def _p(t):
    return None if t is None else t.data_ptr()


def conv_gemm(a, w, epi, n, taps=1, lp=0, klev=0, bias=None, out=None, out_pre=None, resid=None,
              zprev=None, gout=None, outf=None, err=None, stream=None):
    """D[r] = sum_t a[r + t - taps // 2] @ w[t].T with the fused epilogue `epi`.

    a: [rows, k] bf16; w: [taps, n, k] bf16."""
    import torch
    rows, k = a.shape
    d = GemmDesc(_p(a), _p(w), rows, k, n, taps, lp, klev, epi, _p(bias), _p(out), _p(out_pre),
                 _p(resid), _p(zprev), _p(gout), _p(outf), _p(err))
    s = torch.cuda.current_stream().cuda_stream if stream is None else stream
    rc = _lib_fn()(ctypes.byref(d), s)
    if rc != 0:
        raise RuntimeError(f"cs_conv_gemm failed ({rc})")


_mh = None


def mlp_head(a, w1, b1, w2, b2, y, lp=0, klev=0, err=None, stream=None):
    """y = SiLU(a @ w1.T + b1) @ w2.T + b2 in one kernel (cs_mlp_head): the
    hidden activation stays on chip.  a: [rows, k] bf16; w1: [k, k] (or
    [1, k, k]) and w2: [64, k] (or [1, 64, k]) bf16; b1 [k], b2 [64] f32 or
    None; y: f32 with at least rows rows of 64."""
    global _mh
    import torch
    if _mh is None:
        L = cloudsc.lib()
        vp, i32 = ctypes.c_void_p, ctypes.c_int32
        L.cs_mlp_head.argtypes = [vp, vp, vp, vp, vp, i32, i32, i32, i32, vp, vp, vp]
        L.cs_mlp_head.restype = ctypes.c_int
        _mh = L.cs_mlp_head
    rows, k = a.shape
    if y.shape[-1] != 64 or y.numel() < rows * 64:
        raise ValueError("y must hold rows x 64 floats")
    s = torch.cuda.current_stream().cuda_stream if stream is None else stream
    rc = _mh(_p(a), _p(w1), _p(b1), _p(w2), _p(b2), rows, k, lp, klev, _p(y), _p(err), s)
    if rc != 0:
        raise RuntimeError(f"cs_mlp_head failed ({rc})")
