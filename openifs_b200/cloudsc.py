"""Python binding of libcloudsc_b200.so (the C ABI in include/cloudsc_b200.h).

This mirrors the reference's operator interface for the path: one call per
NPROMA block with CLOUDSC's argument list (``cloudsc_block``), or one call for
all blocks (``cloudsc_batched`` on device arrays, ``cloudsc_batched_host`` on
host arrays).  Errors follow the C ABI: a negative return raises
``CloudscError``; a positive return is the number of negative-condensate
warning events the reference would have written to NULOUT
(cloudsc.F90:3794,3802).

There is no CPU fallback: if the library is missing or no GPU is present the
calls raise.
"""
import ctypes
import functools
import os

import numpy as np

from .fields import BATCHED_FIELDS
from .params import CloudscParams

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcloudsc_b200.so")

FP64 = 0
MIXED = 1
PHYS32 = 2  # FP32 process rates; state, solve, saturation adjustment and budgets in FP64


class CloudscError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"CLOUDSC error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise CloudscError(-4, f"{LIB_PATH} not built; run python -m openifs_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER(CloudscParams)
        vp = ctypes.c_void_p
        i32 = ctypes.c_int32
        L.cloudsc_b200_params_default.argtypes = [ctypes.c_double, i32, P]
        L.cloudsc_b200_params_default.restype = ctypes.c_int
        L.cloudsc_b200_ncldtop.argtypes = [i32, vp, ctypes.c_double]
        L.cloudsc_b200_ncldtop.restype = i32
        L.cloudsc_b200_setup.argtypes = [P]
        L.cloudsc_b200_setup.restype = ctypes.c_int
        L.cloudsc_b200_set_launch.argtypes = [i32, i32, i32]
        L.cloudsc_b200_set_launch.restype = ctypes.c_int
        pi32 = ctypes.POINTER(i32)
        L.cloudsc_b200_num_variants.restype = ctypes.c_int
        L.cloudsc_b200_variant_info.argtypes = [i32, i32, pi32, pi32, pi32, pi32]
        L.cloudsc_b200_variant_info.restype = ctypes.c_int
        L.cloudsc_b200_set_schedule.argtypes = [i32, i32, i32, i32]
        L.cloudsc_b200_set_schedule.restype = ctypes.c_int
        L.cloudsc_b200_get_schedule.argtypes = [i32, pi32, pi32, pi32]
        L.cloudsc_b200_get_schedule.restype = ctypes.c_int
        from .fields import DIAG_FIELDS
        L.cloudsc_b200_batched_diag.argtypes = ([P, i32, i32, i32, i32, ctypes.c_double] +
                                                [vp] * (len(BATCHED_FIELDS) + len(DIAG_FIELDS)) + [i32, vp, vp])
        L.cloudsc_b200_batched_diag.restype = ctypes.c_int
        from .fields import SATADJ_FIELDS
        ns = len(SATADJ_FIELDS)
        L.cloudsc_b200_satadj_batched.argtypes = [P, i32, i32, i32, i32, ctypes.c_double] + [vp] * ns + [vp, vp]
        L.cloudsc_b200_satadj_batched.restype = ctypes.c_int
        L.cloudsc_b200_satadj_increment_batched.argtypes = ([P, i32, i32, i32, i32, ctypes.c_double] +
                                                            [vp] * ns + [ctypes.c_uint32, vp, vp])
        L.cloudsc_b200_satadj_increment_batched.restype = ctypes.c_int
        L.cloudsc_b200_state_increment_batched.argtypes = [i32] * 5 + [vp] * 3
        L.cloudsc_b200_state_increment_batched.restype = ctypes.c_int
        L.cloudsc_b200_satadj_block.argtypes = ([P, i32, i32, i32, i32, vp, i32, ctypes.c_double] + [vp] * 16 +
                                                [vp, vp, vp, vp, vp] + [vp] * 5 + [vp, i32])
        L.cloudsc_b200_satadj_block.restype = ctypes.c_int
        from .fields import SLTEND_FIELDS
        L.cloudsc_b200_sltend_supersat_batched.argtypes = ([P, i32, i32, i32, i32, ctypes.c_double] +
                                                           [vp] * len(SLTEND_FIELDS) + [vp])
        L.cloudsc_b200_sltend_supersat_batched.restype = ctypes.c_int
        L.cloudsc_b200_division_check.argtypes = [vp, vp, ctypes.c_int64, vp, vp, vp]
        L.cloudsc_b200_division_check.restype = ctypes.c_int
        L.cloudsc_b200_reciprocal_check.argtypes = [vp, ctypes.c_int64, vp, vp, vp]
        L.cloudsc_b200_reciprocal_check.restype = ctypes.c_int
        L.cloudsc_b200_last_error.restype = ctypes.c_char_p
        L.cloudsc_b200_version.restype = ctypes.c_char_p
        L.cloudsc_b200_params_size.restype = ctypes.c_size_t
        nf = len(BATCHED_FIELDS)
        L.cloudsc_b200_batched.argtypes = [P, i32, i32, i32, i32, ctypes.c_double] + [vp] * nf + [vp, i32, vp]
        L.cloudsc_b200_batched.restype = ctypes.c_int
        L.cloudsc_b200_batched_host.argtypes = [P, i32, i32, i32, i32, ctypes.c_double] + [vp] * nf + [i32, i32]
        L.cloudsc_b200_batched_host.restype = ctypes.c_int
        L.cloudsc_b200_block.argtypes = ([P, i32, i32, i32, i32, i32, ctypes.c_double] +
                                         [vp] * len(BLOCK_ARRAYS_1) + [i32] +
                                         [vp] * len(BLOCK_ARRAYS_2) + [i32])
        L.cloudsc_b200_block.restype = ctypes.c_int
        L.cloudsc_b200_batched_sp.argtypes = [P, i32, i32, i32, i32, ctypes.c_float] + [vp] * nf + [vp, i32, vp]
        L.cloudsc_b200_batched_sp.restype = ctypes.c_int
        L.cloudsc_b200_batched_host_sp.argtypes = [P, i32, i32, i32, i32, ctypes.c_float] + [vp] * nf + [i32, i32]
        L.cloudsc_b200_batched_host_sp.restype = ctypes.c_int
        _lib = L
    return _lib


def _check(rc):
    if rc < 0:
        raise CloudscError(rc, lib().cloudsc_b200_last_error().decode())
    return rc


def default_params(tsphy=3600.0, ncldtop=None):
    """Reference defaults (SUCLDP et al.) for time step ``tsphy``."""
    if ncldtop is None:
        from .inputs import ncldtop_l137
        ncldtop = ncldtop_l137()
    p = CloudscParams()
    _check(lib().cloudsc_b200_params_default(float(tsphy), int(ncldtop), ctypes.byref(p)))
    return p


def setup(params):
    """Upload ``params`` to the GPU(s); required before any CLOUDSC call."""
    return _check(lib().cloudsc_b200_setup(ctypes.byref(params)))


def set_launch(precision, threads_per_cta, ctas_per_sm):
    return _check(lib().cloudsc_b200_set_launch(int(precision), int(threads_per_cta), int(ctas_per_sm)))


def num_variants():
    """Number of compiled (max threads, min CTAs per SM) kernel variants."""
    return int(lib().cloudsc_b200_num_variants())


def variant_info(precision, variant):
    """{"max_threads", "min_ctas", "regs", "local_bytes"} of a compiled
    variant (regs and local_bytes are -1 without a GPU)."""
    v = [ctypes.c_int32() for _ in range(4)]
    _check(lib().cloudsc_b200_variant_info(int(precision), int(variant), *[ctypes.byref(x) for x in v]))
    return dict(zip(("max_threads", "min_ctas", "regs", "local_bytes"), (x.value for x in v)))


def set_schedule(precision, variant, threads_per_cta, ctas_per_sm):
    return _check(lib().cloudsc_b200_set_schedule(int(precision), int(variant), int(threads_per_cta),
                                                  int(ctas_per_sm)))


def get_schedule(precision):
    """(variant, threads_per_cta, ctas_per_sm) used for `precision`."""
    v = [ctypes.c_int32() for _ in range(3)]
    _check(lib().cloudsc_b200_get_schedule(int(precision), *[ctypes.byref(x) for x in v]))
    return tuple(x.value for x in v)


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        if not x.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return x.ctypes.data
    # torch tensor (device or pinned host)
    if not x.is_contiguous():
        raise ValueError("tensors must be contiguous")
    return x.data_ptr()


@functools.lru_cache(maxsize=64)
def _batched_spec(nproma, klev, ngpblks):
    """(name, numpy dtype, element count) of every batched array."""
    from .fields import DTYPE, batched_shape
    return tuple((n, np.dtype(DTYPE[n]), int(np.prod(batched_shape(n, ngpblks, nproma, klev))))
                 for n, *_ in BATCHED_FIELDS)


def _check_batched(arrays, nproma, klev, ngpblks, device):
    """Every array of fields.BATCHED_FIELDS is present with its dtype and its
    (NGPBLKS, ..., NPROMA) element count, on the CUDA device (device=True) or
    in host memory: the C ABI takes bare pointers and cannot check them.
    Raises CloudscError with the C ABI's codes (-1 missing, -2 shape)."""
    for n, dt, want in _batched_spec(int(nproma), int(klev), int(ngpblks)):
        x = arrays.get(n)
        if x is None:
            raise CloudscError(-1, f"{n}: array missing")
        if isinstance(x, np.ndarray):
            if device:
                raise CloudscError(-2, f"{n}: a device tensor is needed, not a numpy array")
            ok_dtype, size = x.dtype == dt, x.size
        else:
            if x.is_cuda != device:
                raise CloudscError(-2, f"{n}: tensor must be on {'the GPU' if device else 'the host'}")
            ok_dtype = x.element_size() == dt.itemsize and x.is_floating_point() == (dt.kind == "f")
            size = x.numel()
        if not ok_dtype:
            raise CloudscError(-2, f"{n}: dtype must be {dt.name}")
        if size < want:
            raise CloudscError(-2, f"{n}: {size} elements, the shape needs {want}")


def cloudsc_batched(params, arrays, nproma, klev, ngpblks, ngptot, ptsphy, precision=FP64,
                    stream=None, counter=None, validate=True):
    """One persistent launch over all blocks; ``arrays`` are CUDA tensors in
    the fields.BATCHED_FIELDS layout.  Asynchronous on ``stream``.
    ``validate=False`` skips the Python-side array checks and leaves only
    the C ABI's own (for callers that pass raw pointers' owners)."""
    if validate:
        _check_batched(arrays, nproma, klev, ngpblks, device=True)
    args = [_ptr(arrays[n]) for n, *_ in BATCHED_FIELDS]
    s = None
    if stream is not None:
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
    return _check(lib().cloudsc_b200_batched(
        ctypes.byref(params), int(nproma), int(klev), int(ngpblks), int(ngptot), float(ptsphy),
        *args, _ptr(counter), int(precision), s))


def _check_sp(arrays, nproma, klev, ngpblks, device):
    """The single-precision interface's arrays: present, float32 (int32 for
    LDCUM and KTYPE), large enough, on the device or the host."""
    from .fields import DTYPE_SP, batched_shape
    for n, *_ in BATCHED_FIELDS:
        x = arrays.get(n)
        if x is None:
            raise CloudscError(-1, f"{n}: array missing")
        want = int(np.prod(batched_shape(n, ngpblks, nproma, klev)))
        dt = np.dtype(DTYPE_SP[n])
        if isinstance(x, np.ndarray):
            if device:
                raise CloudscError(-2, f"{n}: a device tensor is needed, not a numpy array")
            ok, size = x.dtype == dt, x.size
        else:
            if x.is_cuda != device:
                raise CloudscError(-2, f"{n}: tensor must be on {'the GPU' if device else 'the host'}")
            ok = x.element_size() == dt.itemsize and x.is_floating_point() == (dt.kind == "f")
            size = x.numel()
        if not ok:
            raise CloudscError(-2, f"{n}: dtype must be {dt.name}")
        if size < want:
            raise CloudscError(-2, f"{n}: {size} elements, the shape needs {want}")


def cloudsc_batched_sp(params, arrays, nproma, klev, ngpblks, ngptot, ptsphy, precision=FP64, stream=None,
                       counter=None):
    """The single-precision interface (float arrays, fields.DTYPE_SP) on
    the device: one launch over every block, asynchronous on ``stream``;
    ``precision`` selects the arithmetic (FP64, MIXED, PHYS32)."""
    _check_sp(arrays, nproma, klev, ngpblks, device=True)
    args = [_ptr(arrays[n]) for n, *_ in BATCHED_FIELDS]
    s = None
    if stream is not None:
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
    return _check(lib().cloudsc_b200_batched_sp(
        ctypes.byref(params), int(nproma), int(klev), int(ngpblks), int(ngptot), float(ptsphy),
        *args, _ptr(counter), int(precision), s))


def cloudsc_batched_host_sp(params, arrays, nproma, klev, ngpblks, ngptot, ptsphy, precision=FP64,
                            chunk_blocks=0):
    """The single-precision interface from host arrays (numpy float32, or
    pinned torch CPU tensors), pipelined like cloudsc_batched_host.
    Synchronous."""
    _check_sp(arrays, nproma, klev, ngpblks, device=False)
    args = [_ptr(arrays[n]) for n, *_ in BATCHED_FIELDS]
    return _check(lib().cloudsc_b200_batched_host_sp(
        ctypes.byref(params), int(nproma), int(klev), int(ngpblks), int(ngptot), float(ptsphy),
        *args, int(precision), int(chunk_blocks)))


def cloudsc_batched_host(params, arrays, nproma, klev, ngpblks, ngptot, ptsphy, precision=FP64,
                         chunk_blocks=0, validate=True):
    """All blocks from host arrays (numpy, or pinned torch CPU tensors), with
    transfers pipelined against compute.  Synchronous."""
    if validate:
        _check_batched(arrays, nproma, klev, ngpblks, device=False)
    args = [_ptr(arrays[n]) for n, *_ in BATCHED_FIELDS]
    return _check(lib().cloudsc_b200_batched_host(
        ctypes.byref(params), int(nproma), int(klev), int(ngpblks), int(ngptot), float(ptsphy),
        *args, int(precision), int(chunk_blocks)))


# Argument list of SUBROUTINE CLOUDSC (cloudsc.F90:14-44) after the seven
# derived types: (name, is_array); None entries are the unused optional arrays.
BLOCK_ARRAYS_1 = ["pt", "pq", "tendency_cml_t", "tendency_cml_q", "tendency_cml_a",
                  "tendency_cml_cld", "tendency_loc_t", "tendency_loc_q", "tendency_loc_a",
                  "tendency_loc_cld", "pvfa", "pvfl", "pvfi", "pdyna", "pdynl", "pdyni", "pdynr",
                  "pdyns", "phrsw", "phrlw", "pvervel", "pap", "paph", "pgeom", "plsm", "pgaw",
                  "ldcum", "kctop", "ktype", "kpbltype", "peis", "plu", "plude", "pludeli",
                  "psnde", "pmfu", "pmfd", "pgp2dspp"]
BLOCK_ARRAYS_2 = ["pa", "pclv", "plcrit_aer", "picrit_aer", "pre_ice", "pccn", "pnice",
                  "pcovptot", "pfsd", "prainfrac_toprfz", "pfsqlf", "pfsqif", "pfcqnng",
                  "pfcqlng", "pfsqrf", "pfsqsf", "pfcqrng", "pfcqsng", "pfsqltur", "pfsqitur",
                  "pfplsl", "pfplsn", "pfhpsl", "pfhpsn", "pextra"]


def cloudsc_block(params, kidia, kfdia, klon, klev, ptsphy, arrays, lddiag=False, ldslphy=False,
                  kfldx=0):
    """The per-block drop-in: CLOUDSC's argument list with host arrays.

    ``arrays`` maps the reference argument names (lower case, without the
    leading 'p' of PTENDENCY_* spelled as in fields.py) to numpy arrays in
    the (KLON, ...) Fortran layout of one block, i.e. C shape (..., KLON).
    Arrays the default configuration does not read may be omitted.
    """
    a1 = [_ptr(arrays.get(n)) for n in BLOCK_ARRAYS_1]
    a2 = [_ptr(arrays.get(n)) for n in BLOCK_ARRAYS_2]
    return _check(lib().cloudsc_b200_block(
        ctypes.byref(params), int(kidia), int(kfdia), int(klon), int(klev), int(bool(lddiag)),
        float(ptsphy), *a1, int(bool(ldslphy)), *a2, int(kfldx)))


def cloudsc_block_noalloc(params, kidia, kfdia, klon, klev, ptsphy, arrays, stream=None):
    """cloudsc_b200_block_noalloc: the per-block call that allocates no device
    memory (it works in one fixed 16 MiB array inside the library; KLON <= 288
    at KLEV 137).  ``arrays`` as for cloudsc_block (one block, host numpy
    arrays); the arrays the default configuration reads and writes are
    required.  Synchronous on ``stream`` (None = the default stream)."""
    L = lib()
    f = L.cloudsc_b200_block_noalloc
    if f.argtypes is None:
        vp = ctypes.c_void_p
        f.argtypes = ([ctypes.POINTER(CloudscParams), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                       ctypes.c_int32, ctypes.c_double] + [vp] * len(BATCHED_FIELDS) + [vp])
        f.restype = ctypes.c_int
        L.cloudsc_b200_block_noalloc_capacity.restype = ctypes.c_size_t
    args = [_ptr(arrays[n]) for n, *_ in BATCHED_FIELDS]
    s = None
    if stream is not None:
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
    return _check(f(ctypes.byref(params), int(kidia), int(kfdia), int(klon), int(klev), float(ptsphy),
                    *args, s))


def block_noalloc_capacity():
    """Bytes of the fixed device array cloudsc_block_noalloc works in."""
    L = lib()
    L.cloudsc_b200_block_noalloc_capacity.restype = ctypes.c_size_t
    return int(L.cloudsc_b200_block_noalloc_capacity())


def satadj_batched(params, arrays, nproma, klev, ngpblks, ngptot, ptsphy, counter=None, stream=None):
    """CLOUD_SATADJ over every block of ``arrays`` (torch CUDA tensors in the
    fields.SATADJ_FIELDS layout); outputs written in place, asynchronously on
    ``stream``."""
    from .fields import SATADJ_FIELDS
    ptrs = [_ptr(arrays[n]) for n, *_ in SATADJ_FIELDS]
    cnt = _ptr(counter) if counter is not None else None
    st = stream.cuda_stream if stream is not None else None
    return _check(lib().cloudsc_b200_satadj_batched(ctypes.byref(params), int(nproma), int(klev), int(ngpblks),
                                                    int(ngptot), float(ptsphy), *ptrs, cnt, st))


def satadj_block(params, kidia, kfdia, klon, klev, ptsphy, arrays):
    """Per-block drop-in with host (numpy) arrays of one block, shapes as one
    block of fields.SATADJ_FIELDS; returns the warning count."""
    a = arrays

    def h(n):
        x = a[n]
        if not (isinstance(x, np.ndarray) and x.flags["C_CONTIGUOUS"] and x.dtype == np.float64):
            raise ValueError(f"{n}: need a C-contiguous float64 numpy array")
        return x.ctypes.data

    ins = ["pap", "paph", "pt", "pq", "pa", "pl", "pi", "tendency_cml_t", "tendency_cml_q", "tendency_cml_a",
           "tendency_cml_l", "tendency_cml_i", "phrsw", "phrlw", "tendency_vdf_t", "tendency_vdf_q"]
    outs = ["tendency_loc_t", "tendency_loc_q", "tendency_loc_a", "tendency_loc_l", "tendency_loc_i"]
    return _check(lib().cloudsc_b200_satadj_block(
        ctypes.byref(params), int(kidia), int(kfdia), int(klon), int(klev), None, 0, float(ptsphy),
        *[h(n) for n in ins], None, None, h("pludeli"), h("pvervel"), None, *[h(n) for n in outs], None, 0))


def sltend_supersat_batched(params, arrays, nproma, klev, ngpblks, ngptot, tsphy, stream=None, diagnostics=True):
    """SLTEND's supersaturation adjustment over every block of ``arrays``
    (torch CUDA tensors, fields.SLTEND_FIELDS layout); the tendencies are
    updated in place, the rates written when ``diagnostics``."""
    from .fields import SLTEND_FIELDS
    ptrs = []
    for n, *_ in SLTEND_FIELDS:
        ptrs.append(_ptr(arrays[n]) if (diagnostics or not n.startswith("padj")) else None)
    st = stream.cuda_stream if stream is not None else None
    return _check(lib().cloudsc_b200_sltend_supersat_batched(ctypes.byref(params), int(nproma), int(klev),
                                                             int(ngpblks), int(ngptot), float(tsphy), *ptrs, st))


def cloudsc_batched_diag(params, arrays, diag, nproma, klev, ngpblks, ngptot, ptsphy, counter=None, stream=None):
    """cloudsc_batched (FP64) with the optional configurations the params
    switch on (budget diagnostics, SPP, cloud inhomogeneity, the aerosol
    switches LAERICESED and LAERICEAUTO): ``diag`` holds
    the fields.DIAG_FIELDS device tensors (those of options that are off may
    be omitted); PEXTRA, (NGPBLKS, KFLDX, KLEV, NPROMA), is added to and PFSD
    written in place."""
    from .fields import DIAG_FIELDS
    ptrs = [_ptr(arrays[n]) for n, *_ in BATCHED_FIELDS]
    dptrs = [_ptr(diag.get(n)) for n, *_ in DIAG_FIELDS]
    kfldx = int(diag["pextra"].shape[1]) if diag.get("pextra") is not None else 0
    cnt = _ptr(counter) if counter is not None else None
    st = stream.cuda_stream if stream is not None else None
    return _check(lib().cloudsc_b200_batched_diag(ctypes.byref(params), int(nproma), int(klev), int(ngpblks),
                                                  int(ngptot), float(ptsphy), *ptrs, *dptrs, kfldx, cnt, st))


def _species_ptr(x, m):
    """Address of species m of a (NGPBLKS, N, KLEV, NPROMA) array."""
    return _ptr(x) + m * x.shape[2] * x.shape[3] * x.element_size()


def state_increment_batched(state, increments, nproma, klev, ngpblks, ngptot, kidia=1, keymask=None,
                            stream=None):
    """STATE_INCREMENT (state_increment.F90) over every block: each field of
    ``state`` (torch CUDA tensors, keys u, v, t, o3, q, a, cld, tke; CLD
    (NGPBLKS, NCLV, KLEV, NPROMA)) is incremented in place by the increment
    of the same name in ``increments`` (keys u, v, t, o3, q, a, ql, qi, qr,
    qs, tke, or cld for a CLD-shaped array whose four condensate species are
    added), over columns KIDIA..ICEND; Q, O3, A, TKE and the condensates only
    where ``keymask`` (params.KEY_* bits, default all) has their bit.
    Asynchronous on ``stream``."""
    from .params import KEY_ALL, make_increments, make_state
    st = make_state(state, KEY_ALL if keymask is None else keymask, _ptr)
    inc = make_increments(increments, _ptr, _species_ptr)
    s = stream.cuda_stream if stream is not None else None
    f = lib().cloudsc_b200_state_increment_batched
    return _check(f(int(nproma), int(klev), int(ngpblks), int(ngptot), int(kidia), ctypes.byref(st),
                    ctypes.byref(inc), s))


def satadj_increment_batched(params, arrays, nproma, klev, ngpblks, ngptot, ptsphy, keymask=None, counter=None,
                             stream=None):
    """CLOUD_SATADJ followed by the STATE_INCREMENT of its five tendencies
    into the cumulative ones (callpar.F90:1253-1280), one kernel: as
    satadj_batched, and the tendency_cml_t/q/a/l/i tensors of ``arrays`` are
    incremented in place (q, a, l, i only where ``keymask`` has KEY_Q,
    KEY_A, KEY_QL, KEY_QI; default all)."""
    from .fields import SATADJ_FIELDS
    from .params import KEY_ALL
    ptrs = [_ptr(arrays[n]) for n, *_ in SATADJ_FIELDS]
    cnt = _ptr(counter) if counter is not None else None
    st = stream.cuda_stream if stream is not None else None
    f = lib().cloudsc_b200_satadj_increment_batched
    return _check(f(ctypes.byref(params), int(nproma), int(klev), int(ngpblks), int(ngptot), float(ptsphy),
                    *ptrs, int(KEY_ALL if keymask is None else keymask), cnt, st))


def division_check(a, b, stream=None):
    """The column kernels' division on the pairs of two equal-length float64
    CUDA tensors: returns (q, bad), the quotients and an int32 flag, 1 where
    an operand lies outside the division's exact window (the kernels then run
    the column again with IEEE division).  Inside the window q equals IEEE
    a / b bit for bit."""
    import torch
    if a.dtype != torch.float64 or b.dtype != torch.float64 or a.shape != b.shape or not a.is_cuda:
        raise CloudscError(-2, "division_check wants two float64 CUDA tensors of one shape")
    a, b = a.contiguous(), b.contiguous()
    q = torch.empty_like(a)
    bad = torch.empty(a.shape, dtype=torch.int32, device=a.device)
    st = stream.cuda_stream if stream is not None else None
    _check(lib().cloudsc_b200_division_check(_ptr(a), _ptr(b), a.numel(), _ptr(q), _ptr(bad), st))
    return q, bad


def reciprocal_check(b, stream=None):
    """The column kernels' reciprocal on a float64 CUDA tensor: returns
    (y, bad), the reciprocals and an int32 flag, 1 where b lies outside the
    window 2^-256 <= |b| < 2^256.  Inside it y equals IEEE 1 / b bit for
    bit."""
    import torch
    if b.dtype != torch.float64 or not b.is_cuda:
        raise CloudscError(-2, "reciprocal_check wants a float64 CUDA tensor")
    b = b.contiguous()
    y = torch.empty_like(b)
    bad = torch.empty(b.shape, dtype=torch.int32, device=b.device)
    st = stream.cuda_stream if stream is not None else None
    _check(lib().cloudsc_b200_reciprocal_check(_ptr(b), b.numel(), _ptr(y), _ptr(bad), st))
    return y, bad
