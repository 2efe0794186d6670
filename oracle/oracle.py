"""ORACLE -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper of liboracle_cloudsc.so, the CPU restatement of the reference's
double-precision CLOUDSC and CLOUD_SATADJ (cloudsc_oracle.c).  Only tests/, the smoke test and
bench.py's CPU-baseline leg use it, as the checker; the product never calls it.
Parity unpinned: the reference has no CLOUDSC golden vectors and cannot be
compiled here (no Fortran compiler).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATHS = {"glibc": os.path.join(_HERE, "liboracle_cloudsc.so"),
             "plibm": os.path.join(_HERE, "liboracle_cloudsc_plibm.so")}
_libs = {}


def build():
    r = subprocess.run(["make", "-s", "-C", _HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB_PATHS


def lib(libm="glibc"):
    """The oracle linked against the system libm ("glibc", the reference as a
    gfortran/Linux build runs it) or against plibm.h ("plibm", the libm of
    the B200 kernels)."""
    if libm not in _libs:
        if not os.path.exists(LIB_PATHS[libm]):
            build()
        from openifs_b200.params import CloudscParams
        from openifs_b200.fields import BATCHED_FIELDS, DIAG_FIELDS
        L = ctypes.CDLL(LIB_PATHS[libm])
        P = ctypes.POINTER(CloudscParams)
        vp = ctypes.c_void_p
        i32 = ctypes.c_int
        L.oracle_params_default.argtypes = [ctypes.c_double, i32, P]
        L.oracle_params_default.restype = i32
        L.oracle_fcgeneralized_gamma.argtypes = [ctypes.c_double]
        L.oracle_fcgeneralized_gamma.restype = ctypes.c_double
        L.oracle_cloudsc_batched.argtypes = ([P, i32, i32, i32, i32, ctypes.c_double] +
                                             [vp] * len(BATCHED_FIELDS) + [i32])
        L.oracle_cloudsc_batched.restype = i32
        from openifs_b200.fields import SATADJ_FIELDS
        L.oracle_cloud_satadj_batched.argtypes = ([P, i32, i32, i32, i32, ctypes.c_double] +
                                                  [vp] * len(SATADJ_FIELDS) + [i32])
        L.oracle_cloud_satadj_batched.restype = i32
        L.oracle_cloudsc_batched_diag.argtypes = ([P, i32, i32, i32, i32, ctypes.c_double] +
                                                  [vp] * (len(BATCHED_FIELDS) + len(DIAG_FIELDS)) + [i32, i32])
        L.oracle_cloudsc_batched_diag.restype = i32
        from openifs_b200.fields import SLTEND_FIELDS
        L.oracle_sltend_supersat_batched.argtypes = ([P, i32, i32, i32, i32, ctypes.c_double] +
                                                     [vp] * len(SLTEND_FIELDS) + [i32])
        L.oracle_sltend_supersat_batched.restype = i32
        _libs[libm] = L
    return _libs[libm]


def params_default(tsphy, ncldtop):
    from openifs_b200.params import CloudscParams
    p = CloudscParams()
    rc = lib().oracle_params_default(float(tsphy), int(ncldtop), ctypes.byref(p))
    if rc != 0:
        raise RuntimeError(f"oracle_params_default returned {rc}")
    return p


def gamma(x):
    return lib().oracle_fcgeneralized_gamma(float(x))


def cloudsc_batched(params, arrays, nproma, klev, ngpblks, ngptot, ptsphy, nthreads=0, libm="glibc"):
    """Run the oracle over all blocks of ``arrays`` (numpy, fields layout), in
    place.  Returns the number of negative-condensate warning events."""
    from openifs_b200.fields import BATCHED_FIELDS
    ptrs = []
    for n, *_ in BATCHED_FIELDS:
        a = arrays[n]
        if not (isinstance(a, np.ndarray) and a.flags["C_CONTIGUOUS"]):
            raise ValueError(f"{n}: need a C-contiguous numpy array")
        ptrs.append(a.ctypes.data)
    rc = lib(libm).oracle_cloudsc_batched(ctypes.byref(params), int(nproma), int(klev), int(ngpblks),
                                      int(ngptot), float(ptsphy), *ptrs, int(nthreads))
    if rc < 0:
        raise RuntimeError(f"oracle_cloudsc_batched returned {rc}")
    return rc


def satadj_batched(params, arrays, nproma, klev, ngpblks, ngptot, ptsphy, nthreads=0, libm="glibc"):
    """CLOUD_SATADJ over all blocks of ``arrays`` (numpy, fields.SATADJ_FIELDS
    layout), outputs in place.  Returns the negative-condensate warning count."""
    from openifs_b200.fields import SATADJ_FIELDS
    ptrs = []
    for n, *_ in SATADJ_FIELDS:
        a = arrays[n]
        if not (isinstance(a, np.ndarray) and a.flags["C_CONTIGUOUS"]):
            raise ValueError(f"{n}: need a C-contiguous numpy array")
        ptrs.append(a.ctypes.data)
    rc = lib(libm).oracle_cloud_satadj_batched(ctypes.byref(params), int(nproma), int(klev), int(ngpblks),
                                               int(ngptot), float(ptsphy), *ptrs, int(nthreads))
    if rc < 0:
        raise RuntimeError(f"oracle_cloud_satadj_batched returned {rc}")
    return rc


def sltend_supersat_batched(params, arrays, nproma, klev, ngpblks, ngptot, tsphy, nthreads=0, libm="glibc"):
    """SLTEND's supersaturation adjustment over all blocks (numpy,
    fields.SLTEND_FIELDS layout), in place."""
    from openifs_b200.fields import SLTEND_FIELDS
    ptrs = []
    for n, *_ in SLTEND_FIELDS:
        a = arrays[n]
        if not (isinstance(a, np.ndarray) and a.flags["C_CONTIGUOUS"]):
            raise ValueError(f"{n}: need a C-contiguous numpy array")
        ptrs.append(a.ctypes.data)
    rc = lib(libm).oracle_sltend_supersat_batched(ctypes.byref(params), int(nproma), int(klev), int(ngpblks),
                                                  int(ngptot), float(tsphy), *ptrs, int(nthreads))
    if rc < 0:
        raise RuntimeError(f"oracle_sltend_supersat_batched returned {rc}")
    return rc


def cloudsc_batched_diag(params, arrays, diag, nproma, klev, ngpblks, ngptot, ptsphy, nthreads=0, libm="glibc"):
    """oracle cloudsc_batched with the cloud budget diagnostics: ``diag``
    holds the fields.DIAG_FIELDS arrays (PEXTRA updated in place)."""
    from openifs_b200.fields import BATCHED_FIELDS, DIAG_FIELDS
    ptrs = []
    for n, *_ in BATCHED_FIELDS:
        a = arrays[n]
        if not (isinstance(a, np.ndarray) and a.flags["C_CONTIGUOUS"]):
            raise ValueError(f"{n}: need a C-contiguous numpy array")
        ptrs.append(a.ctypes.data)
    for n, *_ in DIAG_FIELDS:
        a = diag.get(n)
        ptrs.append(None if a is None else a.ctypes.data)
    kfldx = diag["pextra"].shape[1] if diag.get("pextra") is not None else 0
    rc = lib(libm).oracle_cloudsc_batched_diag(ctypes.byref(params), int(nproma), int(klev), int(ngpblks),
                                               int(ngptot), float(ptsphy), *ptrs, int(kfldx), int(nthreads))
    if rc < 0:
        raise RuntimeError(f"oracle_cloudsc_batched_diag returned {rc}")
    return rc


def state_increment_batched(state, increments, nproma, klev, ngpblks, ngptot, kidia=1, keymask=None):
    """STATE_INCREMENT over every block of numpy arrays, in place; the
    conventions of openifs_b200.cloudsc.state_increment_batched."""
    from openifs_b200.params import KEY_ALL, make_increments, make_state

    def ptr(x):
        if not (isinstance(x, np.ndarray) and x.flags["C_CONTIGUOUS"] and x.dtype == np.float64):
            raise ValueError("need C-contiguous float64 numpy arrays")
        return x.ctypes.data

    def species(x, m):
        return ptr(x) + m * x.shape[2] * x.shape[3] * 8

    st = make_state(state, KEY_ALL if keymask is None else keymask, ptr)
    inc = make_increments(increments, ptr, species)
    L = lib()
    f = L.oracle_state_increment_batched
    f.argtypes = [ctypes.c_int] * 5 + [ctypes.c_void_p] * 2
    f.restype = ctypes.c_int
    rc = f(int(nproma), int(klev), int(ngpblks), int(ngptot), int(kidia), ctypes.byref(st), ctypes.byref(inc))
    if rc < 0:
        raise RuntimeError(f"oracle_state_increment_batched returned {rc}")
    return rc
