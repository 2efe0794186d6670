"""Shared helpers for the parity tests: run the oracle and the GPU on the same
inputs and compare every defined output."""
import numpy as np

from openifs_b200 import cloudsc, fields, inputs
from oracle import oracle

KLEV = 137
PTSPHY = 3600.0

# Outputs compared.  PTENDENCY_LOC_CLD(:,:,NCLV) is left undefined by the
# reference (cloudsc.F90:971 loops to NCLV-1) and is excluded by slicing.
COMPARED = [n for n in fields.OUTPUT_NAMES]

# Relative-error denominator floor: an element's error is
# |gpu - ref| / max(|ref|, FLOOR_REL * max|ref over the field|).
FLOOR_REL = 1e-6


def params(ncldtop=None):
    nc = inputs.ncldtop_l137() if ncldtop is None else ncldtop
    return cloudsc.default_params(PTSPHY, nc), oracle.params_default(PTSPHY, nc)


def defined(name, a):
    if name == "tendency_loc_cld":
        return a[:, :4]
    return a


def rel_err(g, o):
    g = np.asarray(g, dtype=np.float64)
    o = np.asarray(o, dtype=np.float64)
    scale = np.max(np.abs(o)) if o.size else 0.0
    denom = np.maximum(np.abs(o), FLOOR_REL * scale)
    with np.errstate(invalid="ignore", divide="ignore"):
        e = np.where(denom > 0, np.abs(g - o) / denom, np.where(g == o, 0.0, np.inf))
    return e


def compare(gpu, ref, names=COMPARED, ngptot=None, nproma=None):
    """Per-field max relative error, plus the column-wise maximum used to
    count branch-flip columns."""
    report = {}
    colmax = None
    for n in names:
        g, o = defined(n, gpu[n]), defined(n, ref[n])
        if ngptot is not None:
            g = _valid_cols(g, ngptot, nproma)
            o = _valid_cols(o, ngptot, nproma)
        e = rel_err(g, o)
        report[n] = float(e.max()) if e.size else 0.0
        c = e.reshape(e.shape[0], -1, e.shape[-1]).max(axis=1)  # (blocks, columns)
        colmax = c if colmax is None else np.maximum(colmax, c)
    return report, colmax


def _valid_cols(a, ngptot, nproma):
    nb = a.shape[0]
    last = ngptot - (nb - 1) * nproma
    if last == nproma:
        return a
    a = a.copy()
    a[-1, ..., last:] = 0.0
    return a


def run_oracle(po, arrs, nproma, ngpblks, ngptot, nthreads=0, libm="plibm", klev=KLEV):
    ref = {k: v.copy() for k, v in arrs.items()}
    nwarn = oracle.cloudsc_batched(po, ref, nproma, klev, ngpblks, ngptot, PTSPHY, nthreads, libm=libm)
    return ref, nwarn


def run_hostemu(p, arrs, nproma, ngpblks, ngptot, precision=0, libm="plibm", klev=KLEV):
    """The kernel's own column code built for the host (tests/hostemu)."""
    import ctypes
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hostemu")
    # "redo": every fast division of a FASTDIV column reports bad, so each
    # level also runs its IEEE-division pass
    name = {"plibm": "libcloudsc_hostemu.so", "glibc": "libcloudsc_hostemu_glibc.so",
            "redo": "libcloudsc_hostemu_redo.so"}[libm]
    path = os.path.join(here, name)
    if not os.path.exists(path):
        import subprocess
        subprocess.run(["make", "-s", "-C", here], check=True)
    L = ctypes.CDLL(path)
    out = {k: v.copy() for k, v in arrs.items()}
    ptrs = (ctypes.c_void_p * len(fields.BATCHED_FIELDS))(
        *[out[n].ctypes.data for n, *_ in fields.BATCHED_FIELDS])
    nw = L.hostemu_batched(ctypes.byref(p), int(nproma), int(klev), int(ngpblks), int(ngptot),
                           ctypes.c_double(PTSPHY), ptrs, int(precision))
    return out, nw


EDGE_CASES = ["clear", "overcast", "warm", "cold", "no_convection", "all_convection", "land",
              "sea", "tiny_condensate", "supersaturated", "tiny_cloud_fraction", "negative_condensate"]


def apply_case(arrs, case):
    """Turn a generated input into one of the edge cases the reference's
    branches single out (in place)."""
    cl = arrs["pclv"]
    if case == "clear":
        cl[:] = 0.0
        arrs["pa"][:] = 0.0
        arrs["tendency_cml_cld"][:] = 0.0
    elif case == "overcast":
        arrs["pa"][:] = 1.0
    elif case == "warm":
        arrs["pt"][:] = np.maximum(arrs["pt"], 280.0)
    elif case == "cold":
        arrs["pt"][:] = np.minimum(arrs["pt"], 230.0)
    elif case == "no_convection":
        for n in ("ldcum", "ktype", "plu", "plude", "pludeli", "psnde", "pmfu", "pmfd"):
            arrs[n][:] = 0
    elif case == "all_convection":
        arrs["ldcum"][:] = 1
        arrs["ktype"][:] = np.where(arrs["ktype"] == 0, 2, arrs["ktype"])
    elif case == "land":
        arrs["plsm"][:] = 1.0
    elif case == "sea":
        arrs["plsm"][:] = 0.0
    elif case == "tiny_condensate":
        cl[:, :4] = np.where(cl[:, :4] > 0, 5e-9, 0.0)
    elif case == "supersaturated":
        # 40 % more vapour: most cloudy levels above saturation, so that
        # CLOUD_SUPERSATCHECK and the condensation branches act everywhere
        arrs["pq"][:] = arrs["pq"] * 1.4
    elif case == "tiny_cloud_fraction":
        # cloud fraction below RAMIN (1e-8) wherever there is cloud: the
        # tidy-up evaporates the condensate of every such level
        arrs["pa"][:] = np.where(arrs["pa"] > 0, 5e-9, 0.0)
    elif case == "negative_condensate":
        # negative liquid and ice of about -1e-6 kg/kg on every 7th level
        # (as a dynamics step can leave them): the tidy-up moves them to the
        # vapour, and the tendencies are taken against the negative first
        # guess
        cl[:, 0, ::7] = -np.abs(cl[:, 0, ::7]) * 0.01 - 1e-6
        cl[:, 1, ::7] = -np.abs(cl[:, 1, ::7]) * 0.01 - 1e-6
    else:
        raise ValueError(case)
    return arrs


# fields and slices reported for the FP32-mixed form: the 5 species
# tendencies (4 condensates + vapour), T, surface rain/snow (the bar of 1e-5
# applies to these), and cloud fraction (reported only: it jumps at the
# CLOUD_SUPERSATCHECK branch ZCOND > ZEPSEC, cloud_supersatcheck.F90:183-191)
MIXED_REPORT = [("tendency_loc_t", None), ("tendency_loc_q", None),
                ("tendency_loc_cld:l", 0), ("tendency_loc_cld:i", 1), ("tendency_loc_cld:r", 2),
                ("tendency_loc_cld:s", 3), ("pfplsl:surface", -1), ("pfplsn:surface", -1),
                ("tendency_loc_a", None)]
MIXED_BOUNDED = [n for n, _ in MIXED_REPORT if n != "tendency_loc_a"]
# the FP32-mixed form's error contract on those fields: RMS error / RMS of
# the FP64 field at most 1e-5, and normwise max error (max |err| / max |ref|)
# at most 1e-4 (measured on 262,144 columns: RMS 1e-6, max 7e-5 for the T and
# q tendencies)
MIXED_RMS_TOL = 1e-5
MIXED_MAX_TOL = 1e-4
# the target for both, met by the host build of the same code (C library
# expf/powf instead of the GPU's special-function-unit forms)
MIXED_TOL = 1e-5


def mixed_error_stats(g, o):
    out = {}
    for name, sl in MIXED_REPORT:
        base = name.split(":")[0]
        a, b = g[base], o[base]
        if base == "tendency_loc_cld":
            a, b = a[:, sl], b[:, sl]
        elif sl is not None:
            a, b = a[:, sl], b[:, sl]
        d = np.abs(a - b)
        mref = np.abs(b).max()
        rms_ref = np.sqrt(np.mean(b * b))
        out[name] = {"normwise_max": float(d.max() / mref) if mref > 0 else float(d.max()),
                     "rms_ratio": float(np.sqrt(np.mean(d * d)) / rms_ref) if rms_ref > 0 else 0.0,
                     "max_abs": float(d.max())}
    return out


def run_gpu(p, arrs, nproma, ngpblks, ngptot, precision=cloudsc.FP64, device="cuda:0", klev=KLEV):
    import torch
    cloudsc.setup(p)
    dev = {k: torch.from_numpy(v).to(device) for k, v in arrs.items()}
    cnt = torch.zeros(1, dtype=torch.int32, device=device)
    cloudsc.cloudsc_batched(p, dev, nproma, klev, ngpblks, ngptot, PTSPHY, precision=precision,
                            counter=cnt)
    torch.cuda.synchronize()
    out = {k: v.cpu().numpy() for k, v in dev.items()}
    return out, int(cnt.item())


def run_hostemu_satadj(p, arrs, nproma, ngpblks, ngptot, libm="plibm"):
    """The SATADJ kernel's point code built for the host (tests/hostemu)."""
    import ctypes
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hostemu")
    name = "libcloudsc_hostemu.so" if libm == "plibm" else "libcloudsc_hostemu_glibc.so"
    path = os.path.join(here, name)
    import subprocess
    subprocess.run(["make", "-s", "-C", here], check=True)
    L = ctypes.CDLL(path)
    out = {k: v.copy() for k, v in arrs.items()}
    ptrs = (ctypes.c_void_p * len(fields.SATADJ_FIELDS))(*[out[n].ctypes.data for n, *_ in fields.SATADJ_FIELDS])
    nw = L.hostemu_satadj_batched(ctypes.byref(p), int(nproma), KLEV, int(ngpblks), int(ngptot),
                                  ctypes.c_double(PTSPHY), ptrs)
    return out, nw


def run_oracle_satadj(po, arrs, nproma, ngpblks, ngptot, libm="plibm"):
    from oracle import oracle
    out = {k: v.copy() for k, v in arrs.items()}
    nw = oracle.satadj_batched(po, out, nproma, KLEV, ngpblks, ngptot, PTSPHY, libm=libm)
    return out, nw


def run_hostemu_sltend(p, arrs, nproma, ngpblks, ngptot, libm="plibm"):
    """SLTEND's supersaturation adjustment, the kernel's point code on the host."""
    import ctypes
    import os
    import subprocess
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hostemu")
    subprocess.run(["make", "-s", "-C", here], check=True)
    name = "libcloudsc_hostemu.so" if libm == "plibm" else "libcloudsc_hostemu_glibc.so"
    L = ctypes.CDLL(os.path.join(here, name))
    out = {k: v.copy() for k, v in arrs.items()}
    ptrs = (ctypes.c_void_p * len(fields.SLTEND_FIELDS))(*[out[n].ctypes.data for n, *_ in fields.SLTEND_FIELDS])
    L.hostemu_sltend_batched(ctypes.byref(p), int(nproma), KLEV, int(ngpblks), int(ngptot),
                             ctypes.c_double(PTSPHY), ptrs)
    return out


def run_oracle_sltend(po, arrs, nproma, ngpblks, ngptot, libm="plibm"):
    from oracle import oracle
    out = {k: v.copy() for k, v in arrs.items()}
    oracle.sltend_supersat_batched(po, out, nproma, KLEV, ngpblks, ngptot, PTSPHY, libm=libm)
    return out



def run_hostemu_diag(p, arrs, diag, nproma, ngpblks, ngptot, libm="plibm", flags=0, klev=KLEV):
    """The kernel's column code with the budget diagnostics, on the host;
    flags 0x100 for the GEN column code, 0x200 for the kernels' fast pass with
    its rerun."""
    import ctypes
    import os
    import subprocess
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hostemu")
    subprocess.run(["make", "-s", "-C", here], check=True)
    name = {"plibm": "libcloudsc_hostemu.so", "glibc": "libcloudsc_hostemu_glibc.so",
            "redo": "libcloudsc_hostemu_redo.so"}[libm]
    L = ctypes.CDLL(os.path.join(here, name))
    out = {k: v.copy() for k, v in arrs.items()}
    dout = {k: v.copy() for k, v in diag.items()}
    a = (ctypes.c_void_p * len(fields.BATCHED_FIELDS))(*[out[n].ctypes.data for n, *_ in fields.BATCHED_FIELDS])
    b = (ctypes.c_void_p * len(fields.DIAG_FIELDS))(
        *[(dout[n].ctypes.data if dout.get(n) is not None else None) for n, *_ in fields.DIAG_FIELDS])
    nw = L.hostemu_batched_diag(ctypes.byref(p), int(nproma), int(klev), int(ngpblks), int(ngptot),
                                ctypes.c_double(PTSPHY), a, b, int(dout["pextra"].shape[1]), int(flags))
    return out, dout, nw


def run_oracle_diag(po, arrs, diag, nproma, ngpblks, ngptot, libm="plibm", klev=KLEV):
    from oracle import oracle
    out = {k: v.copy() for k, v in arrs.items()}
    dout = {k: v.copy() for k, v in diag.items()}
    nw = oracle.cloudsc_batched_diag(po, out, dout, nproma, klev, ngpblks, ngptot, PTSPHY, libm=libm)
    return out, dout, nw


BUDGET_CASES = [
    {"lcldbudc": 1},
    {"lcldbudl": 1},
    {"lcldbudi": 1},
    {"lcldbudt": 1},
    {"lcldbud_vertint": 1},
    {"lcldbudc": 1, "lcldbudl": 1, "lcldbudi": 1, "lcldbudt": 1, "lcldbud_vertint": 1, "lcldbud_timeint": 1,
     "lbud23": 1},
]


def with_flags(p, flags):
    """A copy of the params struct ``p`` with ``flags`` set."""
    q = type(p).from_buffer_copy(p)
    for k, v in flags.items():
        setattr(q, k, v)
    return q


def with_spp(p, lramidlimit1=1, nrftotal=10):
    """A copy of ``p`` with LSPP and all eight perturbations on: fields
    MP = 1..8 (CLOUDINHOM also reads MP+1 = 9), MU(i) = -0.05 (n+1) i and
    XMAG(i) = 0.3 + 0.05 n."""
    q = type(p).from_buffer_copy(p)
    q.lspp = 1
    q.spp_nrftotal = nrftotal
    q.spp_lramidlimit1 = lramidlimit1
    for n in range(8):
        q.spp_on[n] = 1
        q.spp_mp[n] = n + 1
        for i in range(2):
            q.spp_mu[2 * n + i] = -0.05 * (n + 1) * (i + 1)
            q.spp_xmag[2 * n + i] = 0.3 + 0.05 * n
    return q


OPT_CASES = ["spp", "inhomog", "radinhomog", "aerosol", "all", "all+budgets"]

# (block, column, level) points given a pressure of 1e80 Pa, outside the fast
# division's window: those columns' fast pass reports at that level (the
# first division by PAP) and they run again with IEEE division; the scheme's
# outputs stay finite
OUT_OF_WINDOW_PAP = [(0, 3, 90), (2, 17, 60), (5, 1, 120)]


def with_out_of_window_pressure(arrs, points=OUT_OF_WINDOW_PAP):
    """A copy of ``arrs`` with PAP = 1e80 at ``points``."""
    out = dict(arrs)
    out["pap"] = arrs["pap"].copy()
    for ib, jl, k in points:
        out["pap"][ib, k, jl] = 1e80
    return out
# the four aerosol switches (NAERCLD > 0); LAERLIQAUTOLSP and LAERLIQCOLL act
# only under IWARMRAIN = 1, which the reference does not use
AEROSOL = {"laericesed": 1, "laericeauto": 1, "laerliqautolsp": 1, "laerliqcoll": 1}


def opt_params(p, case):
    """``p`` with the optional configuration ``case`` of OPT_CASES."""
    if case == "spp":
        return with_spp(p)
    if case == "inhomog":
        return with_flags(p, {"lcloud_inhomog": 1})
    if case == "radinhomog":
        return with_flags(p, {"lrad_cloud_inhomog": 1})
    if case == "aerosol":
        return with_flags(p, AEROSOL)
    q = with_flags(with_spp(p, lramidlimit1=0), dict({"lcloud_inhomog": 1, "lrad_cloud_inhomog": 1}, **AEROSOL))
    if case == "all+budgets":
        q = with_flags(q, BUDGET_CASES[-1])
    return q
