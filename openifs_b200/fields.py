"""The arrays of the batched CLOUDSC call, in C-ABI argument order.

Every array is stored as the Fortran (NPROMA, <dims>, NGPBLKS) block layout of
EC_PHYS_DRV (ifs-source/arpifs/phys_ec/ec_phys_drv.F90:145-185); in numpy /
torch C order that is shape (NGPBLKS, <dims reversed>, NPROMA):

    "2d"  (KLEV, NPROMA)          a (KLON,KLEV) field
    "3dN" (N, KLEV, NPROMA)       a (KLON,KLEV,N) field
    "hl"  (KLEV+1, NPROMA)        a half-level (KLON,KLEV+1) field
    "1d"  (NPROMA,)               a (KLON) field
"""
import numpy as np

# (name, kind, dtype, role) with role in {"in", "out", "inout"}; the order is
# the argument order of cloudsc_b200_batched / cloudsc_b200_batched_host.
BATCHED_FIELDS = [
    ("pt", "2d", np.float64, "in"),
    ("pq", "2d", np.float64, "in"),
    ("tendency_cml_t", "2d", np.float64, "in"),
    ("tendency_cml_q", "2d", np.float64, "in"),
    ("tendency_cml_a", "2d", np.float64, "in"),
    ("tendency_cml_cld", "3d5", np.float64, "in"),
    ("tendency_loc_t", "2d", np.float64, "out"),
    ("tendency_loc_q", "2d", np.float64, "out"),
    ("tendency_loc_a", "2d", np.float64, "out"),
    ("tendency_loc_cld", "3d5", np.float64, "out"),
    ("pvfl", "2d", np.float64, "in"),
    ("pvfi", "2d", np.float64, "in"),
    ("pap", "2d", np.float64, "in"),
    ("paph", "hl", np.float64, "in"),
    ("plsm", "1d", np.float64, "in"),
    ("ldcum", "1d", np.int32, "in"),
    ("ktype", "1d", np.int32, "in"),
    ("peis", "1d", np.float64, "in"),
    ("plu", "2d", np.float64, "in"),
    ("plude", "2d", np.float64, "inout"),
    ("pludeli", "3d4", np.float64, "in"),
    ("psnde", "3d2", np.float64, "in"),
    ("pmfu", "2d", np.float64, "in"),
    ("pmfd", "2d", np.float64, "in"),
    ("pa", "2d", np.float64, "in"),
    ("pclv", "3d5", np.float64, "in"),
    ("pcovptot", "2d", np.float64, "out"),
    ("prainfrac_toprfz", "1d", np.float64, "out"),
    ("pfsqlf", "hl", np.float64, "out"),
    ("pfsqif", "hl", np.float64, "out"),
    ("pfcqnng", "hl", np.float64, "out"),
    ("pfcqlng", "hl", np.float64, "out"),
    ("pfsqrf", "hl", np.float64, "out"),
    ("pfsqsf", "hl", np.float64, "out"),
    ("pfcqrng", "hl", np.float64, "out"),
    ("pfcqsng", "hl", np.float64, "out"),
    ("pfsqltur", "hl", np.float64, "out"),
    ("pfsqitur", "hl", np.float64, "out"),
    ("pfplsl", "hl", np.float64, "out"),
    ("pfplsn", "hl", np.float64, "out"),
    ("pfhpsl", "hl", np.float64, "out"),
    ("pfhpsn", "hl", np.float64, "out"),
]
FIELD_INDEX = {f[0]: i for i, f in enumerate(BATCHED_FIELDS)}
# element type of each array in the single-precision interface (JPRB =
# REAL(4)): every real array float32, the integer ones unchanged
DTYPE_SP = {f[0]: (np.float32 if f[2] == np.float64 else f[2]) for f in BATCHED_FIELDS}
INPUT_NAMES = [f[0] for f in BATCHED_FIELDS if f[3] in ("in", "inout")]
OUTPUT_NAMES = [f[0] for f in BATCHED_FIELDS if f[3] in ("out", "inout")]
KIND = {f[0]: f[1] for f in BATCHED_FIELDS}
DTYPE = {f[0]: f[2] for f in BATCHED_FIELDS}


def block_shape(kind, nproma, klev):
    if kind == "2d":
        return (klev, nproma)
    if kind == "hl":
        return (klev + 1, nproma)
    if kind == "1d":
        return (nproma,)
    if kind.startswith("3d"):
        return (int(kind[2:]), klev, nproma)
    raise ValueError(kind)


def batched_shape(name, ngpblks, nproma, klev):
    return (ngpblks,) + block_shape(KIND[name], nproma, klev)


def alloc(ngpblks, nproma, klev, names=None, alloc_fn=None):
    """Zero-filled arrays for `names` (default: all) in the batched layout."""
    names = names or [f[0] for f in BATCHED_FIELDS]
    out = {}
    for n in names:
        shp = batched_shape(n, ngpblks, nproma, klev)
        out[n] = alloc_fn(shp, DTYPE[n]) if alloc_fn else np.zeros(shp, DTYPE[n])
    return out


# Algorithmic HBM traffic of one FP64 column (bytes): every array element the
# default configuration reads or writes, once.
def bytes_per_column(klev=137, fp=8):
    reads_lv = 26  # PT PQ CML_T CML_Q CML_A CML_CLD*4 PA PCLV*4 PAP PAPH PLU PLUDE
    #                PLUDELI*2 PSNDE*2 PMFU PMFD PVFL PVFI
    read = (reads_lv * klev + 1) * fp + 2 * fp + 2 * 4  # + extra PAPH half level, PLSM PEIS, KTYPE LDCUM
    writes_lv = 9  # LOC_T LOC_Q LOC_A LOC_CLD*4 PCOVPTOT PLUDE
    write = (writes_lv * klev + 14 * (klev + 1) + 1) * fp
    return read, write


def host_copy_bytes(nproma, klev, ngpblks, ngptot=None):
    """Bytes cloudsc_b200_batched_host copies (host to device, device to host).

    Inputs cross PCIe as whole blocks, and only the rows the default
    configuration reads (bytes_per_column's read list: four of the five
    PTENDENCY_CML_CLD and PCLV species, two of the four PLUDELI components);
    outputs come back for the NGPTOT computed columns only."""
    ngptot = nproma * ngpblks if ngptot is None else ngptot
    read, write = bytes_per_column(klev)
    return read * nproma * ngpblks, write * ngptot


# The arrays of the batched CLOUD_SATADJ call (cloudsc_b200_satadj_batched),
# in its argument order: the argument order of cloud_satadj.F90:13-26 without
# the arguments the default configuration does not read (KTYPE, LDDIAG, PMFU,
# PMFD, PGP2DSPP, PEXTRA).  PL/PI and their tendencies are the liquid and ice
# slices of CALLPAR's STATE_T0%CLD / TENDENCY_CML%CLD (callpar.F90:1253-1279).
SATADJ_FIELDS = [
    ("pap", "2d", np.float64, "in"),
    ("paph", "hl", np.float64, "in"),
    ("pt", "2d", np.float64, "in"),
    ("pq", "2d", np.float64, "in"),
    ("pa", "2d", np.float64, "in"),
    ("pl", "2d", np.float64, "in"),
    ("pi", "2d", np.float64, "in"),
    ("tendency_cml_t", "2d", np.float64, "in"),
    ("tendency_cml_q", "2d", np.float64, "in"),
    ("tendency_cml_a", "2d", np.float64, "in"),
    ("tendency_cml_l", "2d", np.float64, "in"),
    ("tendency_cml_i", "2d", np.float64, "in"),
    ("phrsw", "2d", np.float64, "in"),
    ("phrlw", "2d", np.float64, "in"),
    ("tendency_vdf_t", "2d", np.float64, "in"),
    ("tendency_vdf_q", "2d", np.float64, "in"),
    ("pludeli", "3d4", np.float64, "in"),
    ("pvervel", "2d", np.float64, "in"),
    ("tendency_loc_t", "2d", np.float64, "out"),
    ("tendency_loc_q", "2d", np.float64, "out"),
    ("tendency_loc_a", "2d", np.float64, "out"),
    ("tendency_loc_l", "2d", np.float64, "out"),
    ("tendency_loc_i", "2d", np.float64, "out"),
]
SATADJ_INPUTS = [f[0] for f in SATADJ_FIELDS if f[3] == "in"]
SATADJ_OUTPUTS = [f[0] for f in SATADJ_FIELDS if f[3] == "out"]


def satadj_alloc(ngpblks, nproma, klev, alloc_fn=None):
    """Zero-filled CLOUD_SATADJ arrays in the batched layout."""
    out = {}
    for n, kind, dt, _ in SATADJ_FIELDS:
        shp = (ngpblks,) + block_shape(kind, nproma, klev)
        out[n] = alloc_fn(shp, dt) if alloc_fn else np.zeros(shp, dt)
    return out


# Algorithmic HBM traffic of one CLOUD_SATADJ column (bytes, default
# configuration).  Levels NCLDTOP..KLEV read 17 level fields (PT PQ PA PL PI,
# five CML tendencies, PHRSW PHRLW, the two VDF tendencies, PLUDELI(3:4),
# PVERVEL) and PAP, plus PAPH on half levels NCLDTOP..KLEV+1; the levels
# above NCLDTOP read nothing (cloud_satadj.F90:338-345).  All KLEV levels of
# the 5 tendencies are written.
def satadj_bytes_per_column(klev=137, ncldtop=15, fp=8):
    nlev = klev - ncldtop + 1
    read = (18 * nlev + nlev + 1) * fp
    write = 5 * klev * fp
    return read, write


# The arrays of the batched SLTEND supersaturation adjustment
# (cloudsc_b200_sltend_supersat_batched), in its argument order.  "inout"
# tendencies are updated in place.
SLTEND_FIELDS = [
    ("pt", "2d", np.float64, "in"),
    ("pq", "2d", np.float64, "in"),
    ("pa", "2d", np.float64, "in"),
    ("prsf1", "2d", np.float64, "in"),
    ("prs1", "hl", np.float64, "in"),
    ("pcent", "2d", np.float64, "in"),
    ("pcenq", "2d", np.float64, "in"),
    ("pcena", "2d", np.float64, "in"),
    ("ptent", "2d", np.float64, "inout"),
    ("ptenq", "2d", np.float64, "inout"),
    ("ptena", "2d", np.float64, "inout"),
    ("ptencld", "3d5", np.float64, "inout"),
    ("padja", "2d", np.float64, "out"),
    ("padjl", "2d", np.float64, "out"),
    ("padji", "2d", np.float64, "out"),
]
SLTEND_OUTPUTS = [f[0] for f in SLTEND_FIELDS if f[3] in ("out", "inout")]


def sltend_alloc(ngpblks, nproma, klev, alloc_fn=None):
    out = {}
    for n, kind, dt, _ in SLTEND_FIELDS:
        shp = (ngpblks,) + block_shape(kind, nproma, klev)
        out[n] = alloc_fn(shp, dt) if alloc_fn else np.zeros(shp, dt)
    return out


# Algorithmic HBM traffic of one column of the SLTEND adjustment (bytes):
# levels NCLDTOP..KLEV read 12 level fields (PT PQ PA PRSF1, three PCEN, three
# PTEN, PTENCLD liquid and ice) and write 8 (five tendencies, three rates).
def sltend_bytes_per_column(klev=137, ncldtop=15, fp=8):
    nlev = klev - ncldtop + 1
    return 12 * nlev * fp, 8 * nlev * fp


# The arrays that only the optional configurations read or write -- the
# cloud budget diagnostics (LCLDBUDC/L/I/T, LCLDBUD_VERTINT;
# cloudsc.F90:3832-4110), SPP (LSPP) and the cloud-inhomogeneity paths
# (LCLOUD_INHOMOG, LRAD_CLOUD_INHOMOG) -- in the argument order of
# cloudsc_b200_batched_diag after the BATCHED_FIELDS arrays.  PGP2DSPP is
# (KLON, NRFTOTAL) per block: numpy shape (NGPBLKS, NRFTOTAL, NPROMA); PEXTRA
# is (KLON, KLEV, KFLDX) per block: numpy shape (NGPBLKS, KFLDX, KLEV, NPROMA).
DIAG_FIELDS = [
    ("pvfa", "2d", np.float64, "in"),
    ("pdyna", "2d", np.float64, "in"),
    ("pdynl", "2d", np.float64, "in"),
    ("pdyni", "2d", np.float64, "in"),
    ("pdyns", "2d", np.float64, "in"),
    ("phrsw", "2d", np.float64, "in"),
    ("phrlw", "2d", np.float64, "in"),
    ("pgaw", "1d", np.float64, "in"),
    ("kctop", "1d", np.int32, "in"),
    ("kpbltype", "1d", np.int32, "in"),
    ("pgp2dspp", "spp", np.float64, "in"),
    ("pre_ice", "2d", np.float64, "in"),
    ("picrit_aer", "2d", np.float64, "in"),
    ("pnice", "2d", np.float64, "in"),
    ("pfsd", "2d", np.float64, "out"),
    ("pextra", "extra", np.float64, "inout"),
]


def budget_fields_needed(params):
    """PEXTRA fields the budget sections of ``params`` write (cloudsc.F90:3832-4110)."""
    return ((26 if params.lbud23 else 0) + (1 if params.lcldbud_vertint else 0) + (12 if params.lcldbudc else 0) +
            (22 if params.lcldbudl else 0) + (20 if params.lcldbudi else 0) + (13 if params.lcldbudt else 0))


def to_single(arrays):
    """The arrays of the single-precision interface: each real array of
    ``arrays`` (numpy or torch, fields.BATCHED_FIELDS names) rounded to
    float32, the integer arrays as they are."""
    out = {}
    for n, v in arrays.items():
        if n in DTYPE_SP and DTYPE_SP[n] == np.float32:
            out[n] = v.astype(np.float32) if isinstance(v, np.ndarray) else v.float()
        else:
            out[n] = v
    return out


def host_copy_bytes_sp(nproma, klev, ngpblks, ngptot):
    """Bytes per call crossing PCIe in cloudsc_b200_batched_host_sp: those of
    host_copy_bytes with every real element 4 bytes instead of 8."""
    h2d, d2h = host_copy_bytes(nproma, klev, ngpblks, ngptot)
    ints = 2 * 4 * nproma * ngpblks  # LDCUM and KTYPE
    return (h2d - ints) // 2 + ints, d2h // 2
