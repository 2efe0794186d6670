"""ctypes mirror of ``cloudsc_params`` (include/cloudsc_b200.h).

The structure is built by parsing the public header, so the Python view and
the C ABI cannot drift apart; ``tests/test_abi.py`` also checks its size
against ``cloudsc_b200_params_size()``.  The fields are the scalars CLOUDSC
reads through its ASSOCIATE block (ifs-source/arpifs/phys_ec/cloudsc.F90:612-682).
"""
import ctypes
import os
import re

_HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                    "include", "cloudsc_b200.h")
_CTYPES = {"double": ctypes.c_double, "int32_t": ctypes.c_int32, "uint32_t": ctypes.c_uint32}

PARAMS_MAGIC = 0x434C4453


def _parse_fields(path=_HDR):
    text = open(path).read()
    body = text[text.index("typedef struct cloudsc_params {") + len("typedef struct cloudsc_params {"):
                text.index("} cloudsc_params;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    body = re.sub(r"//[^\n]*", "", body)
    fields = []
    for stmt in body.split(";"):
        stmt = stmt.strip()
        if not stmt:
            continue
        typ, rest = stmt.split(None, 1)
        for name in rest.split(","):
            name = name.strip()
            m = re.fullmatch(r"(\w+)\[(\d+)\]", name)
            if m:  # a one-dimensional array member
                fields.append((m.group(1), _CTYPES[typ] * int(m.group(2))))
            else:
                fields.append((name, _CTYPES[typ]))
    return fields


class CloudscParams(ctypes.Structure):
    _fields_ = _parse_fields()

    def as_dict(self):
        out = {}
        for n, _ in self._fields_:
            v = getattr(self, n)
            out[n] = list(v) if isinstance(v, ctypes.Array) else v
        return out

    def copy(self):
        c = CloudscParams()
        ctypes.memmove(ctypes.byref(c), ctypes.byref(self), ctypes.sizeof(self))
        return c

    def tobytes(self):
        return bytes(memoryview(self).cast("B"))


# Species index order of the (KLON,KLEV,NCLV) arrays (yoecldp.F90:102-107).
NCLV = 5
NCLDQL, NCLDQI, NCLDQR, NCLDQS, NCLDQV = 1, 2, 3, 4, 5


# STATE_INCREMENT (state_increment.F90): the state's KEYMASK switches as the
# CLOUDSC_KEY_* bits of include/cloudsc_b200.h, and ctypes mirrors of
# cloudsc_state / cloudsc_increments.
KEY_Q, KEY_O3, KEY_A, KEY_TKE, KEY_QL, KEY_QI, KEY_QR, KEY_QS = 0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x40, 0x80
KEY_ALL = 0xFF
STATE_FIELDS = ("u", "v", "t", "o3", "q", "a", "cld", "tke")
INCREMENT_FIELDS = ("u", "v", "t", "o3", "q", "a", "ql", "qi", "qr", "qs", "tke")


class CloudscState(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in STATE_FIELDS] + [("keymask", ctypes.c_uint32),
                                                                ("nclv", ctypes.c_int32)]


class CloudscIncrements(ctypes.Structure):
    _fields_ = [("pa_" + n, ctypes.c_void_p) for n in INCREMENT_FIELDS] + [("nclv_pa", ctypes.c_int32)]


def make_state(state, keymask, ptr):
    """cloudsc_state from a dict of the state's arrays (keys of STATE_FIELDS;
    CLD shaped (NGPBLKS, NCLV, KLEV, NPROMA)); ``ptr`` gives an array's
    address."""
    s = CloudscState()
    for n in STATE_FIELDS:
        x = state.get(n)
        setattr(s, n, None if x is None else ptr(x))
    s.keymask = int(keymask)
    cld = state.get("cld")
    s.nclv = 0 if cld is None else int(cld.shape[1])
    return s


def make_increments(inc, ptr, species_stride):
    """cloudsc_increments from a dict of increments (keys of
    INCREMENT_FIELDS), or with key "cld" a (NGPBLKS, N, KLEV, NPROMA) array
    whose first four species give PA_QL..PA_QS; ``species_stride(x, m)`` is
    the address of species m of such an array."""
    c = CloudscIncrements()
    for n in INCREMENT_FIELDS:
        x = inc.get(n)
        setattr(c, "pa_" + n, None if x is None else ptr(x))
    c.nclv_pa = 0
    cld = inc.get("cld")
    if cld is not None:
        for m, n in enumerate(("ql", "qi", "qr", "qs")):
            if n in inc:
                raise ValueError(f"give {n} either alone or through cld, not both")
            setattr(c, "pa_" + n, species_stride(cld, m))
        c.nclv_pa = int(cld.shape[1])
    return c
