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
