"""The Fortran side of the boundary, include/cloudsc_b200_mod.F90, checked
mechanically against the C header (no Fortran compiler exists in the build
image, so the module is parsed): the BIND(C) derived types field for field
(names, order, kinds, array lengths) against the header's structs and the
ctypes mirrors' offsets, and every BIND(C) interface argument for argument
(names, order, by-value or by-reference, kind, INTENT against const)
against its C prototype.  CLOUDSC_B200_BLOCK's arguments are also checked
against the dummy-argument list of SUBROUTINE CLOUDSC (cloudsc.F90:14-44),
with the seven derived types collapsed into P."""
import ctypes
import os
import re

import pytest

from openifs_b200 import params as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MOD = os.path.join(ROOT, "include", "cloudsc_b200_mod.F90")
HDR = os.path.join(ROOT, "include", "cloudsc_b200.h")

# SUBROUTINE CLOUDSC's dummy arguments in order (cloudsc.F90:14-44)
CSC_ARGS = """YDECLDP YDECUMF YDEPHLI YDERAD YDEPHY YDVDF YDSPP_CONFIG KIDIA KFDIA KLON KLEV LDDIAG
PTSPHY PT PQ PTENDENCY_CML_T PTENDENCY_CML_Q PTENDENCY_CML_A PTENDENCY_CML_CLD PTENDENCY_LOC_T
PTENDENCY_LOC_Q PTENDENCY_LOC_A PTENDENCY_LOC_CLD PVFA PVFL PVFI PDYNA PDYNL PDYNI PDYNR PDYNS
PHRSW PHRLW PVERVEL PAP PAPH PGEOM PLSM PGAW LDCUM KCTOP KTYPE KPBLTYPE PEIS PLU PLUDE PLUDELI
PSNDE PMFU PMFD PGP2DSPP LDSLPHY PA PCLV PLCRIT_AER PICRIT_AER PRE_ICE PCCN PNICE PCOVPTOT PFSD
PRAINFRAC_TOPRFZ PFSQLF PFSQIF PFCQNNG PFCQLNG PFSQRF PFSQSF PFCQRNG PFCQSNG PFSQLTUR PFSQITUR
PFPLSL PFPLSN PFHPSL PFHPSN PEXTRA KFLDX""".split()


# ---------------------------------------------------------------- Fortran side
def fortran_statements(path=None):
    """Statements of the module: comments removed, continuation lines joined."""
    out, cur = [], ""
    for raw in open(path or MOD):
        line = raw.split("!", 1)[0].rstrip() if "'" not in raw else raw.rstrip()
        if "'" in line and "!" in line:  # a comment after a quoted NAME='...'
            q = line.rfind("'")
            bang = line.find("!", q)
            line = line if bang < 0 else line[:bang].rstrip()
        s = line.strip()
        if not s:
            continue
        if s.startswith("&"):
            s = s[1:].strip()
        if cur:
            cur += " " + s
        else:
            cur = s
        if cur.endswith("&"):
            cur = cur[:-1].rstrip()
            continue
        out.append(cur)
        cur = ""
    return out


def parse_decl(stmt):
    """'KIND, ATTR :: A, B(*), C(8)' -> (kind, attrs, [(name, dim)])."""
    spec, names = stmt.split("::", 1)
    parts = [p.strip() for p in re.split(r",(?![^()]*\))", spec)]
    kind, attrs = parts[0].replace(" ", "").upper(), [a.upper().replace(" ", "") for a in parts[1:]]
    out = []
    for n in re.split(r",(?![^()]*\))", names):
        m = re.fullmatch(r"\s*(\w+)\s*(?:\(([^)]*)\))?\s*", n)
        out.append((m.group(1).upper(), m.group(2)))
    return kind, attrs, out


def fortran_module(path=None):
    st = fortran_statements(path)
    types, funcs, i = {}, {}, 0
    while i < len(st):
        s = st[i]
        m = re.match(r"TYPE\s*,\s*BIND\(C\)\s*::\s*(\w+)", s, re.I)
        if m:
            name, fields = m.group(1).upper(), []
            i += 1
            while not re.match(r"END\s+TYPE", st[i], re.I):
                kind, _, names = parse_decl(st[i])
                fields += [(n, kind, d) for n, d in names]
                i += 1
            types[name] = fields
        m = re.match(r"(.*?)\bFUNCTION\s+(\w+)\s*\(([^)]*)\)\s*BIND\(C\s*,\s*NAME\s*=\s*'(\w+)'\)", s, re.I)
        if m:
            ret = m.group(1).strip().replace(" ", "").upper()
            args = [a.strip().upper() for a in m.group(3).split(",") if a.strip()]
            decls = {}
            i += 1
            while not re.match(r"END\s+FUNCTION", st[i], re.I):
                if "::" in st[i]:
                    kind, attrs, names = parse_decl(st[i])
                    for n, d in names:
                        decls[n] = (kind, attrs, d)
                i += 1
            funcs[m.group(4)] = {"ret": ret, "args": args, "decls": decls, "fname": m.group(2).upper()}
        i += 1
    return types, funcs


# ---------------------------------------------------------------------- C side
def header_text():
    t = open(HDR).read()
    t = re.sub(r"/\*.*?\*/", "", t, flags=re.S)
    return re.sub(r"//[^\n]*", "", t)


def c_struct(name):
    t = header_text()
    body = t[t.index(f"typedef struct {name} {{") + len(f"typedef struct {name} {{"):t.index(f"}} {name};")]
    fields = []
    for stmt in body.split(";"):
        stmt = stmt.strip()
        if not stmt:
            continue
        m = re.match(r"((?:const\s+)?\w+)\s*(.*)", stmt, re.S)
        typ, rest = m.group(1), m.group(2)
        for n in rest.split(","):
            n = n.strip()
            ptr = n.startswith("*")
            n = n.lstrip("*").strip()
            dm = re.fullmatch(r"(\w+)\[(\d+)\]", n)
            fields.append((dm.group(1) if dm else n, typ, ptr, dm.group(2) if dm else None))
    return fields


def c_prototypes():
    t = header_text()
    out = {}
    for m in re.finditer(r"(int|size_t|int32_t|const char\s*\*)\s*(cloudsc_b200_\w+)\s*\(([^;{]*?)\)\s*;", t, re.S):
        args = []
        body = " ".join(m.group(3).split())
        if body and body != "void":
            for a in body.split(","):
                a = a.strip()
                am = re.fullmatch(r"(const\s+)?(\w+)\s*(\*?)\s*(\w+)", a)
                assert am, a
                args.append({"const": bool(am.group(1)), "type": am.group(2), "ptr": bool(am.group(3)),
                             "name": am.group(4).upper()})
        out[m.group(2)] = {"ret": " ".join(m.group(1).split()), "args": args}
    return out


KIND_OF = {"double": "REAL(C_DOUBLE)", "int32_t": "INTEGER(C_INT32_T)", "uint32_t": "INTEGER(C_INT32_T)"}
STRUCT_TYPES = {"cloudsc_params": "TYPE(CLOUDSC_PARAMS)", "cloudsc_state": "TYPE(CLOUDSC_STATE)",
                "cloudsc_increments": "TYPE(CLOUDSC_INCREMENTS)"}


@pytest.fixture(scope="module")
def mod():
    return fortran_module()


def test_params_type_matches_header_and_ctypes(mod):
    types, _ = mod
    f = types["CLOUDSC_PARAMS"]
    c = c_struct("cloudsc_params")
    assert [n for n, *_ in f] == [n.upper() for n, *_ in c]
    for (fn, fkind, fdim), (cn, ctyp, ptr, cdim) in zip(f, c):
        assert not ptr
        assert fkind == KIND_OF[ctyp], (fn, fkind, ctyp)
        assert (fdim or None) == cdim, (fn, fdim, cdim)
    # the ctypes mirror has the same fields in the same order
    assert [n.upper() for n, _ in P.CloudscParams._fields_] == [n for n, *_ in f]


@pytest.mark.parametrize("ftype,cname,mirror", [("CLOUDSC_STATE", "cloudsc_state", P.CloudscState),
                                                ("CLOUDSC_INCREMENTS", "cloudsc_increments", P.CloudscIncrements)])
def test_state_types_match_header(mod, ftype, cname, mirror):
    types, _ = mod
    f, c = types[ftype], c_struct(cname)
    assert [n for n, *_ in f] == [n.upper() for n, *_ in c]
    for (fn, fkind, _), (cn, ctyp, ptr, _) in zip(f, c):
        assert fkind == ("TYPE(C_PTR)" if ptr else KIND_OF[ctyp]), (fn, fkind, ctyp)
    assert [n.upper() for n, _ in mirror._fields_] == [n for n, *_ in f]
    assert ctypes.sizeof(mirror) == (8 * sum(1 for *_, p, _ in c if p) + 4 * sum(1 for *_, p, _ in c if not p) + 7) // 8 * 8


def test_every_interface_matches_its_prototype(mod):
    _, funcs = mod
    protos = c_prototypes()
    assert len(funcs) >= 8
    for cname, fn in funcs.items():
        assert cname in protos, cname
        pr = protos[cname]
        assert fn["args"] == [a["name"] for a in pr["args"]], cname
        want_ret = {"int": "INTEGER(C_INT)", "const char *": "TYPE(C_PTR)"}[pr["ret"]]
        assert fn["ret"] == want_ret, (cname, fn["ret"])
        for a in pr["args"]:
            kind, attrs, dim = fn["decls"][a["name"]]
            where = (cname, a["name"])
            if a["type"] == "void":
                assert a["ptr"] and kind == "TYPE(C_PTR)" and "VALUE" in attrs, where
            elif a["type"] in STRUCT_TYPES:
                assert a["ptr"] and kind == STRUCT_TYPES[a["type"]] and "VALUE" not in attrs, where
                assert ("INTENT(IN)" in attrs) == a["const"], where
            elif a["ptr"]:
                assert kind == KIND_OF[a["type"]] and dim == "*" and "VALUE" not in attrs, where
                assert ("INTENT(IN)" in attrs) == a["const"], where
            else:
                assert kind == KIND_OF[a["type"]] and "VALUE" in attrs and dim is None, where


def test_block_interface_is_cloudsc_argument_list(mod):
    _, funcs = mod
    args = funcs["cloudsc_b200_block"]["args"]
    assert args == ["P"] + CSC_ARGS[7:]
    assert funcs["cloudsc_b200_block"]["fname"] == "CLOUDSC_B200_BLOCK"


def test_key_constants_match_header(mod):
    text = open(MOD).read()
    hdr = header_text()
    for name in ("Q", "O3", "A", "TKE", "QL", "QI", "QR", "QS"):
        c = int(re.search(rf"#define CLOUDSC_KEY_{name}\s+0x([0-9a-fA-F]+)u", hdr).group(1), 16)
        f = int(re.search(rf"CLOUDSC_KEY_{name}\s*=\s*(\d+)", text).group(1))
        assert c == f == getattr(P, f"KEY_{name}"), name
