"""The Fortran ISO_C_BINDING module (senga-versiona_b200/fortran/
senga_gpu_mod.f) against the C header it binds (include/senga_gpu.h).

No Fortran compiler exists in this environment, so the module is checked as
text: every BIND(C) type must list the members of its C struct in the same
order, with matching kinds (int <-> INTEGER(C_INT), double <->
REAL(C_DOUBLE)) and extents in reversed order (C [a][b] = Fortran (b,a)); the
C layout those members imply must equal the size of the ctypes mirror the
Python host uses; the PARAMETER bounds must equal the header's SENGA_*
constants; and every interface's BIND(C, NAME=...) must be a function the
header declares and the library exports. The driver glue beside it may only
call functions the module declares."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MOD = os.path.join(ROOT, "senga-versiona_b200", "fortran", "senga_gpu_mod.f")
DRV = os.path.join(ROOT, "senga-versiona_b200", "fortran", "senga_gpu_drv.f")
HDR = os.path.join(ROOT, "include", "senga_gpu.h")

STRUCTS = {"senga_chem": "SENGA_CHEM", "senga_diff": "SENGA_DIFF", "senga_config": "SENGA_CONFIG",
           "senga_radn": "SENGA_RADN", "senga_nscbc": "SENGA_NSCBC", "senga_synth_inflow": "SENGA_SYNTH_INFLOW"}


def _header():
    with open(HDR) as fh:
        text = fh.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    defines = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define\s+(SENGA_\w+)\s+(\d+)\b", text)}
    structs = {}
    for m in re.finditer(r"typedef struct (\w+) \{(.*?)\} \1;", text, flags=re.S):
        members = []
        for decl in m.group(2).split(";"):
            decl = decl.strip()
            if not decl:
                continue
            ctype, rest = decl.split(None, 1)
            for item in rest.split(","):
                item = item.strip()
                name = item.split("[")[0].strip()
                dims = [defines.get(d, None) if not d.isdigit() else int(d) for d in re.findall(r"\[(\w+)\]", item)]
                members.append((name.upper(), ctype, dims))
        structs[m.group(1)] = members
    funcs = set(re.findall(r"^\s*(?:int|const char\*|void\*)\s+(senga_\w+)\s*\(", text, flags=re.M))
    return defines, structs, funcs


def _fortran_lines(path):
    """Statements of a fixed-form file: comments dropped, continuation
    lines (column 6 non-blank) joined."""
    out = []
    with open(path) as fh:
        for line in fh:
            line = line.rstrip("\n")
            if not line.strip() or line[0] in "Cc*!":
                continue
            if len(line) > 5 and line[5] not in " 0" and out:
                out[-1] += " " + line[6:].strip()
            else:
                out.append(line[6:].strip() if len(line) > 6 else line.strip())
    return out


def _module():
    lines = _fortran_lines(MOD)
    params = {}
    for ln in lines:
        m = re.match(r"INTEGER, PARAMETER :: (.*)", ln)
        if m:
            for a in m.group(1).split(","):
                k, v = a.split("=")
                params[k.strip()] = int(v)
    types, cur = {}, None
    for ln in lines:
        m = re.match(r"TYPE, BIND\(C\) :: (\w+)", ln)
        if m:
            cur = m.group(1)
            types[cur] = []
            continue
        if ln.startswith("END TYPE"):
            cur = None
            continue
        if cur:
            m = re.match(r"(INTEGER\(C_INT\)|REAL\(C_DOUBLE\)) :: (.*)", ln)
            assert m, ln
            kind = "int" if m.group(1).startswith("INTEGER") else "double"
            for name, dims in re.findall(r"(\w+)(?:\(([^)]*)\))?", m.group(2)):
                ds = [params[d.strip()] if d.strip() in params else int(d) for d in dims.split(",")] if dims else []
                types[cur].append((name, kind, ds))
    binds = re.findall(r"BIND\(C, NAME='(\w+)'\)", " ".join(lines))
    funcs = re.findall(r"FUNCTION (\w+)\(", " ".join(lines))
    return params, types, binds, funcs


def _c_size(members):
    off, align = 0, 1
    for _, kind, dims in members:
        sz = 4 if kind == "int" else 8
        align = max(align, sz)
        off = (off + sz - 1) // sz * sz
        n = 1
        for d in dims:
            n *= d
        off += sz * n
    return (off + align - 1) // align * align


def test_parameters_equal_header_constants():
    defines, _, _ = _header()
    params, _, _, _ = _module()
    pairs = {"SNSPCM": "SENGA_NSPCMX", "SNSTPM": "SENGA_NSTPMX", "SNSPIM": "SENGA_NSPIMX", "SNTINM": "SENGA_NTINMX", "SNCOFM": "SENGA_NCOFMX",
             "SNSSMX": "SENGA_NSSMAX", "SNBDYM": "SENGA_NBDYMX", "SNLLMX": "SENGA_NLLMAX", "SNDCFM": "SENGA_NDCFMX",
             "SNCFRM": "SENGA_NCFRMX", "SNOBC": "SENGA_NOBC", "SNBOUN": "SENGA_NBOUND", "SNPERI": "SENGA_NPERI"}
    for f, c in pairs.items():
        assert params[f] == defines[c], (f, c)


@pytest.mark.parametrize("cname", sorted(STRUCTS))
def test_bind_c_types_mirror_the_header_structs(cname):
    _, structs, _ = _header()
    _, types, _, _ = _module()
    cm = structs[cname]
    fm = types[STRUCTS[cname]]
    assert [m[0] for m in fm] == [m[0] for m in cm], "member order"
    for (fn, fk, fd), (cn, ck, cd) in zip(fm, cm):
        assert fk == ck, f"{cname}.{cn}: kind"
        assert fd == cd[::-1], f"{cname}.{cn}: extents {fd} vs C {cd}"


@pytest.mark.parametrize("cname", sorted(STRUCTS))
def test_bind_c_layout_equals_the_ctypes_mirror(cname):
    import senga

    mirror = {"senga_chem": senga.ChemT, "senga_diff": senga.DiffT, "senga_config": senga.ConfigT,
              "senga_nscbc": senga.NscbcT, "senga_radn": senga.RadnT, "senga_synth_inflow": senga.SynthT}[cname]
    _, types, _, _ = _module()
    assert _c_size(types[STRUCTS[cname]]) == C.sizeof(mirror)


def test_interfaces_bind_declared_and_exported_functions():
    import senga

    _, _, header_funcs = _header()
    _, _, binds, _ = _module()
    assert len(binds) >= 15
    for name in binds:
        assert name in header_funcs, f"{name} not declared in include/senga_gpu.h"
        assert hasattr(senga.lib, name), f"{name} not exported by libsenga_gpu.so"


def test_driver_glue_calls_only_module_functions():
    _, _, _, funcs = _module()
    text = " ".join(_fortran_lines(DRV))
    called = set(re.findall(r"\b(SENGA_\w+)\(", text)) - set(STRUCTS.values())
    assert called, "no library calls found"
    assert called <= set(funcs), called - set(funcs)
