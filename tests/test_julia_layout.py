"""The Julia binding's C structs against the C header (CPU).

Julia lays out an isbits `struct` exactly as C does, so a binding struct
whose fields have the header struct's order and types has its size and
offsets.  Julia is not installed here, so this test reads both files as text:
every `struct C…` of julia/HPRSOCPB200.jl that stands for a header struct
must list the same fields, in the same order, with the matching types.  A
slip here would be silent memory corruption inside ccall.
"""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hprsocp_b200.h")
JULIA = os.path.join(ROOT, "hpr-socp_b200", "julia", "HPRSOCPB200.jl")

# Julia struct -> C struct
PAIRS = {"CCSR": "hpr_csr", "CProblem": "hpr_problem", "CParams": "hpr_params", "CResiduals": "hpr_residuals",
         "CResults": "hpr_results", "CCbfData": "hpr_cbf_data"}

# C field type -> Julia field type
SCALARS = {"int64_t": "Int64", "int32_t": "Int32", "int": "Int32", "double": "Float64", "size_t": "UInt64",
           "char": "UInt8"}


def c_structs():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    out = {}
    for m in re.finditer(r"typedef\s+struct\s+(\w+)\s*\{(.*?)\}\s*(\w+)\s*;", text, flags=re.S):
        fields = []
        for decl in m.group(2).split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            decl = decl.replace("const ", "")
            mm = re.fullmatch(r"(\w+)\s*(\*?\s*\w.*)", decl)
            assert mm, f"unparsed C field: {decl!r}"
            for name in mm.group(2).split(","):  # `double a, b;` declares two fields
                nm = re.fullmatch(r"\s*(\*?)\s*(\w+)\s*", name)
                assert nm, f"unparsed C field: {decl!r}"
                fields.append((nm.group(2), mm.group(1), bool(nm.group(1))))
        out[m.group(3)] = fields
    return out


def julia_structs():
    text = open(JULIA).read()
    out = {}
    for m in re.finditer(r"^(?:mutable\s+)?struct\s+(\w+)\s*\n(.*?)^end", text, flags=re.S | re.M):
        fields = []
        for line in m.group(2).splitlines():
            line = line.split("#")[0].strip()
            if "::" in line:
                name, typ = line.split("::", 1)
                fields.append((name.strip(), typ.strip()))
        out[m.group(1)] = fields
    return out


def julia_type_of(ctype, ptr):
    if ctype in PAIRS.values():
        assert not ptr
        return {v: k for k, v in PAIRS.items()}[ctype]
    base = SCALARS[ctype]
    return f"Ptr{{{base}}}" if ptr else base


def test_every_binding_struct_matches_the_header():
    cs, js = c_structs(), julia_structs()
    for jname, cname in PAIRS.items():
        assert jname in js, f"{jname} missing from the Julia binding"
        assert cname in cs, f"{cname} missing from the header"
        cf, jf = cs[cname], js[jname]
        assert [n for n, _, _ in cf] == [n for n, _ in jf], (jname, [n for n, _, _ in cf], [n for n, _ in jf])
        for (n, ct, ptr), (_, jt) in zip(cf, jf):
            assert julia_type_of(ct, ptr) == jt, (jname, n, ct, ptr, jt)


def test_the_parser_sees_the_structs():
    # guards the test itself against a regex that matches nothing
    cs, js = c_structs(), julia_structs()
    assert len(cs["hpr_params"]) >= 20 and len(js["CParams"]) == len(cs["hpr_params"])
    assert len(cs["hpr_results"]) >= 20 and js["CResults"][15] == ("last", "CResiduals")
