"""The Julia package extension (ext/FEMToolsB200Ext.jl) against the C header.

Julia is not installed here, so the extension is checked as text: every isbits
struct it passes to `ccall` must list the fields of its C counterpart in
include/femtools_b200.h in the same order with the same types and array lengths
(Julia lays isbits structs out with the C alignment rules, so equal field lists
give equal layouts), and every library symbol it calls must be declared there.
"""
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "femtools_b200.h")
EXT = os.path.join(ROOT, "ext", "FEMToolsB200Ext.jl")

MIRRORS = {
    "StokesMaterialC": "femb200_stokes_material",
    "StokesProblemC": "femb200_stokes_problem",
    "StokesControlsC": "femb200_stokes_controls",
    "StokesStatsC": "femb200_stokes_stats",
    "ThermalProblemC": "femb200_thermal_problem",
    "ThermalControlsC": "femb200_thermal_controls",
    "ThermalStatsC": "femb200_thermal_stats",
}


def c_structs():
    """{struct name: [(field, kind, count)]} from the header; kind is i32, i64, f64,
    ptr or the name of a nested struct."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    text = text.replace("FEMB200_MAX_PHASES", "16")
    out = {}
    for body, name in re.findall(r"typedef struct \w+ \{(.*?)\} (\w+);", text, re.S):
        fields = []
        for decl in (d.strip() for d in body.split(";")):
            if not decl:
                continue
            m = re.match(r"((?:const\s+)?[\w]+)\s*(.*)", decl, re.S)
            base, rest = m.group(1).replace("const ", "").strip(), m.group(2)
            for item in (x.strip() for x in rest.split(",")):
                im = re.match(r"(\**)\s*(?:const\s+)?(\w+)\s*(?:\[(\d+)\])?$", item)
                assert im, (name, item)
                stars, fname, n = im.groups()
                if stars:
                    kind = "ptr"
                else:
                    kind = {"int32_t": "i32", "int64_t": "i64", "double": "f64"}.get(base, base)
                fields.append((fname, kind, int(n) if n else 1))
        out[name] = fields
    return out


def julia_structs():
    text = open(EXT).read()
    out = {}
    for name, body in re.findall(r"^struct (\w+)[^\n]*\n(.*?)^end", text, re.S | re.M):
        fields = []
        for line in body.splitlines():
            line = line.split("#")[0].strip()
            if not line:
                continue
            fname, typ = (s.strip() for s in line.split("::", 1))
            n = 1
            tm = re.match(r"NTuple\{(\d+),\s*(.+)\}$", typ)
            if tm:
                n, typ = int(tm.group(1)), tm.group(2).strip()
            if typ.startswith("Ptr{"):
                kind = "ptr"
            else:
                kind = {"Int32": "i32", "Int64": "i64", "Float64": "f64"}.get(typ, MIRRORS.get(typ, typ))
            fields.append((fname, kind, n))
        out[name] = fields
    return out


def test_every_mirror_matches_its_c_struct_field_for_field():
    c, jl = c_structs(), julia_structs()
    for jname, cname in MIRRORS.items():
        assert jname in jl, jname
        assert jl[jname] == c[cname], (jname, [x for x in zip(jl[jname], c[cname]) if x[0] != x[1]])


def test_every_called_symbol_is_declared_in_the_header():
    header = open(HEADER).read()
    called = set(re.findall(r"ccall\(\(:(\w+),", open(EXT).read()))
    assert {"femb200_create", "femb200_destroy", "femb200_set_stream", "femb200_last_error",
            "femb200_solve_stokes", "femb200_solve_thermal", "femb200_solve_coupled"} <= called
    for sym in called:
        assert re.search(rf"\b{sym}\s*\(", header), sym


def test_enumerations_match_the_header():
    header = open(HEADER).read()
    ext = open(EXT).read()
    pairs = {"F64": "FEMB200_F64", "F32": "FEMB200_F32", "PHASE_NODAL": "FEMB200_PHASE_NODAL",
             "PHASE_CELL": "FEMB200_PHASE_CELL", "PHASE_ELEMENT_NODE": "FEMB200_PHASE_ELEMENT_NODE",
             "FIELD_NONE": "FEMB200_FIELD_NONE", "FIELD_IP": "FEMB200_FIELD_IP", "FIELD_NODAL": "FEMB200_FIELD_NODAL",
             "PRECISION_FP64": "FEMB200_PRECISION_FP64", "PRECISION_MIXED": "FEMB200_PRECISION_MIXED"}
    c_vals = {k: int(v) for k, v in re.findall(r"(FEMB200_\w+)\s*=\s*(\d+)", header)}
    jl_vals = {}
    for names, vals in re.findall(r"^const ([\w, ]+) = ((?:Int32\(\d+\)(?:, )?)+)$", ext, re.M):
        for n, v in zip(names.split(", "), re.findall(r"Int32\((\d+)\)", vals)):
            jl_vals[n] = int(v)
    for jn, cn in pairs.items():
        assert jl_vals[jn] == c_vals[cn], jn
    assert "const MAX_PHASES = 16" in ext and "#define FEMB200_MAX_PHASES 16" in header
