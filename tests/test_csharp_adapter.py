"""The C# adapter sources (celestial-mechanics-desktop_b200/csharp/) against
the C ABI they bind: every nb_* entry point of include/nbody_b200.h has one
DllImport with the same name, the same number of arguments and matching
types, and every constant the adapter defines has the header's value.  No
.NET toolchain exists here, so the check is textual.  CPU only."""
from __future__ import annotations

import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "nbody_b200.h"
CS_DIR = ROOT / "celestial-mechanics-desktop_b200" / "csharp"

# C type -> accepted C# spellings (P/Invoke blittable equivalents)
C_TO_CS = {
    "int32_t": {"int"}, "int32_t*": {"int*"}, "int64_t*": {"long*"},
    "uint64_t": {"ulong"}, "uint64_t*": {"ulong*"}, "uint8_t*": {"byte*"},
    "double": {"double"}, "double*": {"double*"}, "float*": {"float*"},
    "void*": {"IntPtr"}, "nb_engine*": {"IntPtr"}, "nb_ensemble*": {"IntPtr"},
    "nb_engine**": {"out IntPtr"}, "nb_ensemble**": {"out IntPtr"},
    "const char*": {"IntPtr"},
}


def _norm_c(t: str) -> str:
    t = " ".join(t.replace("*", " * ").split())
    t = t.replace(" *", "*")
    if t.startswith("const ") and t != "const char*":
        t = t[len("const "):]
    return t


def header_functions() -> dict:
    h = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    out = {}
    for m in re.finditer(r"NB_API\s+([\w\s\*]+?)\s*(\w+)\s*\(([^)]*)\)\s*;", h):
        ret, name, params = m.groups()
        ret = _norm_c(ret.strip())
        args = []
        params = " ".join(params.split())
        if params and params != "void":
            for p in params.split(","):
                p = p.strip()
                typ = re.sub(r"\w+$", "", p).strip()  # drop the parameter name
                args.append(_norm_c(typ))
        out[name] = (ret, args)
    return out


def cs_imports() -> dict:
    src = (CS_DIR / "B200Native.cs").read_text()
    src = re.sub(r"//[^\n]*", "", src)
    out = {}
    for m in re.finditer(r"\[DllImport\(Lib\)\]\s*public static extern\s+([\w\*]+)\s+(\w+)\s*"
                         r"\(([^)]*)\)\s*;", src, flags=re.S):
        ret, name, params = m.groups()
        assert name not in out, f"duplicate DllImport {name}"
        args = []
        params = " ".join(params.split())
        if params:
            for p in params.split(","):
                words = p.strip().split()
                args.append(" ".join(words[:-1]))  # drop the parameter name
        out[name] = (ret, args)
    return out


def test_every_entry_point_has_a_matching_dllimport():
    hf, cs = header_functions(), cs_imports()
    assert len(hf) >= 50
    assert set(hf) == set(cs), (sorted(set(hf) - set(cs)), sorted(set(cs) - set(hf)))
    for name, (ret, args) in hf.items():
        cret, cargs = cs[name]
        assert cret in C_TO_CS[ret], (name, ret, cret)
        assert len(cargs) == len(args), (name, args, cargs)
        for k, (a, c) in enumerate(zip(args, cargs)):
            assert c in C_TO_CS[a], (name, k, a, c)


def _header_values() -> dict:
    h = HEADER.read_text()
    vals = {}
    for m in re.finditer(r"#define\s+(NB_\w+)\s+(0x[0-9A-Fa-f]+|\d+)", h):
        vals[m.group(1)] = int(m.group(2), 0)
    for m in re.finditer(r"(NB_\w+)\s*=\s*(-?\d+)", h):
        vals[m.group(1)] = int(m.group(2))
    return vals


def _camel(name: str, prefix: str) -> str:
    return "".join(w.capitalize() for w in name[len(prefix):].lower().split("_"))


@pytest.mark.parametrize("prefix,cs_prefix", [
    ("NB_MODE_", "Mode"), ("NB_FLAG_", "Flag"), ("NB_PARAM_", "Param"), ("NB_T_", "T"),
    ("NB_C_", "C"), ("NB_ERR_", "Err")])
def test_constants_equal_the_header(prefix, cs_prefix):
    src = (CS_DIR / "B200Native.cs").read_text()
    cs = {m.group(1): int(m.group(2), 0)
          for m in re.finditer(r"\b([A-Z]\w*)\s*=\s*(-?0x[0-9A-Fa-f]+|-?\d+)", src)}
    hv = {k: v for k, v in _header_values().items() if k.startswith(prefix)}
    if prefix == "NB_MODE_":
        hv.pop("NB_MODE_MASK", None)
    assert hv
    for k, v in hv.items():
        name = cs_prefix + _camel(k, prefix)
        assert cs.get(name) == v, (k, name, cs.get(name), v)


def test_adapter_uses_only_bound_entry_points():
    """The backend, integrator and selection classes call nb_* functions
    that B200Native declares, and implement the app's interfaces."""
    cs = cs_imports()
    for f in ("B200PhysicsBackend.cs", "B200SoAIntegrator.cs", "B200BackendSelection.cs"):
        src = (CS_DIR / f).read_text()
        for name in re.findall(r"B200Native\.(nb_\w+)", src):
            assert name in cs, (f, name)
    backend = (CS_DIR / "B200PhysicsBackend.cs").read_text()
    assert re.search(r"class B200PhysicsBackend\s*:\s*IPhysicsComputeBackend,\s*"
                     r"IGravityModelAwareBackend", backend)
    for prop in ("EnableShellTheorem", "Theta", "LastBuildTimeMs", "LastTraversalTimeMs",
                 "LastTotalTimeMs"):
        assert re.search(rf"public \w+ {prop} \{{", backend), prop
    assert "public void ComputeForces(BodySoA bodies, double softening)" in backend
    integ = (CS_DIR / "B200SoAIntegrator.cs").read_text()
    assert re.search(r"class B200SoAIntegrator\s*:\s*ISoAIntegrator", integ)
    assert ("public void Step(BodySoA bodies, IPhysicsComputeBackend backend, double softening, "
            "double dt)") in integ
