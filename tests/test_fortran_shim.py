"""The Fortran drop-in module (thesiscode_b200/fortran/PanelVelocityCUDA.f90) against the C ABI it
binds, without a Fortran compiler (neither machine has one): every bind(C) interface names a
function the header declares, with the same number of arguments, passed by value exactly where the
C parameter is a scalar (a C pointer is either a Fortran array or scalar passed by reference, or a
type(c_ptr) passed by value; a pointer to a pointer is a type(c_ptr) passed by reference), with
matching scalar kinds and result type; every procedure is
closed; and the module exports the public names of the reference's PanelVelocityParallelModule
that are on this path."""
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
SHIM = ROOT / "thesiscode_b200" / "fortran" / "PanelVelocityCUDA.f90"
HEADER = ROOT / "include" / "thesiscode_b200.h"

# PanelVelocityParallel.f90:13-20 public names; AdvectionRK4 / DivergentAdvectionRK4 (prescribed
# winds, no Biot-Savart sum) are not on this path
REFERENCE_PUBLIC = {"totalKE", "kineticEnergy", "BVERK4", "StratosphereRK4", "ResetRK4", "ResetArea",
                    "SetSmooth", "GetSmooth", "InitializeMPIRK4", "FinalizeMPIRK4", "LoadBalance"}


def c_prototypes():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(int|const char\*|void)\s+(tc_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", text):
        ret, name, params = m.group(1), m.group(2), m.group(3).strip()
        plist = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
        out[name] = (ret, [("ptrptr" if "**" in p else "ptr" if "*" in p else
                            ("double" if "double" in p else "int")) for p in plist])
    return out


def fortran_interfaces():
    """name -> (result kind, [(arg, by_value, type)]) for each bind(C) function of the interface."""
    src = SHIM.read_text()
    body = src[src.index("interface"):src.index("end interface")]
    # join continuation lines
    body = re.sub(r"&\s*\n\s*", " ", body)
    out = {}
    for m in re.finditer(r"(integer\(c_int\)|type\(c_ptr\))\s+function\s+(\w+)\s*\(([^)]*)\)\s*"
                         r"bind\(C,\s*name=\"(\w+)\"\)(.*?)end function", body, flags=re.S | re.I):
        result, args, cname, decls = m.group(1), m.group(3), m.group(4), m.group(5)
        names = [a.strip() for a in args.split(",") if a.strip()]
        info = {}
        for line in decls.splitlines():
            line = line.strip()
            dm = re.match(r"(integer\(c_int\)|real\(c_double\)|type\(c_ptr\))\s*(,\s*value)?\s*::\s*(.*)", line)
            if not dm:
                continue
            kind, value, rest = dm.group(1), bool(dm.group(2)), dm.group(3)
            for item in re.split(r",\s*(?![^()]*\))", rest):
                nm = item.split("(")[0].strip()
                info[nm] = (value, kind, "(" in item)
        out[cname] = (result, [(n,) + info[n] for n in names])
    return out


def test_every_binding_matches_the_header():
    protos = c_prototypes()
    binds = fortran_interfaces()
    assert len(binds) >= 15
    for cname, (result, args) in binds.items():
        assert cname in protos, f"{cname} is not declared in the header"
        ret, params = protos[cname]
        assert (ret == "int") == (result == "integer(c_int)"), cname
        assert (ret == "const char*") == (result == "type(c_ptr)"), cname
        assert len(args) == len(params), (cname, len(args), len(params))
        for (name, by_value, kind, is_array), ptype in zip(args, params):
            if ptype == "ptrptr":
                # the address of a C pointer: a type(c_ptr) passed by reference
                assert kind == "type(c_ptr)" and not by_value, (cname, name)
            elif ptype == "ptr":
                # a C pointer: c_ptr by value, or an array / scalar by reference
                assert (kind == "type(c_ptr)" and by_value) or (kind != "type(c_ptr)" and not by_value), \
                    (cname, name)
            else:
                assert by_value and not is_array, (cname, name)
                assert kind == ("real(c_double)" if ptype == "double" else "integer(c_int)"), (cname, name)


def test_procedures_are_closed_and_public_names_match_the_reference():
    src = SHIM.read_text()
    code = "\n".join(line.split("!")[0] for line in src.splitlines())
    opened = re.findall(r"^\s*subroutine\s+(\w+)", code, flags=re.M | re.I)
    closed = re.findall(r"^\s*end subroutine", code, flags=re.M | re.I)
    assert len(opened) == len(closed) and len(opened) >= 10
    fn_open = re.findall(r"^\s*function\s+(\w+)", code, flags=re.M | re.I)
    fn_close = [ln for ln in re.findall(r"^\s*end function", code, flags=re.M | re.I)]
    iface = code[code.index("interface"):code.index("end interface")]
    assert len(fn_open) == len(fn_close) - iface.count("end function")
    public = set()
    for line in re.findall(r"^\s*public\s+(.*)$", code, flags=re.M | re.I):
        public |= {w.strip() for w in line.split(",")}
    assert REFERENCE_PUBLIC <= public, REFERENCE_PUBLIC - public
    for name in REFERENCE_PUBLIC - {"totalKE", "kineticEnergy"}:
        assert re.search(rf"^\s*(subroutine|function)\s+{name}\b", code, flags=re.M | re.I), name
    # the sharded step: one MPI_ALLGATHERV per exchange, LoadBalance rows to 0-based ranges
    assert "MPI_ALLGATHERV" in code and "tc_rk4_stage_range" in code
    assert "activePanelsIndexStart(procRank) - 1" in code


def test_dropin_module_translates_and_runs_up_to_the_library():
    """The module goes through the Fortran 90 subset translator (oracle/f90) together with the
    reference's modules it uses; every public procedure exists in the translation. Without a GPU
    its first library call (tc_device_count) fails and CheckStatus stops, as the module is
    written to do; tests/test_fortran_shim_gpu.py runs it on the GPU."""
    import pytest

    from oracle.f90 import reference as REF
    from oracle.f90 import rt

    if not REF.shim_built():
        pytest.skip("the drop-in's translation needs the reference's sources or its build")
    inst = REF.shim_runner().instance(host={"__cdll__": _NoGpuLib()})
    for name in ("bverk4", "stratosphererk4", "initializempirk4", "finalizempirk4", "setsmooth",
                 "getsmooth", "resetrk4", "loadbalance"):
        inst.proc(REF.PVC, name)
    inst.proc(REF.PVC, "setsmooth")(0.07)
    assert inst.proc(REF.PVC, "getsmooth")() == 0.07
    p, _, q = REF.new_grid(inst, 1)
    with pytest.raises(rt.FortranStop):
        inst.proc(REF.PVC, "bverk4")(p, q, 0.01, 0, 1)


class _NoGpuLib:
    """A library whose every call fails, as the real one does on a machine without a GPU."""

    def __getattr__(self, name):
        def f(*args):
            return -2
        return f
