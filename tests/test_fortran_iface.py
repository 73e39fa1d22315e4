"""The iso_c_binding module for IMPACT-Z's Fortran driver
(impact-z_b200/fortran/impz_iface.f90) against include/impz_b200.h, read as
text (no Fortran compiler here): every interface binds an entry point the
header declares and the library exports, with the header's number of
arguments, and each argument is passed the way the C prototype takes it
(by value for a scalar, by reference for a pointer, c_ptr by value for an
opaque handle or a device address).  No GPU needed."""
import os
import re

from conftest import ROOT, load_impz

impz = load_impz()

FORTRAN = os.path.join(ROOT, "impact-z_b200", "fortran", "impz_iface.f90")
HEADER = os.path.join(ROOT, "include", "impz_b200.h")


def _strip_comments(txt):
    return "\n".join(line.split("!")[0] for line in txt.splitlines())


def fortran_interfaces():
    """{bind name: (dummy names in order, {name: (type, value?)}, result type)}."""
    txt = _strip_comments(open(FORTRAN).read())
    txt = re.sub(r"&\s*\n\s*", " ", txt)  # join continuation lines
    out = {}
    pat = re.compile(
        r"^\s*(integer\(c_int\)|integer\(c_long_long\)|type\(c_ptr\)|real\(c_double\))\s+"
        r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)(.*?)end function",
        re.M | re.S)
    for m in pat.finditer(txt):
        result, fname, args, bname, body = m.groups()
        assert fname == bname, (fname, bname)
        names = [a.strip().lower() for a in args.split(",") if a.strip()]
        decl = {}
        for line in body.splitlines():
            if "::" not in line or line.strip().startswith("import"):
                continue
            spec, vars_ = line.split("::")
            base = spec.split(",")[0].strip().lower()
            byval = "value" in spec.lower()
            for v in re.split(r",(?![^(]*\))", vars_):
                v = v.strip().lower()
                if v:
                    decl[re.sub(r"\(.*", "", v)] = (base, byval)
        out[bname] = (names, decl, result)
    return out


def header_prototypes():
    """{name: (return type, [parameter declarations])}."""
    txt = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    txt = "\n".join(line for line in txt.splitlines() if not line.lstrip().startswith("#"))
    out = {}
    for m in re.finditer(r"([\w\s\*]+?)\b(impz_\w+)\s*\(([^;{]*?)\)\s*;", txt):
        ret, name, params = m.groups()
        ps = [p.strip() for p in params.split(",")] if params.strip() not in ("", "void") else []
        out[name] = (" ".join(ret.split()), ps)
    return out


def c_kind(param):
    """How a C parameter is passed: ('ptr',) or ('val', scalar type)."""
    p = " ".join(param.split())
    if "*" in p or "[" in p or p.startswith("impz_bunch_t "):
        return ("ptr",)
    if p.startswith("long long"):
        return ("val", "integer(c_long_long)")
    if p.startswith("double"):
        return ("val", "real(c_double)")
    if p.startswith("int"):
        return ("val", "integer(c_int)")
    raise AssertionError("unclassified C parameter: " + param)


def test_every_interface_binds_a_declared_exported_symbol():
    ifs = fortran_interfaces()
    protos = header_prototypes()
    L = impz.lib()
    assert len(ifs) >= 30
    for name in ifs:
        assert name in protos, name
        assert hasattr(L, name), name


def test_the_driver_facing_entry_points_are_bound():
    ifs = fortran_interfaces()
    for name in ("impz_bunch_create", "impz_run", "impz_map_half", "impz_sc_prepare",
                 "impz_deposit", "impz_poisson_open", "impz_kick", "impz_moments",
                 "impz_wake_set", "impz_set_integrator", "impz_laser_heater",
                 "impz_bunch_geom", "impz_bunch_set_z", "impz_bunch_upload",
                 "impz_run_reference", "impz_error_string", "impz_deposit_static"):
        assert name in ifs, name


def test_arguments_are_passed_as_the_prototypes_take_them():
    ifs = fortran_interfaces()
    protos = header_prototypes()
    for name, (names, decl, result) in ifs.items():
        ret, params = protos[name]
        assert len(names) == len(params), (name, names, params)
        want_ret = {"int": "integer(c_int)", "long long": "integer(c_long_long)"}.get(
            ret, "type(c_ptr)")
        assert result.lower() == want_ret, (name, ret, result)
        for arg, param in zip(names, params):
            assert arg in decl, (name, arg)
            ftype, byval = decl[arg]
            kind = c_kind(param)
            if kind[0] == "val":
                assert byval and ftype == kind[1], (name, arg, param, decl[arg])
            elif ftype == "type(c_ptr)":
                # an opaque handle or a device address goes by value; a
                # handle that the call writes (impz_bunch_t*) by reference
                assert byval != param.rstrip().endswith("* out"), (name, arg, param)
            else:
                assert not byval, (name, arg, param)
