"""The Fortran binding (dftb_fast-ewald_3d_b200/fortran/ewald_b200.f90) against
the C header, without a Fortran compiler: every bind(C) interface names an entry
point the header declares, with the same number of arguments, and each dummy
argument is passed the way the C parameter expects -- by value (the `value`
attribute) for a C scalar or a handle pointer (ewg_context*, void*), by
reference for data pointers with matching interoperable types, or as an address
by value (type(c_ptr), for arrays the caller may leave out)."""

import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "dftb_fast-ewald_3d_b200", "fortran", "ewald_b200.f90")
HEADER = os.path.join(ROOT, "include", "ewald_b200.h")

# C base type of a pointer parameter -> the Fortran declaration's type.
POINTEE = {"double": "real(c_double)", "int": "integer(c_int)", "long long": "integer(c_long_long)",
           "ewg_overrides": "type(tewgoverrides)", "ewg_kernel_shape": "type(tewgkernelshape)",
           "ewg_params": "type(tewgparams)"}
SCALAR = {"int": "integer(c_int)", "double": "real(c_double)", "long long": "integer(c_long_long)"}


def c_prototypes():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    protos = {}
    for m in re.finditer(r"([A-Za-z_][A-Za-z_ ]*?[\s\*]+)(ewg_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", text):
        ret, name, params = m.group(1).strip(), m.group(2), m.group(3).strip()
        plist = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
        protos[name] = (ret, plist)
    return protos


def c_param(p):
    """(base type, pointer depth) of one C parameter declaration."""
    stars = p.count("*")
    words = p.replace("*", " ").split()
    words = [w for w in words if w != "const"][:-1]  # drop the parameter name
    return " ".join(words), stars


def fortran_interfaces():
    text = open(F90).read()
    text = re.sub(r"&\s*\n\s*&?", " ", text)  # join continuation lines
    out = {}
    pat = re.compile(r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)\s*result\((\w+)\)"
                     r"(.*?)end function\s+\1", re.S | re.I)
    for m in pat.finditer(text):
        args = [a.strip().lower() for a in m.group(2).split(",") if a.strip()]
        result = m.group(4).lower()
        decls = {}
        for line in m.group(5).split("\n"):
            if "::" not in line:
                continue
            spec, names = line.split("::", 1)
            spec = spec.strip().lower().replace(" ", "")
            for nm in re.findall(r"(\w+)\s*(?:\([^)]*\))?", names):
                decls[nm.lower()] = spec
        out[m.group(3)] = (args, result, decls)
    return out


def test_every_interface_matches_its_c_prototype():
    protos = c_prototypes()
    ifaces = fortran_interfaces()
    assert len(ifaces) >= 20
    for cname, (args, result, decls) in ifaces.items():
        assert cname in protos, f"{cname}: not declared in the header"
        ret, params = protos[cname]
        assert len(args) == len(params), f"{cname}: {len(args)} Fortran args, {len(params)} in C"
        rspec = decls[result]
        if ret == "int":
            assert rspec.startswith("integer(c_int)"), cname
        elif ret == "long long":
            assert rspec.startswith("integer(c_long_long)"), cname
        else:
            assert rspec.startswith("type(c_ptr)"), (cname, ret)
        for a, p in zip(args, params):
            spec = decls[a]
            base, depth = c_param(p)
            by_value = ",value" in spec
            where = f"{cname}({a}: {p})"
            if depth == 0:
                assert by_value and spec.startswith(SCALAR[base]), where
            elif base in ("ewg_context", "void") and depth == 1:
                assert by_value and spec.startswith("type(c_ptr)"), where
            elif base == "ewg_context" and depth == 2:
                assert not by_value and spec.startswith("type(c_ptr)"), where
            elif spec.startswith("type(c_ptr)"):
                # an optional array: its address by value (C_NULL_PTR or c_loc)
                assert depth == 1 and by_value, where
            else:
                assert depth == 1 and not by_value, where
                assert spec.startswith(POINTEE[base]), where


@pytest.mark.parametrize("name", ["ewg_create", "ewg_potential_force", "ewg_tune_kernels",
                                  "ewg_set_kernel_shape", "ewg_batch_potential_force_ov",
                                  "ewg_xlbomd_gradients", "ewg_external_pot_grad"])
def test_binding_covers(name):
    assert name in fortran_interfaces()


def c_structs():
    """{typedef name: [(member, C type, count)]} of the header's plain structs."""
    text = re.sub(r"/\*.*?\*/", " ", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"typedef struct\s*\{([^}]*)\}\s*(\w+)\s*;", text):
        members = []
        for decl in m.group(1).split(";"):
            decl = decl.strip()
            if not decl:
                continue
            ctype, rest = decl.split(None, 1)
            for item in rest.split(","):
                item = item.strip()
                mm = re.match(r"(\w+)(?:\[(\d+)\])?", item)
                members.append((mm.group(1), ctype, int(mm.group(2) or 1)))
        out[m.group(2)] = members
    return out


def fortran_types():
    """{type name (lower case): [(component, Fortran type, count)]} of bind(C) types."""
    text = re.sub(r"&\s*\n\s*&?", " ", open(F90).read())
    out = {}
    for m in re.finditer(r"type,\s*bind\(C\)\s*::\s*(\w+)(.*?)end type", text, re.S | re.I):
        comps = []
        for line in m.group(2).split("\n"):
            if "::" not in line:
                continue
            spec, names = line.split("::", 1)
            for item in re.findall(r"(\w+)\s*(?:\((\d+)\))?\s*(?:=\s*[^,]+)?", names):
                if item[0]:
                    comps.append((item[0].lower(), spec.strip().lower(), int(item[1] or 1)))
        out[m.group(1).lower()] = comps
    return out


@pytest.mark.parametrize("cname,ftype", [("ewg_overrides", "tewgoverrides"),
                                          ("ewg_params", "tewgparams"),
                                          ("ewg_kernel_shape", "tewgkernelshape")])
def test_derived_types_match_the_c_structs(cname, ftype):
    ctype = {"int": "integer(c_int)", "double": "real(c_double)"}
    c = [(n.lower(), ctype[t], k) for n, t, k in c_structs()[cname]]
    f = fortran_types()[ftype]
    assert f == c

