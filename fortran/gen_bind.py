#!/usr/bin/env python
"""Writes fortran/x3d_b200_bind.f90, the ISO_C_BINDING module of the C ABI,
from include/x3d_b200.h: every integer #define as a named constant and every
entry point as a bind(C) interface, plus the status check that maps a
non-zero status to decomp_2d_abort (the reference's error path).

Run after changing the header:  python fortran/gen_bind.py
tests/test_capi_abi.py checks that the committed module matches the header.

The structs the header defines by value (x3d_work, x3d_box, x3d_block)
become bind(C) derived types with the same members in the same order; the
entry points take them by address (c_loc of an array of them).

Type mapping: handles (x3d_ctx, x3d_op, x3d_batch) and field or array
pointers pass by value as type(c_ptr) -- c_loc of a target array, or a
device address under !$acc host_data use_device; arrays of field pointers
(void *const *) as arrays of type(c_ptr); handles a call returns
(x3d_ctx *, ...) pass by reference; int, double and size_t pass by value;
int * outputs pass by reference (arrays where the header takes several
values); strings pass as character arrays (trim(name) // c_null_char).  A C
parameter whose name is a Fortran keyword is renamed (bind(C) matches by
position).
"""
from __future__ import annotations

import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(os.path.dirname(HERE), "include", "x3d_b200.h")
OUT = os.path.join(HERE, "x3d_b200_bind.f90")

RENAME = {"precision": "prec", "kind": "op_kind", "count": "cnt", "value": "val", "in": "src", "out": "dst"}
ARRAY_INTS = {"ncl", "dims", "meta"}  # int * parameters that carry several values
KIND_ORDER = ["c_ptr", "c_int", "c_double", "c_size_t", "c_long_long", "c_char"]


def declarations(text):
    """(return type, name, [(C type, parameter name)]) of every entry point."""
    out = []
    for ret, name, args in re.findall(r"^(int|const char \*)\s*(x3d_\w+)\(([^;]*?)\);", text, re.M | re.S):
        params = []
        for a in (x.strip() for x in " ".join(args.split()).split(",")):
            m = re.match(r"(.*?)(\w+)$", a)
            params.append((" ".join(m.group(1).split()), m.group(2)))
        out.append((ret, name, params))
    return out


def constants(text):
    return re.findall(r"^#define\s+(X3D_\w+)\s+(-?\d+)\b", text, re.M)


STRUCT_FIELD = {"int": "integer(c_int)", "long long": "integer(c_long_long)", "double": "real(c_double)",
                "x3d_op": "type(c_ptr)", "void *": "type(c_ptr)", "const void *": "type(c_ptr)"}


def structs(text):
    """(name, [(Fortran declaration, member)]) of every struct the header
    defines by value (typedef struct [tag] { ... } name;), members in order."""
    out = []
    for body, name in re.findall(r"^typedef struct(?: \w+)? \{(.*?)\} (x3d_\w+);", text, re.M | re.S):
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        fields = []
        for decl in (d.strip() for d in body.split(";") if d.strip()):
            m = re.match(r"((?:const )?[a-z_0-9 ]+?\s*\*?)\s*(\w+(?:\s*,\s*\w+)*)$", " ".join(decl.split()))
            ctype = " ".join(m.group(1).split())
            for member in (x.strip() for x in m.group(2).split(",")):
                fields.append((STRUCT_FIELD[ctype], member))
        out.append((name, fields))
    return out


def derived_type(name, fields):
    """A bind(C) derived type with the struct's layout (members in order)."""
    lines = [f"  type, bind(C) :: {name}"]
    lines += [f"     {ft} :: {RENAME.get(m, m)}" for ft, m in fields]
    lines.append(f"  end type {name}")
    return lines


def fortran_type(ctype, pname):
    """(declaration, dimension suffix) of one dummy argument."""
    by_value_ptr = {"x3d_ctx", "x3d_op", "x3d_batch", "void *", "const void *", "double *", "const double *",
                    "const x3d_box *", "const x3d_work *", "const x3d_block *"}
    if ctype in by_value_ptr:
        return "type(c_ptr), value", ""
    if ctype in ("x3d_ctx *", "x3d_op *", "x3d_batch *", "void **"):
        return "type(c_ptr)", ""
    if ctype in ("void *const *", "const void *const *"):
        return "type(c_ptr)", "(*)"
    if ctype == "int":
        return "integer(c_int), value", ""
    if ctype in ("int *", "const int *"):
        return "integer(c_int)", "(*)" if pname in ARRAY_INTS else ""
    if ctype == "double":
        return "real(c_double), value", ""
    if ctype == "size_t":
        return "integer(c_size_t), value", ""
    if ctype in ("long long *", "unsigned long long *"):
        return "integer(c_long_long)", ""
    if ctype == "const char *":
        return "character(kind=c_char)", "(*)"
    raise ValueError(f"no Fortran mapping for C type {ctype!r} ({pname})")


def wrap(head, first_indent=5, cont_indent=10, width=96):
    """A Fortran statement split with & continuations at argument commas."""
    if len(head) + first_indent <= width:
        return [" " * first_indent + head]
    lines, cur = [], " " * first_indent
    for p in re.split(r"(?<=, )", head):
        if len(cur) + len(p) > width and cur.strip():
            lines.append(cur.rstrip() + " &")
            cur = " " * cont_indent
        cur += p
    lines.append(cur)
    return lines


def interface(ret, name, params):
    names = [RENAME.get(p, p) for _, p in params]
    fret = "type(c_ptr)" if ret.startswith("const char") else "integer(c_int)"
    lines = wrap(f'{fret} function {name}({", ".join(names)}) bind(C, name="{name}")')
    kinds = {"c_ptr" if fret.startswith("type") else "c_int"}
    body = []
    for (ct, pn), fn in zip(params, names):
        ft, dim = fortran_type(ct, pn)
        kinds.update(k for k in KIND_ORDER if k in ft)
        body.append(f"       {ft} :: {fn}{dim}")
    lines.append("       import :: " + ", ".join(k for k in KIND_ORDER if k in kinds))
    lines += body
    lines.append("     end function")
    return lines


def generate(text):
    out = ["! ISO_C_BINDING module of the B200 hot-path library (include/x3d_b200.h).",
           "! Written by fortran/gen_bind.py from the header; do not edit by hand.",
           "! Not compiled in this repository's image (it has no Fortran compiler).",
           "module x3d_b200_bind",
           "  use iso_c_binding",
           "  implicit none",
           ""]
    for name, val in constants(text):
        out.append(f"  integer(c_int), parameter :: {name} = {val}")
    out += ["", "  ! the structs the entry points take by address (pass c_loc of an array of them)"]
    for name, fields in structs(text):
        out += derived_type(name, fields)
    out += ["",
            "  ! the context the re-pointed routines use (x3d_b200_derive.f90)",
            "  type(c_ptr), save :: x3d_ctx = c_null_ptr",
            "",
            "  interface"]
    for ret, name, params in declarations(text):
        out += interface(ret, name, params)
    out += ["  end interface",
            "",
            "contains",
            "",
            "  ! A non-zero status from the library becomes the reference's abort.",
            "  subroutine x3d_check(rc, where)",
            "    use decomp_2d_mpi, only : decomp_2d_abort",
            "    integer(c_int), intent(in) :: rc",
            "    character(len=*), intent(in) :: where",
            "    if (rc /= 0) call decomp_2d_abort(__FILE__, __LINE__, int(rc), where)",
            "  end subroutine x3d_check",
            "",
            "end module x3d_b200_bind",
            ""]
    return "\n".join(out)


def main():
    with open(HEADER) as f:
        text = f.read()
    with open(OUT, "w") as f:
        f.write(generate(text))
    print(f"wrote {OUT}: {len(declarations(text))} interfaces, {len(constants(text))} constants")


if __name__ == "__main__":
    main()
