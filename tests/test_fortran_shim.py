"""The Fortran side of the boundary (bqcd-r399-quda_b200/fortran/bqcdg_shim.F90)
against the C header, on CPU.  No Fortran compiler is installed here, so the
shim is checked by reading it:

* every bind(c) derived type must have the members of the C struct of the
  same name, in the same order, with the same kinds and array lengths; the
  offsets and sizes those kinds give under C's layout rules must equal the
  ones gcc computes for the header (offsetof / sizeof);
* every bind(c, name=...) interface must name a function that the header
  declares and the library exports, with as many arguments as its C
  prototype.
"""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "bqcd-r399-quda_b200", "fortran", "bqcdg_shim.F90")
HEADER = os.path.join(ROOT, "include", "bqcdg.h")
KINDS = {"real(c_double)": ("double", 8), "real(c_float)": ("float", 4), "integer(c_int)": ("int", 4)}


def fortran_types():
    src = open(SHIM).read()
    types = {}
    for m in re.finditer(r"type, bind\(c\) :: (\w+)\n(.*?)end type", src, flags=re.S):
        members = []
        for line in m.group(2).splitlines():
            line = line.split("!")[0].strip()
            if not line:
                continue
            kind, rest = [x.strip() for x in line.split("::")]
            for name in re.findall(r"(\w+)(?:\((\d+)\))?", rest):
                members.append((name[0], kind, int(name[1] or 1)))
        types[m.group(1)] = members
    return types


def c_layout(name, members, tmp_path):
    prog = ["#include <stdio.h>", "#include <stddef.h>", '#include "bqcdg.h"', "int main(void) {"]
    for mname, _, _ in members:
        prog.append('  printf("%%zu %%zu\\n", offsetof(%s, %s), sizeof(((%s *)0)->%s));' % (name, mname, name, mname))
    prog.append('  printf("%%zu\\n", sizeof(%s));' % name)
    prog.append("  return 0;\n}")
    c = tmp_path / ("%s.c" % name)
    c.write_text("\n".join(prog))
    exe = tmp_path / name
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    return [(int(out[2 * k]), int(out[2 * k + 1])) for k in range(len(members))], int(out[-1])


def fortran_layout(members):
    off, lay, align = 0, [], 1
    for _, kind, n in members:
        _, size = KINDS[kind]
        align = max(align, size)
        off = (off + size - 1) // size * size
        lay.append((off, size * n))
        off += size * n
    return lay, (off + align - 1) // align * align


def test_every_bind_c_type_matches_its_c_struct(tmp_path):
    types = fortran_types()
    assert set(types) >= {"bqcdg_params", "bqcdg_cg_para", "bqcdg_solver_opts", "bqcdg_solve_info",
                          "bqcdg_conf_meta"}
    header = open(HEADER).read()
    for name, members in types.items():
        body = re.search(r"typedef struct \{([^{}]*)\} %s;" % name, header).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        cmembers = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            ctype, names = decl.split(None, 1)
            for nm in names.split(","):
                mm = re.match(r"\s*(\w+)(?:\[(\d+)\])?", nm)
                cmembers.append((mm.group(1), ctype, int(mm.group(2) or 1)))
        assert [(m, KINDS[k][0], n) for m, k, n in members] == cmembers, name
        got, size = c_layout(name, members, tmp_path)
        want, fsize = fortran_layout(members)
        assert got == want and size == fsize, name


def header_prototypes():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(bqcdg_\w+)\s*\(([^)]*)\)\s*;", text):
        args = m.group(2).strip()
        protos[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return protos


def test_every_interface_names_an_exported_function_with_its_arity():
    src = open(SHIM).read()
    lib = C.CDLL(os.path.join(ROOT, "bqcd-r399-quda_b200", "lib", "libbqcdg.so"))
    protos = header_prototypes()
    found = re.findall(r"function (\w+)\(([^)]*)\)\s*(?:&\s*)?bind\(c, name = \"(\w+)\"\)", src)
    assert len(found) >= 15
    for fname, args, cname in found:
        assert fname == cname
        assert cname in protos, cname
        assert hasattr(lib, cname), cname
        assert len([a for a in args.split(",") if a.strip()]) == protos[cname], cname


def test_shim_replaces_the_reference_entry_points():
    src = open(SHIM).read()
    # the hook's own name and argument list (invert_quda.F90:96)
    assert re.search(r"^subroutine quda_solver\(matrix_mult, x, b, para, conf, iterations, rho\)", src, re.M)
    assert re.search(r"^subroutine bqcdg_f_cg\(matrix_mult, x, b, para, conf, iterations\)", src, re.M)
    assert re.search(r"^subroutine bqcdg_f_dsf\(p, conf, step, para, a, b\)", src, re.M)
    for op in ("mtil", "mtil_dag", "mtdagmt", "w_mult", "w_mult_dag", "w_dagger_w"):
        assert re.search(r"^subroutine bqcdg_f_%s\(out, in, para, conf\)" % op, src, re.M)
