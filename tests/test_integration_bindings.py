"""Every symbol that the Fortran module include/ising_gpu.f90 binds (bind(C, name="...")) is
declared in include/ising_gpu.h with the same number of arguments and exported by the built
library, so the module's interfaces name real entry points."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_fortran_bindings_name_real_entry_points():
    doc = open(os.path.join(ROOT, "include", "ising_gpu.f90")).read()
    names = sorted(set(re.findall(r'bind\(C,\s*name="([A-Za-z0-9_]+)"\)', doc)))
    assert len(names) >= 20
    header = open(os.path.join(ROOT, "include", "ising_gpu.h")).read()
    missing_decl = [n for n in names if not re.search(r"\b" + n + r"\s*\(", header)]
    assert not missing_decl, f"bound in the Fortran module but not declared in the header: {missing_decl}"
    so = os.path.join(ROOT, "ising_b200", "libisinggpu.so")
    if not os.path.exists(so):
        pytest.skip("libisinggpu.so not built")
    lib = ctypes.CDLL(so)
    missing_sym = [n for n in names if not hasattr(lib, n)]
    assert not missing_sym, f"not exported by libisinggpu.so: {missing_sym}"


def _c_arg_count(header, name):
    m = re.search(r"\b" + name + r"\s*\(([^;]*?)\)\s*;", header, re.S)
    assert m, name
    args = m.group(1).strip()
    return 0 if args in ("", "void") else args.count(",") + 1


def test_fortran_bindings_take_as_many_arguments_as_the_c_prototypes():
    doc = open(os.path.join(ROOT, "include", "ising_gpu.f90")).read()
    joined = re.sub(r"&\s*\n\s*", " ", doc)          # Fortran continuation lines
    header = open(os.path.join(ROOT, "include", "ising_gpu.h")).read()
    found = re.findall(r'function\s+\w+\(([^)]*)\)\s*bind\(C,\s*name="([A-Za-z0-9_]+)"\)', joined)
    assert len(found) >= 20, len(found)
    bad = []
    for fargs, cname in found:
        n_f = 0 if not fargs.strip() else fargs.count(",") + 1
        n_c = _c_arg_count(header, cname)
        if n_f != n_c:
            bad.append((cname, n_f, n_c))
    assert not bad, f"(symbol, Fortran arguments, C arguments): {bad}"

