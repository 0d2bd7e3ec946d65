"""The ctypes mirrors in ising_b200/_lib.py must lay out every public struct exactly as the C
compiler does from include/ising_gpu.h: same size, same offset for every field.  A small C
program generated from the ctypes field lists prints sizeof/offsetof; no GPU is needed."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _mirrors():
    from ising_b200 import _lib
    return [(_lib.MeshInfo, "ising_mesh_info"), (_lib.Params, "ising_params"), (_lib.PTOptions, "ising_pt_options"),
            (_lib.EnsembleDesc, "ising_ensemble_desc"), (_lib.EnsemblesOptions, "ising_ensembles_options"),
            (_lib.EnsSchedule, "ising_ensembles_schedule_t")]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_mirrors_match_the_c_header(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "ising_gpu.h"', "int main(void) {"]
    expect = []
    for cls, cname in _mirrors():
        lines.append(f'printf("%zu\\n", sizeof({cname}));')
        expect.append((f"sizeof({cname})", C.sizeof(cls)))
        for name, _t in cls._fields_:
            lines.append(f'printf("%zu\\n", offsetof({cname}, {name}));')
            expect.append((f"offsetof({cname}, {name})", getattr(cls, name).offset))
    lines += ["return 0;", "}"]
    src = tmp_path / "abi.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "abi"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert len(got) == len(expect)
    bad = [(what, want, have) for (what, want), have in zip(expect, got) if want != have]
    assert not bad, f"ctypes layout differs from the C header: {bad}"
