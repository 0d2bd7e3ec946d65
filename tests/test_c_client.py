"""A C client (tests/c_client/pt_driver.c) drives the library through include/ising_gpu.h and
libisinggpu.so alone, as the reference's drivers would: it compiles cleanly as C99 and links
(CPU), and on the GPU its PT run gives the same energies and temperature map as the same run
through the Python API, a near-integer winding number and a spins CSV of the right shape."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "ising_b200")
SRC = os.path.join(ROOT, "tests", "c_client", "pt_driver.c")


def _build(tmp_path):
    if shutil.which("gcc") is None:
        pytest.skip("needs gcc")
    if not os.path.exists(os.path.join(LIBDIR, "libisinggpu.so")):
        pytest.skip("libisinggpu.so not built")
    exe = str(tmp_path / "pt_driver")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
                    "-L", LIBDIR, "-lisinggpu", "-lm", f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def test_c_client_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_c_client_runs_pt_like_the_python_api(ib, cuda_ok, tmp_path):
    exe = _build(tmp_path)
    csv = tmp_path / "spins.csv"
    L, n, rounds = 16, 4, 5
    out = subprocess.run([exe, str(L), str(n), str(rounds), str(csv)], check=True, capture_output=True, text=True)
    head, e_part, perm_part, q_part = out.stdout.split(" ", 1)[0], *out.stdout.split(" ", 1)[1].split("|")
    assert head == "ok"
    e_c = np.array([float(v) for v in e_part.split()])
    t2r_c = np.array([int(v) for v in perm_part.split()])
    q = float(q_part)
    assert sorted(t2r_c) == list(range(n))
    assert abs(q - round(q)) < 1e-6
    lines = csv.read_text().splitlines()
    assert lines[0].replace(" ", "") == "x,y,z,Sx,Sy,Sz" and len(lines) == 1 + L ** 3
    # the same run through the Python API
    m = ib.ChainMesh.simple_cubic(L, n_replicas=n)
    m.init_uniform(0x15196, 0)
    betas = 1.0 / (0.1 * 15.0 ** (np.arange(n) / (n - 1)))
    p = ib.params(J=-1.0, Dz=0.7, B=0.3, dmi="bulk", include_Jp=False)
    pt = ib.ParallelTempering(m, betas, p, seed=0x15196, move=1, r=0.2)
    pt.run(10, rounds)
    e, _ = pt.energies()
    t2r = pt.permutation()
    np.testing.assert_array_equal(t2r_c, t2r)
    np.testing.assert_allclose(e_c, e[t2r], rtol=1e-8, atol=1e-8)
