"""ising_total_energy_noalloc: the total energy without device allocation.

Some callers cannot call cudaMalloc (a loop that must not stall other streams, since
cudaFree synchronises the device; work issued while another thread captures a CUDA graph;
an application that reserves device memory up front).  The entry point keeps its scratch in
a fixed array inside the library; this test checks it through the C-ABI against
ising_total_energy on two calls in a row, and that oversized replicas are rejected.
The file is named to run last in a pytest session."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _spins(n, seed):
    rng = np.random.default_rng(seed)
    s = rng.normal(size=(n, 3))
    s /= np.linalg.norm(s, axis=1, keepdims=True)
    return s.astype(np.float32).astype(np.float64)


def _energy(L, fn, mesh, replica, p):
    e = C.c_double()
    st = getattr(L, fn)(mesh.handle, replica, C.byref(p), C.byref(e))
    return st, e.value


def test_noalloc_matches_allocating_entry_point(ib, cuda_ok):
    L = ib._lib.load()
    frac = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.5]], np.float32)
    meshes = [ib.ChainMesh.simple_cubic(12, n_replicas=2), ib.ChainMesh(5, 4, 6, frac, 2.0, 2.0, 2.0, n_replicas=2)]
    params = [ib.reference_params("total", -1.0, 0.0, 0.4, 0.0, 0.2),
              ib.params(J=-1.0, J_prime=0.2, Dz=0.7, B=0.3, K=0.05, dmi="bulk")]
    for mi, m in enumerate(meshes):
        for r in range(2):
            m.set_spins(_spins(m.numAtoms, 10 * mi + r), r)
        n1 = len(m.neighbours(0, 0))
        # two calls in a row on different replicas and Hamiltonians: the shared scratch
        # keeps the previous call's contents, which must not leak into the next result
        for r, p in ((0, params[0]), (1, params[1]), (0, params[1]), (1, params[0])):
            st_a, e_a = _energy(L, "ising_total_energy", m, r, p)
            st_b, e_b = _energy(L, "ising_total_energy_noalloc", m, r, p)
            assert st_a == 0 and st_b == 0, (st_a, st_b, L.ising_last_error())
            scale = m.numAtoms * (abs(p.J) * n1 + abs(p.Dz) * n1 + abs(p.J_prime) * 12 + abs(p.B) * 2 + abs(p.K))
            assert abs(e_a - e_b) <= 1e-6 * scale, (mi, r, e_a, e_b)
        m.close()


def test_noalloc_rejects_oversized_replica(ib, cuda_ok):
    L = ib._lib.load()
    # 257 x 256 x 256 = 16,842,752 atoms, one past the 4096 x 4096 limit
    m = ib.ChainMesh(257, 256, 256, np.zeros((1, 3), np.float32), 1.0, 1.0, 1.0)
    p = ib.params(J=-1.0)
    st, _ = _energy(L, "ising_total_energy_noalloc", m, 0, p)
    assert st == 1
    assert b"16777216" in L.ising_last_error()
    m.close()
