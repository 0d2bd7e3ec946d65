"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates the reference's FP64 Fortran routines in C (``ising_oracle.c``).
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline /
reference arm may import this module; the CUDA product never does.

Parity is unpinned by the reference itself (it ships no golden vectors and cannot be
built in this image); the oracle is pinned by analytic known answers and by the
fixtures under ``tests/golden`` that ``tests/golden/make_golden.py`` generates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libising_oracle.so")


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    src = os.path.join(_HERE, "ising_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        d, i, l, f = C.c_double, C.c_int, C.c_long, C.c_float
        P = C.POINTER
        L.ora_mesh_create.restype = C.c_void_p
        L.ora_mesh_create.argtypes = [P(f), i, i, i, i, d, d, d, d, d, d, d, i]
        L.ora_mesh_destroy.argtypes = [C.c_void_p]
        L.ora_mesh_natoms.restype = l
        L.ora_mesh_natoms.argtypes = [C.c_void_p]
        L.ora_mesh_vectors.argtypes = [C.c_void_p, P(d)]
        L.ora_mesh_positions.argtypes = [C.c_void_p, P(f)]
        L.ora_mesh_first_atom.restype = i
        L.ora_mesh_first_atom.argtypes = [C.c_void_p, l]
        L.ora_mesh_shell_size.restype = i
        L.ora_mesh_shell_size.argtypes = [C.c_void_p, l, i]
        L.ora_mesh_shell_list.restype = i
        L.ora_mesh_shell_list.argtypes = [C.c_void_p, l, i, P(i)]
        L.ora_mesh_nl_size.restype = i
        L.ora_mesh_nl_size.argtypes = [C.c_void_p, l]
        L.ora_mesh_nl_list.restype = i
        L.ora_mesh_nl_list.argtypes = [C.c_void_p, l, P(i)]
        L.ora_mesh_deriv.restype = i
        L.ora_mesh_deriv.argtypes = [C.c_void_p, l, i, i]
        L.ora_mesh_spins.restype = P(d)
        L.ora_mesh_spins.argtypes = [C.c_void_p]
        L.ora_mesh_min_image.argtypes = [C.c_void_p, l, l, P(d)]
        L.ora_local_energy.argtypes = [C.c_void_p, l, C.c_void_p, P(d), P(d), P(d)]
        L.ora_total_energy.restype = d
        L.ora_total_energy.argtypes = [C.c_void_p, C.c_void_p, d]
        L.ora_canonical_energy.restype = d
        L.ora_canonical_energy.argtypes = [C.c_void_p, C.c_void_p]
        L.ora_arc_winding.restype = d
        L.ora_arc_winding.argtypes = [P(d), P(d), P(d)]
        L.ora_winding_number.restype = d
        L.ora_winding_number.argtypes = [C.c_void_p, i]
        L.ora_winding_density.argtypes = [C.c_void_p, i, P(d)]
        L.ora_statistics.argtypes = [C.c_void_p, P(d), P(d), P(d)]
        L.ora_cb_sweeps_f32.restype = l
        L.ora_cb_sweeps_f32.argtypes = [P(C.c_float), P(C.c_float), P(C.c_float), i, i, C.c_uint32, d,
                                        C.c_void_p, C.c_void_p, i]
        L.ora_gaussian_kernel.argtypes = [d, P(d)]
        L.ora_gaussian_filter_2d.restype = i
        L.ora_gaussian_filter_2d.argtypes = [P(d), i, i, d]
        L.ora_skyrmion_number.restype = i
        L.ora_skyrmion_number.argtypes = [P(d), i, i, i, i, d, i, d, P(i)]
        L.ora_skyrmion_distribution.restype = i
        L.ora_skyrmion_distribution.argtypes = [P(d), i, i, i, i, d, i, d, d, i, P(i)]
        L.ora_metropolis_mcs_ref.argtypes = [C.c_void_p, d, i, C.c_void_p, d]
        L.ora_metropolis_mcs_omp.argtypes = [C.c_void_p, d, i, C.c_void_p, d, i, i]
        L.ora_colour_pass.restype = l
        L.ora_colour_pass.argtypes = [C.c_void_p, P(i), i, C.c_uint32, d, C.c_void_p,
                                      C.c_void_p, P(d), P(C.c_uint8), P(d)]
        L.ora_colour_sweeps_omp.restype = l
        L.ora_colour_sweeps_omp.argtypes = [C.c_void_p, P(i), i, C.c_uint32, i, d,
                                            C.c_void_p, C.c_void_p, i]
        L.ora_init_uniform.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32]
        L.ora_init_skyrmion.argtypes = [C.c_void_p, d, d, d, d, i]
        L.ora_temperature_ladder.argtypes = [d, d, i, P(d)]
        L.ora_pt_swaps_ref.argtypes = [C.c_void_p, i, i, P(d), P(d), P(i)]
        L.ora_pt_exchange.restype = i
        L.ora_pt_exchange.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, i, P(d), P(d), P(i), i]
        L.ora_make_random.restype = _Random
        L.ora_make_random.argtypes = [C.c_int32]
        L.ora_uniform.restype = d
        L.ora_uniform.argtypes = [P(_Random)]
        L.ora_uniform_stream.argtypes = [C.c_int32, i, P(d)]
        L.ora_philox4x32.argtypes = [P(C.c_uint32), P(C.c_uint32), i, P(C.c_uint32)]
        L.ora_u01.restype = d
        L.ora_u01.argtypes = [C.c_uint32]
        L.ora_tau_int.restype = d
        L.ora_tau_int.argtypes = [P(d), l, d]
        for name in ("ora_const_kb", "ora_const_pi_f", "ora_const_g", "ora_const_mu_b"):
            getattr(L, name).restype = d
        for name in ("ora_fmt_F0", "ora_fmt_E0"):
            getattr(L, name).restype = i
            getattr(L, name).argtypes = [C.c_char_p, d, i]
        L.ora_fmt_I0m.restype = i
        L.ora_fmt_I0m.argtypes = [C.c_char_p, l, i]
        L.ora_fmt_ES.restype = i
        L.ora_fmt_ES.argtypes = [C.c_char_p, d, i, i]
        _lib = L
    return _lib


class _Random(C.Structure):
    _fields_ = [("seed", C.c_int32), ("ix", C.c_int32), ("iy", C.c_int32)]


class Params(C.Structure):
    """Hamiltonian arguments of calculateHeisenbergEnergy (src/energyMin.f90:86-87)
    plus the anisotropy extension and the DMI form selector."""
    _fields_ = [("J", C.c_double), ("J_prime", C.c_double), ("Dz", C.c_double),
                ("Dz_prime", C.c_double), ("B", C.c_double), ("K", C.c_double),
                ("K_axis", C.c_double * 3), ("dmi_bulk", C.c_int)]

    def __init__(self, J=0.0, J_prime=0.0, Dz=0.0, Dz_prime=0.0, B=0.0, K=0.0,
                 K_axis=(0.0, 0.0, 1.0), dmi_bulk=False):
        super().__init__(J, J_prime, Dz, Dz_prime, B, K, (C.c_double * 3)(*K_axis), int(dmi_bulk))


class SweepKey(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("ensemble", C.c_uint32), ("replica", C.c_uint32),
                ("move", C.c_int), ("r", C.c_double), ("philox_rounds", C.c_int)]


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


# unit cells (src/unit_cells.f90:7-77) plus the simple cubic cell the build adds
SC_CELL = (np.array([[0.0, 0.0, 0.0]], np.float32), (1.0, 1.0, 1.0, 90.0, 90.0, 90.0))
BCC_CELL = (np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.5]], np.float32), (2.0, 2.0, 2.0, 90.0, 90.0, 90.0))
HYPER_KAGOME_CELL = (np.array([
    [-0.5, 0.0, 0.5], [-0.25, 0.75, 0.5], [-0.5, 0.75, 0.25], [-0.25, 0.25, 0.0],
    [-0.5, 0.25, 0.75], [-0.25, 0.5, 0.75], [-0.75, 0.5, 0.25], [0.0, 0.5, 0.5],
    [0.0, 0.25, 0.25], [-0.75, 0.75, 0.0], [0.0, 0.0, 0.0], [-0.75, 0.0, 0.75]], np.float32),
    (6.0, 6.0, 6.0, 90.0, 90.0, 90.0))


class Mesh:
    """makeChainMesh (src/chainMesh.f90:729-911) restated; spins FP64 column-major."""

    def __init__(self, frac, nx, ny, nz, a, b, c, ab=90.0, bc=90.0, ca=90.0,
                 shell_tol=0.0, n_shells=2):
        L = lib()
        frac = np.ascontiguousarray(frac, dtype=np.float32)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.a, self.b, self.c = float(a), float(b), float(c)   # chainMesh%a, %b, %c
        self.nsub = frac.shape[0]
        self.n_shells = n_shells if n_shells > 0 else 2
        self._h = L.ora_mesh_create(frac.ctypes.data_as(C.POINTER(C.c_float)), self.nsub,
                                    nx, ny, nz, a, b, c, ab, bc, ca, shell_tol, n_shells)
        if not self._h:
            raise ValueError("ora_mesh_create failed (lattice too small for the derivative list)")
        self.natoms = L.ora_mesh_natoms(self._h)

    @classmethod
    def sc(cls, L_, ny=None, nz=None, a=1.0, **kw):
        return cls(SC_CELL[0], L_, ny or L_, nz or L_, a, a, a, **kw)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ora_mesh_destroy(self._h)
            self._h = None

    @property
    def spins(self) -> np.ndarray:
        """(natoms, 3) view in Fortran order over the oracle's atomSpins."""
        p = lib().ora_mesh_spins(self._h)
        flat = np.ctypeslib.as_array(p, shape=(3 * self.natoms,))
        return flat.reshape((3, self.natoms)).T

    def set_spins(self, s):
        s = np.asarray(s, dtype=np.float64).reshape(self.natoms, 3)
        self.spins[:, :] = s

    def vectors(self):
        out = np.zeros(18)
        lib().ora_mesh_vectors(self._h, _dp(out))
        return out.reshape(6, 3)

    def positions(self):
        out = np.zeros((self.natoms, 3), np.float32)
        lib().ora_mesh_positions(self._h, out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def shell(self, atom, s):
        n = lib().ora_mesh_shell_size(self._h, atom, s)
        out = np.zeros(max(n, 1), np.int32)
        lib().ora_mesh_shell_list(self._h, atom, s, _ip(out))
        return out[:n]

    def neighbor_list(self, atom):
        n = lib().ora_mesh_nl_size(self._h, atom)
        out = np.zeros(max(n, 1), np.int32)
        lib().ora_mesh_nl_list(self._h, atom, _ip(out))
        return out[:n]

    def deriv(self, atom, d, side):
        return lib().ora_mesh_deriv(self._h, atom, d, side)

    def derivative_table(self):
        t = np.zeros((self.natoms, 3, 2), np.int32)
        for a in range(self.natoms):
            for d in range(3):
                for s in range(2):
                    t[a, d, s] = self.deriv(a, d, s)
        return t

    def first_atom(self, cell):
        return lib().ora_mesh_first_atom(self._h, cell)

    def min_image(self, i, j):
        out = np.zeros(3)
        lib().ora_mesh_min_image(self._h, i, j, _dp(out))
        return out

    def local_energy(self, atom, params: Params, s_prop):
        sp = np.ascontiguousarray(s_prop, dtype=np.float64)
        o, n = C.c_double(), C.c_double()
        lib().ora_local_energy(self._h, atom, C.byref(params), _dp(sp), C.byref(o), C.byref(n))
        return o.value, n.value

    def total_energy(self, params: Params, zeeman_gmu=2.0):
        return lib().ora_total_energy(self._h, C.byref(params), zeeman_gmu)

    def canonical_energy(self, params: Params):
        return lib().ora_canonical_energy(self._h, C.byref(params))

    def winding_number(self, z1):
        return lib().ora_winding_number(self._h, z1)

    def winding_density(self, z1):
        out = np.zeros(self.nx * self.ny)
        lib().ora_winding_density(self._h, z1, _dp(out))
        return out.reshape((self.ny, self.nx)).T

    def statistics(self):
        wm, ws, m = C.c_double(), C.c_double(), np.zeros(3)
        lib().ora_statistics(self._h, C.byref(wm), C.byref(ws), _dp(m))
        return wm.value, ws.value, m

    def metropolis_mcs_ref(self, beta, n_sweeps, params, r=0.2):
        lib().ora_metropolis_mcs_ref(self._h, beta, n_sweeps, C.byref(params), r)

    def metropolis_mcs_omp(self, beta, n_sweeps, params, r=0.2, n_threads=1, time_seed=1):
        lib().ora_metropolis_mcs_omp(self._h, beta, n_sweeps, C.byref(params), r, n_threads, time_seed)

    def colour_pass(self, colour_of, colour, sweep, beta, params, key: SweepKey,
                    want_detail=False):
        col = np.ascontiguousarray(colour_of, dtype=np.int32)
        de = C.c_double(0.0)
        acc = marg = None
        if want_detail:
            acc = np.zeros(self.natoms, np.uint8)
            marg = np.zeros(self.natoms)
        n = lib().ora_colour_pass(self._h, _ip(col), colour, sweep, beta, C.byref(params),
                                  C.byref(key), C.byref(de),
                                  acc.ctypes.data_as(C.POINTER(C.c_uint8)) if want_detail else None,
                                  _dp(marg) if want_detail else None)
        if want_detail:
            return n, de.value, acc, marg
        return n, de.value

    def colour_sweeps_omp(self, colour_of, n_colours, sweep0, n_sweeps, beta, params,
                          key: SweepKey, n_threads=1):
        col = np.ascontiguousarray(colour_of, dtype=np.int32)
        return lib().ora_colour_sweeps_omp(self._h, _ip(col), n_colours, sweep0, n_sweeps, beta,
                                           C.byref(params), C.byref(key), n_threads)

    def init_uniform(self, seed, ensemble=0, replica=0):
        lib().ora_init_uniform(self._h, seed, ensemble, replica)

    def init_skyrmion(self, rx, ry, R_s, chi=1.56, N=1):
        lib().ora_init_skyrmion(self._h, rx, ry, R_s, chi, N)


def checkerboard(nx, ny, nz, nsub=1):
    """Two-colour class (x+y+z) & 1 for the simple cubic atom order (z fastest)."""
    x, y, z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    return ((x + y + z) & 1).astype(np.int32).reshape(-1)


def uniform_stream(seed, n):
    out = np.zeros(n)
    lib().ora_uniform_stream(seed, n, _dp(out))
    return out


def philox(ctr, key, rounds=10):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().ora_philox4x32(c, k, rounds, o)
    return list(o)


def temperature_ladder(tmin, tmax, n):
    out = np.zeros(n)
    lib().ora_temperature_ladder(tmin, tmax, n, _dp(out))
    return out


def pt_exchange(seed, ensemble, rnd, betas, e_rep, t2r, rounds=10):
    b = np.ascontiguousarray(betas, np.float64)
    e = np.ascontiguousarray(e_rep, np.float64)
    t = np.ascontiguousarray(t2r, np.int32).copy()
    n = lib().ora_pt_exchange(seed, ensemble, rnd, len(b), _dp(b), _dp(e), _ip(t), rounds)
    return n, t


def pt_swaps_ref(seed, n_swaps, T, energies, temp_mesh, warmup=50):
    """PT.f90:214-217 (makeRandom(rank) + 50 warm-up draws) then :235-272."""
    L = lib()
    rng = L.ora_make_random(seed)
    for _ in range(warmup):
        L.ora_uniform(C.byref(rng))
    T = np.ascontiguousarray(T, np.float64)
    E = np.ascontiguousarray(energies, np.float64)
    tm = np.ascontiguousarray(temp_mesh, np.int32).copy()
    L.ora_pt_swaps_ref(C.byref(rng), len(T), n_swaps, _dp(T), _dp(E), _ip(tm))
    return tm


def arc_winding(s1, s2, s3):
    a, b, c = (np.ascontiguousarray(v, np.float64) for v in (s1, s2, s3))
    return lib().ora_arc_winding(_dp(a), _dp(b), _dp(c))


def tau_int(x, c=5.0):
    x = np.ascontiguousarray(x, np.float64)
    return lib().ora_tau_int(_dp(x), len(x), c)


def fmt_F0(x, d):
    b = C.create_string_buffer(512)
    lib().ora_fmt_F0(b, x, d)
    return b.value.decode()


def fmt_E0(x, d):
    b = C.create_string_buffer(512)
    lib().ora_fmt_E0(b, x, d)
    return b.value.decode()


def fmt_ES(x, w, d):
    b = C.create_string_buffer(512)
    lib().ora_fmt_ES(b, x, w, d)
    return b.value.decode()


def fmt_I0m(v, m):
    b = C.create_string_buffer(64)
    lib().ora_fmt_I0m(b, v, m)
    return b.value.decode()


# ---------------------------------------------------------------- skyrmion counting
def gaussian_kernel(sigma):
    """The normalised 5x5 kernel of Gaussian_filter_2d (rsp:814-834), G[l-1, m-1]."""
    G = np.zeros(25)
    lib().ora_gaussian_kernel(sigma, _dp(G))
    return G.reshape(5, 5)


def gaussian_filter_2d(a, sigma):
    """Gaussian_filter_2d (rsp:814-859) on a copy of the (nx, ny) array a."""
    b = np.asfortranarray(np.array(a, dtype=np.float64))
    st = lib().ora_gaussian_filter_2d(b.ctypes.data_as(C.POINTER(C.c_double)), b.shape[0], b.shape[1], sigma)
    if st:
        raise ValueError(f"gaussian_filter_2d status {st}")
    return b


def skyrmion_number(dens, ncx, ncy, q_threshold, particle_number, sigma):
    """calculate_skyrmion_number (rsp:627-812) after its interpolation step, on the (fx, fy)
    fine density; returns (status, count)."""
    b = np.asfortranarray(np.array(dens, dtype=np.float64))
    out = C.c_int(0)
    st = lib().ora_skyrmion_number(b.ctypes.data_as(C.POINTER(C.c_double)), b.shape[0], b.shape[1], ncx, ncy,
                                   q_threshold, particle_number, sigma, C.byref(out))
    return st, out.value


def skyrmion_distribution(dens, ncx, ncy, total_charge, N, min_t, max_t, num_thresholds):
    """compute_skyrmion_distribution (rsp:930-983) on a fixed fine density; returns
    (status, counts of particles 1..N)."""
    b = np.asfortranarray(np.array(dens, dtype=np.float64))
    out = (C.c_int * N)()
    st = lib().ora_skyrmion_distribution(b.ctypes.data_as(C.POINTER(C.c_double)), b.shape[0], b.shape[1], ncx, ncy,
                                         total_charge, N, min_t, max_t, num_thresholds, out)
    return st, list(out)


def spectral_upsample(f, sclx, scly):
    """Band-limited periodic interpolation of the (nx, ny, 3) grid f onto (sclx*nx, scly*ny):
    the 2-D DFT zero-padded in the middle of each axis, an even axis's Nyquist bin split
    between +N/2 and -N/2, scaled so that the fine grid passes through the coarse samples.
    This is the operation spectral_interpolate_to_fine (rsp:12-70) names; the reference's own
    FFTW plans (src/fft.f90:80-84,128-155) take the padded row length 2(nx/2+1) as the
    transform length and write rows of nx/2+2 bins at a pitch of nx/2+1, so its values are
    not reproducible and this restatement follows the stated intent."""
    f = np.asarray(f, dtype=np.float64)
    nx, ny = f.shape[:2]
    Mx, My = sclx * nx, scly * ny

    def pad(F, n, M, axis):
        F = np.moveaxis(F, axis, 0)
        G = np.zeros((M,) + F.shape[1:], dtype=complex)
        h = n // 2
        if n % 2 == 0:
            G[:h] = F[:h]
            if h > 0:
                G[M - h + 1:] = F[h + 1:]
            G[h] += F[h] / 2
            G[M - h] += F[h] / 2
        else:
            G[:h + 1] = F[:h + 1]
            if h > 0:
                G[M - h:] = F[h + 1:]
        return np.moveaxis(G, 0, axis)

    F = np.fft.fft2(f, axes=(0, 1))
    G = pad(pad(F, nx, Mx, 0), ny, My, 1)
    return np.real(np.fft.ifft2(G, axes=(0, 1))) * (Mx * My) / (nx * ny)


def fine_winding_density(g):
    """The density loop of calculate_winding_density_interpolated (rsp:409-434) on the
    (fx, fy, 3) fine grid: triangles (s1,s2,s3) and (s1,s3,s4) of the periodic plaquette
    (i,j), (i+1,j), (i+1,j+1), (i,j+1), normalised spins, divided by 4 pi (float pi)."""
    s1 = g / np.linalg.norm(g, axis=2, keepdims=True)
    s2 = np.roll(s1, -1, axis=0)
    s3 = np.roll(s2, -1, axis=1)
    s4 = np.roll(s1, -1, axis=1)

    def arc(a, b, c):
        d12 = (a * b).sum(2)
        d23 = (b * c).sum(2)
        d31 = (c * a).sum(2)
        im = (a * np.cross(b, c)).sum(2)
        re = 1.0 + d12 + d23 + d31
        nrm = np.sqrt(2.0 * (1.0 + d12) * (1.0 + d23) * (1.0 + d31))
        return 2.0 * np.arctan2(im / nrm, re / nrm)

    return (arc(s1, s2, s3) + arc(s1, s3, s4)) / (4.0 * float(np.float32(np.pi)))


def std_grid(mesh, z1):
    """map_spins_to_std_grid (src/chainMesh.f90:54-83): the spin of the first atom (the
    linked-list head) of every cell of slice z1, as an (nx, ny, 3) array."""
    out = np.zeros((mesh.nx, mesh.ny, 3))
    s = mesh.spins
    for i in range(mesh.nx):
        for j in range(mesh.ny):
            out[i, j] = s[mesh.first_atom((i * mesh.ny + j) * mesh.nz + (z1 - 1))]
    return out


def winding_density_interpolated(mesh, z1, sclx=10, scly=10):
    """calculate_winding_density_interpolated (rsp:366-436) with the band-limited
    interpolation of spectral_upsample."""
    return fine_winding_density(spectral_upsample(std_grid(mesh, z1), sclx, scly))


def cb_sweeps_f32(planes, L, n_sweeps, sweep0, beta, params, key, n_threads=1):
    """The optimised FP32 checkerboard sweep (CPU baseline) on planes = float32 array (3, L^3)
    in reference atom order, updated in place; returns the accepted count."""
    assert planes.dtype == np.float32 and planes.flags["C_CONTIGUOUS"] and planes.shape == (3, L ** 3)
    f = C.POINTER(C.c_float)
    return lib().ora_cb_sweeps_f32(planes[0].ctypes.data_as(f), planes[1].ctypes.data_as(f),
                                   planes[2].ctypes.data_as(f), L, n_sweeps, sweep0, beta,
                                   C.byref(params), C.byref(key), n_threads)
