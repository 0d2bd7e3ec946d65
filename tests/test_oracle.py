"""CPU tests of the oracle (the FP64 restatement of the reference) against analytic known
answers.  The reference ships no golden vectors, so these pin the oracle."""
import math

import numpy as np
import pytest


def test_constants_are_float_rounded(oracle):
    L = oracle.lib()
    assert L.ora_const_pi_f() == float(np.float32(math.pi))
    assert L.ora_const_kb() == float(np.float32(8.6173303e-5))
    assert L.ora_const_g() == 2.0 and L.ora_const_mu_b() == 1.0


def test_reference_rng_stream(oracle):
    a = oracle.uniform_stream(0, 1000)
    b = oracle.uniform_stream(0, 1000)
    assert np.array_equal(a, b)
    assert np.all(a > 0) and np.all(a <= 1)
    c = oracle.uniform_stream(12345, 1000)
    assert not np.array_equal(a, c)
    # (0,1] mask with the low bit set: every draw is an odd multiple of 1/(2^31-1)
    k = np.rint(a * 2147483647.0).astype(np.int64)
    assert np.all(k % 2 == 1)
    # uniformity
    h, _ = np.histogram(oracle.uniform_stream(7, 100000), bins=20, range=(0, 1))
    chi2 = ((h - 5000) ** 2 / 5000).sum()
    assert chi2 < 45  # 19 dof, p ~ 1e-3


def test_philox_properties(oracle):
    a = oracle.philox([1, 2, 3, 4], [5, 6])
    assert a == oracle.philox([1, 2, 3, 4], [5, 6])
    assert a != oracle.philox([1, 2, 3, 5], [5, 6])
    assert a != oracle.philox([1, 2, 3, 4], [5, 7])
    # fewer rounds differ
    assert a != oracle.philox([1, 2, 3, 4], [5, 6], rounds=7)
    # bit balance over many counters
    bits = 0
    n = 4000
    for i in range(n):
        for w in oracle.philox([i, 0, 0, 0], [0x15196, 0]):
            bits += bin(w).count("1")
    frac = bits / (n * 128)
    assert abs(frac - 0.5) < 0.005
    # u01 is an odd multiple of 2^-24 in (0,1)
    L = oracle.lib()
    for x in (0, 1, 0xFFFFFFFF, 0x80000000, 12345):
        u = L.ora_u01(x)
        assert 0 < u < 1
        assert (u * 2 ** 24) % 2 == 1


def test_sc_mesh_geometry(oracle):
    m = oracle.Mesh.sc(6)
    assert m.natoms == 216
    for a in (0, 7, 100, 215):
        assert len(m.shell(a, 0)) == 6
        assert len(m.shell(a, 1)) == 12
        assert len(m.neighbor_list(a)) == 6
        assert sorted(m.shell(a, 0)) == sorted(m.neighbor_list(a))
    # atom order: z fastest (chainMesh.f90:684); derivative list = axis neighbours
    assert m.deriv(0, 2, 1) == 1 and m.deriv(0, 1, 1) == 6 and m.deriv(0, 0, 1) == 36
    assert m.deriv(0, 2, 0) == 5 and m.deriv(0, 0, 0) == 180
    v = m.vectors()
    assert np.allclose(v[0], [1, 0, 0]) and np.allclose(v[1], [0, 1, 0]) and np.allclose(v[2], [0, 0, 1])


def test_bcc_and_hyper_kagome_shells(oracle):
    f, (a, b, c, ab, bc, ca) = oracle.BCC_CELL
    m = oracle.Mesh(f, 4, 4, 4, a, b, c, ab, bc, ca)
    assert m.natoms == 128
    assert all(len(m.shell(i, 0)) == 8 for i in range(m.natoms))
    assert all(len(m.shell(i, 1)) == 6 for i in range(m.natoms))
    f, (a, b, c, ab, bc, ca) = oracle.HYPER_KAGOME_CELL
    h = oracle.Mesh(f, 4, 4, 4, a, b, c, ab, bc, ca)
    assert h.natoms == 768
    assert all(len(h.shell(i, 0)) == 4 for i in range(h.natoms))
    assert all(len(h.neighbor_list(i)) == 4 for i in range(h.natoms))


def test_small_mesh_shell_duplicates(oracle):
    # initAtomShells scans (2N+1)^3 cells with modulo wrap (src/chainMesh.f90:618-634): on a
    # 3-cell axis the +-2 cells alias the +-1 cells, so shell 1 lists each neighbour twice.
    # The legacy NeighborList de-duplicates (src/chainMesh.f90:331).
    m = oracle.Mesh.sc(3)
    assert len(m.shell(0, 0)) == 12 and len(set(m.shell(0, 0))) == 6
    assert len(m.neighbor_list(0)) == 6


@pytest.mark.parametrize("J,B,Dz", [(-1.0, 0.1, 0.3), (1.0, -0.2, 0.7), (-0.5, 0.0, 0.0)])
def test_uniform_state_energies(oracle, J, B, Dz):
    m = oracle.Mesh.sc(6)
    m.spins[:, :] = 0.0
    m.spins[:, 2] = 1.0
    N = m.natoms
    p = oracle.Params(J=J, Dz=Dz, B=B)
    # TotalHeisenbergEnergy: N*(z/2)*J - N*g*muB*B, DMI cancels for a uniform state
    assert m.total_energy(p, 2.0) == pytest.approx(N * 3 * J - N * 2 * B, abs=1e-9)
    assert m.canonical_energy(p) == pytest.approx(N * 3 * J - N * B, abs=1e-9)
    # local routine: S . (sum of neighbours) J - B S_z
    o, n = m.local_energy(5, p, np.array([0.0, 0.0, -1.0]))
    assert o == pytest.approx(6 * J - B, abs=1e-12)
    assert n == pytest.approx(-6 * J + B, abs=1e-12)


def _spiral(positions, q, kind):
    """Commensurate spiral along x: a Bloch helix (0, cos qx, sin qx) for bulk DMI, a Neel
    cycloid (sin qx, 0, cos qx) for interfacial DMI about z."""
    x = np.rint(positions[:, 0]).astype(np.float64)
    c, s = np.cos(q * x), np.sin(q * x)
    z = np.zeros_like(x)
    return np.stack([z, c, s], axis=1) if kind == "bulk" else np.stack([s, z, c], axis=1)


@pytest.mark.parametrize("kind", ["bulk", "interfacial"])
@pytest.mark.parametrize("m_q", [1, -1, 3])
def test_spin_spiral_dmi_known_answers(oracle, kind, m_q):
    """DMI sign and bond-vector convention pinned by a closed form.  With the bond vector
    r = -(r_j - r_i)/|r_j - r_i| and D = Dz r (bulk) or Dz z x r (interfacial), both x-bonds of
    a site of the spiral give D.(S_i x S_j) = -Dz sin q and J cos q, the y and z bonds J:
    energy per site J cos q - Dz sin q + 2J (the Zeeman sum vanishes over whole periods), local
    sum 2J cos q - 2 Dz sin q + 4J - B S_z."""
    L = 8
    m = oracle.Mesh.sc(L)
    q = 2.0 * np.pi * m_q / L
    m.set_spins(_spiral(m.positions(), q, kind))
    J, Dz, B = -1.0, 0.7, 0.3
    p = oracle.Params(J=J, Dz=Dz, B=B, dmi_bulk=(kind == "bulk"))
    N = m.natoms
    per_site = J * np.cos(q) - Dz * np.sin(q) + 2.0 * J
    assert m.canonical_energy(p) == pytest.approx(N * per_site, abs=1e-9)
    assert m.total_energy(p, 2.0) == pytest.approx(N * per_site, abs=1e-9)
    for atom in (0, 9, 77, N - 1):
        S = m.spins[atom].copy()
        o, n = m.local_energy(atom, p, S)
        want = 2.0 * J * np.cos(q) - 2.0 * Dz * np.sin(q) + 4.0 * J - B * S[2]
        assert o == pytest.approx(want, abs=1e-12) and n == pytest.approx(want, abs=1e-12)
    # the opposite chirality costs 2 Dz sin q more (or less) per site: DMI selects one hand
    m.set_spins(_spiral(m.positions(), -q, kind))
    assert m.canonical_energy(p) - N * per_site == pytest.approx(N * 2.0 * Dz * np.sin(q), abs=1e-9)


def test_local_delta_equals_total_difference(oracle):
    m = oracle.Mesh.sc(6)
    m.init_uniform(0x15196)
    p = oracle.Params(J=-1.0, J_prime=0.13, Dz=0.4, B=0.2, K=0.05, K_axis=(0.0, 0.6, 0.8))
    rng = np.random.default_rng(1)
    for atom in (0, 17, 101):
        sp = rng.normal(size=3)
        sp /= np.linalg.norm(sp)
        e0 = m.canonical_energy(p)
        o, n = m.local_energy(atom, p, sp)
        old = m.spins[atom].copy()
        m.spins[atom] = sp
        e1 = m.canonical_energy(p)
        m.spins[atom] = old
        assert (e1 - e0) == pytest.approx(n - o, abs=1e-10)


def test_arc_winding_octant(oracle):
    x, y, z = np.eye(3)
    assert oracle.arc_winding(x, y, z) == pytest.approx(math.pi / 2, abs=1e-14)
    assert oracle.arc_winding(x, z, y) == pytest.approx(-math.pi / 2, abs=1e-14)


def test_winding_known_answers(oracle):
    m = oracle.Mesh.sc(16, nz=4)
    m.spins[:, :] = 0.0
    m.spins[:, 2] = 1.0
    assert all(m.winding_number(z) == 0.0 for z in range(1, 5))
    # stereographic skyrmion (src/LLG.f90:28-73, N=1, chi=1.56) -> Q = -1 on every slice
    m.init_skyrmion(8.0, 8.0, 3.0, 1.56, 1)
    q = [m.winding_number(z) for z in range(1, 5)]
    assert all(round(v) == -1 for v in q)
    # mirror z -> -z of the texture flips the sign
    m.spins[:, 2] *= -1.0
    assert all(round(m.winding_number(z)) == 1 for z in range(1, 5))
    wm, ws, mag = m.statistics()
    assert round(wm) == 1 and ws < 1e-9


def test_metropolis_reference_deterministic(oracle):
    p = oracle.Params(J=-1.0, Dz=0.3, B=0.1)
    a = oracle.Mesh.sc(6)
    b = oracle.Mesh.sc(6)
    a.init_uniform(3)
    b.init_uniform(3)
    a.metropolis_mcs_ref(4.0, 5, p, 0.2)
    b.metropolis_mcs_ref(4.0, 5, p, 0.2)
    assert np.array_equal(a.spins, b.spins)
    assert np.allclose(np.linalg.norm(a.spins, axis=1), 1.0, atol=1e-12)
    e0 = b.canonical_energy(p)
    b.metropolis_mcs_ref(20.0, 30, p, 0.2)
    assert b.canonical_energy(p) < e0


def test_colour_pass_is_exact_metropolis(oracle):
    # the same key replays the same pass; accepted dE sums to the energy change
    p = oracle.Params(J=-1.0, Dz=0.3, B=0.1, dmi_bulk=True)
    m = oracle.Mesh.sc(6)
    m.init_uniform(9)
    col = oracle.checkerboard(6, 6, 6)
    key = oracle.SweepKey(seed=0x15196, ensemble=0, replica=0, move=0, r=0.0, philox_rounds=10)
    e0 = m.canonical_energy(p)
    n, de = m.colour_pass(col, 0, 0, 2.0, p, key)
    n2, de2 = m.colour_pass(col, 1, 0, 2.0, p, key)
    assert 0 < n + n2 < m.natoms
    assert m.canonical_energy(p) - e0 == pytest.approx(de + de2, abs=1e-9)


def test_pt_exchange_criterion(oracle):
    betas = np.array([2.0, 1.0, 0.5, 0.25])
    # lower energy at the hotter slot -> always swap (d >= 0)
    e = np.array([0.0, -10.0, 5.0, 4.0])
    n, t2r = oracle.pt_exchange(1, 0, 0, betas, e, [0, 1, 2, 3])
    assert n >= 1 and t2r[0] == 1 and t2r[1] == 0
    # reference block is deterministic for a seed
    T = oracle.temperature_ladder(400.0, 20000.0, 10)
    assert T[0] == pytest.approx(400.0) and T[-1] == pytest.approx(20000.0)
    tm1 = oracle.pt_swaps_ref(0, 10, T, np.linspace(-5, 5, 10), np.arange(10))
    tm2 = oracle.pt_swaps_ref(0, 10, T, np.linspace(-5, 5, 10), np.arange(10))
    assert np.array_equal(tm1, tm2) and sorted(tm1) == list(range(10))


def test_tau_int_ar1(oracle):
    rng = np.random.default_rng(0)
    rho = 0.8
    n = 200000
    x = np.empty(n)
    x[0] = 0.0
    eps = rng.normal(size=n)
    for i in range(1, n):
        x[i] = rho * x[i - 1] + eps[i]
    tau = oracle.tau_int(x[:20000])
    assert tau == pytest.approx((1 + rho) / (2 * (1 - rho)), rel=0.15)


def test_fortran_formats(oracle):
    assert oracle.fmt_F0(0.5, 4) == ".5000"
    assert oracle.fmt_F0(-0.5, 4) == "-.5000"
    assert oracle.fmt_F0(-2.5, 4) == "-2.5000"
    assert oracle.fmt_F0(400.0, 10) == "400.0000000000"
    assert oracle.fmt_E0(400.0, 4) == "0.4000E+3"
    assert oracle.fmt_E0(20000.0, 4) == "0.2000E+5"
    assert oracle.fmt_ES(2.8, 22, 14) == "  2.80000000000000E+00"
    assert oracle.fmt_ES(-1.0, 22, 14) == " -1.00000000000000E+00"
    assert oracle.fmt_I0m(0, 4) == "0000" and oracle.fmt_I0m(-3, 4) == "-0003"


def _consumer_tag(x, d=4):
    """The file-name rule of the reference's analysis script (F0.4 without the leading zero,
    E0.4 as a 0.dddd mantissa with an unpadded exponent), restated for the check."""
    s = f"{x:.{d}f}"
    if s.startswith("0"):
        s = s[1:]
    elif s.startswith("-0"):
        s = "-" + s[2:]
    return s


def test_fortran_formats_match_consumer_rule(oracle):
    for v in (-2.5, -1.25, 0.0, 0.5, 1.5, 2.0, -0.1):
        assert oracle.fmt_F0(v, 4) == _consumer_tag(v) or (v == 0.0 and oracle.fmt_F0(v, 4) == ".0000")
    for T in (400.0, 612.3, 1234.5678, 20000.0):
        e = math.floor(math.log10(T)) + 1
        assert oracle.fmt_E0(T, 4) == f"{round(T / 10 ** e, 4):.4f}E+{e}"


def test_philox_stream_statistics(oracle):
    """The device's keyed Philox4x32-10 stream (same algorithm as the oracle's, replayed
    decision for decision by the GPU parity tests): uniformity of the (0,1) floats over 64
    bins, no lag-1 correlation along sites, independence of neighbouring keys (seeds) and of
    the four words of one call."""
    L = oracle.lib()
    n = 40000
    w = np.array([oracle.philox([i, 7, 3, (5 << 8) | 0], [0x15196, 0]) for i in range(n)], dtype=np.uint64)
    w2 = np.array([oracle.philox([i, 7, 3, (5 << 8) | 0], [0x15197, 0]) for i in range(n)], dtype=np.uint64)
    u = np.array([L.ora_u01(int(x)) for x in w[:, 0]])
    h, _ = np.histogram(u, bins=64, range=(0.0, 1.0))
    chi2 = ((h - n / 64) ** 2 / (n / 64)).sum()
    assert chi2 < 120, chi2                       # 63 dof: mean 63, sd 11
    lim = 5.0 / np.sqrt(n)
    uf = (w.astype(np.float64) + 0.5) / 2.0 ** 32
    uf2 = (w2.astype(np.float64) + 0.5) / 2.0 ** 32
    assert abs(np.corrcoef(uf[:-1, 0], uf[1:, 0])[0, 1]) < lim
    assert abs(np.corrcoef(uf[:, 0], uf2[:, 0])[0, 1]) < lim
    for a in range(4):
        for b in range(a + 1, 4):
            assert abs(np.corrcoef(uf[:, a], uf[:, b])[0, 1]) < lim
    assert abs(uf.mean() - 0.5) < 5 * np.sqrt(1 / 12 / (4 * n))


@pytest.mark.parametrize("bulk,move", [(True, 1), (True, 0), (False, 1), (False, 0)])
def test_fast_cpu_checkerboard_replays_colour_pass(oracle, bulk, move):
    """The optimised FP32 CPU sweep (the fastest CPU baseline) takes the same decisions as the
    FP64 colour-class sweep with the same Philox keys: spins equal to FP32 rounding."""
    L = 8
    om = oracle.Mesh.sc(L)
    om.init_uniform(5)
    s0 = om.spins.copy()
    p = oracle.Params(J=-1.0, Dz=0.7, B=0.3, K=0.05, dmi_bulk=bulk)
    key = oracle.SweepKey(seed=0x15196, ensemble=0, replica=0, move=move, r=0.2, philox_rounds=10)
    col = oracle.checkerboard(L, L, L)
    for sw in range(2):
        om.colour_pass(col, 0, sw, 2.0, p, key)
        om.colour_pass(col, 1, sw, 2.0, p, key)
    planes = np.ascontiguousarray(s0.T.astype(np.float32))
    acc = oracle.cb_sweeps_f32(planes, L, 2, 0, 2.0, p, key, 2)
    assert acc > 0
    d = np.abs(planes.T.astype(np.float64) - om.spins).max(axis=1)
    assert (d > 1e-4).sum() <= 2 and np.median(d) < 1e-6
