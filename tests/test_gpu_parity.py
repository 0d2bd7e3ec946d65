"""GPU parity of the CUDA path (through the C-ABI) against the FP64 oracle.

Tolerances: per-site energies within 1e-6 of the site's energy scale
(|J| z1 + |Dz| z1 + |J'| z2 + |B| + |K|); total energies within 1e-6 of the sum of the
per-site scales; winding numbers within 1e-9 per slice (FP64 on the device) and rounded Q
exactly equal; sweep replays identical except at near-threshold accept decisions."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cell(oracle, kind):
    return {"SC": oracle.SC_CELL, "BCC": oracle.BCC_CELL, "HK": oracle.HYPER_KAGOME_CELL}[kind]


def _pair(oracle, ib, kind, dims, n_replicas=1):
    frac, (a, b, c, ab, bc, ca) = _cell(oracle, kind)
    om = oracle.Mesh(frac, *dims, a, b, c, ab, bc, ca)
    pm = ib.ChainMesh(*dims, frac, a, b, c, ab, bc, ca, n_replicas=n_replicas)
    return om, pm


def _random_spins(n, seed):
    rng = np.random.default_rng(seed)
    s = rng.normal(size=(n, 3))
    s /= np.linalg.norm(s, axis=1, keepdims=True)
    return s.astype(np.float32).astype(np.float64)


def _both_params(oracle, ib, J=-1.0, Jp=0.0, Dz=0.0, B=0.0, K=0.0, Kax=(0.0, 0.0, 1.0), bulk=False):
    return (oracle.Params(J=J, J_prime=Jp, Dz=Dz, B=B, K=K, K_axis=Kax, dmi_bulk=bulk),
            ib.params(J=J, J_prime=Jp, Dz=Dz, B=B, K=K, K_axis=Kax, dmi="bulk" if bulk else "interfacial"))


HAMS = [
    dict(J=-1.0, Dz=0.3, B=0.1, bulk=True),
    dict(J=-1.0, Dz=0.7, B=0.3, K=0.05, bulk=True),
    dict(J=1.0, Dz=0.5, B=-0.2, bulk=False),
    dict(J=-1.0, Jp=0.25, Dz=0.4, B=0.15, K=0.1, Kax=(0.6, 0.0, 0.8), bulk=False),
]
MESHES = [("SC", (8, 8, 8)), ("SC", (5, 6, 7)), ("BCC", (4, 4, 4)), ("HK", (3, 3, 3))]


@pytest.mark.parametrize("kind,dims", MESHES, ids=["sc8", "sc567", "bcc4", "hk3"])
@pytest.mark.parametrize("hi", range(len(HAMS)))
def test_local_energy_parity(oracle, ib, cuda_ok, kind, dims, hi):
    h = HAMS[hi]
    om, pm = _pair(oracle, ib, kind, dims)
    s = _random_spins(om.natoms, 11 + hi)
    om.set_spins(s)
    pm.set_spins(s)
    op, pp = _both_params(oracle, ib, **h)
    rng = np.random.default_rng(5)
    atoms = rng.choice(om.natoms, size=min(om.natoms, 200), replace=False)
    sp = _random_spins(len(atoms), 99)
    go, gn = ib.local_energy_batch(pm, atoms, sp, pp)
    z1 = len(om.shell(0, 0))
    z2 = len(om.shell(0, 1))
    scale = abs(h["J"]) * z1 + abs(h.get("Dz", 0)) * z1 + abs(h.get("Jp", 0)) * z2 + abs(h.get("B", 0)) + abs(h.get("K", 0))
    for k, a in enumerate(atoms):
        o, n = om.local_energy(int(a), op, sp[k])
        assert abs(go[k] - o) <= 1e-6 * scale, (a, go[k], o)
        assert abs(gn[k] - n) <= 1e-6 * scale, (a, gn[k], n)
    # the 1-based single-site entry point (calculateHeisenbergEnergy signature)
    o1, n1 = ib.calculate_heisenberg_energy(pm, int(atoms[0]) + 1, 0, 0, 0, 0, 0, sp[0], p=pp)
    assert o1 == pytest.approx(go[0], abs=0) and n1 == pytest.approx(gn[0], abs=0)


@pytest.mark.parametrize("kind,dims", MESHES, ids=["sc8", "sc567", "bcc4", "hk3"])
def test_total_energy_parity(oracle, ib, cuda_ok, kind, dims):
    om, pm = _pair(oracle, ib, kind, dims)
    s = _random_spins(om.natoms, 3)
    om.set_spins(s)
    pm.set_spins(s)
    # reference TotalHeisenbergEnergy convention: legacy list, D axis z, g*muB*B, no J'
    op = oracle.Params(J=-1.0, Dz=0.4, B=0.2)
    e_ref = om.total_energy(op, 2.0)
    e_gpu = ib.total_heisenberg_energy(pm, -1.0, 0.0, 0.4, 0.0, 0.2)
    z = len(om.neighbor_list(0))
    tol = 1e-6 * om.natoms * (1.0 * z + 0.4 * z + 0.4)
    assert abs(e_gpu - e_ref) <= tol
    # canonical form (the Hamiltonian the sweep samples)
    for h in HAMS:
        op, pp = _both_params(oracle, ib, **h)
        e_ref = om.canonical_energy(op)
        e, m = ib.observables(pm, pp)
        z1, z2 = len(om.shell(0, 0)), len(om.shell(0, 1))
        scale = abs(h["J"]) * z1 + abs(h.get("Dz", 0)) * z1 + abs(h.get("Jp", 0)) * z2 + abs(h.get("B", 0)) + abs(h.get("K", 0))
        assert abs(e[0] - e_ref) <= 1e-6 * om.natoms * scale
        assert np.allclose(m[0], s.sum(axis=0), atol=1e-9 * om.natoms)


def _random_energy_cases(n=8, seed=4242):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        kind = ["SC", "BCC", "HK", "SC"][i % 4]
        hi = 5 if kind == "HK" else 8
        dims = tuple(int(v) for v in rng.integers(3, hi, size=3))
        ax = rng.normal(size=3)
        ax /= np.linalg.norm(ax)
        h = dict(J=float(rng.choice([-1.0, 1.0]) * rng.uniform(0.5, 1.5)), Jp=float(rng.uniform(-0.3, 0.3)),
                 Dz=float(rng.uniform(0.0, 1.0)), B=float(rng.uniform(-0.5, 0.5)), K=float(rng.uniform(0.0, 0.2)),
                 Kax=tuple(float(v) for v in ax), bulk=bool(i % 2))
        out.append((kind, dims, h))
    return out


@pytest.mark.parametrize("case", range(8))
def test_energy_parity_on_random_shapes_and_hamiltonians(oracle, ib, cuda_ok, case):
    """Seeded random meshes (SC, BCC, hyper-kagome; 3-7 cells per side, odd sizes taking the
    general-colouring path) and random Hamiltonians: per-site energies of 200 random proposals
    and the canonical total energy equal the oracle's within 1e-6 of the energy scale."""
    kind, dims, h = _random_energy_cases()[case]
    om, pm = _pair(oracle, ib, kind, dims)
    s = _random_spins(om.natoms, 100 + case)
    om.set_spins(s)
    pm.set_spins(s)
    op, pp = _both_params(oracle, ib, **h)
    rng = np.random.default_rng(case)
    atoms = rng.choice(om.natoms, size=min(om.natoms, 200), replace=False)
    sp = _random_spins(len(atoms), 300 + case)
    go, gn = ib.local_energy_batch(pm, atoms, sp, pp)
    z1, z2 = len(om.shell(0, 0)), len(om.shell(0, 1))
    scale = abs(h["J"]) * z1 + h["Dz"] * z1 + abs(h["Jp"]) * z2 + abs(h["B"]) + h["K"]
    for k, a in enumerate(atoms):
        o, n = om.local_energy(int(a), op, sp[k])
        assert abs(go[k] - o) <= 1e-6 * scale and abs(gn[k] - n) <= 1e-6 * scale, (a, go[k], o, gn[k], n)
    e, _m = ib.observables(pm, pp)
    assert abs(e[0] - om.canonical_energy(op)) <= 1e-6 * om.natoms * scale


def test_init_uniform_matches_oracle(oracle, ib, cuda_ok):
    om, pm = _pair(oracle, ib, "SC", (6, 6, 6), n_replicas=3)
    pm.init_uniform(0x15196, ensemble=5)
    for r in range(3):
        om.init_uniform(0x15196, 5, r)
        g = pm.get_spins(r)
        assert np.allclose(g, om.spins, atol=2e-6)
        assert np.allclose(np.linalg.norm(g, axis=1), 1.0, atol=1e-6)


@pytest.mark.parametrize("kind", ["bulk", "interfacial"])
def test_spin_spiral_energy_known_answer_at_l128(ib, cuda_ok, kind):
    """The device energy of a commensurate spiral at L=128 equals the closed form
    N (J cos q - Dz sin q + 2J) that pins the oracle's DMI convention (tests/test_oracle.py)."""
    L = 128
    pm = ib.ChainMesh.simple_cubic(L)
    q = 2.0 * np.pi * 5 / L
    x = np.rint(pm.positions()[:, 0]).astype(np.float64)
    c, s_, z = np.cos(q * x), np.sin(q * x), np.zeros_like(x)
    spins = np.stack([z, c, s_], axis=1) if kind == "bulk" else np.stack([s_, z, c], axis=1)
    pm.set_spins(spins)
    J, Dz, B = -1.0, 0.7, 0.3
    e, _m = ib.observables(pm, ib.params(J=J, Dz=Dz, B=B, dmi=kind, include_Jp=False))
    N = pm.numAtoms
    want = N * (J * np.cos(q) - Dz * np.sin(q) + 2.0 * J)
    assert abs(e[0] - want) <= 1e-6 * N * (6 * abs(J) + 6 * Dz + B)


@pytest.mark.parametrize("kind,dims", [("SC", (8, 8, 6)), ("BCC", (4, 4, 4)), ("HK", (3, 3, 4))])
def test_winding_parity(oracle, ib, cuda_ok, kind, dims):
    om, pm = _pair(oracle, ib, kind, dims)
    s = _random_spins(om.natoms, 21)
    om.set_spins(s)
    pm.set_spins(s)
    q = ib.winding_all_slices(pm)
    for z in range(1, dims[2] + 1):
        assert abs(q[z - 1] - om.winding_number(z)) <= 1e-9
        assert ib.calculate_winding_number2(pm, z) == q[z - 1]
    wm, ws, mag = ib.chain_mesh_statistics(pm)
    owm, ows, omag = om.statistics()
    assert abs(wm - owm) <= 1e-9 and abs(ws - ows) <= 1e-9
    assert np.allclose(mag, omag, atol=1e-9)
    d = ib.calculate_winding_number_density(pm, 2)
    assert np.allclose(d, om.winding_density(2), atol=1e-12)


@pytest.mark.parametrize("kind,dims", [("SC", (8, 6, 5)), ("BCC", (4, 5, 3)), ("HK", (3, 3, 4))])
def test_winding_density_all_slices(oracle, ib, cuda_ok, kind, dims):
    """All slices in one launch equal the oracle's per-slice density (rsp:438-500), and each
    slice sums to that slice's winding number."""
    om, pm = _pair(oracle, ib, kind, dims)
    s = _random_spins(om.natoms, 33)
    om.set_spins(s)
    pm.set_spins(s)
    d = ib.winding_density_all_slices(pm)
    assert d.shape == dims
    q = ib.winding_all_slices(pm)
    for z in range(1, dims[2] + 1):
        assert np.allclose(d[:, :, z - 1], om.winding_density(z), rtol=0, atol=1e-12)
        assert np.array_equal(d[:, :, z - 1], ib.calculate_winding_number_density(pm, z))
        assert abs(d[:, :, z - 1].sum() - q[z - 1]) <= 1e-9


def test_winding_density_csv_bytes(oracle, ib, cuda_ok, tmp_path):
    """write_winding_number_density (rsp:544-580): header, "x,y,z,d" records in F0.8 with the
    record's own new_line plus the trimmed buffer's, in (z, x, y) order, and a terminator."""
    dims = (5, 4, 3)
    om, pm = _pair(oracle, ib, "BCC", dims)
    s = _random_spins(om.natoms, 4)
    om.set_spins(s)
    pm.set_spins(s)
    path = tmp_path / "density.csv"
    ib.write_winding_number_density(pm, str(path))
    av, bv, cv = om.vectors()[:3]
    out = ["x,y,z,Winding_Density\n"]
    for i in range(1, dims[2] + 1):
        dens = om.winding_density(i)
        for j in range(1, dims[0] + 1):
            for k in range(1, dims[1] + 1):
                pos = (j * av + k * bv) + i * cv
                f = [oracle.fmt_F0(float(v), 8) for v in (*pos, dens[j - 1, k - 1])]
                out.append(",".join(f) + "\n\n")
    out.append("\n")
    assert path.read_text() == "".join(out)


def test_skyrmion_winding_rounds_exactly(oracle, ib, cuda_ok):
    om, pm = _pair(oracle, ib, "SC", (16, 16, 4))
    om.init_skyrmion(8.0, 8.0, 3.0, 1.56, 1)
    pm.set_spins(om.spins.copy())
    q = ib.winding_all_slices(pm)
    assert [round(v) for v in q] == [round(om.winding_number(z)) for z in range(1, 5)] == [-1] * 4
    with pytest.raises(ib.IsingError) as e:
        ib.calculate_winding_number2(pm, 5)
    assert e.value.status == 3


REPLAYS = [("SC", (8, 8, 8), dict(J=-1.0, Dz=0.3, B=0.1, bulk=True), 0, 0.0, 1.5),
           ("SC", (8, 8, 8), dict(J=-1.0, Dz=0.5, B=0.2, bulk=True), 1, 0.2, 2.0),
           ("SC", (8, 8, 8), dict(J=-1.0, Dz=0.7, B=0.3, K=0.05, bulk=False), 0, 0.0, 3.0),
           ("SC", (6, 6, 6), dict(J=-1.0, Jp=0.2, Dz=0.3, B=0.1, bulk=True), 1, 0.3, 1.0),
           ("SC", (5, 5, 5), dict(J=-1.0, Dz=0.3, B=0.1, bulk=True), 0, 0.0, 1.0),
           ("BCC", (4, 4, 4), dict(J=-1.0, Dz=0.3, B=0.1, bulk=True), 0, 0.0, 1.0),
           ("HK", (3, 3, 3), dict(J=-1.0, Dz=0.3, B=0.1, bulk=False), 1, 0.2, 1.0)]


def _random_replays(n=6, seed=777):
    """Seeded random replay cases: cell, shape (odd sizes take the general colouring),
    Hamiltonian, move, ball radius and beta."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        kind = ["SC", "BCC", "SC", "HK", "SC", "BCC"][i]
        hi = 5 if kind == "HK" else 9
        dims = tuple(int(v) for v in rng.integers(3, hi, size=3))
        h = dict(J=-float(rng.uniform(0.5, 1.5)), Jp=float(rng.uniform(0.0, 0.2)) if i % 3 == 0 else 0.0,
                 Dz=float(rng.uniform(0.1, 0.8)), B=float(rng.uniform(0.0, 0.4)), K=float(rng.uniform(0.0, 0.1)),
                 bulk=bool(i % 2))
        move = int(i % 2)
        out.append((kind, dims, h, move, 0.25 if move else 0.0, float(rng.uniform(0.5, 3.0))))
    return out


REPLAYS = REPLAYS + _random_replays()


@pytest.mark.parametrize("case", range(len(REPLAYS)))
def test_sweep_replay(oracle, ib, cuda_ok, case):
    """One GPU sweep against the oracle's colour passes with the same Philox keys and the
    product's colouring; decisions may differ only where |ln u + beta dE| is tiny."""
    kind, dims, h, move, r, beta = REPLAYS[case]
    om, pm = _pair(oracle, ib, kind, dims)
    s = _random_spins(om.natoms, 40 + case)
    om.set_spins(s)
    pm.set_spins(s)
    op, pp = _both_params(oracle, ib, **h)
    col, ncol = pm.colouring(pp)
    seed = 0xBEEF + case
    ib.metropolis_mcs(pm, beta, 1, 0, 0, 0, 0, 0, r if move == 1 else 0.0, seed=seed, p=pp)
    key = oracle.SweepKey(seed=seed, ensemble=0, replica=0, move=move, r=r, philox_rounds=10)
    margins = np.full(om.natoms, np.inf)
    for c in range(ncol):
        _, _, acc, marg = om.colour_pass(col, c, 0, beta, op, key, want_detail=True)
        sel = col == c
        margins[sel] = marg[sel]
    g = pm.get_spins(0)
    diff = np.abs(g - om.spins).max(axis=1)
    bad = np.nonzero(diff > 2e-5)[0]
    assert len(bad) <= max(2, om.natoms // 500), (len(bad), diff.max())
    first_class_bad = [a for a in bad if col[a] == 0]
    assert all(abs(margins[a]) < 1e-3 for a in first_class_bad)
    # second run continues the counter (sweep 1): the stream must not repeat sweep 0
    before = pm.get_spins(0)
    ib.metropolis_mcs(pm, beta, 1, 0, 0, 0, 0, 0, r if move == 1 else 0.0, seed=seed, p=pp)
    assert not np.array_equal(before, pm.get_spins(0))


def test_pt_exchange_and_accumulators(oracle, ib, cuda_ok):
    om, pm = _pair(oracle, ib, "SC", (8, 8, 8), n_replicas=6)
    pm.init_uniform(7)
    op, pp = _both_params(oracle, ib, J=-1.0, Dz=0.5, B=0.2, bulk=True)
    T = ib.temperature_ladder(0.2, 2.0, 6)
    betas = 1.0 / T
    pt = ib.ParallelTempering(pm, betas, pp, seed=77, move=ib._lib.MOVE_BALL, r=0.2)
    perm = np.arange(6)
    for rnd in range(6):
        pt.run(3, 1)
        e, m = pt.energies()
        n, perm = oracle.pt_exchange(77, 0, rnd, betas, e, perm)
        assert np.array_equal(pt.permutation(), perm), rnd
    # running FP64 accumulators agree with a fresh reduction of the spins
    e_run, m_run = pt.energies()
    e_new, m_new = ib.observables(pm, pp)
    assert np.allclose(e_run, e_new[:6], atol=1e-3) and np.allclose(m_run, m_new[:6], atol=1e-3)
    for r_ in range(6):
        om.set_spins(pm.get_spins(r_))
        assert abs(om.canonical_energy(op) - e_new[r_]) <= 1e-6 * om.natoms * (6 + 3 + 0.2)
    att, acc = pt.swap_stats()
    assert att.sum() > 0 and np.all(acc <= att)


def test_error_paths(ib, cuda_ok):
    pm = ib.ChainMesh.simple_cubic(6)
    s = _random_spins(pm.numAtoms, 1)
    s[10] = np.nan
    with pytest.raises(ib.IsingError) as e:
        pm.set_spins(s)
    assert e.value.status == 2
    s[10] = 0.0
    with pytest.raises(ib.IsingError) as e:
        pm.set_spins(s)
    assert e.value.status == 2
    with pytest.raises(ib.IsingError) as e:
        pm.get_spins(3)
    assert e.value.status == 3
    with pytest.raises(ib.IsingError) as e:
        ib.calculate_heisenberg_energy(pm, pm.numAtoms + 1, -1, 0, 0, 0, 0, [0, 0, 1.0])
    assert e.value.status == 3


def test_async_spin_transfers(ib, cuda_ok):
    """Queued downloads and uploads equal the synchronous ones; an upload after a download of
    the same replica and host array waits for it; later calls wait for queued transfers;
    invalid uploads are reported by the wait."""
    import torch
    L, R = 8, 3
    pm = ib.ChainMesh.simple_cubic(L, n_replicas=R)
    pm.init_uniform(11, 2)
    N = pm.numAtoms
    ref = [pm.get_spins(r).copy() for r in range(R)]
    host = [torch.empty(3 * N, dtype=torch.float64, pin_memory=True) for _ in range(R)]
    for r in range(R):
        pm.get_spins_async(host[r].data_ptr(), r)
    pm.wait_spins()
    for r in range(R):
        np.testing.assert_array_equal(host[r].numpy().reshape(3, N).T, ref[r])
    # download and upload again from the same host arrays without a host wait: a round trip
    new = _random_spins(N, 5)
    pm.set_spins(new, 1)
    for r in range(R):
        pm.get_spins_async(host[r].data_ptr(), r)
    for r in range(R):
        pm.set_spins_async(host[r].data_ptr(), (r + 1) % R)     # rotate replicas r -> r+1
    got = [pm.get_spins(r) for r in range(R)]                   # waits for the queued transfers
    want = [ref[0], new, ref[2]]
    for r in range(R):
        np.testing.assert_array_equal(got[(r + 1) % R], want[r])
    # an upload followed by a download of the same replica sees the upload
    h2 = torch.from_numpy(np.ascontiguousarray(ref[2].T).reshape(-1)).pin_memory()
    pm.set_spins_async(h2.data_ptr(), 0)
    pm.get_spins_async(host[0].data_ptr(), 0)
    pm.wait_spins()
    np.testing.assert_array_equal(host[0].numpy().reshape(3, N).T, ref[2])
    # an invalid upload is reported by the wait
    bad = h2.clone().pin_memory()
    bad[7] = float("nan")
    pm.set_spins_async(bad.data_ptr(), 2)
    with pytest.raises(ib.IsingError) as e:
        pm.wait_spins()
    assert e.value.status == 2


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_async_transfers_follow_program_order_per_replica(ib, cuda_ok, seed):
    """Random sequences of queued downloads and uploads (one pinned host array per replica),
    waits, host edits after a wait and synchronous reads leave the device spins and every
    host array exactly as executing the calls one by one would."""
    import torch
    R, L = 4, 8
    pm = ib.ChainMesh.simple_cubic(L, n_replicas=R)
    pm.init_uniform(seed, 1)
    N = pm.numAtoms
    rng = np.random.default_rng(seed)
    dev = [pm.get_spins(r).copy() for r in range(R)]                  # model of the device
    host_t = [torch.zeros(3 * N, dtype=torch.float64).pin_memory() for _ in range(R)]
    host = [np.zeros((N, 3)) for _ in range(R)]                        # model of the host arrays
    view = lambda r: host_t[r].numpy().reshape(3, N).T
    for r in range(R):                     # every host array starts as a copy of its replica
        pm.get_spins_async(host_t[r].data_ptr(), r)
        host[r] = dev[r].copy()
    pm.wait_spins()
    for _ in range(60):
        op = rng.choice(["get", "set", "wait", "sync_get"], p=[0.4, 0.35, 0.15, 0.1])
        r = int(rng.integers(R))
        if op == "get":
            pm.get_spins_async(host_t[r].data_ptr(), r)
            host[r] = dev[r].copy()
        elif op == "set":
            pm.set_spins_async(host_t[r].data_ptr(), r)
            dev[r] = host[r].copy()
        elif op == "wait":
            pm.wait_spins()
            for q in range(R):
                np.testing.assert_array_equal(view(q), host[q])
            q = int(rng.integers(R))                                  # the host edits an array
            new = _random_spins(N, int(rng.integers(1 << 30)))
            view(q)[:] = new
            host[q] = new
        else:
            np.testing.assert_array_equal(pm.get_spins(r), dev[r])   # waits for the queue
    pm.wait_spins()
    for r in range(R):
        np.testing.assert_array_equal(view(r), host[r])
        np.testing.assert_array_equal(pm.get_spins(r), dev[r])


def test_async_uploads_feed_the_engine(ib, cuda_ok):
    """An engine run after queued uploads (no explicit wait) sweeps the uploaded spins: the
    result equals the run after synchronous uploads."""
    import torch
    spec_p = ib.params(J=-1.0, Dz=0.5, B=0.2, dmi="bulk", include_Jp=False)
    betas = 1.0 / ib.temperature_ladder(0.3, 1.5, 2)
    out = []
    for use_async in (False, True):
        m = ib.ChainMesh.simple_cubic(8, n_replicas=2)
        m.init_uniform(3, 9)
        s = [_random_spins(m.numAtoms, 40 + r) for r in range(2)]
        if use_async:
            hs = [torch.from_numpy(np.ascontiguousarray(v.T).reshape(-1)).pin_memory() for v in s]
            for r in range(2):
                m.set_spins_async(hs[r].data_ptr(), r)
        else:
            for r in range(2):
                m.set_spins(s[r], r)
        eng = ib.Ensembles([(m, betas, spec_p, 9)], seed=21)
        eng.run(2, 2)
        out.append([m.get_spins(r) for r in range(2)])
        eng.close()
    for r in range(2):
        np.testing.assert_array_equal(out[0][r], out[1][r])


def test_empty_and_null_inputs(ib, cuda_ok):
    """Empty batches are no-ops; NULL buffers and out-of-range replicas are argument errors."""
    from ising_b200 import _lib
    pm = ib.ChainMesh.simple_cubic(6)
    old, new = ib.local_energy_batch(pm, np.zeros(0, np.int64), np.zeros((0, 3)), ib.params(J=-1.0))
    assert old.shape == (0,) and new.shape == (0,)
    L = _lib.load()
    assert L.ising_spins_set(pm.handle, 0, None) == 1
    assert L.ising_spins_get(pm.handle, 0, None) == 1
    assert L.ising_spins_set(pm.handle, 1, None) in (1, 3)
    em = ib.ChainMesh.simple_cubic(8)           # the engine needs nz % 4 == 0
    em.init_uniform(7, 1)
    spec = [(em, 1.0 / ib.temperature_ladder(0.5, 1.0, 1), ib.params(J=-1.0, Dz=0.3, dmi="bulk", include_Jp=False), 1)]
    before = em.get_spins(0).copy()
    eng = ib.Ensembles(spec, seed=7)
    eng.run(2, 0)                       # zero rounds: nothing runs, nothing changes
    np.testing.assert_array_equal(em.get_spins(0), before)
    eng.close()


def test_spins_csv_bytes(oracle, ib, cuda_ok, tmp_path):
    om, pm = _pair(oracle, ib, "BCC", (3, 3, 3))
    s = _random_spins(om.natoms, 8)
    pm.set_spins(s)
    path = tmp_path / "spins.csv"
    ib.write_spins_to_file(pm, str(path), frame_index=3)
    g = pm.get_spins(0)
    pos = om.positions()
    lines = ["# Frame: 3", "x,y,z,Sx,Sy,Sz"]
    for i in range(om.natoms):
        vals = [float(pos[i, 0]), float(pos[i, 1]), float(pos[i, 2]), g[i, 0], g[i, 1], g[i, 2]]
        lines.append(",".join(oracle.fmt_ES(v, 22, 14) for v in vals))
    assert path.read_text() == "\n".join(lines) + "\n"
    ib.write_spins_to_file(pm, str(path), append=True, include_header=False)
    assert path.read_text().count("\n") == 2 + 2 * om.natoms


def test_spins_csv_bytes_threaded(oracle, ib, cuda_ok, tmp_path):
    """A mesh large enough for the writer to split its records over several host threads:
    the file is still the sequential ES22.14 text."""
    om, pm = _pair(oracle, ib, "SC", (24, 24, 24))
    s = _random_spins(om.natoms, 12)
    pm.set_spins(s)
    path = tmp_path / "spins.csv"
    ib.write_spins_to_file(pm, str(path))
    g = pm.get_spins(0)
    pos = om.positions()
    lines = ["x,y,z,Sx,Sy,Sz"]
    for i in range(om.natoms):
        vals = [float(pos[i, 0]), float(pos[i, 1]), float(pos[i, 2]), g[i, 0], g[i, 1], g[i, 2]]
        lines.append(",".join(oracle.fmt_ES(v, 22, 14) for v in vals))
    assert path.read_text() == "\n".join(lines) + "\n"


def test_observables_match_oracle_statistically(oracle, ib, cuda_ok):
    """Plain single-spin Metropolis at equal observables: GPU chain vs the FP64 oracle chain
    (independent seeds), <E>/N and <|M|>/N within 3 combined binning standard errors."""
    from ising_b200.analysis import binning_error
    L, beta = 8, 1.0
    op, pp = _both_params(oracle, ib, J=-1.0, Dz=0.3, B=0.1, bulk=True)
    om = oracle.Mesh.sc(L)
    pm = ib.ChainMesh.simple_cubic(L)
    om.init_uniform(1)
    pm.init_uniform(2)
    n_therm, n_meas = 300, 3000
    pt = ib.ParallelTempering(pm, [beta], pp, seed=5, move=ib._lib.MOVE_UNIFORM, record=True,
                              record_capacity=n_therm + n_meas)
    pt.run(1, n_therm + n_meas)
    ser = pt.series()[0]
    eg = ser[n_therm:, 0] / om.natoms
    mg = ser[n_therm:, 1]
    col = oracle.checkerboard(L, L, L)
    key = oracle.SweepKey(seed=12345, ensemble=0, replica=0, move=0, r=0.0, philox_rounds=10)
    eo, mo = [], []
    for sw in range(n_therm + n_meas):
        om.colour_pass(col, 0, sw, beta, op, key)
        om.colour_pass(col, 1, sw, beta, op, key)
        if sw >= n_therm:
            eo.append(om.canonical_energy(op) / om.natoms)
            mo.append(np.linalg.norm(om.spins.sum(axis=0)) / om.natoms)
    for a, b in ((eg, np.array(eo)), (mg, np.array(mo))):
        z = abs(a.mean() - b.mean()) / np.hypot(binning_error(a), binning_error(b))
        assert z < 3.0, z
