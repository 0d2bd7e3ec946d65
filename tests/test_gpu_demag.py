"""The demagnetising field on the device (ising_demag_field, calculate_demagnetisation_field of
src/reciprocalSpaceProcesses.f90:202-281) against the FP64 numpy restatement in the oracle, on
simple-cubic, BCC and hyper-kagome meshes with odd and even extents; its energy terms in the
total energy (-1/2 mu_0 S.H) and the local energy (-mu_0 S.H); Metropolis sweeps with the
field on; parallel tempering refusing it."""
import numpy as np
import pytest

from test_gpu_parity import _both_params, _pair, _random_spins

pytestmark = pytest.mark.gpu

MESHES = [("SC", (8, 8, 8)), ("SC", (5, 6, 7)), ("BCC", (6, 4, 4)), ("HK", (3, 4, 3)), ("HK", (4, 4, 4))]


@pytest.mark.parametrize("kind,dims", MESHES, ids=["sc8", "sc567", "bcc644", "hk343", "hk444"])
def test_demag_field_matches_oracle(oracle, ib, cuda_ok, kind, dims):
    from oracle import demag_ref as D
    om, pm = _pair(oracle, ib, kind, dims, n_replicas=2)
    s = _random_spins(om.natoms, 71)
    pm.set_spins(s, 1)
    H = ib.demag_field(pm, 1)
    Href = D.demag_field(om, s)
    scale = np.abs(Href).max()
    assert scale > 1e-3
    np.testing.assert_allclose(H, Href, rtol=0, atol=1e-10 * scale)
    again = ib.demag_field(pm, 1)          # the workspace is reused: the same field again
    np.testing.assert_array_equal(again, H)


def test_demag_energy_terms(oracle, ib, cuda_ok):
    from oracle import demag_ref as D
    om, pm = _pair(oracle, ib, "BCC", (6, 6, 4))
    s = _random_spins(om.natoms, 72)
    pm.set_spins(s)
    op, pp = _both_params(oracle, ib, J=-1.0, Dz=0.3, B=0.1)
    _, pd = _both_params(oracle, ib, J=-1.0, Dz=0.3, B=0.1)
    pd.demag = 1
    e_off, _ = ib.observables(pm, pp)
    e_on, _ = ib.observables(pm, pd)
    Href = D.demag_field(om, s)
    de = D.demag_energy(s, Href)
    assert abs((e_on[0] - e_off[0]) - de) < 1e-9 * abs(de) + 1e-15
    atoms = np.arange(0, om.natoms, 5)
    sp = _random_spins(len(atoms), 73)
    o0, n0 = ib.local_energy_batch(pm, atoms, sp, pp)
    o1, n1 = ib.local_energy_batch(pm, atoms, sp, pd)
    mu0 = D.MU_0
    np.testing.assert_allclose(o1 - o0, -mu0 * (s[atoms] * Href[atoms]).sum(1), rtol=1e-6, atol=1e-18)
    np.testing.assert_allclose(n1 - n0, -mu0 * (sp * Href[atoms]).sum(1), rtol=1e-6, atol=1e-18)


def test_metropolis_with_demag_and_pt_refusal(oracle, ib, cuda_ok):
    om, pm = _pair(oracle, ib, "SC", (8, 8, 8), n_replicas=2)
    pm.init_uniform(5)
    _, pd = _both_params(oracle, ib, J=-1.0, Dz=0.3, B=0.1, bulk=True)
    pd.demag = 1
    before = pm.get_spins(0)
    ib.metropolis_mcs(pm, 2.0, 40, 0, 0, 0, 0, 0, 0.2, seed=9, p=pd)     # field recomputed every 17 sweeps
    after = pm.get_spins(0)
    assert not np.array_equal(before, after)
    assert np.max(np.abs(np.linalg.norm(after, axis=1) - 1.0)) < 1e-5
    with pytest.raises(ib.IsingError) as e:
        ib.ParallelTempering(pm, [1.0, 2.0], pd)
    assert e.value.status == 5           # ISING_ERR_UNSUPPORTED


def test_demag_csv_bytes(oracle, ib, cuda_ok, tmp_path):
    """write_demagnetisation_field_to_file: header and one F8.4 record per atom (position as
    stored in single precision, field components), asterisks where a value does not fit."""
    om, pm = _pair(oracle, ib, "BCC", (4, 4, 4))
    s = _random_spins(om.natoms, 74)
    pm.set_spins(s)
    path = tmp_path / "demag.csv"
    ib.write_demagnetisation_field_to_file(pm, str(path))
    H = ib.demag_field(pm, 0)
    pos = om.positions().astype(np.float64)

    def f84(v):
        t = "%8.4f" % v
        return "*" * 8 if len(t) > 8 else t
    lines = ["x,y,z,fx,fy,fz"]
    for i in range(om.natoms):
        lines.append(",".join(f84(v) for v in (pos[i, 0], pos[i, 1], pos[i, 2], H[i, 0], H[i, 1], H[i, 2])))
    assert path.read_text() == "\n".join(lines) + "\n"
