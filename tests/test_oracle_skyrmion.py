"""CPU tests of the oracle's skyrmion-counting restatement (rsp:366-436,582-983) against
known answers: the interpolation through the coarse samples, exact band-limited signals, the
integer charge of a closed fine lattice, the filter kernel, and hand-checked region counts."""
import math

import numpy as np
import pytest


def test_spectral_upsample_passes_through_samples(oracle):
    rng = np.random.default_rng(3)
    for nx, ny, sx, sy in ((6, 5, 3, 4), (7, 8, 2, 2), (4, 4, 10, 10)):
        f = rng.normal(size=(nx, ny, 3))
        g = oracle.spectral_upsample(f, sx, sy)
        assert g.shape == (nx * sx, ny * sy, 3)
        assert np.abs(g[::sx, ::sy] - f).max() < 1e-12


def test_spectral_upsample_is_exact_on_band_limited_signals(oracle):
    nx, ny, sx, sy = 8, 6, 3, 5
    X = np.arange(nx * sx) / (nx * sx)
    Y = np.arange(ny * sy) / (ny * sy)
    x, y = np.arange(nx) / nx, np.arange(ny) / ny
    # frequencies strictly below Nyquist on both axes
    f = np.cos(2 * np.pi * 3 * x)[:, None] * np.sin(2 * np.pi * 2 * y)[None, :] + 0.5
    g = oracle.spectral_upsample(np.repeat(f[:, :, None], 3, axis=2), sx, sy)[:, :, 0]
    ref = np.cos(2 * np.pi * 3 * X)[:, None] * np.sin(2 * np.pi * 2 * Y)[None, :] + 0.5
    assert np.abs(g - ref).max() < 1e-12


def test_fine_density_charge_is_the_coarse_charge(oracle):
    """A closed periodic lattice's Berg-Luscher charges sum to an integer; for a smooth
    skyrmion the fine grid keeps the coarse slice's charge."""
    m = oracle.Mesh.sc(16, 16, 4)
    m.init_skyrmion(8.0, 8.0, 3.0, 1.56, 1)
    q = m.winding_number(2)
    pi_ratio = float(np.float32(math.pi)) / math.pi   # densities divide by 4 pi with float pi
    for s in (2, 3, 5):
        d = oracle.winding_density_interpolated(m, 2, s, s)
        assert d.shape == (16 * s, 16 * s)
        t = d.sum() * pi_ratio
        assert abs(t - round(t)) < 1e-9
        assert round(t) == round(q) == -1


def test_gaussian_kernel(oracle):
    for sigma in (1.0, 0.5, 0.05, 1e-5):
        G = oracle.gaussian_kernel(sigma)
        assert abs(G.sum() - 1.0) < 1e-15
        assert np.array_equal(G, G.T) and np.array_equal(G, G[::-1, ::-1])
        num = np.add.outer((np.arange(5) - 2) ** 2, (np.arange(5) - 2) ** 2)
        e = np.exp(-num / (2 * sigma ** 2))
        assert np.allclose(G, e / e.sum(), rtol=1e-14, atol=0)
    # sigma -> 0: the centre weight only
    assert oracle.gaussian_kernel(1e-5)[2, 2] == 1.0


def test_gaussian_filter_is_shifted_by_three(oracle):
    """buffer(i,j) = sum array(i-l, j-m) G(l,m), l,m = 1..5: a delta at (a,b) lands centred on
    (a+3, b+3) (periodic), the reference's offset."""
    a = np.zeros((9, 7))
    a[2, 1] = 1.0
    b = oracle.gaussian_filter_2d(a, 0.7)
    assert np.unravel_index(np.argmax(b), b.shape) == ((2 + 3) % 9, (1 + 3) % 7)
    assert abs(b.sum() - 1.0) < 1e-15
    with pytest.raises(ValueError):
        oracle.gaussian_filter_2d(np.zeros((4, 9)), 0.5)


def test_skyrmion_number_hand_cases(oracle):
    # all-zero density: no cell passes the mask
    assert oracle.skyrmion_number(np.zeros((20, 20)), 10, 10, 0.3, 1, 0.5) == (0, 0)
    # q_threshold outside [0, 1]
    assert oracle.skyrmion_number(np.zeros((20, 20)), 10, 10, 1.5, 1, 0.5)[0] == 1
    assert oracle.skyrmion_number(np.zeros((20, 20)), 10, 10, -0.1, 1, 0.5)[0] == 1
    # one cell of charge 1 inside the first coarse block, sigma -> 0 (the filter moves it by
    # (3,3)): one region of one cell with sum 1 -> one skyrmion; charge -1 -> -1
    for sgn in (1.0, -1.0):
        d = np.zeros((20, 20))
        d[1, 2] = sgn
        assert oracle.skyrmion_number(d, 10, 10, 0.5, 1, 1e-5) == (0, int(sgn))
    # the same cell outside the first block: the local-maximum test compares it with cells of
    # the coarse block (all zero), it starts a region of its own and still counts
    d = np.zeros((20, 20))
    d[14, 12] = 1.0
    assert oracle.skyrmion_number(d, 10, 10, 0.5, 1, 1e-5) == (0, 1)
    # two half charges on neighbouring cells in the first block: the second is downhill of
    # the first, so one region of two cells with sum 1, counted once per cell -> 2
    d = np.zeros((20, 20))
    d[2, 2] = 0.5
    d[2, 3] = 0.5
    assert oracle.skyrmion_number(d, 10, 10, 0.5, 1, 1e-5) == (0, 2)


def test_skyrmion_distribution_on_hand_case(oracle):
    d = np.zeros((20, 20))
    d[1, 2] = 1.0
    st, w = oracle.skyrmion_distribution(d, 10, 10, 1.0, 2, 1e-5, 0.95, 60)
    assert st == 0 and w == [1, 0]
    st, _ = oracle.skyrmion_distribution(d, 10, 10, 1.0, 1, 0.9, 0.1, 60)
    assert st == 5


def _bloch_texture(L, nz, R, centres):
    """z-uniform Bloch skyrmions of radius R (theta = pi (1 - r/R) inside, core down) on a
    uniform background: total winding number +1 per skyrmion."""
    x, y = np.meshgrid(np.arange(L, dtype=np.float64), np.arange(L, dtype=np.float64), indexing="ij")
    theta, phi = np.zeros((L, L)), np.zeros((L, L))
    for cx, cy in centres:
        dx = (x - cx + L / 2) % L - L / 2
        dy = (y - cy + L / 2) % L - L / 2
        r = np.hypot(dx, dy)
        inside = r < R
        theta = np.where(inside, np.pi * (1.0 - r / R), theta)
        phi = np.where(inside, np.arctan2(dy, dx) + np.pi / 2, phi)
    s = np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), -np.cos(theta)], axis=-1)
    return np.repeat(s[:, :, None, :], nz, axis=2).reshape(-1, 3)


KNOWN_TEXTURES = {
    # the reference's own test skyrmion (src/ISING.f90:131-137: centre mid-mesh, R_s = a,
    # chi = 3.12/2, N = 1; src/LLG.f90:28-73): winding number -1
    "stereographic": (24, -1),
    # three Bloch skyrmions of radius L/6: winding number +3
    "bloch3": (24, 3),
}


def known_texture(oracle, name):
    L, q = KNOWN_TEXTURES[name]
    om = oracle.Mesh.sc(L, L, 4)
    if name == "stereographic":
        om.init_skyrmion(L / 2, L / 2, 1.0, 1.56, 1)
    else:
        om.set_spins(_bloch_texture(L, 4, L / 6, [(L / 4, L / 4), (3 * L / 4, L / 3), (L / 2, 3 * L / 4)]))
    return om, q


@pytest.mark.parametrize("name", sorted(KNOWN_TEXTURES))
def test_counting_on_known_textures_matches_second_restatement(oracle, name):
    """The C oracle's count equals an independent restatement written from the Fortran text on
    textures of known winding number.  The counts are the reference's, not the number of
    skyrmions: the last loop adds one per CELL of a matching region, and regions of a filtered
    density rarely integrate to within 0.05 of 1."""
    from oracle import skyrmion_count_ref as S
    om, q = known_texture(oracle, name)
    L = om.nx
    z = 2
    assert round(om.winding_number(z)) == q
    seen = set()
    for scale in (1, 2):   # at 2 the fine grid is wider than the coarse wraps of the search
        dens = oracle.winding_density_interpolated(om, z, scale, scale)
        assert abs(dens.sum() - q) < 1e-6
        for thr in (0.5, 0.1, 0.01):
            for sigma in (1.0, 0.5, 1e-5):
                want, accs = S.skyrmion_number(dens, L, L, thr, 1, sigma)
                assert oracle.skyrmion_number(dens, L, L, thr, 1, sigma) == (0, want), (scale, thr, sigma)
                seen.add(want)
    assert seen - {0} or name == "stereographic"   # the Bloch texture reaches the per-cell count
