"""CPU tests of the product's host lattice compiler (meshes built with device = -1) against
the oracle's per-atom restatement of makeChainMesh / initAtomShells / assignNearestNeighbors /
DerivativeList (src/chainMesh.f90)."""
import numpy as np
import pytest

CASES = [
    ("sc3", "SC", (3, 3, 3)), ("sc4", "SC", (4, 4, 4)), ("sc5", "SC", (5, 5, 5)),
    ("sc_rect", "SC", (4, 6, 8)), ("sc_odd", "SC", (5, 3, 7)),
    ("bcc4", "BCC", (4, 4, 4)), ("bcc3", "BCC", (3, 4, 3)),
    ("hk3", "HK", (3, 3, 3)), ("hk4", "HK", (4, 4, 4)),
]


FCC_CELL = (np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]], np.float32),
            (1.0, 1.0, 1.0, 90.0, 90.0, 90.0))


def _cell(oracle, kind):
    if kind == "FCC":   # not one of the reference's cells: a 4-sublattice check of the colourings
        return FCC_CELL
    if kind == "SC":
        return oracle.SC_CELL
    if kind == "BCC":
        return oracle.BCC_CELL
    return oracle.HYPER_KAGOME_CELL


@pytest.mark.parametrize("name,kind,dims", CASES, ids=[c[0] for c in CASES])
def test_lattice_tables_match_oracle(oracle, ib, name, kind, dims):
    frac, (a, b, c, ab, bc, ca) = _cell(oracle, kind)
    om = oracle.Mesh(frac, *dims, a, b, c, ab, bc, ca)
    pm = ib.ChainMesh(*dims, frac, a, b, c, ab, bc, ca, device=-1)
    assert pm.numAtoms == om.natoms
    assert np.array_equal(pm.positions(), om.positions())
    # shells as ordered lists (positions are exact here, so the order is identical)
    for atom in range(om.natoms):
        for s in (0, 1):
            assert np.array_equal(pm.neighbours(atom, s), om.shell(atom, s)), (atom, s)
        assert np.array_equal(pm.neighbours(atom, -1), om.neighbor_list(atom)), atom
    assert np.array_equal(pm.derivative_list(), om.derivative_table())
    v = om.vectors()
    assert np.allclose(pm.a_vec, v[0]) and np.allclose(pm.b_vec, v[1]) and np.allclose(pm.c_vec, v[2])


def _random_cases(n=12, seed=20261204):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        kind = ["SC", "BCC", "HK"][i % 3]
        hi = 5 if kind == "HK" else 8            # the hyper-kagome cell holds 12 atoms
        dims = tuple(int(v) for v in rng.integers(3, hi, size=3))
        shells = int(rng.integers(1, 3))
        out.append((f"{kind.lower()}_{dims[0]}{dims[1]}{dims[2]}_s{shells}", kind, dims, shells))
    return out


@pytest.mark.parametrize("name,kind,dims,shells", _random_cases(), ids=[c[0] for c in _random_cases()])
def test_lattice_tables_match_oracle_on_random_shapes(oracle, ib, name, kind, dims, shells):
    """Seeded random shapes (3-7 cells per side, odd and even, non-cubic) and shell counts:
    the same element-by-element comparison as above."""
    frac, (a, b, c, ab, bc, ca) = _cell(oracle, kind)
    om = oracle.Mesh(frac, *dims, a, b, c, ab, bc, ca, n_shells=shells)
    pm = ib.ChainMesh(*dims, frac, a, b, c, ab, bc, ca, numShells=shells, device=-1)
    assert pm.numAtoms == om.natoms
    assert np.array_equal(pm.positions(), om.positions())
    for atom in range(om.natoms):
        for s in range(shells):
            assert np.array_equal(pm.neighbours(atom, s), om.shell(atom, s)), (atom, s)
        assert np.array_equal(pm.neighbours(atom, -1), om.neighbor_list(atom)), atom
    assert np.array_equal(pm.derivative_list(), om.derivative_table())


def test_non_orthogonal_cell_sets(oracle, ib):
    # monoclinic cell with an inexact lattice constant: neighbour SETS must agree
    frac = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0]], np.float32)
    args = (5, 5, 4, frac, 2.8, 3.1, 2.9, 90.0, 90.0, 100.0)
    om = oracle.Mesh(frac, 5, 5, 4, 2.8, 3.1, 2.9, 90.0, 90.0, 100.0)
    pm = ib.ChainMesh(*args, device=-1)
    for atom in range(0, om.natoms, 7):
        for s in (0, 1):
            assert sorted(pm.neighbours(atom, s)) == sorted(om.shell(atom, s))
        assert sorted(pm.neighbours(atom, -1)) == sorted(om.neighbor_list(atom))


def test_colouring_is_independent(oracle, ib):
    """Every colour class is an independent set of the active shells' bonds (a bond of a site
    to itself, which the reference's shell search gives BCC cells in shell 2, excepted).  BCC
    meshes of at least 4 cells per axis take sublattice planes, whose classes without J' are
    the two sublattices; even hyper-kagome meshes classes of whole octant blocks (cell octant
    (x&1, y&1, z&1), sublattice): without J' its three shell-1 classes (4 of the 12 sublattices
    each, in every octant), with J' the 15 classes of a DSatur colouring of the 96 blocks (72
    octant x sublattice-group classes before); other meshes a greedy colouring.  An FCC cell
    (4 sublattices, not a reference cell) with even extents takes octant order too: without J'
    its 4 sublattices are the classes, with J' 10 block classes."""
    cases = (("SC", (6, 6, 6)), ("SC", (5, 5, 5)), ("BCC", (4, 4, 4)), ("BCC", (6, 4, 8)), ("BCC", (3, 4, 3)),
             ("BCC", (5, 6, 7)), ("HK", (4, 4, 4)), ("HK", (4, 6, 4)), ("HK", (3, 3, 3)),
             ("FCC", (4, 4, 4)), ("FCC", (6, 4, 6)), ("FCC", (5, 5, 5)))
    n_classes = {("HK", False): 3, ("HK", True): 15, ("FCC", False): 4, ("FCC", True): 10}
    for kind, dims in cases:
        frac, (a, b, c, ab, bc, ca) = _cell(oracle, kind)
        pm = ib.ChainMesh(*dims, frac, a, b, c, ab, bc, ca, device=-1)
        even = all(d % 2 == 0 for d in dims)
        want = ("checkerboard" if kind == "SC" and dims[2] % 4 == 0 and even
                else "sublattice" if kind == "BCC" and min(dims) >= 4
                else "octant" if kind in ("HK", "FCC") and even else "reference")
        assert pm.layout == want, (kind, dims, pm.layout)
        for Jp in (0.0, 0.2):
            col, n = pm.colouring(ib.params(J=-1.0, J_prime=Jp))
            shells = (0, 1) if Jp else (0,)
            for atom in range(pm.numAtoms):
                for s in shells:
                    nb = pm.neighbours(atom, s)
                    nb = nb[nb != atom]
                    assert np.all(col[nb] != col[atom]), (kind, dims, Jp, atom)
            if kind == "SC" and dims[0] % 4 == 0 and Jp == 0.0:
                assert n == 2 and pm.checkerboard
            if pm.layout == "sublattice" and Jp == 0.0:
                assert n == 2 and np.array_equal(col, np.arange(pm.numAtoms) % 2)
            elif pm.layout == "octant" and Jp == 0.0:   # whole sublattices, every octant
                assert n == n_classes[(kind, False)]
                nsub = len(frac)
                subs = [sorted(set(np.flatnonzero(col == k) % nsub)) for k in range(n)]
                assert sorted(sum(subs, [])) == list(range(nsub))
                if kind == "HK":
                    assert sorted(len(x) for x in subs) == [4, 4, 4]
            elif pm.layout == "octant":
                assert n == n_classes[(kind, True)]
                nsub = len(frac)
                of_block = {}
                for atom in range(pm.numAtoms):   # the colour is a function of the block
                    cell, sub = divmod(atom, nsub)
                    iz = cell % dims[2]
                    iy = (cell // dims[2]) % dims[1]
                    ix = cell // (dims[1] * dims[2])
                    blk = ((ix & 1) << 2 | (iy & 1) << 1 | (iz & 1), sub)
                    assert of_block.setdefault(blk, col[atom]) == col[atom]
                assert len(of_block) == 8 * nsub
            else:
                deg = sum(len(pm.neighbours(0, s)) for s in shells)
                assert n <= deg + 1  # greedy bound


def test_mesh_argument_errors(ib):
    with pytest.raises(ib.IsingError) as e:
        ib.ChainMesh.simple_cubic(2, device=-1)
    assert e.value.status == 1
    with pytest.raises(ib.IsingError):
        ib.ChainMesh(4, 4, 4, np.zeros((17, 3), np.float32), 1, 1, 1, device=-1)
    with pytest.raises(ib.IsingError) as e:
        ib.ChainMesh(4, 4, 4, np.array([[np.nan, 0, 0]], np.float32), 1, 1, 1, device=-1)
    assert e.value.status == 2
    m = ib.ChainMesh.simple_cubic(4, device=-1)
    with pytest.raises(ib.IsingError) as e:
        m.get_spins(0)  # no device state on a lattice-only mesh
    assert e.value.status == 1
    # maximum size: 1300^3 > 2^31-1 atoms is refused before any table is allocated
    with pytest.raises(ib.IsingError) as e:
        ib.ChainMesh.simple_cubic(1300, device=-1)
    assert e.value.status == 1 and "2^31" in str(e.value)
    for kw in ({"n_replicas": 0}, {"numShells": 5}):
        with pytest.raises(ib.IsingError) as e:
            ib.ChainMesh.simple_cubic(4, device=-1, **kw)
        assert e.value.status == 1
    with pytest.raises(ib.IsingError) as e:
        ib.ChainMesh.simple_cubic(4, a=0.0, device=-1)
    assert e.value.status == 1
