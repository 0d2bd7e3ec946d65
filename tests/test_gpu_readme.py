"""The README's Python example, shortened (SC L=16 x 4 replicas, 3 rounds), runs as written:
the documented calls keep their names, arguments and return shapes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_readme_example_runs(ib, cuda_ok):
    m = ib.ChainMesh.simple_cubic(16, n_replicas=4)
    m.init_uniform(seed=0x15196)
    betas = 1.0 / ib.temperature_ladder(0.1, 1.5, 4)
    p = ib.params(J=-1.0, Dz=0.7, B=0.3, dmi="bulk", include_Jp=False)
    eng = ib.Ensembles([(m, betas, p, 0)])
    eng.autotune(2)
    eng.run(2, 3)
    energies, magnetisation = eng.energies(0)
    assert energies.shape == (4,) and magnetisation.shape == (4, 3)
    assert np.all(np.isfinite(energies))
    coldest = int(eng.permutation(0)[0])
    q = ib.winding_all_slices(m, coldest)
    assert q.shape == (16,)
    assert np.allclose(q, np.round(q), atol=1e-6)     # integer charge per periodic slice
    eng.close()
