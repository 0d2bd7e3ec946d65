"""The committed fixtures of tests/golden are reproduced by the oracle (CPU)."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ["sc4", "sc6", "sc8", "sc16", "bcc3", "hk3"]


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_fixture(oracle, name):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    fresh = mg.make(name)
    ref = np.load(os.path.join(GOLD, f"{name}.npz"))
    assert set(fresh) == set(ref.files)
    for k in ref.files:
        assert np.allclose(fresh[k], ref[k], rtol=1e-13, atol=1e-13), k
