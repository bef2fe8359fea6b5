"""The committed golden vectors (tests/golden/oracle_vectors.npz, written by
tests/golden/make_golden.py) against the oracle run now: the same seeded
inputs give the same outputs for every periodic operator family and
direction, the Poisson solve, one Euler step, and the non-periodic first
derivatives and staggered branches."""
import importlib.util
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _maker():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_golden_vectors_reproduce():
    mk = _maker()
    stored = np.load(mk.FILE)
    fresh = mk.build()
    assert sorted(stored.files) == sorted(fresh)
    # 18 operator outputs, the Poisson solve, the step's u, du, divergence, pressure
    assert len([k for k in fresh if k.rsplit("_", 1)[-1] in "xyz"]) == 18
    for k, v in fresh.items():
        g = stored[k]
        assert g.shape == v.shape, k
        if k.endswith("input") or k.endswith("rhs") or k == "step_u0" or k in ("lengths", "dt"):
            assert np.array_equal(g, v), k  # the seeded inputs regenerate exactly
        else:
            scale = max(np.abs(g).max(), 1e-300)
            assert np.abs(g - v).max() / scale < 1e-12, k
