"""Golden vectors for the hot path, written by the CPU oracle (oracle/):
seeded inputs with the outputs of every periodic operator family along
every direction, of the Poisson solve and of one Euler step, and of the
non-periodic first derivatives and staggered branches, on boxes small
enough to commit.

The reference (Fortran + MPI + 2decomp&FFT) cannot be built here and ships
no vectors of its own.  These freeze the oracle, which
tests/test_oracle_pins.py pins to the reference's own known-answer formulas
(modified wavenumbers, test_du/dv/dw, projection to round-off), so a change
to the oracle that moves any output shows up in tests/test_golden.py.

Run from anywhere:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle  # noqa: E402

FILE = os.path.join(HERE, "oracle_vectors.npz")
SEED = 20261203
OPS_SHAPE = (12, 10, 9)     # (nx, ny, nz): every direction a different length
STEP_SHAPE = (16, 12, 10)
LENGTHS = (2 * np.pi, 1.5, 3.0)
KINDS = ("der", "der2", "dervp", "derpv", "intvp", "intpv")
DT = 1e-3
# non-periodic first derivatives: ((ncl1, ncln), npaire) along each direction
DER_NP = (((1, 1), 0), ((1, 1), 1), ((2, 2), 0), ((1, 2), 1))
# non-periodic staggered branches the reference has: (kind, direction, (ncl1, ncln), npaire)
STAG_NP = (("dervp", 0, (1, 1), 1), ("dervp", 1, (1, 1), 0), ("dervp", 2, (2, 2), 0),
           ("intvp", 1, (1, 1), 1), ("derpv", 2, (1, 1), 1), ("intpv", 0, (2, 2), 1))


def _taylor_green(shape, rng, noise):
    """Taylor-Green velocity on the box plus N(0, noise^2), Fortran order."""
    nx, ny, nz = shape
    x, y, z = (np.arange(n) * (L / n) * (2 * np.pi / L) for n, L in zip(shape, LENGTHS))
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    comps = (np.sin(X) * np.cos(Y) * np.cos(Z), -np.cos(X) * np.sin(Y) * np.cos(Z), np.zeros(shape))
    return [np.asfortranarray(c + noise * rng.standard_normal(shape)) for c in comps]


def build():
    """The vectors, recomputed from the seed: {name: array}."""
    rng = np.random.default_rng(SEED)
    out = {"lengths": np.array(LENGTHS), "dt": np.array(DT)}
    u = np.asfortranarray(rng.standard_normal(OPS_SHAPE))
    out["ops_input"] = u
    for kind in KINDS:
        for d in range(3):
            out[f"{kind}_{'xyz'[d]}"] = oracle.apply(kind, d, u, LENGTHS[d] / OPS_SHAPE[d])
    rhs = np.asfortranarray(rng.standard_normal(STEP_SHAPE))
    out["poisson_rhs"] = rhs
    out["poisson_out"] = oracle.poisson(rhs, *LENGTHS)
    ux, uy, uz = _taylor_green(STEP_SHAPE, rng, 0.1)
    out["step_u0"] = np.stack([ux, uy, uz])
    du, div, pp3 = oracle.euler_step(ux, uy, uz, DT, lengths=LENGTHS)
    out["step_u1"] = np.stack([ux, uy, uz])
    out["step_du"] = np.stack(du)
    out["step_div_before"] = div
    out["step_pp3"] = pp3
    # non-periodic directions: the velocity grid has n points, spacing L/(n-1)
    uv = np.asfortranarray(rng.standard_normal(OPS_SHAPE))
    out["np_vel_input"] = uv
    h = [L / (n - 1) for L, n in zip(LENGTHS, OPS_SHAPE)]
    for d in range(3):
        for (n1, nn), npaire in DER_NP:
            out[f"dernp_{'xyz'[d]}_{n1}{nn}_p{npaire}"] = oracle.der_np(d, uv, h[d], n1, nn, npaire)
    for kind, d, (n1, nn), npaire in STAG_NP:
        if kind.endswith("vp"):
            src = uv
        else:  # pressure-grid input: one point fewer along d
            shape = list(OPS_SHAPE)
            shape[d] -= 1
            src = np.asfortranarray(rng.standard_normal(shape))
            out[f"np_pre_{kind}_{'xyz'[d]}_input"] = src
        out[f"stagnp_{kind}_{'xyz'[d]}_{n1}{nn}_p{npaire}"] = oracle.stag_np(kind, d, src, h[d], n1, nn, npaire)
    return out


if __name__ == "__main__":
    np.savez_compressed(FILE, **build())
    print("wrote", FILE, os.path.getsize(FILE), "bytes")
