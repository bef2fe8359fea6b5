"""The oracle's Poisson solve with non-periodic directions (oracle.poisson_bc):
the bc = 1 case of decomp_2d_poisson_init (src/poisson.f90:85-99), Neumann
conditions on the pressure, which x3div itself stops on (:104-108).

poisson_bc solves the periodic problem (the pinned poisson_000 restatement)
on the box mirrored about the walls.  It is held here to an independent
formulation built from the reference's bc = 1 tables: a DCT-II along each
non-periodic direction, FFTs along the periodic ones, each mode divided by
-K from waves()'s bc = 1 modified wavenumbers (:539-553, :573-588), and the
inverse transforms."""
import numpy as np
import pytest

LENGTHS = (2 * np.pi, 1.5, 3.0)


def test_bc1_tables_are_the_doubled_periodic_tables(oracle):
    """waves()'s bc = 1 table of m points (w = pi i / m, spacing L / m) is the
    periodic table of the doubled line (2 m points over 2 L) at modes
    0 .. m: the fact the mirrored solve rests on."""
    for m, L in ((16, 2 * np.pi), (12, 1.5), (9, 3.0)):
        k2, tt = oracle.poisson_tables_bc1(m, L)
        t = oracle.poisson_tables(2 * m, 2 * m, 2 * m, 2 * L, 2 * L, 2 * L)
        assert np.allclose(k2, t["k2x"][:m + 1], rtol=1e-13, atol=0), m
        assert np.allclose(tt, t["tx"][:m + 1], rtol=1e-13, atol=1e-15), m
        assert k2[0] == 0.0


@pytest.mark.parametrize("shape,per", [((16, 12, 10), (False, True, True)), ((12, 9, 10), (True, False, True)),
                                       ((12, 10, 9), (True, True, False)), ((9, 9, 12), (False, False, True)),
                                       ((9, 11, 10), (False, False, False)), ((10, 9, 16), (True, False, False))])
def test_mirrored_solve_matches_the_cosine_solve(oracle, shape, per):
    g = np.random.default_rng(7).standard_normal(shape)
    a = oracle.poisson_bc(g, LENGTHS, per)
    b = oracle.poisson_bc_dct(g, LENGTHS, per)
    assert np.abs(a - b).max() / np.abs(b).max() < 1e-12


def test_cosine_mode_is_divided_by_its_symbol(oracle):
    """A single mode, cosine in the non-periodic x (cell centres, Neumann),
    Fourier in y and z: the solve returns it divided by -K."""
    m, ny, nz = 12, 10, 8
    kx, ky, kz = 3, 2, 1
    x = (np.arange(m) + 0.5) / m
    y = np.arange(ny) / ny
    z = np.arange(nz) / nz
    f = (np.cos(np.pi * kx * x)[:, None, None] * np.cos(2 * np.pi * ky * y)[None, :, None]
         * np.cos(2 * np.pi * kz * z)[None, None, :])
    k2x, tx = oracle.poisson_tables_bc1(m, LENGTHS[0])
    t = oracle.poisson_tables(ny, ny, nz, LENGTHS[1], LENGTHS[1], LENGTHS[2])
    K = (k2x[kx] * (t["ty"][ky] * t["tz"][kz]) ** 2 + t["k2y"][ky] * (tx[kx] * t["tz"][kz]) ** 2
         + t["k2z"][kz] * (tx[kx] * t["ty"][ky]) ** 2)
    got = oracle.poisson_bc(f, LENGTHS, (False, True, True))
    assert np.abs(got - (-f / K)).max() < 1e-12 * np.abs(f / K).max()


def test_mean_mode_is_removed(oracle):
    """The K = 0 mode is set to zero, as poisson_000 does (:362-370)."""
    g = np.ones((9, 8, 10))
    out = oracle.poisson_bc(g, LENGTHS, (False, True, False))
    assert np.abs(out).max() < 1e-12
