"""The device generators of the benchmark inputs reproduce BQCD's: the RNG
stream position (exactly), hot-start links, Gaussian spinors, cooling sweeps
and the plaquette action, against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L", [(4, 4, 4, 4), (6, 4, 8, 4)])
def test_hot_start_relax_and_sg(oracle, bq, L):
    g = oracle.Geom(L)
    oracle.ranset(4711)
    u = g.hot()
    with bq.Lattice(L) as lat:
        lat.ranset(4711)
        lat.conf_hot()
        assert lat.ranget() == oracle.ranget()          # same number of draws
        ud = lat.get_gauge(flipped=False)
        assert np.abs(ud - u).max() < 1e-13
        g.relax(u, 2)
        lat.conf_relax(2)
        ud = lat.get_gauge(flipped=False)
        assert np.abs(ud - u).max() < 1e-11
        assert abs(lat.sg() - g.sg(u)) < 1e-10 * g.sg(u)


def test_gaussian_spinor_stream(oracle, bq):
    L = (4, 4, 4, 8)
    g = oracle.Geom(L)
    oracle.ranset(0)
    ref = g.gauss_spinor(0, 0.5)
    with bq.Lattice(L) as lat:
        lat.ranset(0)
        h = lat.field()
        lat.field_gauss(h, 0.5)
        assert lat.ranget() == oracle.ranget()
        assert np.abs(lat.field_get(h) - ref).max() < 1e-13


def test_cold_start(bq):
    with bq.Lattice((4, 4, 4, 4)) as lat:
        lat.conf_cold()
        assert lat.sg() == 0.0
