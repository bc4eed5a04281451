"""GPU parity of the pseudofermion force (dsf.F90 with d/DSFxyzt.F90,
clover_bsa/clover_d) and of the clover determinant force (clover_dsd with
clover_ts) against the oracle, to 1e-10 relative."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOLF = 1e-10


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module", params=[(4, 4, 4, 4), (6, 4, 8, 4)], ids=lambda L: "x".join(map(str, L)))
def setup(request, oracle, bq):
    L = request.param
    g = oracle.Geom(L, (1, 1, 1, -1))
    oracle.ranset(777)
    u = g.hot()
    kappa, csw = 0.13, 1.9192
    clov = g.clover_init(u, csw * kappa)
    lat = bq.Lattice(L, (1, 1, 1, -1))
    yield dict(g=g, u=u, clov=clov, lat=lat, kappa=kappa, csw=csw)
    lat.close()


@pytest.mark.parametrize("csw", [0.0, 1.9192])
def test_dsf(setup, bq, csw):
    g, lat = setup["g"], setup["lat"]
    kappa = setup["kappa"]
    clov = setup["clov"] if csw else None
    a = g.gauss_spinor(0)
    b = g.gauss_spinor(0)
    p0 = g.gauss_momenta()
    step = 0.037
    uf = g.flip_bc(setup["u"].copy())
    lat.load_gauge(uf, flipped=True)
    if clov is not None:
        lat.load_clover(*clov)
    pref = g.dsf(p0.copy(), uf, clov, step, kappa, csw * kappa, a, b)     # uf comes back unflipped
    pgpu = lat.dsf(p0.copy(), step, bq.HmcPara(kappa=kappa, csw=csw), a, b)
    assert rel(pgpu - p0, pref - p0) < TOLF


@pytest.mark.parametrize("eo", [0, 1])
def test_clover_dsf(setup, eo):
    g, lat = setup["g"], setup["lat"]
    lat.load_gauge(setup["u"], flipped=False)
    a = g.gauss_spinor(eo)
    b = g.gauss_spinor(eo)
    p0 = g.gauss_momenta()
    pref = g.clover_dsf(eo, p0.copy(), b, a, -0.0123, setup["u"])
    pgpu = lat.clover_dsf(eo, p0.copy(), b, a, -0.0123)
    assert rel(pgpu - p0, pref - p0) < TOLF


@pytest.mark.parametrize("eo", [0, 1])
def test_clover_dsd(setup, eo):
    g, lat = setup["g"], setup["lat"]
    lat.load_gauge(setup["u"], flipped=False)
    lat.load_clover(*setup["clov"])
    p0 = g.gauss_momenta()
    pref = g.clover_dsd(eo, p0.copy(), setup["clov"][2], -0.0211, setup["u"])
    pgpu = lat.clover_dsd(eo, p0.copy(), -0.0211)
    assert rel(pgpu - p0, pref - p0) < TOLF
