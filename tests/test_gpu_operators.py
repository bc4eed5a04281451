"""GPU parity of the operator rows against the CPU oracle, through the C ABI.

FP64 operators must agree with the restated reference to 1e-13 (relative,
norm-wise) on seeded hot-start links, both parities, d and d_dag, with the
fermion boundary sign given either inside the links (flip_bc applied, as at
BQCD's call sites) or applied by the library.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (6,6,6,6): volh = 648, not a multiple of the 128-site blocks, odd x/2;
# (2,4,6,4): extent 2, where the forward and backward x-neighbours coincide
LATTICES = [(4, 4, 4, 4), (6, 4, 8, 4), (8, 8, 8, 8), (6, 6, 6, 6), (2, 4, 6, 4)]
TOL64 = 1e-13


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module", params=LATTICES, ids=lambda L: "x".join(map(str, L)))
def setup(request, oracle, bq):
    L = request.param
    g = oracle.Geom(L, (1, 1, 1, -1))
    oracle.ranset(0)
    u = g.hot()
    uf = g.flip_bc(u.copy())
    csw, kappa = 1.9192, 0.13
    clov = g.clover_init(u, csw * kappa)
    lat = bq.Lattice(L, (1, 1, 1, -1))
    lat.load_gauge(uf, flipped=True)
    lat.load_clover(*clov)
    yield dict(g=g, u=u, uf=uf, clov=clov, lat=lat, kappa=kappa, csw=csw)
    lat.close()


@pytest.mark.parametrize("e", [0, 1])
@pytest.mark.parametrize("dag", [False, True])
def test_dslash(setup, oracle, e, dag):
    g, lat = setup["g"], setup["lat"]
    psi = g.gauss_spinor(1 - e)
    ref = g.d(e, 1 - e, psi, setup["uf"], dag)
    got = (lat.d_dag if dag else lat.d)(e, 1 - e, psi)
    assert rel(got, ref) < TOL64


def test_dslash_bc_in_kernel_equals_flipped_links(setup, bq):
    """Periodic links + in-kernel boundary sign == BQCD's flipped links."""
    g = setup["g"]
    psi = g.gauss_spinor(1)
    a = setup["lat"].d(0, 1, psi)
    with bq.Lattice(g.L, (1, 1, 1, -1)) as lat2:
        lat2.load_gauge(setup["u"], flipped=False)
        b = lat2.d(0, 1, psi)
        back = lat2.get_gauge(flipped=True)
    assert rel(a, b) < 1e-15
    assert np.array_equal(back, setup["uf"])


@pytest.mark.parametrize("eo", [0, 1])
def test_clover_mult(setup, eo):
    g, lat = setup["g"], setup["lat"]
    a, ai, b = setup["clov"]
    psi = g.gauss_spinor(eo)
    assert rel(lat.clover_mult_a(eo, psi), g.clover_mult(0, a[eo], psi)) < TOL64
    assert rel(lat.clover_mult_ao(eo, psi), g.clover_mult(1, ai[eo], psi)) < TOL64
    assert rel(lat.clover_mult_b(eo, psi), g.clover_mult(2, b[eo], psi)) < TOL64


def test_clover_init_on_device(setup, bq):
    g = setup["g"]
    a, ai, b = setup["clov"]
    with bq.Lattice(g.L, (1, 1, 1, -1)) as lat2:
        lat2.load_gauge(setup["u"], flipped=False)
        lat2.clover_init(setup["csw"] * setup["kappa"])
        da, dai, db = lat2.get_clover()
        assert rel(da, a) < 1e-14
        assert rel(dai, ai) < 1e-13
        assert rel(db, b) < 1e-13
        assert abs(lat2.clover_action(1) - g.clover_action(b[1])) < 1e-11 * abs(g.clover_action(b[1]))


OPS = ["mtil", "mtil_dag", "mtdagmt", "w_mult", "w_mult_dag", "w_dagger_w"]


@pytest.mark.parametrize("name", OPS)
def test_clover_operators(setup, bq, name):
    g, lat = setup["g"], setup["lat"]
    rho = 0.1
    para = bq.HmcPara(kappa=setup["kappa"], csw=setup["csw"], rho=rho)
    psi = g.gauss_spinor(0)
    ref = g.op(name, psi, setup["uf"], setup["clov"], setup["kappa"], para.csw_kappa, 0.0, rho)
    got = getattr(lat, name)(psi, para)
    assert rel(got, ref) < TOL64


@pytest.mark.parametrize("name", OPS)
def test_clover_operators_with_h(setup, bq, name):
    """Clover and h together (m_tilde.F90:55-58, 92-95): h_mult_b after
    A_oo^-1 in the first half, b = -kappa^2/(1+h^2) in the second."""
    g, lat = setup["g"], setup["lat"]
    h, rho = 0.05, 0.1
    para = bq.HmcPara(kappa=setup["kappa"], csw=setup["csw"], h=h, rho=rho)
    psi = g.gauss_spinor(0)
    ref = g.op(name, psi, setup["uf"], setup["clov"], setup["kappa"], para.csw_kappa, h, rho)
    got = getattr(lat, name)(psi, para)
    assert rel(got, ref) < TOL64


@pytest.mark.parametrize("name", OPS)
def test_wilson_operators_with_h(setup, bq, name):
    """csw = 0 selects the Wilson operator, where h_mult adds i h gamma_5."""
    g, lat = setup["g"], setup["lat"]
    para = bq.HmcPara(kappa=0.12, csw=0.0, h=0.05, rho=0.2)
    psi = g.gauss_spinor(0)
    ref = g.op(name, psi, setup["uf"], None, 0.12, 0.0, 0.05, 0.2)
    got = getattr(lat, name)(psi, para)
    assert rel(got, ref) < TOL64
