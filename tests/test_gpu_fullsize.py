"""The operator, the forces and the benchmark solve at the benchmark's own
size, 32^3x64, on the benchmark's own system: the device hot start (BQCD's
ranf, default seed) cooled by one conf_relax sweep (plaquette 0.6127), the
clover term at kappa 0.13, c_sw 1.9192.

Element-wise parity with the oracle on that system: the links and clover
blocks built on the device are copied to the host, and the oracle's
mtil / mtil_dag / mtdagmt / w_dagger_w (m_tilde.F90:43-114, mtdagmt.F90:28,
w_mult.F90:28-84) must agree to 1e-13 relative, dsf (dsf.F90:28-110) and
clover_dsf (clover/clover_d.F90:78-107) to 1e-10.  The mixed-precision
solve must reach a true |b - A x|/|b| < 1e-10 measured by the oracle's own
operator, the stopping rule of the benchmark.

Beside them, size-independent properties on device-resident fields: M~^+
is the adjoint of M~, W^+W is Hermitian positive definite, and one
application is linear.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L = (32, 32, 32, 64)
KAPPA, CSW = 0.13, 1.9192
TOL64, TOLF = 1e-13, 1e-10


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def system(bq, oracle):
    lt = bq.Lattice(L, (1, 1, 1, -1))
    lt.ranset(0)
    lt.conf_hot()
    lt.conf_relax(1)
    lt.clover_init(CSW * KAPPA)
    g = oracle.Geom(L, (1, 1, 1, -1))
    host = dict(uf=lt.get_gauge(flipped=True), clov=lt.get_clover())
    yield lt, g, host
    lt.close()


def test_benchmark_configuration(system):
    lat, _, _ = system
    assert abs((1.0 - lat.plaq_energy()) - 0.612665) < 5e-7


@pytest.mark.parametrize("name,rho", [("mtil", 0.0), ("mtil_dag", 0.0), ("mtdagmt", 0.0), ("w_dagger_w", 0.1)])
def test_operator_matches_oracle_elementwise(system, bq, oracle, name, rho):
    lat, g, host = system
    para = bq.HmcPara(kappa=KAPPA, csw=CSW, rho=rho)
    oracle.ranset(11)
    psi = g.gauss_spinor(0)
    ref = g.op(name, psi, host["uf"], host["clov"], KAPPA, para.csw_kappa, 0.0, rho)
    got = getattr(lat, name)(psi, para)
    assert rel(got, ref) < TOL64


def test_dsf_matches_oracle(system, bq, oracle):
    lat, g, host = system
    oracle.ranset(12)
    a, b = g.gauss_spinor(0), g.gauss_spinor(0)
    p0 = g.gauss_momenta()
    step = 0.037
    uf = host["uf"].copy()          # the oracle's dsf un-flips its links in place
    pref = g.dsf(p0.copy(), uf, host["clov"], step, KAPPA, CSW * KAPPA, a, b)
    pgpu = lat.dsf(p0.copy(), step, bq.HmcPara(kappa=KAPPA, csw=CSW), a, b)
    assert rel(pgpu - p0, pref - p0) < TOLF


@pytest.mark.parametrize("eo", [0, 1])
def test_clover_dsf_matches_oracle(system, oracle, eo):
    lat, g, host = system
    oracle.ranset(13 + eo)
    a, b = g.gauss_spinor(eo), g.gauss_spinor(eo)
    p0 = g.gauss_momenta()
    u = g.flip_bc(host["uf"].copy())     # clover_dsf runs on periodic links
    pref = g.clover_dsf(eo, p0.copy(), b, a, -0.0123, u)
    pgpu = lat.clover_dsf(eo, p0.copy(), b, a, -0.0123)
    assert rel(pgpu - p0, pref - p0) < TOLF


def test_mixed_solve_true_residual_by_oracle(system, bq, oracle):
    """The benchmark's solve (int16 iterations, FP64 reliable updates) from
    x = 0 to |r|/|b| < 1e-10; the residual is recomputed with the oracle's
    FP64 M~^+M~ on the host."""
    lat, g, host = system
    para = bq.HmcPara(kappa=KAPPA, csw=CSW)
    lat.ranset(0)
    hb = lat.field()
    lat.field_gauss(hb, 0.5)
    b = lat.field_get(hb)
    x, info = lat.solve(np.zeros_like(b), b, para, precision=bq.PREC_HALF, tol=1e-10)
    assert info.converged
    ax = g.op("mtdagmt", x, host["uf"], host["clov"], KAPPA, CSW * KAPPA)
    assert np.linalg.norm(b - ax) / np.linalg.norm(b) < 1e-10


def gauss(lat, seed):
    h = lat.field()
    lat.ranset(seed)
    lat.field_gauss(h, 0.5)
    return h


def test_mtil_dag_is_the_adjoint(system, bq):
    lat = system[0]
    para = bq.HmcPara(kappa=KAPPA, csw=CSW)
    a, b = gauss(lat, 1), gauss(lat, 2)
    ma, mb = lat.field(), lat.field()
    lat.op_dev("mtil", mb, b, para)
    lat.op_dev("mtil_dag", ma, a, para)
    lhs = lat.field_cdot(a, mb)     # <a, M b>
    rhs = lat.field_cdot(ma, b)     # <M^+ a, b>
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_w_dagger_w_hermitian_positive_and_linear(system, bq):
    lat = system[0]
    para = bq.HmcPara(kappa=KAPPA, csw=CSW, rho=0.1)
    a, b = gauss(lat, 3), gauss(lat, 4)
    wa, wb = lat.field(), lat.field()
    lat.op_dev("w_dagger_w", wa, a, para)
    lat.op_dev("w_dagger_w", wb, b, para)
    ab, ba = lat.field_cdot(a, wb), lat.field_cdot(b, wa)
    assert abs(ab - np.conj(ba)) <= 1e-12 * abs(ab)
    aa = lat.field_cdot(a, wa)
    assert aa.real > 0 and abs(aa.imag) <= 1e-12 * aa.real
    # linearity: A(a + 2i b) = A a + 2i A b
    s, ws = lat.field(), lat.field()
    lat.field_copy(s, a)
    lat.field_caxpby(s, 1.0, 2.0j, b)
    lat.op_dev("w_dagger_w", ws, s, para)
    want = lat.field_get(wa) + 2j * lat.field_get(wb)
    got = lat.field_get(ws)
    assert np.linalg.norm(got - want) <= 1e-13 * np.linalg.norm(want)
