"""Size-independent properties of the operator at the benchmark's full size,
32^3x64, where the oracle is too slow to compare element by element: M~^+
is the adjoint of M~ and W^+W is Hermitian positive definite, both to
rounding (FP64 on device-resident fields, hot links cooled by one sweep);
and one M~^+M~ application is linear in its input."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L = (32, 32, 32, 64)


@pytest.fixture(scope="module")
def lat(bq):
    lt = bq.Lattice(L, (1, 1, 1, -1))
    lt.ranset(9)
    lt.conf_hot()
    lt.conf_relax(1)
    lt.clover_init(1.9192 * 0.13)
    yield lt
    lt.close()


def gauss(lat, seed):
    h = lat.field()
    lat.ranset(seed)
    lat.field_gauss(h, 0.5)
    return h


def test_mtil_dag_is_the_adjoint(lat, bq):
    para = bq.HmcPara(kappa=0.13, csw=1.9192)
    a, b = gauss(lat, 1), gauss(lat, 2)
    ma, mb = lat.field(), lat.field()
    lat.op_dev("mtil", mb, b, para)
    lat.op_dev("mtil_dag", ma, a, para)
    lhs = lat.field_cdot(a, mb)     # <a, M b>
    rhs = lat.field_cdot(ma, b)     # <M^+ a, b>
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_w_dagger_w_hermitian_positive_and_linear(lat, bq):
    para = bq.HmcPara(kappa=0.13, csw=1.9192, rho=0.1)
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
