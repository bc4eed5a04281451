"""Batched multi-RHS mixed-precision CG: every right-hand side meets the FP64
criterion and equals its independent single-RHS FP64 solution; blocks that do
not divide the number of right-hand sides and the autotuned block work."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(oracle, bq):
    L = (8, 8, 8, 8)
    lat = bq.Lattice(L, (1, 1, 1, -1))
    lat.ranset(0)
    lat.conf_hot()
    lat.conf_relax(2)
    lat.clover_init(1.9192 * 0.13)
    yield lat
    lat.close()


@pytest.mark.parametrize("block", [4, 1, 0])
def test_batch_matches_single_solves(setup, bq, block):
    lat = setup
    para = bq.HmcPara(kappa=0.13, csw=1.9192, rho=0.05)
    n = 5
    lat.ranset(99)
    hb = []
    for _ in range(n):
        h = lat.field()
        lat.field_gauss(h, 0.5)
        hb.append(h)
    zero = np.zeros((lat.volh, 3, 4), np.complex128)
    hx = [lat.field(zero) for _ in range(n)]
    infos = lat.solve_batch(hx, hb, para, tol=1e-10, block=block)
    for k in range(n):
        b = lat.field_get(hb[k])
        assert infos[k].converged == 1
        assert infos[k].true_rtr <= 1e-20 * infos[k].b2
        x_ref, info = lat.solve(zero, b, para, precision=bq.PREC_DOUBLE, tol=1e-12)
        x = lat.field_get(hx[k])
        assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)


def test_batch_retires_converged_rhs(setup, bq):
    """A right-hand side that starts converged (b = 0) retires at once; the
    others still converge in the same batch."""
    lat = setup
    para = bq.HmcPara(kappa=0.13, csw=1.9192)
    zero = np.zeros((lat.volh, 3, 4), np.complex128)
    h0 = lat.field(zero)
    h1 = lat.field()
    lat.field_gauss(h1, 0.5)
    hx = [lat.field(zero), lat.field(zero)]
    infos = lat.solve_batch(hx, [h0, h1], para, tol=1e-10, relative=False, block=2)
    assert infos[0].niter == 0 and infos[0].converged == 1, infos[0].as_dict()
    assert infos[1].converged == 1 and infos[1].niter > 0, infos[1].as_dict()
