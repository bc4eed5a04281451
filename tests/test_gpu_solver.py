"""GPU parity of the M^+M CG (cg.F90) and of the QUDA-hook replacement
(invert_quda.F90) against the oracle's CG, through the C ABI."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module", params=[(4, 4, 4, 4), (8, 8, 8, 8)], ids=lambda L: "x".join(map(str, L)))
def setup(request, oracle, bq):
    L = request.param
    g = oracle.Geom(L, (1, 1, 1, -1))
    oracle.ranset(12345)
    u = g.hot()
    uf = g.flip_bc(u.copy())
    kappa, csw = 0.13, 1.9192
    clov = g.clover_init(u, csw * kappa)
    lat = bq.Lattice(L, (1, 1, 1, -1))
    lat.load_gauge(uf, flipped=True)
    lat.load_clover(*clov)
    yield dict(g=g, uf=uf, clov=clov, lat=lat, kappa=kappa, csw=csw)
    lat.close()


@pytest.mark.parametrize("rho", [0.0, 0.1])
def test_fp64_cg_matches_reference_cg(setup, bq, rho):
    """Same algorithm, same absolute stop: same iteration count (+-1 for
    rounding at the threshold) and solutions within the residual's reach."""
    g, lat = setup["g"], setup["lat"]
    b = g.gauss_spinor(0)
    x0 = g.gauss_spinor(0) * 0.1           # x is also an input (cg.F90:81)
    name = "w_dagger_w" if rho else "mtdagmt"
    rest = np.float32(1e-16 * 12 * g.volh)
    xr, itr, rtr, rc = g.cg(name, x0, b, setup["uf"], setup["clov"], setup["kappa"], setup["csw"] * setup["kappa"],
                            0.0, rho, rest=rest, maxiter=2000, log=0)
    assert rc == 0
    para = bq.HmcPara(kappa=setup["kappa"], csw=setup["csw"], rho=rho)
    xg, itg, info = lat.cg(x0, b, para, rest=rest, maxiter=2000, log=0)
    assert abs(itg - itr) <= 1
    assert info.rtr <= rest
    assert rel(xg, xr) < 1e-8
    # the solution solves the system
    ax = getattr(lat, name)(xg, para)
    assert np.linalg.norm(ax - b) ** 2 < 10 * rest


def test_cg_no_convergence_semantics(setup, bq):
    g, lat = setup["g"], setup["lat"]
    b = g.gauss_spinor(0)
    para = bq.HmcPara(kappa=setup["kappa"], csw=setup["csw"])
    with pytest.raises(bq.BqcdgError) as e:
        lat.cg(np.zeros_like(b), b, para, rest=1e-30, maxiter=3, log=0)
    assert e.value.status == bq.ENOCONV
    x, it, info = lat.cg(np.zeros_like(b), b, para, rest=1e-30, maxiter=3, log=2)   # log == 2: ignore
    assert it == 3 and info.converged == 0


@pytest.mark.parametrize("prec", [0, 2])
def test_nan_input_reports_status_and_context_survives(setup, bq, prec):
    """A NaN planted on the host in b ends the solve with BQCDG_ENAN (no
    fault, no hang), and the same context then solves a clean system."""
    g, lat = setup["g"], setup["lat"]
    b = g.gauss_spinor(0)
    bad = b.copy()
    bad[3, 1, 2] = np.nan
    para = bq.HmcPara(kappa=setup["kappa"], csw=setup["csw"])
    with pytest.raises(bq.BqcdgError) as e:
        lat.solve(np.zeros_like(b), bad, para, precision=prec, tol=1e-10, relative=False)
    assert e.value.status == bq.ENAN
    x, info = lat.solve(np.zeros_like(b), b, para, precision=prec, tol=1e-10)
    assert info.converged == 1


@pytest.mark.parametrize("rho", [0.0, 0.1])
def test_quda_solver_mixed_precision(setup, bq, rho):
    """The hook's replacement: int16 sloppy iterations + FP64 reliable updates
    must meet the absolute FP64 criterion and agree with the FP64 solution."""
    g, lat = setup["g"], setup["lat"]
    b = g.gauss_spinor(0)
    name = "w_dagger_w" if rho else "mtdagmt"
    rest = np.float32(1e-18 * 12 * g.volh)
    xr, _, _, rc = g.cg(name, np.zeros_like(b), b, setup["uf"], setup["clov"], setup["kappa"],
                        setup["csw"] * setup["kappa"], 0.0, rho, rest=rest, maxiter=4000, log=0)
    para = bq.HmcPara(kappa=setup["kappa"], csw=setup["csw"], rho=rho)
    xg, it, info = lat.quda_solver(np.zeros_like(b), b, para, rest=rest, maxiter=4000, log=0)
    assert info.converged == 1 and info.true_rtr <= rest
    assert info.reliable_updates >= 1
    assert rel(xg, xr) < 1e-7


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_relative_tolerance_1e10(setup, bq, prec):
    g, lat = setup["g"], setup["lat"]
    b = g.gauss_spinor(0)
    para = bq.HmcPara(kappa=setup["kappa"], csw=setup["csw"])
    x, info = lat.solve(np.zeros_like(b), b, para, precision=prec, tol=1e-10)
    assert info.converged == 1
    assert info.true_rtr <= 1e-20 * info.b2
    r = lat.mtdagmt(x, para) - b
    assert np.linalg.norm(r) <= 1.01e-10 * np.linalg.norm(b)


def test_solver_only_clover_upload(setup, bq):
    """load_clover_solver takes the same Fortran arrays and keeps A (even) and
    A^-1 (odd) only: the solve is bit-identical to one with the full upload,
    and the force-side parts report their absence."""
    g, lat = setup["g"], setup["lat"]
    para = bq.HmcPara(kappa=setup["kappa"], csw=setup["csw"], rho=0.1)
    b = g.gauss_spinor(0)
    x_full, info = lat.solve(np.zeros_like(b), b, para, precision=bq.PREC_DOUBLE, tol=1e-12)
    a, ai, bb = setup["clov"]
    lat.load_clover_solver(a, ai)
    x_lean, info2 = lat.solve(np.zeros_like(b), b, para, precision=bq.PREC_DOUBLE, tol=1e-12)
    assert info.converged and info2.converged
    assert np.array_equal(x_full, x_lean)
    with pytest.raises(bq.BqcdgError) as e:
        lat.clover_action(1)
    assert e.value.status == bq.ENOCLOVER
    lat.load_clover(*setup["clov"])   # restore the full set for the other tests
