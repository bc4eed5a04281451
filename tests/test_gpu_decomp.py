"""The time-slab domain decomposition on the device (bqcdg_dd_*): all slabs of
the lattice in one process on one GPU, the faces exchanged between them on
the device.  Every operator equals the oracle's single-domain one to 1e-13
(FP64), and the decomposed CG -- global sums of its scalars over the slabs,
as the reference's MPI build does (cg.F90:91,97,109) -- matches the oracle's
CG: iterations +-1, solution to 1e-8.  The NCCL form of the same slabs (one
process per GPU) is not run here: every run of this project has one GPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# one slab (its faces come back to itself), two and four slabs of 8^4, and
# three slabs of a ragged lattice (V3h = 72)
CASES = [((8, 8, 8, 8), 1), ((8, 8, 8, 8), 2), ((8, 8, 8, 8), 4), ((6, 4, 6, 12), 3)]


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module", params=CASES, ids=lambda c: "%s_%dslabs" % ("x".join(map(str, c[0])), c[1]))
def setup(request, oracle, bq):
    L, n = request.param
    g = oracle.Geom(L, (1, 1, 1, -1))
    oracle.ranset(4242)
    u = g.hot()
    g.relax(u, 1)
    uf = g.flip_bc(u.copy())
    kappa, csw = 0.13, 1.9192
    clov = g.clover_init(u, csw * kappa)
    dd = bq.SlabDecomposition.local(L, n)
    dd.load_gauge(uf, flipped=True)
    dd.load_clover(clov[0], clov[1])
    yield dict(g=g, uf=uf, clov=clov, dd=dd, kappa=kappa, csw=csw)
    dd.close()


@pytest.mark.parametrize("dag", [False, True])
def test_decomposed_dslash(setup, bq, dag):
    g, dd = setup["g"], setup["dd"]
    psi = g.gauss_spinor(1)
    ref = g.d(0, 1, psi, setup["uf"], dag)
    got = dd.op("d_dag" if dag else "d", psi, bq.HmcPara(kappa=setup["kappa"]))
    assert rel(got, ref) < 1e-13


@pytest.mark.parametrize("name", ["mtil", "mtil_dag", "mtdagmt", "w_mult", "w_mult_dag", "w_dagger_w"])
def test_decomposed_operators(setup, bq, name):
    g, dd = setup["g"], setup["dd"]
    rho = 0.1
    para = bq.HmcPara(kappa=setup["kappa"], csw=setup["csw"], rho=rho)
    psi = g.gauss_spinor(0)
    ref = g.op(name, psi, setup["uf"], setup["clov"], setup["kappa"], para.csw_kappa, 0.0, rho)
    assert rel(dd.op(name, psi, para), ref) < 1e-13


@pytest.mark.parametrize("rho", [0.0, 0.1])
def test_decomposed_cg_matches_reference_cg(setup, bq, rho):
    g, dd = setup["g"], setup["dd"]
    b = g.gauss_spinor(0)
    x0 = g.gauss_spinor(0) * 0.1
    name = "w_dagger_w" if rho else "mtdagmt"
    rest = np.float32(1e-16 * 12 * g.volh)
    xr, itr, rtr, rc = g.cg(name, x0, b, setup["uf"], setup["clov"], setup["kappa"], setup["csw"] * setup["kappa"],
                            0.0, rho, rest=rest, maxiter=2000, log=0)
    assert rc == 0
    para = bq.HmcPara(kappa=setup["kappa"], csw=setup["csw"], rho=rho)
    xg, itg, info = dd.cg(x0, b, para, rest=rest, maxiter=2000, log=0)
    assert abs(itg - itr) <= 1 and info.converged
    assert rel(xg, xr) < 1e-8


def test_decomposed_cg_no_convergence_semantics(setup, bq):
    g, dd = setup["g"], setup["dd"]
    b = g.gauss_spinor(0)
    para = bq.HmcPara(kappa=setup["kappa"], csw=setup["csw"])
    with pytest.raises(bq.BqcdgError) as e:
        dd.cg(np.zeros_like(b), b, para, rest=1e-30, maxiter=3, log=0)
    assert e.value.status == bq.ENOCONV
    x, it, info = dd.cg(np.zeros_like(b), b, para, rest=1e-30, maxiter=3, log=2)
    assert it == 3 and info.converged == 0



@pytest.mark.parametrize("rho,clover", [(0.0, True), (0.1, True), (0.0, False)], ids=["mtdagmt", "w_dagger_w", "wilson"])
def test_decomposed_mixed_solve(setup, bq, rho, clover):
    """bqcdg_dd_solve: int16 slab passes with FP32 ghost faces, FP64 reliable
    updates, the two reductions of an iteration summed over the slabs on the
    device.  The solution must reach a true |b - A x|/|b| < 1e-10 measured by
    the oracle's operator, and agree with the single-domain mixed solve of the
    same system (solution to 1e-8, iterations within 15 %)."""
    g, dd = setup["g"], setup["dd"]
    kappa, csw = setup["kappa"], (setup["csw"] if clover else 0.0)
    para = bq.HmcPara(kappa=kappa, csw=csw, rho=rho)
    b = g.gauss_spinor(0)
    x, info = dd.solve(np.zeros_like(b), b, para, tol=1e-10)
    assert info.converged, info.as_dict()
    name = "w_dagger_w" if rho else "mtdagmt"
    ax = g.op(name, x, setup["uf"], setup["clov"] if clover else None, kappa, csw * kappa, 0.0, rho)
    assert rel(ax, b) < 1e-10
    with bq.Lattice(g.L, (1, 1, 1, -1)) as lat:
        lat.load_gauge(setup["uf"], flipped=True)
        lat.load_clover(*setup["clov"])
        x1, i1 = lat.solve(np.zeros_like(b), b, para, precision=bq.PREC_HALF, tol=1e-10)
    print("slabs %d: %d iterations (%d reliable updates) against %d on one domain"
          % (dd.nranks, info.niter, info.reliable_updates, i1.niter))
    assert abs(info.niter - i1.niter) <= max(8, 0.15 * i1.niter)
    assert rel(x, x1) < 1e-8
