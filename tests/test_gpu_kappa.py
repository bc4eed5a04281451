"""Operators and batched solves at several hopping parameters on one gauge
field.  clover_init.F90:46-77 builds each chiral block as
1 + (-c_sw kappa / 8)(p +- q); bqcdg_clover_init_t stores T = (-c_sw/8)(p +- q)
once and the kernels form A(kappa) and its inverse per site.  At every kappa
the FP64 operators must equal the oracle's, built with clover_init at that
kappa, to 1e-13; a batched int16 solve with one kappa per system must reach
|r|/|b| < 1e-10 on each system and agree with the oracle's FP64 CG of that
system."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KAPPAS = [0.120, 0.125, 0.130, 0.1355]
CSW = 1.9192


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module", params=[(8, 8, 8, 8), (6, 4, 8, 4)], ids=lambda L: "x".join(map(str, L)))
def setup(request, oracle, bq):
    L = request.param
    g = oracle.Geom(L, (1, 1, 1, -1))
    oracle.ranset(99)
    u = g.hot()
    g.relax(u, 1)
    uf = g.flip_bc(u.copy())
    lat = bq.Lattice(L, (1, 1, 1, -1))
    lat.load_gauge(uf, flipped=True)
    lat.clover_init_t(CSW)
    clov = {k: g.clover_init(u, CSW * k) for k in KAPPAS}
    yield dict(g=g, u=u, uf=uf, lat=lat, clov=clov)
    lat.close()


@pytest.mark.parametrize("kappa", KAPPAS)
@pytest.mark.parametrize("name", ["mtil", "mtil_dag", "mtdagmt", "w_mult", "w_mult_dag", "w_dagger_w"])
def test_operator_at_each_kappa(setup, bq, name, kappa):
    g, lat = setup["g"], setup["lat"]
    rho = 0.1
    para = bq.HmcPara(kappa=kappa, csw=CSW, rho=rho)
    psi = g.gauss_spinor(0)
    ref = g.op(name, psi, setup["uf"], setup["clov"][kappa], kappa, CSW * kappa, 0.0, rho)
    assert rel(getattr(lat, name)(psi, para), ref) < 1e-13


@pytest.mark.parametrize("csw", [CSW, 0.0])
def test_batched_solve_one_kappa_per_system(setup, bq, oracle, csw):
    g, lat = setup["g"], setup["lat"]
    n = len(KAPPAS)
    bs = [g.gauss_spinor(0) for _ in range(n)]
    hbs = [lat.field(b) for b in bs]
    hxs = [lat.field() for _ in range(n)]
    infos = lat.solve_batch_kappa(hxs, hbs, bq.HmcPara(kappa=0.13, csw=csw), KAPPAS, precision=bq.PREC_HALF,
                                  tol=1e-10)
    for k, kap in enumerate(KAPPAS):
        assert infos[k].converged, infos[k].as_dict()
        assert infos[k].true_rtr <= 1e-20 * infos[k].b2
        x = lat.field_get(hxs[k])
        b2 = float(np.vdot(bs[k], bs[k]).real)
        clov = setup["clov"][kap] if csw else None
        xr, itr, rtr, rc = g.cg("mtdagmt", np.zeros_like(bs[k]), bs[k], setup["uf"], clov, kap, csw * kap, 0.0, 0.0,
                                rest=np.float32(1e-22 * b2), maxiter=5000, log=0)
        assert rc == 0
        assert rel(x, xr) < 1e-7, (kap, rel(x, xr))


def test_fp64_solve_at_a_kappa(setup, bq):
    g, lat = setup["g"], setup["lat"]
    kap = KAPPAS[-1]
    para = bq.HmcPara(kappa=kap, csw=CSW)
    b = g.gauss_spinor(0)
    x, info = lat.solve(np.zeros_like(b), b, para, precision=bq.PREC_DOUBLE, tol=1e-12)
    assert info.converged
    ax = g.op("mtdagmt", x, setup["uf"], setup["clov"][kap], kap, CSW * kap)
    assert rel(ax, b) < 1e-11


def test_entry_points_that_read_the_blocks_refuse_t(setup, bq, oracle):
    g, lat = setup["g"], setup["lat"]
    psi = g.gauss_spinor(0)
    with pytest.raises(bq.BqcdgError) as e:
        lat.clover_mult_a(0, psi)
    assert e.value.status == bq.EUNSUPPORTED
    with pytest.raises(bq.BqcdgError) as e:
        lat.get_clover()
    assert e.value.status == bq.EUNSUPPORTED
    # a clover_init at one kappa replaces T, and the blocks are BQCD's again
    with bq.Lattice(g.L, (1, 1, 1, -1)) as lat2:
        lat2.load_gauge(setup["uf"], flipped=True)
        lat2.clover_init_t(CSW)
        lat2.clover_init(CSW * 0.13)
        a, ai, bb = lat2.get_clover()
        assert rel(a, setup["clov"][0.13][0]) < 1e-14
        para = bq.HmcPara(kappa=0.13, csw=CSW)
        ref = g.op("mtdagmt", psi, setup["uf"], setup["clov"][0.13], 0.13, CSW * 0.13)
        assert rel(lat2.mtdagmt(psi, para), ref) < 1e-13
