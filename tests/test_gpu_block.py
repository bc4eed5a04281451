"""Block CG (bqcdg_solve_block) against the oracle and against single
solves: every system of the block reaches |r|/|b| < 1e-10, measured again
with the oracle's FP64 operator, and the block needs fewer iterations than
the slowest of the same systems solved alone (it searches along all their
directions at once)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KAPPA, CSW = 0.13, 1.9192


@pytest.fixture(scope="module", params=[(8, 8, 8, 8), (6, 4, 6, 4)], ids=lambda L: "x".join(map(str, L)))
def setup(request, oracle, bq):
    L = request.param
    g = oracle.Geom(L, (1, 1, 1, -1))
    oracle.ranset(77)
    u = g.hot()
    g.relax(u, 1)
    uf = g.flip_bc(u.copy())
    clov = g.clover_init(u, CSW * KAPPA)
    lat = bq.Lattice(L, (1, 1, 1, -1))
    lat.load_gauge(uf, flipped=True)
    lat.load_clover(*clov)
    yield dict(g=g, uf=uf, clov=clov, lat=lat)
    lat.close()


def sources(g, n):
    """point sources at site 0 (spin-colour s % 12), then Gaussian vectors"""
    out = []
    for s in range(n):
        if s < min(n // 2, 12):
            b = np.zeros((g.volh, 3, 4), complex)
            b[0, (s % 12) // 4, s % 4] = 1.0
        else:
            b = g.gauss_spinor(0)
        out.append(b)
    return out


@pytest.mark.parametrize("n,rho", [(6, 0.0), (6, 0.1), (16, 0.0), (1, 0.0)])
def test_block_solutions_and_iterations(setup, bq, oracle, n, rho):
    g, lat = setup["g"], setup["lat"]
    name = "w_dagger_w" if rho else "mtdagmt"
    para = bq.HmcPara(kappa=KAPPA, csw=CSW, rho=rho)
    bs = sources(g, n)
    hbs = [lat.field(b) for b in bs]
    hxs = [lat.field() for _ in bs]
    infos = lat.solve_block(hxs, hbs, para, tol=1e-10)
    single = []
    for k, b in enumerate(bs):
        assert infos[k].converged, (k, infos[k].as_dict())
        x = lat.field_get(hxs[k])
        ax = g.op(name, x, setup["uf"], setup["clov"], KAPPA, CSW * KAPPA, 0.0, rho)
        assert np.linalg.norm(b - ax) / np.linalg.norm(b) < 1.01e-10
        h = lat.field()
        single.append(lat.solve_dev(h, hbs[k], para, precision=bq.PREC_SINGLE, tol=1e-10).niter)
    block = max(i.niter for i in infos)
    print("block CG, %d systems, rho %g: block iterations %s (restarts %d), alone %s"
          % (n, rho, [i.niter for i in infos], infos[0].reliable_updates, single))
    if n > 1:
        assert block < max(single), (block, single)
