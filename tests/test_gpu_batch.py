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


@pytest.fixture(scope="module")
def oracle_setup(oracle, bq):
    L = (8, 8, 8, 8)
    g = oracle.Geom(L, (1, 1, 1, -1))
    oracle.ranset(2468)
    u = g.hot()
    uf = g.flip_bc(u.copy())
    kappa, csw = 0.13, 1.9192
    clov = g.clover_init(u, csw * kappa)
    lat = bq.Lattice(L, (1, 1, 1, -1))
    lat.load_gauge(uf, flipped=True)
    lat.load_clover(*clov)
    yield dict(g=g, uf=uf, clov=clov, lat=lat, kappa=kappa, csw=csw)
    lat.close()


@pytest.mark.parametrize("block", [3, 0])
def test_shifted_batch_matches_oracle_cg(oracle_setup, bq, block):
    """System k is (W^+W) x = b with W = M~ + rho_k (m_tilde.F90:63-73): each
    solution equals the oracle's FP64 CG of w_dagger_w at that rho, one
    right-hand side appears twice with different shifts, and rho = 0 gives
    the mtdagmt system of dsf2.F90:64."""
    s = oracle_setup
    g, lat = s["g"], s["lat"]
    para = bq.HmcPara(kappa=s["kappa"], csw=s["csw"])
    rhos = [0.0, 0.05, 0.3, 0.05, 1.0]
    bs = [g.gauss_spinor(0) for _ in range(4)]
    bs.append(bs[1].copy())                  # the same b as system 1, another rho
    rhos[4] = 0.3
    hb = [lat.field(b) for b in bs]
    zero = np.zeros_like(bs[0])
    hx = [lat.field(zero) for _ in bs]
    infos = lat.solve_batch_shifted(hx, hb, para, rhos, tol=1e-10, block=block)
    xs = []
    for k, (b, rho) in enumerate(zip(bs, rhos)):
        assert infos[k].converged == 1, infos[k].as_dict()
        assert infos[k].true_rtr <= 1e-20 * infos[k].b2
        name = "w_dagger_w" if rho else "mtdagmt"
        xr, _, _, rc = g.cg(name, zero, b, s["uf"], s["clov"], s["kappa"], s["csw"] * s["kappa"], 0.0, rho,
                            rest=1e-22 * float(np.vdot(b, b).real), maxiter=5000, log=0)
        assert rc == 0
        x = lat.field_get(hx[k])
        assert np.linalg.norm(x - xr) <= 1e-8 * np.linalg.norm(xr), (k, rho)
        xs.append(x)
    # the shift is applied per system: same b, rho 0.05 vs 0.3
    assert np.linalg.norm(xs[1] - xs[4]) > 1e-3 * np.linalg.norm(xs[1])


def test_shifted_batch_rejects_missing_rho(oracle_setup, bq):
    lat = oracle_setup["lat"]
    para = bq.HmcPara(kappa=0.13, csw=1.9192)
    h = lat.field()
    with pytest.raises(ValueError):
        lat.solve_batch_shifted([h], [h], para, [0.1, 0.2])


def test_solver_only_clover_gives_the_same_solution(bq):
    """clover_init_solver keeps A (even) and A^-1 (odd) only: the solver's
    result is unchanged, the context holds less memory, and the entry points
    that need the released parts say so."""
    L = (8, 8, 8, 8)
    para = bq.HmcPara(kappa=0.13, csw=1.9192, rho=0.1)
    out = []
    for solver_only in (False, True):
        lat = bq.Lattice(L, (1, 1, 1, -1))
        lat.ranset(5)
        lat.conf_hot()
        lat.conf_relax(1)
        if solver_only:
            lat.clover_init_solver(para.csw_kappa)
        else:
            lat.clover_init(para.csw_kappa)
        lat.ranset(77)
        hb = lat.field()
        lat.field_gauss(hb, 0.5)
        hx = lat.field(np.zeros((lat.volh, 3, 4), np.complex128))
        info = lat.solve_dev(hx, hb, para, precision=bq.PREC_DOUBLE, tol=1e-12)
        assert info.converged == 1
        out.append((lat.field_get(hx), lat.device_bytes))
        if solver_only:
            with pytest.raises(bq.BqcdgError) as e:
                lat.clover_action(1)
            assert e.value.status == bq.ENOCLOVER
        lat.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert out[1][1] < out[0][1]


def test_release_scratch_frees_and_recreates(bq):
    """release_scratch gives back the work buffers; the next solve re-creates
    them and returns the same solution, and released momenta must be made
    again before the momentum entry points accept a call."""
    L = (8, 8, 8, 8)
    para = bq.HmcPara(kappa=0.13, csw=1.9192, rho=0.1)
    lat = bq.Lattice(L, (1, 1, 1, -1))
    lat.ranset(3)
    lat.conf_hot()
    lat.clover_init(para.csw_kappa)
    lat.ranset(4)
    hb = lat.field()
    lat.field_gauss(hb, 0.5)
    zero = np.zeros((lat.volh, 3, 4), np.complex128)
    hx = lat.field(zero)
    lat.solve_batch([hx], [hb], para, tol=1e-10, block=1)
    x1 = lat.field_get(hx)
    lat.mom_gauss()
    before = lat.device_bytes
    lat.release_scratch(solver=True, hmc=True)
    after = lat.device_bytes
    assert after < before
    with pytest.raises(bq.BqcdgError) as e:
        lat.mom_action()
    assert e.value.status == bq.EINVAL
    lat.field_set(hx, zero)
    lat.solve_batch([hx], [hb], para, tol=1e-10, block=1)
    assert np.array_equal(lat.field_get(hx), x1)
    lat.mom_gauss()
    assert lat.mom_action() > 0
    lat.close()


@pytest.mark.parametrize("prec", ["half", "single"])
@pytest.mark.parametrize("nbt", [2, 4])
def test_register_blocked_batch_matches_fp64(oracle_setup, bq, prec, nbt):
    """The register-blocked passes (nbt right-hand sides per stencil thread,
    one link and clover load for all of them) solve every system of a batch
    whose size nbt does not divide (5: groups of 2+2+1 or 4+1, so some threads
    carry absent RHS), with a shift per system: each solution equals the
    single-system FP64 solve, and the iteration counts stay those of one RHS
    per thread."""
    s = oracle_setup
    g, lat = s["g"], s["lat"]
    para = bq.HmcPara(kappa=s["kappa"], csw=s["csw"])
    precision = bq.PREC_HALF if prec == "half" else bq.PREC_SINGLE
    rhos = [0.0, 0.1, 0.02, 0.3, 0.0]
    bs = [g.gauss_spinor(0) for _ in rhos]
    hb = [lat.field(b) for b in bs]
    zero = np.zeros_like(bs[0])
    runs = {}
    for k in (1, nbt):
        hx = [lat.field(zero) for _ in bs]
        infos = lat.solve_batch_shifted(hx, hb, para, rhos, precision=precision, tol=1e-10, block=5,
                                        rhs_per_thread=k)
        runs[k] = (infos, [lat.field_get(h) for h in hx])
    for j, rho in enumerate(rhos):
        info = runs[nbt][0][j]
        assert info.converged == 1 and info.true_rtr <= 1e-20 * info.b2, info.as_dict()
        x_ref, _ = lat.solve(zero, bs[j], para, precision=bq.PREC_DOUBLE, tol=1e-12, rho=rho)
        assert np.linalg.norm(runs[nbt][1][j] - x_ref) <= 1e-8 * np.linalg.norm(x_ref), (j, rho)
        assert abs(info.niter - runs[1][0][j].niter) <= max(3, runs[1][0][j].niter // 20)


@pytest.mark.parametrize("nbt", [2, 4])
def test_register_blocked_batch_wilson(bq, nbt):
    """c_sw = 0: the register-blocked second pass without a clover block
    ((1 + rho) x + b D t) matches the FP64 solve of each system."""
    L = (8, 8, 8, 8)
    lat = bq.Lattice(L, (1, 1, 1, -1))
    lat.ranset(11)
    lat.conf_hot()
    lat.conf_relax(2)
    para = bq.HmcPara(kappa=0.12, csw=0.0)
    rhos = [0.05, 0.0, 0.2, 0.1]
    zero = np.zeros((lat.volh, 3, 4), np.complex128)
    hb = []
    for _ in rhos:
        h = lat.field()
        lat.field_gauss(h, 0.5)
        hb.append(h)
    hx = [lat.field(zero) for _ in rhos]
    infos = lat.solve_batch_shifted(hx, hb, para, rhos, precision=bq.PREC_SINGLE, tol=1e-10, block=4,
                                    rhs_per_thread=nbt)
    for j, rho in enumerate(rhos):
        assert infos[j].converged == 1, infos[j].as_dict()
        b = lat.field_get(hb[j])
        x_ref, _ = lat.solve(zero, b, para, precision=bq.PREC_DOUBLE, tol=1e-12, rho=rho)
        assert np.linalg.norm(lat.field_get(hx[j]) - x_ref) <= 1e-8 * np.linalg.norm(x_ref), (j, rho)
    # the timed batched pass runs for every choice of RHS per thread
    for k in (0, 1, 2, 4):
        assert lat.time_pass_batch(hx, para, bq.PREC_HALF, 2, rhs_per_thread=k) > 0
    lat.close()


def test_shifted_batch_per_rhs_tolerance(oracle_setup, bq):
    """One tolerance per system: each stops at its own |r|/|b|, so a looser
    system retires earlier while the others go on in the same launches."""
    s = oracle_setup
    g, lat = s["g"], s["lat"]
    para = bq.HmcPara(kappa=s["kappa"], csw=s["csw"])
    tols = [1e-5, 1e-10, 1e-7]
    bs = [g.gauss_spinor(0) for _ in tols]
    hb = [lat.field(b) for b in bs]
    hx = [lat.field(np.zeros_like(bs[0])) for _ in tols]
    infos = lat.solve_batch_shifted(hx, hb, para, [0.1] * 3, tol=tols, block=3)
    for info, t in zip(infos, tols):
        assert info.converged == 1 and info.true_rtr <= t * t * info.b2, info.as_dict()
    assert infos[0].niter < infos[2].niter < infos[1].niter


@pytest.mark.parametrize("nbt", [1, 2, 4])
def test_batch_on_a_ragged_lattice(bq, oracle, nbt):
    """6^4: 648 sites per parity, so the last block of every launch is partly
    empty, and 3 right-hand sides leave absent lanes in the register-blocked
    groups.  Every batched solution equals its FP64 solve."""
    L = (6, 6, 6, 6)
    g = oracle.Geom(L, (1, 1, 1, -1))
    oracle.ranset(31)
    u = g.hot()
    clov = g.clover_init(u, 1.9192 * 0.13)
    lat = bq.Lattice(L, (1, 1, 1, -1))
    lat.load_gauge(g.flip_bc(u.copy()), flipped=True)
    lat.load_clover(*clov)
    para = bq.HmcPara(kappa=0.13, csw=1.9192)
    rhos = [0.0, 0.2, 0.05]
    bs = [g.gauss_spinor(0) for _ in rhos]
    hb = [lat.field(b) for b in bs]
    zero = np.zeros_like(bs[0])
    hx = [lat.field(zero) for _ in rhos]
    infos = lat.solve_batch_shifted(hx, hb, para, rhos, tol=1e-10, block=3, rhs_per_thread=nbt)
    for j, rho in enumerate(rhos):
        assert infos[j].converged == 1, infos[j].as_dict()
        x_ref, _ = lat.solve(zero, bs[j], para, precision=bq.PREC_DOUBLE, tol=1e-12, rho=rho)
        assert np.linalg.norm(lat.field_get(hx[j]) - x_ref) <= 1e-8 * np.linalg.norm(x_ref), (j, rho)
    lat.close()
