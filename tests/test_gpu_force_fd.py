"""The pseudofermion force against finite differences of the action.

S_f1 = phi^+ (W^+W)^-1 phi with W = M~ + rho (the clover operator on the
flipped links; the clover blocks are rebuilt on the device from each perturbed
gauge field).  dsf (dsf.F90:28) adds p -= step * dS/domega_j for
U -> exp(i omega_j lambda_j) U (hmc_u.F90:53-60), so along a direction h
(h_j per link) the derivative is  dS/deps = -(p_new - p_old).h / step.
Two checks, both along 16 random su(3) directions and to 1e-7 relative:

* 24^3x48, the HMC configuration's system (hot start, one conf_relax
  sweep, 10 forced-accept pure-gauge trajectories at beta 5.29; kappa
  0.1355, c_sw 1.9192, rho = 0.1355/0.13 - 1): central differences at
  eps = 1e-5, (S(+eps) - S(-eps)) / (2 eps);
* 4^4, Wilson and clover: a fourth-order quotient at eps = 1e-4.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def gell_mann():
    lam = np.zeros((8, 3, 3), complex)
    lam[0][0, 1] = lam[0][1, 0] = 1
    lam[1][0, 1], lam[1][1, 0] = -1j, 1j
    lam[2][0, 0], lam[2][1, 1] = 1, -1
    lam[3][0, 2] = lam[3][2, 0] = 1
    lam[4][0, 2], lam[4][2, 0] = -1j, 1j
    lam[5][1, 2] = lam[5][2, 1] = 1
    lam[6][1, 2], lam[6][2, 1] = -1j, 1j
    lam[7] = np.diag([1, 1, -2]) / np.sqrt(3)
    return lam


def perturb(oracle, u, h, eps):
    """U -> exp(i eps h_j lambda_j) U on every link -- the update of hmc_u.F90
    (gen2u, su3.F90:28, whose generators are the Gell-Mann matrices of
    im_tr_j).  The exponential is taken exactly from the eigen-decomposition
    of the Hermitian H = h.lambda: gen2u's closed form loses accuracy (and is
    undefined at h = 0) for arguments as small as eps = 1e-5.  Links are
    stored [col][row], so a stored block is the transposed matrix."""
    H = np.einsum("...j,jab->...ab", h, gell_mann())
    w, V = np.linalg.eigh(H)
    E = (V * np.exp(1j * eps * w)[..., None, :]) @ np.conj(np.swapaxes(V, -1, -2))
    M = np.swapaxes(u, -1, -2)
    return np.swapaxes(E @ M, -1, -2).copy()


def perturb_taylor(u, h, eps):
    """perturb() with exp(i eps H) summed as its Taylor series to the fifth
    power: |eps H| is below 1e-4 here, so the omitted terms are under 1e-22
    and the result is unitary to rounding (vectorised, for 2.6M links)."""
    H = np.einsum("...j,jab->...ab", h, gell_mann())
    X = 1j * eps * H
    E = np.broadcast_to(np.eye(3, dtype=complex), X.shape).copy()
    term = E.copy()
    for k in range(1, 6):
        term = term @ X / k
        E += term
    M = np.swapaxes(u, -1, -2)
    return np.swapaxes(E @ M, -1, -2).copy()


def xdot(a, b):
    """Re <a, b> summed in extended precision: over 4M sites the rounding of
    a double-precision sum would be comparable to S(+eps) - S(-eps)."""
    return np.sum((a.real * b.real + a.imag * b.imag).astype(np.longdouble), dtype=np.longdouble)


def action(lat, g, oracle, u, phi, para, csw_kappa):
    """S = phi^+ A^-1 phi (A = W^+W) from the Galerkin estimate
    2 Re <phi,x> - <x,Ax>, whose error is quadratic in the solver's: the
    fourth-order difference quotient at eps = 1e-4 needs S to ~1e-15 relative."""
    uf = g.flip_bc(u.copy())
    lat.load_gauge(uf, flipped=True)
    lat.clover_init(csw_kappa)
    x, info = lat.solve(np.zeros_like(phi), phi, para, precision=0, tol=1e-13, rho=para.rho)
    assert info.converged
    ax = lat.w_dagger_w(x, para)
    return float(2.0 * np.vdot(phi, x).real - np.vdot(x, ax).real)


@pytest.mark.parametrize("csw", [0.0, 1.9192])
def test_dsf_matches_finite_differences(oracle, bq, csw):
    L = (4, 4, 4, 4)
    g = oracle.Geom(L, (1, 1, 1, -1))
    oracle.ranset(2024)
    u = g.hot()
    g.relax(u, 2)
    kappa, rho = 0.12, 0.1
    para = bq.HmcPara(kappa=kappa, csw=csw, rho=rho)
    phi = g.gauss_spinor(0)
    rng = np.random.default_rng(7)
    with bq.Lattice(L, (1, 1, 1, -1)) as lat:
        # force at U: a = (W^+W)^-1 phi, b = W a  (dsf1.F90:64-71)
        uf = g.flip_bc(u.copy())
        lat.load_gauge(uf, flipped=True)
        lat.clover_init(csw * kappa)
        a, info = lat.solve(np.zeros_like(phi), phi, para, precision=0, tol=1e-13)
        b = lat.w_mult(a, para)
        step = 1.0
        p0 = np.zeros((4, 2, lat.volh, 8))
        dS = -lat.dsf(p0.copy(), step, para, a, b) / step          # dS/domega_j per link
        # fourth-order central difference: truncation O(eps^4) is negligible,
        # and eps = 1e-4 keeps the rounding noise of S (~1e-12 absolute)
        # divided by eps well under the tolerance
        eps = 1e-4
        errs = []
        for _ in range(16):
            h = rng.standard_normal((4, 2, lat.volh, 8))
            s = {k: action(lat, g, oracle, perturb(oracle, u, h, k * eps), phi, para, csw * kappa)
                 for k in (-2, -1, 1, 2)}
            fd = (8.0 * (s[1] - s[-1]) - (s[2] - s[-2])) / (12.0 * eps)
            an = float(np.sum(dS * h))
            errs.append(abs(fd - an) / abs(an))
        print("finite differences 4^4, csw %g: relative errors" % csw, ["%.2e" % e for e in errs])
        assert max(errs) < 1e-7, errs


@pytest.mark.slow
def test_dsf_matches_central_differences_24x24x24x48(bq):
    from bqcdg.hmc import quenched_trajectory
    L = (24, 24, 24, 48)
    kappa, csw, beta = 0.1355, 1.9192, 5.29
    rho = kappa / 0.13 - 1.0
    para = bq.HmcPara(kappa=kappa, csw=csw, rho=rho)
    with bq.Lattice(L, (1, 1, 1, -1)) as lat:
        lat.ranset(0)
        lat.conf_hot()
        lat.conf_relax(1)
        for _ in range(10):
            quenched_trajectory(lat, beta, 1.0, 50, force_accept=True)
        u = lat.get_gauge(flipped=False)
        lat.clover_init(csw * kappa)
        lat.ranset(5)
        hphi = lat.field()
        lat.field_gauss(hphi, 0.5)
        phi = lat.field_get(hphi)

        def S(links):
            lat.load_gauge(links, flipped=False)
            lat.clover_init(csw * kappa)
            x, info = lat.solve(np.zeros_like(phi), phi, para, precision=0, tol=1e-13)
            assert info.converged
            ax = lat.w_dagger_w(x, para)
            return float(2.0 * xdot(phi, x) - xdot(x, ax))

        lat.load_gauge(u, flipped=False)
        lat.clover_init(csw * kappa)
        a, info = lat.solve(np.zeros_like(phi), phi, para, precision=0, tol=1e-13)
        assert info.converged
        b = lat.w_mult(a, para)
        p0 = np.zeros((4, 2, lat.volh, 8))
        dS = -lat.dsf(p0.copy(), 1.0, para, a, b)
        eps = 1e-5
        rng = np.random.default_rng(11)
        errs = []
        for _ in range(16):
            h = rng.standard_normal((4, 2, lat.volh, 8))
            fd = (S(perturb_taylor(u, h, eps)) - S(perturb_taylor(u, h, -eps))) / (2.0 * eps)
            an = float(np.sum(dS * h))
            errs.append(abs(fd - an) / abs(an))
        print("finite differences 24^3x48, eps 1e-5: relative errors", ["%.2e" % e for e in errs])
        assert max(errs) < 1e-7, errs
