"""The reduced-precision operators against the FP64 one.

The sloppy iterations of the mixed-precision solver apply M~^+M~ with FP32 or
int16 fields (int16: offset-binary fixed point, one float norm per site for
spinors and clover blocks, links scaled by 32767).  Applied once to the same
input, each must equal the FP64 operator to its storage precision: FP32 to a
few 1e-7, int16 to a few 1e-5 relative in the 2-norm (its quantisation step is
2^-15 of the largest component of a site).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {1: 2e-6, 2: 2e-4}


@pytest.fixture(scope="module", params=[(8, 8, 8, 16), (6, 6, 6, 6), (2, 4, 6, 4)],
                ids=lambda L: "x".join(map(str, L)))
def lat(request, bq):
    lt = bq.Lattice(request.param, (1, 1, 1, -1))
    lt.ranset(5)
    lt.conf_hot()
    lt.conf_relax(1)
    lt.clover_init(1.9192 * 0.13)
    yield lt
    lt.close()


def apply_both(lat, bq, para, prec, x):
    hin = lat.field(x)
    h64, hs = lat.field(), lat.field()
    lat.mdagm_dev(h64, hin, para, bq.PREC_DOUBLE, 1)
    lat.mdagm_dev(hs, hin, para, prec, 1)
    return lat.field_get(h64), lat.field_get(hs)


def gauss(lat, seed):
    h = lat.field()
    lat.ranset(seed)
    lat.field_gauss(h, 0.5)
    return lat.field_get(h)


@pytest.mark.parametrize("csw", [0.0, 1.9192])
@pytest.mark.parametrize("rho", [0.0, 0.1])
@pytest.mark.parametrize("prec", [1, 2])
def test_sloppy_mdagm_matches_fp64(lat, bq, prec, csw, rho):
    para = bq.HmcPara(kappa=0.13, csw=csw, rho=rho)
    lat.clover_init(csw * 0.13)
    ref, got = apply_both(lat, bq, para, prec, gauss(lat, 17))
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < TOL[prec], err
    assert err > 1e-12  # the reduced precision is really in use


def test_int16_keeps_relative_accuracy_per_site(lat, bq):
    """One norm per site: an input whose sites span 12 orders of magnitude
    keeps its accuracy on the sites that dominate the result."""
    para = bq.HmcPara(kappa=0.13, csw=1.9192)
    lat.clover_init(1.9192 * 0.13)
    x = gauss(lat, 23)
    scale = 10.0 ** np.linspace(-6, 6, lat.volh)
    ref, got = apply_both(lat, bq, para, bq.PREC_HALF, x * scale[:, None, None])
    big = scale > 1e3
    err = np.linalg.norm((got - ref)[big]) / np.linalg.norm(ref[big])
    assert err < 2e-4, err
