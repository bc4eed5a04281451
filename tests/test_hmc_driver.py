"""Host logic of the device HMC driver (bqcdg/hmc.py), on CPU.

The driver only sequences calls into the C ABI, so its control flow can be
checked without a GPU against a recording stand-in for the Lattice: the
nested leapfrog of hmc_leap_frog.F90 (step sizes, the halved last steps, the
action evaluation on the last one), the model switches of hmc_integrator.F90,
and the Gauss-Jordan solve of the MRE Gram system (mre.F90:215-279).
"""
import math
import types

import numpy as np
import pytest

from bqcdg.hmc import Hmc, Mre


class FakeLattice:
    """Records the ABI calls of a trajectory; fields are handles only."""

    def __init__(self):
        self.volh = 128
        self.calls = []
        self._next = 1

    def field(self, host=None):
        self._next += 1
        return self._next

    def __getattr__(self, name):
        def rec(*args, **kw):
            self.calls.append((name, args, kw))
            if name in ("field_cdot",):
                return complex(1.0, 0.0)
            if name in ("mom_action", "sg", "clover_action", "mom_change"):
                return 1.0
            if name == "cg_dev":
                return 10, types.SimpleNamespace(seconds=1e-3, converged=1, niter=10)
            if name == "ranf":
                return 0.5
        return rec


def run(model, ntau=3, m_scale=2, tau_len=0.6, csw=1.9192):
    lat = FakeLattice()
    h = Hmc(lat, beta=5.29, kappa=0.13, csw=csw, rho=0.1, traj_length=tau_len, ntau=ntau, m_scale=m_scale,
            model=model, mre_n_vec=0)
    lat.calls.clear()
    rec = h.trajectory(force_accept=True)
    return lat.calls, rec


def steps(calls, name):
    return [c[1][0] for c in calls if c[0] == name]


@pytest.mark.parametrize("model", ["A", "B", "C"])
def test_leapfrog_schedule(model):
    ntau, m, tau_len = 3, 2, 0.6
    calls, _ = run(model, ntau, m, tau_len)
    tau = tau_len / ntau
    # gauge updates: ntau * m inner steps of tau / m, total = trajectory length
    u = steps(calls, "hmc_u_dev")
    assert len(u) == ntau * m and all(abs(s - tau / m) < 1e-15 for s in u)
    assert abs(sum(u) - tau_len) < 1e-12
    # gauge force: the inner scale, half steps at both ends
    g = steps(calls, "dsg_dev")
    want = [0.5 * tau / m] + [tau / m] * (ntau * m - 1) + [0.5 * tau / m]
    assert np.allclose(g, want)
    assert abs(sum(g) - tau_len) < 1e-12
    # fermion forces: S_f1 on the inner scale for model C, outer otherwise;
    # S_f2 on the outer scale (not present in model A)
    n_f1 = len([c for c in calls if c[0] == "dsf_dev"])
    outer = ntau + 1
    if model == "A":
        assert n_f1 == outer
    elif model == "B":
        assert n_f1 == 2 * outer
    else:
        assert n_f1 == (ntau * m + 1) + outer


def test_actions_measured_at_the_last_step_only():
    calls, rec = run("C")
    # the action is evaluated from |b|^2 only with calc_sf: the halved last
    # steps, one dsf1 and one dsf2 (field_cdot(b, b) besides init_phi's two)
    cdots = [c for c in calls if c[0] == "field_cdot"]
    assert len(cdots) == 2 + 2
    assert rec["accepted"] and rec["cg_calls"] > 0


def test_no_clover_skips_the_det_force():
    calls, _ = run("A", csw=0.0)
    assert not [c for c in calls if c[0] == "dsd_dev"]


def test_solver_choice_is_checked():
    with pytest.raises(ValueError):
        Hmc(FakeLattice(), 5.29, 0.13, 1.9192, 0.1, 1.0, 2, 2, solver="bicgstab")


def test_mre_gauss_jordan_matches_numpy():
    rng = np.random.default_rng(0)
    for n in (2, 3, 5, 7):
        a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        a = a @ np.conj(a.T) + n * np.eye(n)          # a Hermitian positive Gram matrix
        b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        x = Mre._gauss_jordan(a, b)
        assert np.allclose(x, np.linalg.solve(a, b), rtol=1e-12, atol=1e-12)
    with pytest.raises(ArithmeticError):
        Mre._gauss_jordan(np.zeros((2, 2), complex), np.ones(2, complex))
