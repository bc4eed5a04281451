"""Host logic of the MRE initial guess (bqcdg/hmc.py Mre, mre.F90:29-279) on CPU.

Mre reads its scalar products back in batches (Lattice.field_cdot_pairs).
Against a numpy stand-in for the resident fields it must give the same trial
vector as the step-by-step form of mre.F90 (one product per read-back),
restated here.
"""
import math

import numpy as np
import pytest

from bqcdg.hmc import Mre


class NumpyLattice:
    """Resident fields as numpy vectors; op_dev applies one fixed matrix."""

    MAX_DOT_PAIRS = 8

    def __init__(self, n=48, seed=0):
        rng = np.random.default_rng(seed)
        self.n = n
        self.m = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 4 * np.eye(n)
        self.f = {}
        self.pair_calls = []

    def field(self, host=None):
        h = len(self.f) + 1
        self.f[h] = np.zeros(self.n, complex)
        return h

    def field_cdot(self, a, b):
        return complex(np.vdot(self.f[a], self.f[b]))

    def field_cdot_pairs(self, pairs):
        # as Lattice.field_cdot_pairs: launches of up to MAX_DOT_PAIRS, none
        # for an empty list
        for k in range(0, len(pairs), self.MAX_DOT_PAIRS):
            self.pair_calls.append(len(pairs[k:k + self.MAX_DOT_PAIRS]))
        return [self.field_cdot(a, b) for a, b in pairs]

    def field_caxpby(self, hy, ay, a, hx):
        self.f[hy] = ay * self.f[hy] + complex(a) * self.f[hx] if ay != 0 else complex(a) * self.f[hx]

    def field_copy(self, dst, src):
        self.f[dst] = self.f[src].copy()

    def op_dev(self, which, hout, hin, para, rho=None):
        self.f[hout] = self.m @ self.f[hin]


def stepwise_get(lat, vecs, phi):
    """mre.F90:68-213 one scalar product at a time (the loop order of the
    reference), on copies of the stored vectors."""
    v = [lat.f[h].copy() for h in vecs]
    r = len(v)
    for k in range(r):
        v[k] = v[k] * (1.0 / math.sqrt(np.vdot(v[k], v[k]).real))
        for j in range(k + 1, r):
            v[j] = v[j] - np.vdot(v[k], v[j]).real * v[k]
    mv = [lat.m @ x for x in v]
    bb = np.array([np.vdot(x, phi) for x in v])
    ga = np.zeros((r, r), complex)
    for i in range(r):
        ga[i, i] = np.vdot(mv[i], mv[i]).real
        for j in range(i + 1, r):
            ga[i, j] = np.vdot(mv[i], mv[j])
            ga[j, i] = np.conj(ga[i, j])
    x = Mre._gauss_jordan(ga, bb)
    trial = x[0] * v[0]
    for i in range(1, r):
        trial = trial + x[i] * v[i]
    return trial, ga, bb


@pytest.mark.parametrize("nput", [2, 3, 7, 9])
def test_batched_products_give_the_stepwise_guess(nput):
    lat = NumpyLattice()
    rng = np.random.default_rng(nput)
    mre = Mre(lat, 7)
    h = lat.field()
    for _ in range(nput):
        lat.f[h] = rng.standard_normal(lat.n) + 1j * rng.standard_normal(lat.n)
        mre.put(h, False)
    assert mre.rank == min(nput, 7)
    stored = list(mre.vec[:mre.rank])
    phi_h, trial_h = lat.field(), lat.field()
    lat.f[phi_h] = rng.standard_normal(lat.n) + 1j * rng.standard_normal(lat.n)
    want, ga, bb = stepwise_get(lat, stored, lat.f[phi_h])
    mre.get("mtil", trial_h, phi_h, None)
    got = lat.f[trial_h]
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12)
    # the Gram matrix is Hermitian positive, as mre.F90's elimination assumes
    assert np.allclose(ga, np.conj(ga.T)) and np.all(np.linalg.eigvalsh(ga) > 0)
    # every batch fits one launch, and the whole guess takes a few read-backs
    r = mre.rank
    assert max(lat.pair_calls) <= lat.MAX_DOT_PAIRS
    assert len(lat.pair_calls) <= (r - 1) + 1 + math.ceil(r * (r + 1) / 2 / lat.MAX_DOT_PAIRS)


def test_rank_one_and_reset():
    lat = NumpyLattice()
    mre = Mre(lat, 4)
    h, phi_h, trial_h = lat.field(), lat.field(), lat.field()
    lat.f[h] = np.arange(lat.n) + 1j
    lat.f[phi_h] = np.ones(lat.n, complex)
    mre.get("mtil", trial_h, phi_h, None)            # nothing stored: phi itself
    assert np.array_equal(lat.f[trial_h], lat.f[phi_h])
    mre.put(h, False)
    mre.get("mtil", trial_h, phi_h, None)            # one stored: that solution
    assert np.array_equal(lat.f[trial_h], lat.f[h])
    mre.put(h, True)
    assert mre.rank == 0


def test_lattice_wrapper_splits_pairs_into_launches(bq, monkeypatch):
    """Lattice.field_cdot_pairs against a stand-in for the library call: at
    most MAX_DOT_PAIRS pairs per call, in order, results in order."""
    calls = []

    class FakeLib:
        def bqcdg_field_cdot_pairs(self, h, n, ha, hb, re, im):
            calls.append((h, n, list(ha)[:n], list(hb)[:n]))
            for j in range(n):
                re[j] = 10.0 * ha[j] + hb[j]
                im[j] = -float(ha[j])
            return 0

    monkeypatch.setattr(bq, "lib", lambda: FakeLib())
    lat = object.__new__(bq.Lattice)
    lat.h = "ctx"
    pairs = [(a, a + 1) for a in range(11)]
    got = lat.field_cdot_pairs(pairs)
    assert [c[1] for c in calls] == [8, 3] and all(c[0] == "ctx" for c in calls)
    assert [c[2] for c in calls] == [list(range(8)), [8, 9, 10]]
    assert got == [complex(10.0 * a + a + 1, -a) for a in range(11)]
    calls.clear()
    assert lat.field_cdot_pairs([]) == [] and not calls
