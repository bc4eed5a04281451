"""The resident HMC pieces against the oracle, and one device trajectory
against the reference's golden quick-test record.

Links are stored [col][row] (Fortran u(row,col)), so a stored block is the
transposed matrix: U -> G U reads u_stored -> u_stored @ g_stored, with
g_stored the transposed gen2u as the oracle returns it.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
L = (4, 4, 4, 4)
BC = (1, 1, 1, -1)


@pytest.fixture
def pair(oracle, bq):
    g = oracle.Geom(L, BC)
    oracle.ranset(11)
    u = g.hot()
    g.relax(u, 1)
    lat = bq.Lattice(L, BC)
    lat.load_gauge(u, flipped=False)
    yield g, u, lat
    lat.close()


def test_momentum_draw_and_kinetic_term(oracle, bq, pair):
    g, u, lat = pair
    oracle.ranset(99)
    p_ref = g.gauss_momenta()
    lat.ranset(99)
    lat.mom_gauss()
    # same random stream exactly; the Box-Muller transcendentals of the
    # device and the host libm differ in the last bits
    assert np.abs(lat.mom_get() - p_ref).max() <= 1e-13
    assert lat.ranget() == oracle.ranget()
    assert abs(lat.mom_action() - 0.5 * np.sum(p_ref ** 2)) <= 1e-13 * np.sum(p_ref ** 2)


def test_gauge_update_matches_gen2u(oracle, bq, pair):
    g, u, lat = pair
    rng = np.random.default_rng(3)
    p = rng.standard_normal((4, 2, g.volh, 8))
    step = 0.07
    lat.mom_set(p)
    lat.hmc_u_dev(step, 0.0)
    got = lat.get_gauge(flipped=False)
    want = np.empty_like(u)
    for mu in range(4):
        for eo in range(2):
            for i in range(g.volh):
                want[mu, eo, i] = u[mu, eo, i] @ oracle.gen2u(step * p[mu, eo, i])
    assert np.abs(got - want).max() < 1e-13
    # unitary to rounding after u_normalize
    m = np.swapaxes(got, -1, -2)
    eye = np.eye(3)
    assert np.abs(m @ np.conj(np.swapaxes(m, -1, -2)) - eye).max() < 1e-14


def test_gauge_force_matches_oracle(oracle, bq, pair):
    g, u, lat = pair
    rng = np.random.default_rng(5)
    p = rng.standard_normal((4, 2, g.volh, 8))
    lat.mom_set(p)
    lat.dsg_dev(0.1, 5.29)
    want = g.dsg(p.copy(), u, 0.1, 5.29)
    got = lat.mom_get()
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


def test_resident_forces_and_ops_match_host_entry_points(oracle, bq, pair):
    g, u, lat = pair
    para = bq.HmcPara(kappa=0.13, csw=1.9192, rho=0.1)
    lat.clover_init(para.csw_kappa)
    a, b = g.gauss_spinor(0), g.gauss_spinor(0)
    p = np.random.default_rng(8).standard_normal((4, 2, g.volh, 8))
    want = lat.dsf(p.copy(), 0.3, para, a, b)
    ha, hb, hc = lat.field(a), lat.field(b), lat.field()
    lat.mom_set(p)
    lat.dsf_dev(0.3, para, ha, hb)
    assert np.abs(lat.mom_get() - want).max() <= 1e-13 * np.abs(want).max()
    want = lat.clover_dsd(1, p.copy(), -2 * 0.3 * para.csw_kappa / 8)
    lat.mom_set(p)
    lat.dsd_dev(0.3, para)
    assert np.abs(lat.mom_get() - want).max() <= 1e-13 * np.abs(want).max()
    for name in ("mtil", "mtil_dag", "mtdagmt", "w_mult", "w_mult_dag", "w_dagger_w"):
        lat.op_dev(name, hc, ha, para)
        ref = getattr(lat, name)(a, para)
        assert np.linalg.norm(lat.field_get(hc) - ref) <= 1e-14 * np.linalg.norm(ref), name
    z = lat.field_cdot(ha, hb)
    zr = np.vdot(a, b)
    assert abs(z - zr) <= 1e-13 * abs(zr)
    lat.field_caxpby(hc, 0.5, 0.25 - 2j, ha)
    ref = 0.5 * lat.w_dagger_w(a, para) + (0.25 - 2j) * a
    assert np.linalg.norm(lat.field_get(hc) - ref) <= 1e-14 * np.linalg.norm(ref)
    # the batched products of the MRE guess: each equal to field_cdot's bit
    # for bit, in launches of 1 to 8 pairs (ragged last launch of 11 pairs)
    hs = [ha, hb, hc, lat.field(g.gauss_spinor(0))]
    pairs = [(hs[i % 4], hs[(3 * i + 1) % 4]) for i in range(11)]
    for n in (1, 2, 5, 8, 11):
        got = lat.field_cdot_pairs(pairs[:n])
        assert got == [lat.field_cdot(x, y) for x, y in pairs[:n]]


def test_resident_cg_matches_reference_cg(oracle, bq, pair):
    g, u, lat = pair
    para = bq.HmcPara(kappa=0.13, csw=1.9192, rho=0.1)
    lat.clover_init(para.csw_kappa)
    uf = g.flip_bc(u.copy())
    clov = g.clover_init(u, para.csw_kappa)
    bvec = g.gauss_spinor(0)
    x_ref, it_ref, _, rc = g.cg("w_dagger_w", np.zeros_like(bvec), bvec, uf, clov, 0.13, para.csw_kappa,
                                rho=0.1, rest=1e-10)
    hx, hb = lat.field(np.zeros_like(bvec)), lat.field(bvec)
    it, info = lat.cg_dev(hx, hb, para, 1e-10)
    assert rc == 0 and info.converged and abs(it - it_ref) <= 1
    assert np.linalg.norm(lat.field_get(hx) - x_ref) <= 1e-8 * np.linalg.norm(x_ref)


def test_quick_test_trajectory_on_device(bq):
    """work/out.quick-test.reference: one 4^4 model-C trajectory (Hasenbusch
    rho 0.1, kappa 0.13, c_sw 2.3327, beta 5.0, tau 0.2 in 10 steps of 3 inner
    steps, MRE with 7 vectors, CG to rtr <= 1e-5) from a cold start with the
    default seed, forced accept: every printed digit of the iteration counts, the
    force monitors, the plaquette, exp(-dH) and the final RNG seed."""
    from bqcdg.hmc import Hmc
    with open(os.path.join(HERE, "golden", "quick_test.json")) as f:
        gold = json.load(f)
    lat = bq.Lattice(L, BC)
    try:
        lat.ranset(0)
        lat.conf_cold()
        hmc = Hmc(lat, beta=5.0, kappa=0.13, csw=2.3327, rho=0.1, traj_length=0.2, ntau=10, m_scale=3,
                  model="C", rest=1e-5, maxiter=1000, mre_n_vec=7)
        rec = hmc.trajectory(force_accept=True)
        assert (rec["it_f1"], rec["it_f2"]) == (gold["it"]["f1"], gold["it"]["f2"]), rec
        for key, got in (("Favg", rec["f_avg"]), ("Fmax", rec["f_max"])):
            for a, b in zip(got, gold[key]["values"]):
                assert abs(a - b) <= 6e-10 * abs(b), (key, a, b)
        assert abs(rec["plaq_energy"] - gold["fa"]["plaq_energy"]) <= 6e-11
        assert abs(rec["exp_dh"] - gold["fa"]["exp_mdh"]) <= 6e-11
        assert (rec["cg_calls"], rec["cg_it_tot"], rec["cg_it_max"]) == \
            (gold["fa"]["cg_calls"], gold["fa"]["cg_it_tot"], gold["fa"]["cg_it_max"])
        assert lat.ranget() == gold["final_seed"]
    finally:
        lat.close()


def test_twenty_trajectories_on_device(bq):
    """work/out.test.reference: the quick-test system for 20 trajectories on
    the device, the first 10 force-accepted and the next 10 through the
    Metropolis test with the context's RNG stream; every record to the
    reference's printed precision (iteration counts and CG statistics
    exactly) and the final seed exactly."""
    from bqcdg.hmc import Hmc
    from test_oracle_golden import check_test20
    with open(os.path.join(HERE, "golden", "test20.json")) as f:
        gold = json.load(f)
    lat = bq.Lattice(L, BC)
    try:
        lat.ranset(0)
        lat.conf_cold()
        hmc = Hmc(lat, beta=5.0, kappa=0.13, csw=2.3327, rho=0.1, traj_length=0.2, ntau=10, m_scale=3,
                  model="C", rest=1e-5, maxiter=1000, mre_n_vec=7)
        recs = []
        for traj in range(-9, 11):
            r = hmc.trajectory(force_accept=traj <= 0)
            recs.append({"traj": traj, "f1": r["it_f1"], "f2": r["it_f2"], "plaq_energy": r["plaq_energy"],
                         "exp_mdh": r["exp_dh"], "accepted": int(r["accepted"]), "cg_calls": r["cg_calls"],
                         "cg_it_tot": r["cg_it_tot"], "cg_it_max": r["cg_it_max"]})
        check_test20(recs, gold)
        assert lat.ranget() == gold["final_seed"]
    finally:
        lat.close()


def test_smp_benchmark_trajectory_on_device(bq):
    """work/out.smp.reference: the reference's SMP benchmark (work/input.smp),
    24^3x48, model A, c_sw 1.923076923076923, kappa 0.13, beta 5: one
    force-accepted trajectory of 10 steps from a cold start with the default
    seed, the CG capped at 100 iterations (solver_rest 1e-99, no convergence
    ignored) and no MRE vectors.  The device run reproduces its %fa record
    (CG statistics exactly, the plaquette to the printed precision) and the
    final seed."""
    from bqcdg.hmc import Hmc
    with open(os.path.join(HERE, "golden", "smp.json")) as f:
        gold = json.load(f)
    lat = bq.Lattice((24, 24, 24, 48), BC)
    try:
        lat.ranset(0)
        lat.conf_cold()
        hmc = Hmc(lat, beta=5.0, kappa=0.13, csw=1.923076923076923, rho=0.0, traj_length=0.2, ntau=10, m_scale=1,
                  model="A", rest=1e-99, maxiter=100, mre_n_vec=0, cg_log=2)
        rec = hmc.trajectory(force_accept=True)
        fa = gold["fa"]
        assert (rec["cg_calls"], rec["cg_it_tot"], rec["cg_it_max"]) == (fa["cg_calls"], fa["cg_it_tot"],
                                                                          fa["cg_it_max"]), rec
        assert abs(rec["plaq_energy"] - fa["plaq_energy"]) <= 2e-9, rec
        assert rec["exp_dh"] < 5e-11
        assert lat.ranget() == gold["final_seed"]
    finally:
        lat.close()


def test_mpp_benchmark_job_on_device(bq):
    """work/out.mpp.reference: the reference's MPP benchmark (work/input.mpp,
    run there on 6912 MPI processes), 48^3x96, model A, c_sw
    1.923076923076923, kappa 0.13, beta 5: a force-accepted trajectory of 20
    steps, then one through the Metropolis test, which rejects it (the links
    go back); CG capped at 100 iterations, no MRE.  On one GPU the device run
    reproduces both records and the final seed."""
    from bqcdg.hmc import Hmc
    with open(os.path.join(HERE, "golden", "mpp.json")) as f:
        gold = json.load(f)
    want = [dict(gold["fa"], accepted=1)] + gold["mc"]
    lat = bq.Lattice((48, 48, 48, 96), BC)
    try:
        lat.ranset(0)
        lat.conf_cold()
        hmc = Hmc(lat, beta=5.0, kappa=0.13, csw=1.923076923076923, rho=0.0, traj_length=0.2, ntau=20, m_scale=1,
                  model="A", rest=1e-99, maxiter=100, mre_n_vec=0, cg_log=2)
        for k, w in enumerate(want):
            rec = hmc.trajectory(force_accept=(k == 0))
            assert (rec["cg_calls"], rec["cg_it_tot"], rec["cg_it_max"]) == (w["cg_calls"], w["cg_it_tot"],
                                                                              w["cg_it_max"]), rec
            assert int(rec["accepted"]) == w["accepted"]
            assert abs(rec["plaq_energy"] - w["plaq_energy"]) <= 2e-9, rec
            assert rec["exp_dh"] < 5e-11
        assert lat.ranget() == gold["final_seed"]
    finally:
        lat.close()


@pytest.mark.parametrize("solver", ["cg", "mixed"])
def test_leapfrog_is_reversible(bq, solver):
    """The nested leapfrog (hmc_leap_frog.F90) with the device forces is
    reversible: integrate a model-C system (Hasenbusch, clover) forward,
    negate the momenta and integrate again, and the links and momenta return
    to their start, to the accuracy of the solves (the MRE guesses differ
    between the two legs, so each solve contributes its tolerance); the
    fermion and gauge actions, and so H, return with them.  A leapfrog that
    is not reversible, or a force that is not the gradient of the action it
    is paired with, leaves an O(step^2) difference."""
    from bqcdg.hmc import Hmc, quenched_trajectory
    with bq.Lattice((8, 8, 8, 8), BC) as lat:
        lat.ranset(5)
        lat.conf_hot()
        lat.conf_relax(2)
        for _ in range(3):
            quenched_trajectory(lat, 5.29, 1.0, 20, force_accept=True)
        rest = 1e-24 * 12 * 2 * lat.volh   # |r|/|b| about 1e-12 for these pseudofermions
        hmc = Hmc(lat, beta=5.29, kappa=0.13, csw=1.9192, rho=0.1, traj_length=0.5, ntau=5, m_scale=2, model="C",
                  rest=rest, maxiter=20000, solver=solver)
        lat.mom_gauss()
        sf0 = hmc.init_phi()
        u0, p0 = lat.get_gauge(), lat.mom_get()
        h0 = lat.mom_action() + 5.29 * lat.sg() + sum(sf0)
        hmc.md_evolve()
        u1 = lat.get_gauge()
        lat.mom_set(-lat.mom_get())
        sf2 = hmc.md_evolve()
        u2, p2 = lat.get_gauge(), lat.mom_get()
        h2 = lat.mom_action() + 5.29 * lat.sg() + sum(sf2)
        moved = np.linalg.norm(u1 - u0) / np.linalg.norm(u0)
        du = np.linalg.norm(u2 - u0) / np.linalg.norm(u0)
        dp = np.linalg.norm(p2 + p0) / np.linalg.norm(p0)
        print("reversibility (%s): links moved %.2e, back to %.2e; momenta %.2e; H %.6e -> %.6e"
              % (solver, moved, du, dp, h0, h2))
        assert moved > 1e-3
        tol = 1e-9 if solver == "cg" else 1e-6
        assert du < tol and dp < tol
        assert abs(h2 - h0) < (1e-6 if solver == "cg" else 1e-3) * abs(h0)
