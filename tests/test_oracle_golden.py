"""Pin the CPU oracle to the reference's own golden outputs.

ranf_test.reference      : bit-exact known answers of the 48-bit LCG (ranf.F90)
out.quick-test.reference : one 4^4 model-C HMC trajectory (work/input.quick-test)
                           exercising D21, the clover term, W/M~, CG, MRE, all
                           four forces, plaquette and exp(-dH).
"""
import json
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden(name):
    with open(os.path.join(HERE, "golden", name)) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def oracle_exe():
    from oracle import build
    _, exe = build.build()
    return exe


def test_ranf_known_answers(oracle_exe):
    g = _golden("ranf_test.json")
    out = subprocess.run([oracle_exe, "ranf_test"], capture_output=True, text=True, check=True).stdout
    recs = [l.split() for l in out.splitlines() if l.strip() and not l.strip().endswith(":")]
    want = [r for s in g["sections"] for r in s["records"]]
    assert len(recs) == len(want) == 10 + 10 + 31 + 31 + 48 + 48
    for got, exp in zip(recs, want):
        assert int(got[0]) == exp[0]
        assert int(got[1]) == exp[1]          # the 48-bit seed, exactly
        assert got[2] == exp[2]               # f24.16 text of the double, exactly


def test_quick_test_trajectory(oracle_exe):
    g = _golden("quick_test.json")
    env = dict(os.environ, OMP_NUM_THREADS="2")
    out = subprocess.run([oracle_exe, "quick_test"], capture_output=True, text=True, check=True, env=env).stdout
    rec = {l.split()[0]: l.split()[1:] for l in out.splitlines()}
    it = rec["%it"]
    assert (int(it[1]), int(it[2])) == (g["it"]["f1"], g["it"]["f2"])
    # force norms: printed with 10 significant digits (g20.10)
    for key in ("Favg", "Fmax"):
        got = [float(v) for v in rec["%" + key][1:5]]
        for a, b in zip(got, g[key]["values"]):
            assert abs(a - b) <= 6e-10 * abs(b), (key, a, b)
    fa = rec["%fa"]
    assert abs(float(fa[2]) - g["fa"]["plaq_energy"]) <= 6e-11
    assert abs(float(fa[3]) - g["fa"]["exp_mdh"]) <= 6e-11
    assert (int(fa[4]), int(fa[5]), int(fa[6])) == (g["fa"]["cg_calls"], g["fa"]["cg_it_tot"], g["fa"]["cg_it_max"])
    assert int(rec["Seed"][0]) == g["final_seed"]


def test_oracle_thread_independent(oracle_exe):
    outs = []
    for n in ("1", "4"):
        env = dict(os.environ, OMP_NUM_THREADS=n)
        outs.append(subprocess.run([oracle_exe, "quick_test"], capture_output=True, text=True, check=True,
                                   env=env).stdout)
    assert outs[0] == outs[1]


def check_test20(records, gold):
    """Compare 20 trajectory records with work/out.test.reference: iteration
    counts and CG statistics exactly, the 10-decimal plaquette and exp(-dH)
    to the last or second-last digit (README:235-262)."""
    assert len(records) == len(gold["records"]) == 20
    for got, want in zip(records, gold["records"]):
        assert got["traj"] == want["traj"]
        assert (got["f1"], got["f2"]) == (want["f1"], want["f2"]), (got, want)
        assert (got["cg_calls"], got["cg_it_tot"], got["cg_it_max"]) == \
            (want["cg_calls"], want["cg_it_tot"], want["cg_it_max"]), (got, want)
        assert got["accepted"] == want["accepted"]
        assert abs(got["plaq_energy"] - want["plaq_energy"]) <= 2e-9, (got, want)
        assert abs(got["exp_mdh"] - want["exp_mdh"]) <= 2e-9, (got, want)


def test_twenty_trajectories(oracle_exe):
    """work/out.test.reference: 10 force-accepted and 10 Metropolis
    trajectories of the quick-test system, and the final RNG seed."""
    gold = _golden("test20.json")
    env = dict(os.environ, OMP_NUM_THREADS="4")
    out = subprocess.run([oracle_exe, "test20"], capture_output=True, text=True, check=True, env=env).stdout
    recs, seed = [], None
    for line in out.splitlines():
        f = line.split()
        if f[0] == "%it":
            recs.append({"traj": int(f[1]), "f1": int(f[2]), "f2": int(f[3])})
        elif f[0] == "%fa":
            recs[-1].update(plaq_energy=float(f[3]), exp_mdh=float(f[4]), accepted=1, cg_calls=int(f[5]),
                            cg_it_tot=int(f[6]), cg_it_max=int(f[7]))
        elif f[0] == "%mc":
            recs[-1].update(plaq_energy=float(f[4]), exp_mdh=float(f[5]), accepted=int(f[6]), cg_calls=int(f[7]),
                            cg_it_tot=int(f[8]), cg_it_max=int(f[9]))
        elif f[0] == "Seed":
            seed = int(f[1])
    check_test20(recs, gold)
    assert seed == gold["final_seed"]
