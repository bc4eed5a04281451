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
