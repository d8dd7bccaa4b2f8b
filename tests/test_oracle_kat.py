"""End-to-end known-answer test of the oracle against the reference's own P5.9 run records
(tests/golden/p5_9_kat.json, extracted from output/p5_9_ako_apples_to_apples.json by
tests/golden/make_golden.py).  Protocol: src/bin/p5_9_ako_apples_to_apples.rs:175-207."""
import json
import os

import pytest

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "p5_9_kat.json")))
FULL = bool(os.environ.get("CY3Q_FULL_KAT"))


def _records():
    out = []
    for r in GOLD["records"]:
        quick = r["k"] == 3 and r["seed"] in (42, 7)
        out.append(pytest.param(r, id=f"k{r['k']}-seed{r['seed']}",
                                marks=() if quick else pytest.mark.skipif(not FULL, reason="set CY3Q_FULL_KAT=1")))
    return out


@pytest.mark.parametrize("rec", _records())
def test_p5_9_known_answer(orc, rec):
    s = orc.OracleSolver.new_with_sampler(rec["k"], rec["n_pts"], rec["seed"], 1e-12, "sz")
    assert s.n_points == rec["n_pts"] and s.n_basis == rec["n_basis"]
    s.orthonormalise_basis_fs_gram()
    sig_fs = s.sigma()
    it = s.donaldson_solve(GOLD["donaldson_iters"], GOLD["donaldson_tol"])
    sig_d = s.sigma()
    assert sig_fs == pytest.approx(rec["sigma_fs_identity"], rel=1e-12, abs=0)
    assert sig_d == pytest.approx(rec["sigma_donaldson"], rel=1e-12, abs=0)
    assert it == rec["donaldson_iters_run"]
