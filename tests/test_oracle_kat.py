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


# ---- P5.3 records (tests/golden/p5_3_kat.json): 20 seeds x k = 2, 3, 4 at n = 10,000 ----
# sigma at h = I after FS-Gram for every record; the earlier (non-inverting) Donaldson step and 20 Adam steps
# with the analytic gradient (sigma_refine_analytic, quintic.rs:453-514) for a few records by default and all
# of them with CY3Q_FULL_KAT=1.  Together they pin the oracle's sigma gradient and its restatement of the
# Adam update of the missing pwos-math crate against the reference's own output.
GOLD3 = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "p5_3_kat.json")))


def _records3(quick_seeds):
    out = []
    for r in GOLD3["records"]:
        quick = r["seed"] in quick_seeds
        out.append(pytest.param(r, id=f"k{r['k']}-seed{r['seed']}",
                                marks=() if quick else pytest.mark.skipif(not FULL, reason="set CY3Q_FULL_KAT=1")))
    return out


@pytest.mark.parametrize("rec", _records3((42, 100, 12345, 7, 99, 1, 2, 3, 4, 5)))
def test_p5_3_sigma_fs_identity(orc, rec):
    s = orc.OracleSolver.new_with_sampler(rec["k"], GOLD3["n_pts"], rec["seed"], GOLD3["newton_tol"], "sz")
    assert s.n_basis == rec["n_basis"]
    s.orthonormalise_basis_fs_gram()
    assert s.sigma() == pytest.approx(rec["sigma_fs_identity"], rel=1e-12, abs=0)


@pytest.mark.parametrize("rec", _records3((42,)))
def test_p5_3_refinement_known_answer(orc, rec):
    s = orc.OracleSolver.new_with_sampler(rec["k"], GOLD3["n_pts"], rec["seed"], GOLD3["newton_tol"], "sz")
    s.orthonormalise_basis_fs_gram()
    s.donaldson_solve(GOLD3["donaldson_iters"], GOLD3["donaldson_tol"], unfixed=True)
    sig_d = s.sigma()
    assert sig_d == pytest.approx(rec["sigma_donaldson"], rel=1e-12, abs=0)
    hist = s.sigma_refine_analytic(GOLD3["refine_iters"], GOLD3["refine_lr"])
    vals = [sig_d] + list(hist)
    best = min(vals)
    assert best == pytest.approx(rec["sigma_post_refine"], rel=1e-12, abs=0)
    assert vals.index(best) == rec["refine_min_idx"]
