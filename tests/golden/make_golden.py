"""Extract the reference's known-answer records for the quintic path into small fixtures.

    python tests/golden/make_golden.py <reference cy3_solver/output directory>

Reads two of the reference's own run artefacts from that directory and writes only the fields the tests
use next to this script; the fixtures are committed, so the tests never read the reference at run time.

* p5_9_ako_apples_to_apples.json -> p5_9_kat.json.  Protocol (src/bin/p5_9_ako_apples_to_apples.rs:175-207):
  Fermat quintic, Shiffman-Zelditch sampler, FS-Gram orthonormalisation, sigma at h = I,
  donaldson_solve(50, 1e-12), sigma again.
* p5_3_multi_seed_ensemble.json -> p5_3_kat.json.  Protocol (src/bin/p5_3_multi_seed_ensemble.rs:180-215):
  the same sampler and FS-Gram at n = 10,000 for k = 2, 3, 4 and 20 seeds, sigma at h = I,
  donaldson_solve(50, 1e-10), sigma, then sigma_refine_analytic(20, 1e-3) and the running minimum of sigma
  over the post-Donaldson value and the refinement history.  These records were made before the reference
  fixed its Donaldson step (they store T(h) without inverting it, quintic.rs:1722-1726), so the Donaldson
  and refinement values pin the oracle's restatement of that earlier step and, through it, the analytic
  sigma gradient and the Adam update; sigma at h = I does not depend on the step.
* p5_10_ty_schoen_5sigma.json, bit_exact_fix/p5_10_xoshiro_reduced.json and
  ../tests/data/p5_10_determinism_golden.json -> ty_kat.json: the Tian-Yau records of the reference's
  solve_ty_metric (src/route34/ty_metric.rs:461; spec of src/route34/cy3_metric_unified.rs:242-261): k = 3,
  20 seeds at n = 40,000 and 3 seeds at n = 2,000 (100 and 30 iterations, tolerance 1e-6), the 20-seed runs
  at k = 4 and k = 5 (p5_10_k4_adaptive.json, p5_10_k5_damped.json: 40,000 points, 100 / 200 iterations), and
  the determinism record at n = 200 (5 iterations; bit patterns decoded to floats).
* the same three files -> schoen_kat.json: the Schoen records of solve_schoen_metric
  (src/route34/schoen_metric.rs:766; spec of src/route34/cy3_metric_unified.rs:289-320) at (d_x, d_y, d_t) =
  (3, 3, 1), the tuple the reference uses for k = 3.
"""
import json
import struct
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def p5_9(src_dir):
    ref = json.load(open(os.path.join(src_dir, "p5_9_ako_apples_to_apples.json")))
    out = {
        "source": "substrate_sm_derivation/cy3_solver/output/p5_9_ako_apples_to_apples.json",
        "protocol": "QuinticSolver::new_with_sampler(k, n_pts, seed, 1e-12, ShiffmanZelditch); "
                    "orthonormalise_basis_fs_gram(); sigma(); donaldson_solve(50, 1e-12); sigma()",
        "donaldson_iters": ref["donaldson_iters"],
        "donaldson_tol": ref["donaldson_tol"],
        "records": [],
    }
    for ke in ref["ks"]:
        for rec in ke["per_seed"]:
            out["records"].append({
                "k": ke["k"], "n_pts": ke["n_pts"], "n_basis": ke["n_basis"], "seed": rec["seed"],
                "sigma_fs_identity": rec["sigma_fs_identity"], "sigma_donaldson": rec["sigma_donaldson"],
                "donaldson_iters_run": rec["donaldson_iters_run"],
            })
    return "p5_9_kat.json", out


def p5_3(src_dir):
    ref = json.load(open(os.path.join(src_dir, "p5_3_multi_seed_ensemble.json")))
    out = {
        "source": "substrate_sm_derivation/cy3_solver/output/p5_3_multi_seed_ensemble.json",
        "protocol": "QuinticSolver::new_with_sampler(k, n_pts, seed, newton_tol, ShiffmanZelditch); "
                    "orthonormalise_basis_fs_gram(); sigma(); donaldson_solve(donaldson_iters, donaldson_tol) "
                    "with the earlier step h <- T(h); sigma(); sigma_refine_analytic(refine_iters, refine_lr); "
                    "running minimum of sigma over the post-Donaldson value and the history",
        "n_pts": ref["n_pts"], "donaldson_iters": ref["donaldson_iters"], "donaldson_tol": ref["donaldson_tol"],
        "refine_iters": ref["refine_iters"], "refine_lr": ref["refine_lr"], "newton_tol": ref["newton_tol"],
        "records": [],
    }
    for ke in ref["ks"]:
        for rec in ke["per_seed"]:
            out["records"].append({
                "k": ke["k"], "n_pts": ke["n_pts"], "n_basis": ke["n_basis"], "seed": rec["seed"],
                "sigma_fs_identity": rec["sigma_fs_identity"], "sigma_donaldson": rec["sigma_donaldson"],
                "sigma_post_refine": rec["sigma_post_refine"], "refine_min_idx": rec["refine_min_idx"],
            })
    return "p5_3_kat.json", out


def ty(src_dir, candidate="TY"):
    out = {
        "source": ["substrate_sm_derivation/cy3_solver/output/p5_10_ty_schoen_5sigma.json",
                   "substrate_sm_derivation/cy3_solver/output/bit_exact_fix/p5_10_xoshiro_reduced.json",
                   "substrate_sm_derivation/cy3_solver/tests/data/p5_10_determinism_golden.json"],
        "protocol": "TianYauSolver.solve_metric(Cy3MetricSpec::TianYau { k, n_sample, max_iter, donaldson_tol, seed }): "
                    "CicySampler::sample_batch + Z/3 quotient, invariant Groebner-reduced basis, h = I, "
                    "donaldson_iteration until residual < tol, sigma after every iteration",
        "records": [],
    }
    for name, max_iter in (("p5_10_ty_schoen_5sigma.json", None), (os.path.join("bit_exact_fix", "p5_10_xoshiro_reduced.json"), 30),
                           ("p5_10_k4_adaptive.json", None), ("p5_10_k5_damped.json", None)):
        ref = json.load(open(os.path.join(src_dir, name)))
        for cand in ref["candidates"]:
            if cand["candidate"] != candidate:
                continue
            for rec in cand["per_seed"]:
                out["records"].append({
                    "k": rec["k"], "n_pts": ref["n_pts"], "seed": rec["seed"],
                    "max_iter": max_iter or ref["donaldson_iters"], "tol": ref["donaldson_tol"],
                    "n_basis": rec["n_basis"], "iterations_run": rec["iterations_run"],
                    "sigma_fs_identity": rec["sigma_fs_identity"], "sigma_final": rec["sigma_final"],
                    "final_donaldson_residual": rec["final_donaldson_residual"],
                    "elapsed_s": rec.get("elapsed_s"), "source_file": name,
                })
    gold = json.load(open(os.path.join(src_dir, os.pardir, "tests", "data", "p5_10_determinism_golden.json")))
    f64 = lambda b: struct.unpack("<d", struct.pack("<Q", b))[0]
    for rec in gold["records"]:
        if rec["candidate"] != candidate:
            continue
        out["records"].append({
            "k": rec["k"], "n_pts": rec["n_pts"], "seed": rec["seed"], "max_iter": rec["donaldson_iters"],
            "tol": rec["donaldson_tol"], "n_basis": rec["n_basis"], "iterations_run": rec["iterations_run"],
            "sigma_fs_identity": f64(rec["sigma_fs_identity_bits"]), "sigma_final": f64(rec["sigma_final_bits"]),
            "final_donaldson_residual": f64(rec["final_donaldson_residual_bits"]),
        })
    if candidate != "TY":
        out["protocol"] = ("SchoenSolver.solve_metric(Cy3MetricSpec::Schoen { d_x: 3, d_y: 3, d_t: 1, n_sample, max_iter, "
                           "donaldson_tol, seed }): SchoenSampler::sample_points + Z/3 x Z/3 quotient, invariant "
                           "Groebner-reduced basis, h = I, donaldson_iteration until residual < tol, sigma after every "
                           "iteration")
        return "schoen_kat.json", out
    return "ty_kat.json", out


def schoen(src_dir):
    return ty(src_dir, "Schoen")


def main(src_dir):
    for make in (p5_9, p5_3, ty, schoen):
        name, out = make(src_dir)
        dst = os.path.join(HERE, name)
        json.dump(out, open(dst, "w"), indent=1)
        print("wrote", dst, len(out["records"]), "records")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    main(sys.argv[1])
