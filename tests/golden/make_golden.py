"""Extract the reference's known-answer records for the quintic path into a small fixture.

Reads the reference's own run artefact
    substrate_sm_derivation/cy3_solver/output/p5_9_ako_apples_to_apples.json
(protocol: src/bin/p5_9_ako_apples_to_apples.rs:175-207 -- Fermat quintic, Shiffman-Zelditch sampler,
FS-Gram orthonormalisation, sigma at h = I, donaldson_solve(50, 1e-12), sigma again) and writes
tests/golden/p5_9_kat.json with only the fields the tests use.  Run it where the reference tree is
mounted; the fixture is committed so the tests never read the reference at run time.
"""
import json
import os
import sys

REF = "/root/reference/substrate_sm_derivation/cy3_solver/output/p5_9_ako_apples_to_apples.json"


def main(path=REF):
    ref = json.load(open(path))
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
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "p5_9_kat.json")
    json.dump(out, open(dst, "w"), indent=1)
    print("wrote", dst, len(out["records"]), "records")


if __name__ == "__main__":
    main(*sys.argv[1:])
