"""Metric cache on the CPU (no device work): the library's SHA-256 against hashlib on the padding boundary
cases, and cache file names as route34/metric_cache.rs builds them (ty_cache_path :175-193): the readable
fields plus the first 16 hex digits of the SHA-256 of the canonical key text, so that every key field
changes the name (the reference's ty_path_includes_all_key_fields test, metric_cache.rs:355-385)."""
import hashlib
import struct

import numpy as np
import pytest


@pytest.fixture(scope="module")
def cy():
    from papers_b200 import build as b

    b.build()
    from papers_b200 import cy3q

    cy3q.lib()
    return cy3q


@pytest.mark.parametrize("n", [0, 1, 3, 55, 56, 57, 63, 64, 65, 119, 120, 128, 1000, 100003])
def test_sha256_matches_hashlib(cy, n):
    data = np.random.default_rng(n).integers(0, 256, n, dtype=np.uint8).tobytes()
    assert cy.sha256_hex(data) == hashlib.sha256(data).hexdigest()


def test_sha256_fips_example(cy):
    assert cy.sha256_hex(b"abc") == hashlib.sha256(b"abc").hexdigest()


def _key(cy, **kw):
    base = dict(k=6, psi_re=0.5, psi_im=0.0, n_points=500000, seed=42, sampler=1, fermat_variant=0, dk_iters=50,
                newton_polish=0, reduced_basis=1, precision=1, max_iter=20, tol=0.0)
    base.update(kw)
    return cy.CacheKey(**base)


def _bits(x):
    return "0x%016x" % struct.unpack("<Q", struct.pack("<d", x))[0]


def _text(k):
    return (f"cy3q metric cache v1;manifold=quintic;k={k.k};psi_re={_bits(k.psi_re)};psi_im={_bits(k.psi_im)};"
            f"n_points={k.n_points};seed={k.seed};sampler={k.sampler};fermat_variant={k.fermat_variant};"
            f"dk_iters={k.dk_iters};newton_polish={k.newton_polish};reduced_basis={k.reduced_basis};"
            f"precision={k.precision};max_iter={k.max_iter};tol={_bits(k.tol)}")


def test_cache_path_format(cy):
    k = _key(cy)
    p = cy.cache_path("/tmp/cache", k)
    h = hashlib.sha256(_text(k).encode()).hexdigest()[:16]
    assert p == f"/tmp/cache/quintic_k6_n500000_i20_seed42_{h}.cy3m"


def test_every_key_field_changes_the_path(cy):
    base = cy.cache_path("c", _key(cy))
    changes = [dict(k=5), dict(psi_re=0.25), dict(psi_im=1e-300), dict(n_points=499999), dict(seed=43),
               dict(sampler=0), dict(fermat_variant=1), dict(dk_iters=60), dict(newton_polish=2),
               dict(reduced_basis=0), dict(precision=0), dict(max_iter=21), dict(tol=1e-12)]
    paths = {cy.cache_path("c", _key(cy, **c)) for c in changes}
    assert base not in paths and len(paths) == len(changes)


def test_ty_and_schoen_cache_names_follow_the_reference():
    """ty_cache_path / schoen_cache_path (route34/metric_cache.rs:174-226): readable fields and the first 16 hex
    digits of SHA-256 of the serde_json encoding of the key material (field order, no spaces)."""
    import hashlib
    import json
    import struct

    from papers_b200 import ty

    def ref_name(kind, fields, stem):
        js = json.dumps(fields, separators=(",", ":"))
        return f"{stem}_{hashlib.sha256(js.encode()).hexdigest()[:16]}.cy3m"

    tolbits = struct.unpack("<Q", struct.pack("<d", 1e-6))[0]
    c = ty.TyMetricConfig(k_degree=3, n_sample=40000, max_iter=100, donaldson_tol=1e-6, seed=42)
    want = ref_name("ty", {"schema_version": 1, "manifold": "tian_yau_z3", "k_degree": 3, "n_sample": 40000,
                           "max_iter": 100, "donaldson_tol_bits": tolbits, "seed": 42, "apply_z3_quotient": True},
                    "ty_k3_n40000_i100_seed42")
    assert ty.cache_path("/tmp/cc", c) == "/tmp/cc/" + want
    s = ty.SchoenMetricConfig(d_x=3, d_y=3, d_t=1, n_sample=2000, max_iter=30, donaldson_tol=1e-6, seed=7)
    want = ref_name("schoen", {"schema_version": 1, "manifold": "schoen_z3xz3", "d_x": 3, "d_y": 3, "d_t": 1,
                               "n_sample": 2000, "max_iter": 30, "donaldson_tol_bits": tolbits, "seed": 7,
                               "apply_z3xz3_quotient": True, "schoen_bundle_canonical": False},
                    "schoen_dx3_dy3_dt1_n2000_i30_seed7")
    assert ty.cache_path("", s) == want
    assert ty.cache_path("/x", ty.TyMetricConfig(k_degree=3, n_sample=40000, max_iter=100, donaldson_tol=1e-6,
                                                 seed=43)) != "/x/" + want
