"""Metric cache on the GPU: a stored balanced h comes back bit for bit into a handle holding the same points
(load_or_solve_ty's hit path, route34/metric_cache.rs:254-261); a handle holding other points, a damaged
file or another key misses; strict mode refuses a metric whose sigma is not below the 1e-3 quality
threshold (check_sigma_quality, :318-340) and leaves h alone; the server's warm start returns the cached h
with no iteration run."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cy():
    from papers_b200 import build as b

    b.build()
    import papers_b200

    return papers_b200


def _solved(cy, seed=5, iters=6):
    s = cy.QuinticSolver.new_with_psi_sz(3, 6000, seed, 0.3 + 0.1j, reduced_basis=False)
    r = None
    for _ in range(iters):
        r = s.donaldson_step()
    return s, r


def test_store_then_load_bitwise(cy, tmp_path):
    from papers_b200 import cy3q

    s, r = _solved(cy)
    sig = s.sigma()
    key = s.cache_key(6)
    s.cache_store(str(tmp_path), key, sig, r)
    path = cy3q.cache_path(str(tmp_path), key)
    assert os.path.exists(path) and not os.path.exists(path + ".tmp")
    t = cy.QuinticSolver.new_with_psi_sz(3, 6000, 5, 0.3 + 0.1j, reduced_basis=False)
    got = t.cache_load(str(tmp_path), key)
    assert got is not None and got[0] == sig and got[1] == r
    assert np.array_equal(t.h_block, s.h_block)
    # the loaded metric gives the same sigma on the same points
    assert t.sigma() == sig


def test_misses_and_quality_guard(cy, tmp_path):
    from papers_b200 import cy3q

    s, r = _solved(cy)
    key = s.cache_key(6)
    s.cache_store(str(tmp_path), key, s.sigma(), r)
    # other points under the same key: the recorded sample-cloud hash differs
    other = cy.QuinticSolver.new_with_psi_sz(3, 6000, 6, 0.3 + 0.1j, reduced_basis=False)
    assert other.cache_load(str(tmp_path), key) is None
    # another key: no file
    assert other.cache_load(str(tmp_path), other.cache_key(7)) is None
    # strict: sigma of a k = 3 metric (about 0.1) is far above 1e-3; h is left unchanged
    t = cy.QuinticSolver.new_with_psi_sz(3, 6000, 5, 0.3 + 0.1j, reduced_basis=False)
    h0 = t.h_block
    with pytest.raises(cy3q.Cy3qError) as e:
        t.cache_load(str(tmp_path), key, strict=True)
    assert e.value.status == cy3q.ERR_STALE
    assert np.array_equal(t.h_block, h0)
    # a damaged file misses
    path = cy3q.cache_path(str(tmp_path), key)
    b = bytearray(open(path, "rb").read())
    b[len(b) // 2] ^= 0x01
    open(path, "wb").write(bytes(b))
    assert t.cache_load(str(tmp_path), key) is None


def test_server_warm_start(cy, tmp_path):
    req = dict(k=4, n_points=20000, seed=11, psi=0.2 + 0.3j, iterations=4, precision="fp16x3")
    srv = cy.Server(0, 0, 2, cache_root=str(tmp_path))
    t = srv.submit(**req)
    res = srv.wait(t, 120000)
    assert res.status == 0 and res.cache_hit == 0 and res.iterations == 4
    h1 = srv.h_block(t, res.n_basis)
    srv.close()  # joins the cache writer
    srv = cy.Server(0, 0, 2, cache_root=str(tmp_path))
    t2 = srv.submit(**req)
    res2 = srv.wait(t2, 120000)
    assert res2.status == 0 and res2.cache_hit == 1 and res2.iterations == 0
    assert res2.residual == res.residual
    assert np.array_equal(srv.h_block(t2, res2.n_basis), h1)
    # a request with another seed is solved
    t3 = srv.submit(**dict(req, seed=12))
    res3 = srv.wait(t3, 120000)
    assert res3.status == 0 and res3.cache_hit == 0 and res3.iterations == 4
    srv.close()
