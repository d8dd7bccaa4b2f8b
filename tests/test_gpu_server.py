"""Continuous-batching server (cy3q_server_*): results in a concurrent mix equal the same requests run
alone, cancellation, deadlines and admission by HBM bytes.  Tolerance for 'alone vs in the mix': the
balancing kernels reduce in fixed orders, so the h blocks must agree to 1e-12 relative Frobenius."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MIX_TOL = 1e-12


@pytest.fixture(scope="module")
def cy():
    from papers_b200 import build as b

    b.build()
    import papers_b200
    from papers_b200 import cy3q

    return cy3q


def _requests():
    rng = np.random.default_rng(3)
    out = []
    for i, k in enumerate([2, 3, 4, 5, 6, 3, 2, 4, 5, 3, 6, 2]):
        u, v = rng.random(), rng.random()
        psi = np.sqrt(u) * 0.9 * np.exp(2j * np.pi * v)
        n = {2: 15, 3: 35, 4: 70, 5: 125, 6: 205}[k]
        out.append(dict(k=k, n_points=min(10 * n * n, 60000), seed=100 + i, psi=psi, iterations=4,
                        precision="fp16x3" if i % 3 else "fp64"))
    return out


def test_mix_equals_alone(cy):
    reqs = _requests()
    srv = cy.Server(0, 0, 4)
    tickets = [srv.submit(**r) for r in reqs]
    mix = []
    for t in tickets:
        res = srv.wait(t, 120000)
        assert res.status == 0
        mix.append((res, srv.h_block(t, res.n_basis)))
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert np.isfinite(st["p50_ms"]) and st["p99_ms"] >= st["p50_ms"]
    assert st["iters_per_s"] > 0
    srv.close()
    alone_srv = cy.Server(0, 0, 1)
    for r, (res_m, h_m) in zip(reqs, mix):
        t = alone_srv.submit(**r)
        res_a = alone_srv.wait(t, 120000)
        assert res_a.status == 0
        h_a = alone_srv.h_block(t, res_a.n_basis)
        assert np.linalg.norm(h_a - h_m) <= MIX_TOL * np.linalg.norm(h_a), r
        assert res_a.residual == pytest.approx(res_m.residual, rel=1e-12)
    alone_srv.close()


def test_server_matches_solver(cy):
    r = dict(k=4, n_points=20000, seed=7, psi=0.3 + 0.4j, iterations=3, precision="fp16x3")
    srv = cy.Server(0, 0, 2)
    t = srv.submit(**r)
    res = srv.wait(t, 60000)
    h_srv = srv.h_block(t, res.n_basis)
    srv.close()
    s = cy.QuinticSolver.new_with_psi_sz(4, 20000, 7, 0.3 + 0.4j, reduced_basis=True, precision="fp16x3",
                                         with_derivs=False)
    for _ in range(3):
        s.donaldson_step()
    assert np.linalg.norm(s.h_block - h_srv) <= MIX_TOL * np.linalg.norm(h_srv)


def test_cancel_timeout_and_budget(cy):
    srv = cy.Server(0, 0, 1)
    # long enough that the cancel below always lands while it runs (it ends at the next iteration)
    long_t = srv.submit(k=6, n_points=400000, seed=1, psi=0.5, iterations=100000, precision="fp16x3")
    queued = srv.submit(k=3, n_points=5000, seed=2, psi=0.5, iterations=2)
    # deadline: the long request cannot finish within 1 ms
    with pytest.raises(cy.Cy3qError) as e:
        srv.wait(long_t, 1)
    assert "ERR_TIMEOUT" in str(e.value)
    srv.cancel(queued)  # still queued behind the long one
    assert srv.wait(queued, 10000).status == cy.ERR_CANCELLED
    srv.cancel(long_t)  # running: stops between iterations
    res = srv.wait(long_t, 120000)
    assert res.status == cy.ERR_CANCELLED and res.iterations < 100000
    st = srv.stats()
    assert st["cancelled"] == 2 and st["hbm_in_use"] == 0
    srv.close()
    small = cy.Server(0, 64 << 20, 1)  # 64 MiB budget
    with pytest.raises(cy.Cy3qError) as e:
        small.submit(k=6, n_points=400000, seed=1, psi=0.5)
    assert "ERR_OOM" in str(e.value)
    small.close()


def test_large_bases_in_the_mix_equal_alone(cy):
    """k = 7 and k = 8 requests (N = 315 and 460) at reduced point counts share the grouped steps with
    k = 2..4 requests; every request's h and residual equal the same request served alone, bit for bit."""
    rng = np.random.default_rng(11)
    reqs = []
    for i, k in enumerate([2, 8, 3, 7, 4, 2, 8, 3, 7]):
        u, v = rng.random(), rng.random()
        psi = np.sqrt(u) * 0.9 * np.exp(2j * np.pi * v)
        n = {2: 15, 3: 35, 4: 70, 7: 315, 8: 460}[k]
        reqs.append(dict(k=k, n_points=min(10 * n * n, 30000), seed=300 + i, psi=psi, iterations=3,
                         precision="fp16x3"))
    srv = cy.Server(0, 0, 4)
    tickets = [srv.submit(**r) for r in reqs]
    mix = []
    for t in tickets:
        res = srv.wait(t, 300000)
        assert res.status == 0
        mix.append((res.residual, srv.h_block(t, res.n_basis)))
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0 and st["hbm_in_use"] == 0
    srv.close()
    alone = cy.Server(0, 0, 1)
    for r, (res_m, h_m) in zip(reqs, mix):
        t = alone.submit(**r)
        res_a = alone.wait(t, 300000)
        assert res_a.status == 0
        assert res_a.residual == res_m, r
        assert np.array_equal(alone.h_block(t, res_a.n_basis), h_m), r
    alone.close()
