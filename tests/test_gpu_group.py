"""Grouped balancing (cy3q_group_*): one step of several split-precision solves of different (psi, k, P)
with shared persistent tensor-core launches replayed from CUDA graphs.

Each member's h and residual must equal the same solve stepped alone (cy3q_donaldson_step) bit for bit:
the grouped kernels run every member's own work items in the same order, so the mix changes nothing.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(2, 0.3 + 0.4j, 3000), (3, 0.0, 20000), (4, 0.5, 30000), (6, 0.1 + 0.2j, 40000)]


@pytest.fixture(scope="module")
def cy():
    from papers_b200 import build as b

    b.build()
    from papers_b200 import cy3q

    return cy3q


@pytest.fixture(scope="module")
def clouds(orc):
    out = []
    for i, (k, psi, P) in enumerate(SHAPES):
        if psi == 0:
            o = orc.OracleSolver.new_with_sampler(k, P, 40 + i, 1e-12, "sz", reduced=True)
        else:
            o = orc.OracleSolver.new_with_psi_sz(k, P, 40 + i, psi, reduced=True)
        out.append((k, psi, o.points, o.weights, o.log_omega_sq))
    return out


def make(cy, c, prec="fp16x3"):
    k, psi, pts, w, lo = c
    return cy.QuinticSolver.from_points(k, pts, w, lo, psi=psi, reduced_basis=True, precision=prec)


def test_group_equals_alone(cy, clouds):
    alone = [make(cy, c) for c in clouds]
    grouped = [make(cy, c) for c in clouds]
    g = cy.Group(0, capacity=4)
    for _ in range(4):
        res, st = g.step(grouped)
        ref = [s.donaldson_step() for s in alone]
        assert list(st) == [0] * len(clouds)
        assert list(res) == ref
    for a, b in zip(alone, grouped):
        assert np.array_equal(a.h_block, b.h_block)
    g.close()


def test_group_membership_changes(cy, clouds):
    """Members join and leave between steps (continuous batching); each trajectory is unchanged."""
    alone = [make(cy, c) for c in clouds]
    grouped = [make(cy, c) for c in clouds]
    g = cy.Group(0, capacity=4)
    schedule = [[0, 1], [0, 1, 2], [1, 2, 3], [3], [0, 2, 3], [0, 1, 2, 3]]
    for members in schedule:
        res, st = g.step([grouped[i] for i in members])
        for j, i in enumerate(members):
            assert res[j] == alone[i].donaldson_step()
    for a, b in zip(alone, grouped):
        assert np.array_equal(a.h_block, b.h_block)
    g.close()


def test_group_isolates_a_failing_member(cy, clouds, orc):
    """A member whose T-operator is singular (the full k = 6 basis holds multiples of the quintic) fails
    alone; the other members step normally and the failed one keeps its previous h."""
    k, psi, pts, w, lo = clouds[3]
    bad = cy.QuinticSolver.from_points(k, pts, w, lo, psi=psi, reduced_basis=False, precision="fp16x3")
    h0 = bad.h_block
    ok = [make(cy, c) for c in clouds[:2]]
    ref = [make(cy, c) for c in clouds[:2]]
    g = cy.Group(0, capacity=4)
    res, st = g.step([ok[0], bad, ok[1]], raise_on_error=False)
    assert st[0] == 0 and st[2] == 0
    assert st[1] == cy.ERR_SINGULAR
    assert np.array_equal(bad.h_block, h0)
    assert res[0] == ref[0].donaldson_step() and res[2] == ref[1].donaldson_step()
    g.close()


def test_group_capacity_and_arguments(cy, clouds):
    g = cy.Group(0, capacity=2)
    s = [make(cy, c) for c in clouds[:3]]
    with pytest.raises(cy.Cy3qError):
        g.step(s)  # more members than the capacity
    with pytest.raises(cy.Cy3qError):
        g.step([s[0], s[0]])  # the same handle twice
    k, psi, pts, w, lo = clouds[0]
    f = cy.QuinticSolver.from_points(k, pts, w, lo, psi=psi, reduced_basis=True, precision="fp64")
    with pytest.raises(cy.Cy3qError):
        g.step([f])  # FP64 handles are not grouped
    g.close()


# Large bases next to small ones: k = 7 (N = 315, 2N mod 128 = 118, ldk 640, T-operator tail of 128
# columns) and k = 8 (N = 460, 2N mod 128 = 24, ldk 960, tail of 32 columns, 36 T tiles) at reduced point
# counts, mixed with k = 2..4 in one group whose capacity is larger than any earlier membership, so the
# tables grow while members of every width share them.
LARGE = [(2, 0.3 + 0.4j, 3000, 51), (7, 0.2 - 0.1j, 30000, 52), (3, 0.5, 20000, 53), (8, 0.1 + 0.2j, 30000, 54),
         (4, -0.4 + 0.1j, 20000, 55)]


def _sampled(cy, k, psi, P, seed):
    return cy.QuinticSolver.new_with_psi_sz(k, P, seed, psi, reduced_basis=True, precision="fp16x3",
                                            with_derivs=False)


def test_group_large_bases_mix_equals_alone(cy):
    alone = [_sampled(cy, *x) for x in LARGE]
    grouped = [_sampled(cy, *x) for x in LARGE]
    assert [s.n_basis for s in grouped] == [15, 315, 35, 460, 70]
    g = cy.Group(0, capacity=6)
    schedule = [[0, 2], [0, 1, 2], [1, 3], [0, 1, 2, 3, 4], [3, 4], [0, 1, 2, 3, 4]]
    for members in schedule:
        res, st = g.step([grouped[i] for i in members])
        assert list(st) == [0] * len(members)
        for j, i in enumerate(members):
            assert res[j] == alone[i].donaldson_step(), (members, i)
    for a, b in zip(alone, grouped):
        assert np.array_equal(a.h_block, b.h_block)
    g.close()
