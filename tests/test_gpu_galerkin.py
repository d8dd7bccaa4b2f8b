"""GPU parity of the Laplacian Galerkin assembly, its spectrum and the Yukawa overlap (C ABI).

Tolerances:
  * FP64 assembly vs the oracle on identical points and h: relative Frobenius error <= 1e-10 on M and K
  * FP64 spectrum vs the oracle's (scipy eigh of the oracle matrices): |dlambda| <= 1e-9 max(lambda, 1)
  * tensor-core assembly (int8 digits, exact int32 accumulation; used for either split precision) vs
    the FP64 assembly on the same GPU: eigenvalues within 1e-8 relative (the null mode within 1e-8
    absolute), M and K within 1e-8 relative Frobenius
  * Yukawa overlap vs the oracle: relative error <= 1e-10
"""
import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def relf(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def cy():
    from papers_b200 import build as b

    b.build()
    import papers_b200

    return papers_b200


@pytest.fixture(scope="module")
def pair(cy, orc):
    """GPU solver and oracle on the same points, both at the GPU's h after three balancing steps."""
    psi = 0.1 + 0.2j
    o = orc.OracleSolver.new_with_psi_sz(4, 8000, 21, psi)
    g = cy.QuinticSolver.from_points(4, o.points, o.weights, o.log_omega_sq, psi=psi)
    for _ in range(3):
        g.donaldson_step()
    o.h_block = np.ascontiguousarray(g.h_block)
    return g, o


def _eig_close(ev, ref, rel):
    scale = np.maximum(np.abs(ref), 1.0)
    scale[0] = 1.0  # null mode: absolute
    return float(np.max(np.abs(ev - ref) / scale))


@pytest.mark.parametrize("d", [1, 2])
def test_fp64_matrices_match_oracle(pair, d):
    g, o = pair
    M, K = g.laplacian_matrices(d)
    Mo, Ko = o.laplacian_matrices(d)
    assert M.shape == Mo.shape
    assert relf(M, Mo) <= 1e-10
    assert relf(K, Ko) <= 1e-10


def test_fp64_spectrum_matches_oracle(pair, orc):
    g, o = pair
    ev = g.laplacian(40, 2, reg=1e-12)
    ref = o.laplacian_eigs(40, 2, reg=1e-12)
    assert _eig_close(ev, ref, 1e-9) <= 1e-9


def test_degree1_embeds_in_degree2_on_gpu(pair, orc):
    g, _ = pair
    m1, m2 = orc.monomials(1), orc.monomials(2)
    n1, n2 = len(m1), len(m2)
    pos2 = {tuple(int(x) for x in e): a for a, e in enumerate(m2)}
    var = [int(np.argmax(e)) for e in m1]

    def idx2(i, k):
        e = [0] * 5
        e[i] += 1
        e[k] += 1
        return pos2[tuple(e)]

    A = np.zeros((n1 * n1, n2 * n2))
    for a, b in itertools.product(range(n1), repeat=2):
        for k in range(5):
            A[a * n1 + b, idx2(var[a], k) * n2 + idx2(var[b], k)] += 1.0
    M1, K1 = g.laplacian_matrices(1)
    M2, K2 = g.laplacian_matrices(2)
    assert relf(A @ M2 @ A.T, M1) <= 1e-12
    assert relf(A @ K2 @ A.T, K1) <= 1e-12


@pytest.mark.parametrize("prec", ["fp16x3", "bf16x3"])
def test_tensor_core_assembly_matches_fp64(cy, orc, prec):
    tol = 1e-8
    # balanced k = 6 metric on the reduced basis (the shape of the full-size run), 100k points
    g = cy.QuinticSolver(6, 100_000, 3, 0.5, reduced_basis=True)
    for _ in range(4):
        g.donaldson_step()
    ref = g.laplacian(40, 2, reg=1e-12)
    g.set_precision(prec)
    ev = g.laplacian(40, 2, reg=1e-12)
    err = _eig_close(ev, ref, tol)
    assert err <= tol, err
    M, K = g.laplacian_matrices(2)
    g.set_precision("fp64")
    M64, K64 = g.laplacian_matrices(2)
    assert relf(M, M64) <= 1e-8
    assert relf(K, K64) <= 1e-8


def test_yukawa_matches_oracle(pair):
    g, o = pair
    rng = np.random.default_rng(9)
    c = (rng.standard_normal((3, 225)) + 1j * rng.standard_normal((3, 225))) / np.sqrt(2)
    y = g.yukawa(c)
    yo = o.yukawa(c)
    assert y.shape == (3, 3, 3)
    assert relf(y, yo) <= 1e-10


def test_argument_errors(pair, cy):
    from papers_b200 import cy3q

    g, _ = pair
    with pytest.raises(cy3q.Cy3qError) as e:
        g.laplacian(40, 3)
    assert e.value.status == cy3q.ERR_ARG
    with pytest.raises(cy3q.Cy3qError) as e:
        g.laplacian(226, 2)
    assert e.value.status == cy3q.ERR_ARG
    with pytest.raises(cy3q.Cy3qError) as e:
        g.yukawa(np.zeros((5, 225), np.complex128))
    assert e.value.status == cy3q.ERR_ARG
