"""Oracle self-consistency of the Laplacian Galerkin assembly and the Yukawa overlap (CPU).

The reference has no quintic Laplacian / Yukawa and no golden vectors for them, so the oracle is
pinned by identities that hold exactly for the discrete sums:
  * M and K are Hermitian, M is positive definite and K positive semi-definite;
  * the constant function lies in the span (1 = sum_a m_a |s_a|^2 / (z^H z)^d with the multinomial
    coefficients m_a), so K v = 0 and v^H M v = 1 for its coefficient vector v;
  * every degree-1 test function is a sum of degree-2 ones, z_i conj(z_j) / |z|^2 =
    sum_k (z_i z_k) conj(z_j z_k) / |z|^4, so M1 = A M2 A^T and K1 = A K2 A^T for the 0/1 matrix A
    of that embedding -- this pins the quotient-rule derivatives and the frame contraction;
  * Y_ijk is symmetric in (i, j, k) and trilinear; for psi = 1 it is sum w conj(Omega) / sum w, checked
    against Omega = z_chart / (df/dz_elim) from the quintic gradient.
"""
import itertools
import math

import numpy as np
import pytest


@pytest.fixture(scope="module")
def balanced(orc):
    o = orc.OracleSolver.new_with_psi_sz(3, 3000, 11, 0.1 + 0.2j)
    o.donaldson_solve(6, 1e-12)
    return o


def _const_vector(orc, d):
    mono = orc.monomials(d)
    nd = len(mono)
    v = np.zeros(nd * nd)
    for a, e in enumerate(mono):
        v[a * nd + a] = math.factorial(d) / np.prod([math.factorial(int(x)) for x in e])
    return v


def test_matrices_hermitian_and_definite(orc, balanced):
    M, K = balanced.laplacian_matrices(2)
    assert M.shape == (225, 225)
    assert np.abs(M - M.conj().T).max() <= 1e-15 * np.abs(M).max()
    assert np.abs(K - K.conj().T).max() <= 1e-15 * np.abs(K).max()
    assert np.linalg.eigvalsh(M).min() > 0
    assert np.linalg.eigvalsh(K).min() > -1e-12 * np.abs(K).max()


@pytest.mark.parametrize("d", [1, 2])
def test_constant_function_is_harmonic(orc, balanced, d):
    M, K = balanced.laplacian_matrices(d)
    v = _const_vector(orc, d)
    assert abs(v @ M @ v - 1.0) < 1e-12
    assert np.abs(K @ v).max() < 1e-12 * np.abs(K).max() * np.abs(v).sum()


def test_degree1_functions_embed_in_degree2(orc, balanced):
    m1, m2 = orc.monomials(1), orc.monomials(2)
    n1, n2 = len(m1), len(m2)
    pos2 = {tuple(int(x) for x in e): a for a, e in enumerate(m2)}
    var = [int(np.argmax(e)) for e in m1]  # degree-1 monomial a = z_var[a]

    def idx2(i, k):
        e = [0] * 5
        e[i] += 1
        e[k] += 1
        return pos2[tuple(e)]

    A = np.zeros((n1 * n1, n2 * n2))
    for a, b in itertools.product(range(n1), repeat=2):
        for k in range(5):
            A[a * n1 + b, idx2(var[a], k) * n2 + idx2(var[b], k)] += 1.0
    M1, K1 = balanced.laplacian_matrices(1)
    M2, K2 = balanced.laplacian_matrices(2)
    assert np.abs(A @ M2 @ A.T - M1).max() < 1e-12 * np.abs(M1).max()
    assert np.abs(A @ K2 @ A.T - K1).max() < 1e-12 * np.abs(K1).max()


def test_spectrum_nonnegative_with_one_null_mode(orc, balanced):
    ev = balanced.laplacian_eigs(40, 2)
    assert ev.shape == (40,)
    assert np.all(np.diff(ev) >= 0)
    assert ev[0] < 1e-9
    assert ev[1] > 1e-2


def test_yukawa_symmetric_and_trilinear(orc, balanced):
    rng = np.random.default_rng(5)
    c = rng.standard_normal((3, 225)) + 1j * rng.standard_normal((3, 225))
    y = balanced.yukawa(c)
    for perm in itertools.permutations(range(3)):
        assert np.abs(y - y.transpose(perm)).max() <= 1e-13 * np.abs(y).max()
    y2 = balanced.yukawa(2.0 * c)
    assert np.abs(y2 - 8.0 * y).max() <= 1e-13 * np.abs(y2).max()


def test_yukawa_constant_mode_is_mean_conj_omega(orc, balanced):
    v = _const_vector(orc, 2).astype(np.complex128)[None, :]
    y = balanced.yukawa(v)[0, 0, 0]
    pts = balanced.points
    psi = balanced.psi
    _, chart, elim = orc.log_omega(pts, psi)
    z = pts.view(np.complex128)
    g = np.array([orc.quintic_gradient(p, psi) for p in pts]).view(np.complex128)
    rows = np.arange(len(z))
    om = z[rows, chart] / g[rows, elim]
    w = balanced.weights
    ok = np.isfinite(w) & (w > 0)
    ref = np.sum(w[ok] * np.conj(om[ok])) / np.sum(w[ok])
    assert abs(y - ref) <= 1e-12 * abs(ref)
