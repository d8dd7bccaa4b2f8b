"""Unit known-answer tests of the FP64 oracle, mirroring the reference's own quintic tests
(substrate_sm_derivation/cy3_solver/src/quintic.rs:5467-9120) on CPU."""
import numpy as np
import pytest


def test_n_sections_correct(orc):  # quintic.rs:5472
    assert [len(orc.monomials(k)) for k in (2, 3, 4)] == [15, 35, 70]


def test_reduced_basis_sizes(orc):
    # ideal-reduced basis: drop multiples of z0^5; N_6 = 205, N_8 = 460 (and = full basis for k <= 4)
    assert len(orc.monomials(6, True)) == 205
    assert len(orc.monomials(8, True)) == 460
    for k in (2, 3, 4):
        np.testing.assert_array_equal(orc.monomials(k, True), orc.monomials(k, False))
    full, red = orc.monomials(6), orc.monomials(6, True)
    assert all(m[0] < 5 for m in red)
    # order preserved (subsequence of the lex order, quintic.rs:3192-3209)
    keep = [tuple(m) for m in full if m[0] < 5]
    assert keep == [tuple(m) for m in red]


def test_fermat_quintic_zero_at_known_root(orc):  # quintic.rs:5487
    z = np.array([1.0, 0, 0, 0, 0, 0, 0, 0, -1.0, 0])
    f = orc.quintic_value(z)
    assert abs(f) < 1e-12


def test_lcg_stream_first_values(orc):
    # LCG::new(s) = s*6364136223846793005 + 1; next_f64 uses the top 53 bits (lib.rs:225-236)
    M = (1 << 64) - 1
    s = (42 * 6364136223846793005 + 1) & M
    exp = []
    for _ in range(4):
        s = (s * 6364136223846793005 + 1442695040888963407) & M
        exp.append(((s >> 11) & ((1 << 53) - 1)) / float(1 << 53))
    np.testing.assert_array_equal(orc.lcg_uniforms(42, 4), np.array(exp))


def test_newton_sampled_points_lie_on_quintic(orc):  # quintic.rs:5522
    pts = orc.sample_newton(50, 7, 0.0, True, 1e-10)
    assert pts.shape == (50, 10)
    for z in pts:
        assert abs(orc.quintic_value(z)) ** 2 < 1e-15


@pytest.mark.parametrize("psi", [0.0, 0.5, 0.1 + 0.2j])
def test_sz_points_on_variety(orc, psi):
    pts, tried = orc.sample_sz(2000, 3, psi, fermat_variant=(psi == 0.0))
    assert len(pts) == 2000
    assert tried >= 400
    np.testing.assert_allclose(np.sum(pts ** 2, axis=1), 1.0, atol=1e-14)
    thr = 1e-3 if psi == 0.0 else 1e-2
    for z in pts[:200]:
        assert abs(orc.quintic_value(z, psi)) <= thr


def test_psi_complex_with_zero_imag_matches_real_path(orc):
    # complex-psi extension reduces bit-for-bit to the real-psi reference arithmetic
    a, _ = orc.sample_sz(500, 11, 0.5 + 0.0j, fermat_variant=False)
    b, _ = orc.sample_sz(500, 11, 0.5, fermat_variant=False)
    np.testing.assert_array_equal(a, b)


def test_psi_zero_deformed_matches_fermat_prefix(orc):  # quintic.rs:6018-6048 (psi=0 == Fermat)
    a, _ = orc.sample_sz(1000, 5, 0.0, fermat_variant=False)
    b, _ = orc.sample_sz(1000, 5, 0.0, fermat_variant=True)
    # same lines, same roots; thresholds differ (1e-2 vs 1e-3) so compare the common accepted prefix
    n = 0
    while n < 1000 and np.array_equal(a[n], b[n]):
        n += 1
    assert n > 900


def test_newton_polish_improves_roots(orc):
    a, _ = orc.sample_sz(500, 9, 0.5, fermat_variant=False)
    b, _ = orc.sample_sz(500, 9, 0.5, fermat_variant=False, newton_iters=3)
    fa = np.array([abs(orc.quintic_value(z, 0.5)) for z in a])
    fb = np.array([abs(orc.quintic_value(z, 0.5)) for z in b])
    assert fb.max() <= fa.max() + 1e-15
    assert np.max(np.abs(a - b)) < 1e-6


def test_weights_and_log_omega(orc):
    pts, _ = orc.sample_sz(300, 1, 0.5, fermat_variant=False)
    w = orc.weights(pts, 0.5)
    lo, ch, el = orc.log_omega(pts, 0.5)
    for p in range(0, 300, 37):
        g = orc.quintic_gradient(pts[p], 0.5)
        assert w[p] == pytest.approx(1.0 / np.sum(g * g), rel=1e-15)
        zz = pts[p][0::2] ** 2 + pts[p][1::2] ** 2
        gg = g[0::2] ** 2 + g[1::2] ** 2
        c = int(np.argmax(zz))
        assert ch[p] == c and el[p] != c
        assert lo[p] == pytest.approx(np.log(zz[c]) - np.log(gg[el[p]]), rel=1e-12)


def test_basis_derivatives_match_finite_difference(orc):
    pts, _ = orc.sample_sz(5, 2, 0.0)
    mono = orc.monomials(3)
    ds = orc.basis_derivs(pts, mono)
    h = 1e-6
    for i in range(5):
        zp = pts.copy()
        zm = pts.copy()
        zp[:, 2 * i] += h
        zm[:, 2 * i] -= h
        fd = (orc.basis(zp, mono) - orc.basis(zm, mono)) / (2 * h)
        np.testing.assert_allclose(ds[:, i, :], fd, atol=1e-8)


def test_fs_gram_orthonormalisation_makes_identity(orc):  # quintic.rs:5721
    s = orc.OracleSolver.new_with_sampler(2, 1500, 17, 1e-11, "newton")
    s.orthonormalise_basis_fs_gram()
    gr, gi = orc.fs_gram_matrix(s.section_values, s.weights)
    n = s.n_basis
    assert np.max(np.abs(gr - np.eye(n))) < 1e-6
    assert np.max(np.abs(gi)) < 1e-6


def test_donaldson_residual_decreases(orc):  # quintic.rs:5536
    s = orc.OracleSolver.new_with_sampler(2, 2000, 17, 1e-10, "sz")
    it = s.donaldson_solve(20, 1e-6)
    r = s.donaldson_residuals
    assert it >= 2 and r[-1] < r[0]


def test_donaldson_output_hermitian_block(orc):
    s = orc.OracleSolver.new_with_psi_sz(3, 3000, 4, 0.1 + 0.2j, reduced=True)
    s.donaldson_step()
    h = s.h_block
    np.testing.assert_allclose(h, h.T, atol=1e-14)
    np.testing.assert_array_equal(h[0::2, 0::2], h[1::2, 1::2])
    np.testing.assert_array_equal(h[0::2, 1::2], -h[1::2, 0::2])
    assert np.all(np.linalg.eigvalsh(h) > 0)


def test_analytic_gradient_matches_finite_difference(orc):  # quintic.rs:5646
    s = orc.OracleSolver.new_with_sampler(2, 600, 41, 1e-11, "newton")
    s.donaldson_solve(20, 1e-7)
    l2, g, _ = s.sigma_squared_and_gradient()
    n = s.n_basis
    eps = 1e-5
    h0 = s.h_block.copy()
    errs = []
    for a in range(3):
        s.h_block = h0.copy()
        s.h_block[2 * a, 2 * a] += eps
        s.h_block[2 * a + 1, 2 * a + 1] += eps
        lp, _, _ = s.sigma_squared_and_gradient()
        fd = (lp - l2) / eps
        errs.append(abs(fd - g[a * n + a]) / max(abs(fd), 1e-10))
    s.h_block = h0
    assert max(errs) < 0.05


def test_analytic_gradient_offdiag_complex_psi(orc):
    # off-diagonal real and imaginary directions at complex psi (central differences)
    s = orc.OracleSolver.new_with_psi_sz(2, 800, 6, 0.1 + 0.2j)
    s.donaldson_solve(10, 1e-9)
    _, g, _ = s.sigma_squared_and_gradient()
    n = s.n_basis
    h0 = s.h_block.copy()
    eps = 1e-6
    for (a, b) in [(0, 3), (2, 7), (5, 11)]:
        for part in ("re", "im"):
            def val(sign):
                hb = h0.copy()
                if part == "re":
                    for (i, j) in [(a, b), (b, a)]:
                        hb[2 * i, 2 * j] += sign * eps
                        hb[2 * i + 1, 2 * j + 1] += sign * eps
                else:  # h_im[a,b] += eps, h_im[b,a] -= eps ; block (2a,2b+1) = -h_im
                    hb[2 * a, 2 * b + 1] -= sign * eps
                    hb[2 * a + 1, 2 * b] += sign * eps
                    hb[2 * b, 2 * a + 1] += sign * eps
                    hb[2 * b + 1, 2 * a] -= sign * eps
                s.h_block = hb
                return s.sigma_squared_and_gradient()[0]
            fd = (val(1) - val(-1)) / (2 * eps)
            an = g[a * n + b] if part == "re" else g[n * n + a * n + b]
            assert an == pytest.approx(fd, rel=2e-3, abs=1e-9)
    s.h_block = h0


def test_adam_reduces_sigma(orc):  # quintic.rs analytic_adam_converges
    s = orc.OracleSolver.new_with_sampler(2, 1500, 51, 1e-11, "newton")
    s.donaldson_solve(50, 1e-8)
    s0 = s.sigma()
    hist = s.sigma_refine_analytic(30, 0.005)
    assert len(hist) == 30
    assert hist[0] == pytest.approx(s0, rel=1e-12)
    assert min(hist) < s0


def test_sigma_decreases_with_k(orc):  # quintic.rs:8603
    sig = []
    for k in (2, 3):
        s = orc.OracleSolver.new_with_sampler(k, 4000, 8, 1e-12, "sz")
        s.orthonormalise_basis_fs_gram()
        s.donaldson_solve(15, 1e-10)
        sig.append(s.sigma())
    assert sig[1] < sig[0]


def test_lbfgs_refinement_oracle(orc):
    """The oracle's restatement of the reference L-BFGS refinement (quintic.rs:678-890): sigma falls from the
    balanced metric, every recorded value is finite, and the handle is left at the lowest sigma seen."""
    o = orc.OracleSolver.new_with_sampler(2, 3000, 13, 1e-12, "sz")
    o.donaldson_solve(10, 1e-10)
    s0 = o.sigma()
    hist = orc.lbfgs_refine(o, 6, 5)
    assert len(hist) == 7 and all(np.isfinite(hist))
    assert hist[0] == pytest.approx(s0, rel=1e-12)
    assert min(hist) < 0.5 * s0
    assert o.sigma() == pytest.approx(min(hist), rel=1e-12)
    # restarts keep the best run
    o2 = orc.OracleSolver.new_with_sampler(2, 3000, 13, 1e-12, "sz")
    o2.donaldson_solve(10, 1e-10)
    best, runs = orc.lbfgs_refine_restarts(o2, 2, 3, 5, 1e-3, 7)
    assert len(runs) == 3 and best == min(runs)
    assert o2.sigma() == pytest.approx(best, rel=1e-12)
