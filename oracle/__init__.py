"""ctypes binding of the FP64 CPU oracle (oracle/cy3_oracle.cpp).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by ``__graft_entry__.smoke()`` and by the
CPU-baseline leg of ``bench.py`` -- never by the product package ``papers_b200``.

The oracle restates the reference crate ``substrate_sm_derivation/cy3_solver`` (Rust) function
by function; each wrapper below names the reference function it mirrors.  ``OracleSolver``
mirrors the reference workspace ``QuinticSolver`` (src/quintic.rs:117-165) so tests read like
the reference's own tests.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (gcc, -ffp-contract=off)."""
    srcs = [os.path.join(_HERE, f) for f in ("cy3_oracle.cpp", "cicy_oracle.cpp", "Makefile")]
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < max(map(os.path.getmtime, srcs)):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    sz = C.c_size_t
    d = C.c_double
    L.orc_set_threads.argtypes = [C.c_int]
    L.orc_get_threads.restype = C.c_int
    L.orc_quintic_value.argtypes = [_dp, d, d, _dp]
    L.orc_quintic_gradient.argtypes = [_dp, d, d, _dp]
    L.orc_lcg_normals.argtypes = [C.c_uint64, sz, _dp]
    L.orc_lcg_uniforms.argtypes = [C.c_uint64, sz, _dp]
    L.orc_sample_sz.argtypes = [sz, C.c_uint64, d, d, C.c_int, C.c_int, C.c_int, _dp, C.POINTER(sz)]
    L.orc_sample_sz.restype = sz
    L.orc_sample_newton.argtypes = [sz, C.c_uint64, d, d, C.c_int, d, _dp]
    L.orc_sample_newton.restype = sz
    L.orc_weights.argtypes = [_dp, sz, d, d, _dp]
    L.orc_log_omega.argtypes = [_dp, sz, d, d, _dp, _ip, _ip]
    L.orc_monomials.argtypes = [C.c_int, C.c_int, C.c_void_p]
    L.orc_monomials.restype = C.c_int
    L.orc_basis.argtypes = [_dp, sz, _up, C.c_int, _dp]
    L.orc_basis_derivs.argtypes = [_dp, sz, _up, C.c_int, _dp]
    L.orc_fs_gram_matrix.argtypes = [_dp, _dp, sz, C.c_int, _dp, _dp]
    L.orc_cholesky.argtypes = [_dp, _dp, C.c_int, _dp, _dp]
    L.orc_cholesky.restype = C.c_int
    L.orc_fs_gram_orthonormalise.argtypes = [_dp, C.c_void_p, _dp, sz, C.c_int]
    L.orc_fs_gram_orthonormalise.restype = C.c_int
    L.orc_invert_real.argtypes = [_dp, C.c_int, _dp]
    L.orc_invert_real.restype = C.c_int
    L.orc_inv_k.argtypes = [_dp, sz, C.c_int, _dp, _dp]
    L.orc_t_operator.argtypes = [_dp, _dp, sz, C.c_int, _dp, _dp, C.c_void_p, C.c_void_p]
    L.orc_donaldson_step.argtypes = [_dp, _dp, sz, C.c_int, _dp, C.POINTER(d)]
    L.orc_donaldson_step.restype = C.c_int
    L.orc_sigma.argtypes = [_dp, _dp, _dp, _dp, _dp, sz, C.c_int, d, d, _dp, C.c_void_p]
    L.orc_sigma.restype = d
    L.orc_point_grad.argtypes = [_dp, _dp, _dp, _dp, d, C.c_int, d, d, _dp, C.POINTER(d), C.POINTER(d)]
    L.orc_sigma_grad.argtypes = [_dp, _dp, _dp, _dp, _dp, sz, C.c_int, d, d, _dp, C.POINTER(d), _dp, C.POINTER(d)]
    L.orc_sigma_grad.restype = C.c_int
    L.orc_adam_refine.argtypes = [_dp, _dp, _dp, _dp, _dp, sz, C.c_int, d, d, _dp, C.c_int, d, d, d, d, _dp]
    L.orc_adam_refine.restype = C.c_int
    L.orc_laplacian_rows.argtypes = [_dp, _dp, _dp, _dp, _dp, sz, C.c_int, d, d, _dp, C.c_int, _dp, _dp, _dp]
    L.orc_laplacian_rows.restype = C.c_int
    L.orc_laplacian_gram.argtypes = [_dp, _dp, _dp, sz, C.c_int, _dp, _dp]
    L.orc_laplacian_gram.restype = d
    L.orc_yukawa.argtypes = [_dp, _dp, sz, d, d, C.c_int, _dp, C.c_int, _dp]
    L.orc_yukawa.restype = C.c_int
    vp = C.c_void_p
    L.orc_ty_rng_u64.argtypes = [C.c_uint64, sz, vp]
    L.orc_ty_normals.argtypes = [C.c_uint64, sz, _dp]
    L.orc_ty_sample.argtypes = [C.c_uint64, sz, C.c_int, C.c_int, _dp, _dp, _dp, _ip]
    L.orc_ty_sample.restype = sz
    L.orc_ty_post_process.argtypes = [_dp, _dp, _dp, _dp, _ip]
    L.orc_ty_post_process.restype = C.c_int
    L.orc_ty_groebner_lms.argtypes = [_ip, C.c_int]
    L.orc_ty_groebner_lms.restype = C.c_int
    L.orc_ty_basis.argtypes = [C.c_int, _ip, C.c_int]
    L.orc_ty_basis.restype = C.c_int
    L.orc_ty_sections.argtypes = [_dp, sz, _ip, C.c_int, _dp, vp]
    L.orc_ty_frames.argtypes = [_dp, _ip, sz, _dp]
    L.orc_ty_donaldson_step.argtypes = [_dp, _dp, sz, C.c_int, _dp, _dp, d]
    L.orc_ty_donaldson_step.restype = d
    L.orc_ty_sigma.argtypes = [_dp, _dp, _dp, sz, C.c_int, _dp, _dp, vp]
    L.orc_ty_sigma.restype = d
    L.orc_ty_solve.argtypes = [C.c_int, sz, C.c_int, d, C.c_uint64, _dp, _dp, _dp, C.c_int, vp, vp, sz]
    L.orc_ty_solve.restype = C.c_int
    L.orc_schoen_sample.argtypes = [C.c_uint64, sz, C.c_int, C.c_int, _dp, _dp, _dp, _ip]
    L.orc_schoen_sample.restype = sz
    L.orc_schoen_groebner_lms.argtypes = [_ip, C.c_int]
    L.orc_schoen_groebner_lms.restype = C.c_int
    L.orc_schoen_basis.argtypes = [C.c_int, C.c_int, C.c_int, _ip, C.c_int]
    L.orc_schoen_basis.restype = C.c_int
    L.orc_schoen_frames.argtypes = [_dp, sz, _dp]
    L.orc_schoen_sigma.argtypes = [_dp, _dp, _dp, sz, C.c_int, C.c_int, C.c_int, _dp, _dp, vp]
    L.orc_schoen_sigma.restype = d
    L.orc_schoen_solve.argtypes = [C.c_int, C.c_int, C.c_int, sz, C.c_int, d, C.c_uint64, _dp, _dp, _dp, C.c_int,
                                   vp, vp, sz]
    L.orc_schoen_solve.restype = C.c_int
    L.orc_cicy_adam_refine.argtypes = [C.c_int, _ip, _dp, _dp, _dp, sz, _dp, _dp, C.c_int, d, d, d, _dp, C.c_int]
    L.orc_cicy_adam_refine.restype = C.c_int
    _lib = L
    return L


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def threads() -> int:
    return int(lib().orc_get_threads())


# ---------------------------------------------------------------------------------------------
# free functions
# ---------------------------------------------------------------------------------------------
def quintic_value(z: np.ndarray, psi: complex = 0.0) -> complex:
    """deformed_fermat_quintic (quintic.rs:3248) at one point z [10]."""
    psi = complex(psi)
    out = np.empty(2)
    lib().orc_quintic_value(np.ascontiguousarray(z, dtype=np.float64), psi.real, psi.imag, out)
    return complex(out[0], out[1])


def quintic_gradient(z: np.ndarray, psi: complex = 0.0) -> np.ndarray:
    """deformed_fermat_quintic_gradient (quintic.rs:3276): 10 reals."""
    psi = complex(psi)
    out = np.empty(10)
    lib().orc_quintic_gradient(np.ascontiguousarray(z, dtype=np.float64), psi.real, psi.imag, out)
    return out


def lcg_normals(seed: int, n: int) -> np.ndarray:
    """LCG(seed).next_normal() stream (src/lib.rs:225-246)."""
    out = np.empty(n)
    lib().orc_lcg_normals(seed, n, out)
    return out


def lcg_uniforms(seed: int, n: int) -> np.ndarray:
    out = np.empty(n)
    lib().orc_lcg_uniforms(seed, n, out)
    return out


def sample_sz(n: int, seed: int, psi: complex = 0.0, fermat_variant: bool = True, dk_iters: int = 50,
              newton_iters: int = 0):
    """Line-intersection sampler: sample_quintic_points_sz (quintic.rs:3633) when fermat_variant,
    else sample_deformed_quintic_points_sz (quintic.rs:3810) with complex psi.
    Returns (points [P,10], lines_tried)."""
    out = np.empty((n, 10))
    tried = C.c_size_t(0)
    psi = complex(psi)
    got = lib().orc_sample_sz(n, seed, psi.real, psi.imag, 0 if fermat_variant else 1, dk_iters, newton_iters,
                              out.reshape(-1), C.byref(tried))
    return np.ascontiguousarray(out[:got]), int(tried.value)


def sample_newton(n: int, seed: int, psi: complex = 0.0, fermat_variant: bool = True, tol: float = 1e-12):
    """Newton-projection sampler (quintic.rs:3568 / 3448)."""
    out = np.empty((n, 10))
    psi = complex(psi)
    got = lib().orc_sample_newton(n, seed, psi.real, psi.imag, 0 if fermat_variant else 1, tol, out.reshape(-1))
    return np.ascontiguousarray(out[:got])


def weights(pts: np.ndarray, psi: complex = 0.0) -> np.ndarray:
    """cy_measure_weights(_psi) (quintic.rs:3507-3563)."""
    psi = complex(psi)
    w = np.empty(len(pts))
    lib().orc_weights(np.ascontiguousarray(pts).reshape(-1), len(pts), psi.real, psi.imag, w)
    return w


def log_omega(pts: np.ndarray, psi: complex = 0.0):
    """log|Omega|^2, chart, elim (quintic.rs:4858-4916). Returns (log_om, chart, elim)."""
    psi = complex(psi)
    P = len(pts)
    lo = np.empty(P)
    ch = np.empty(P, np.int32)
    el = np.empty(P, np.int32)
    lib().orc_log_omega(np.ascontiguousarray(pts).reshape(-1), P, psi.real, psi.imag, lo, ch, el)
    return lo, ch, el


def monomials(k: int, reduced: bool = False) -> np.ndarray:
    """build_degree_k_quintic_monomials (quintic.rs:3192); reduced drops e0 >= 5."""
    n = lib().orc_monomials(k, int(reduced), None)
    out = np.empty((n, 5), np.uint32)
    lib().orc_monomials(k, int(reduced), out.ctypes.data)
    return out


def basis(pts: np.ndarray, mono: np.ndarray) -> np.ndarray:
    """evaluate_quintic_basis (quintic.rs:4021): [P, 2N] interleaved (re, im)."""
    P, N = len(pts), len(mono)
    s = np.empty((P, 2 * N))
    lib().orc_basis(np.ascontiguousarray(pts).reshape(-1), P, np.ascontiguousarray(mono).reshape(-1), N, s.reshape(-1))
    return s


def basis_derivs(pts: np.ndarray, mono: np.ndarray) -> np.ndarray:
    """evaluate_quintic_basis_derivs_soa (quintic.rs:1231): [P, 5, 2N]."""
    P, N = len(pts), len(mono)
    d = np.empty((P, 5, 2 * N))
    lib().orc_basis_derivs(np.ascontiguousarray(pts).reshape(-1), P, np.ascontiguousarray(mono).reshape(-1), N,
                           d.reshape(-1))
    return d


def fs_gram_matrix(s: np.ndarray, w: np.ndarray):
    """compute_fs_gram_matrix (quintic.rs:2957)."""
    P, N = s.shape[0], s.shape[1] // 2
    gr = np.empty((N, N))
    gi = np.empty((N, N))
    lib().orc_fs_gram_matrix(s.reshape(-1), w, P, N, gr.reshape(-1), gi.reshape(-1))
    return gr, gi


def invert_real(a: np.ndarray) -> np.ndarray:
    n = a.shape[0]
    out = np.empty_like(a)
    rc = lib().orc_invert_real(np.ascontiguousarray(a).reshape(-1), n, out.reshape(-1))
    if rc != 0:
        raise np.linalg.LinAlgError("singular")
    return out


def t_operator(s: np.ndarray, w: np.ndarray, h_block: np.ndarray) -> np.ndarray:
    """Trace-renormalised lower-index T(h) packed as a 2N x 2N block (quintic.rs:1761-1826)."""
    P, N = s.shape[0], s.shape[1] // 2
    tb = np.empty((2 * N, 2 * N))
    lib().orc_t_operator(s.reshape(-1), w, P, N, np.ascontiguousarray(h_block).reshape(-1), tb.reshape(-1), None, None)
    return tb


def identity_h(N: int) -> np.ndarray:
    """init_h_block_identity (quintic.rs:4120)."""
    return np.eye(2 * N)


# ---------------------------------------------------------------------------------------------
# QuinticSolver mirror
# ---------------------------------------------------------------------------------------------
class OracleSolver:
    """Mirror of the reference workspace `QuinticSolver` (quintic.rs:117-165) on the oracle."""

    def __init__(self, points, weights_, log_om, monomials_, psi=0.0, k_degree=None, with_derivs=True):
        self.points = np.ascontiguousarray(points, dtype=np.float64)
        self.n_points = len(self.points)
        self.weights = np.ascontiguousarray(weights_, dtype=np.float64)
        self.log_omega_sq = np.ascontiguousarray(log_om, dtype=np.float64)
        self.monomials = np.ascontiguousarray(monomials_, dtype=np.uint32)
        self.n_basis = len(self.monomials)
        self.k_degree = k_degree
        self.psi = complex(psi)
        self.section_values = basis(self.points, self.monomials)
        # the balancing step needs the values only; sigma and its gradient need the derivatives too
        self.section_derivs = basis_derivs(self.points, self.monomials) if with_derivs else None
        self.h_block = identity_h(self.n_basis)
        self.donaldson_residuals: list[float] = []

    # constructors (quintic.rs:174-322)
    @classmethod
    def new_with_sampler(cls, k, n_points, seed, newton_tol=1e-12, sampler="sz", reduced=False):
        """QuinticSolver::new_with_sampler (quintic.rs:281), Fermat quintic."""
        if sampler == "sz":
            pts, _ = sample_sz(n_points, seed, 0.0, fermat_variant=True)
        else:
            pts = sample_newton(n_points, seed, 0.0, True, newton_tol)
        if len(pts) == 0:
            return None
        lo, _, _ = log_omega(pts, 0.0)
        return cls(pts, weights(pts, 0.0), lo, monomials(k, reduced), 0.0, k)

    @classmethod
    def new_with_psi_sz(cls, k, n_points, seed, psi, reduced=False, newton_iters=0):
        """QuinticSolver::new_with_psi_sz (quintic.rs:240), extended to complex psi."""
        pts, _ = sample_sz(n_points, seed, psi, fermat_variant=False, newton_iters=newton_iters)
        if len(pts) == 0:
            return None
        lo, _, _ = log_omega(pts, psi)
        return cls(pts, weights(pts, psi), lo, monomials(k, reduced), psi, k)

    # methods
    def orthonormalise_basis_fs_gram(self):
        """quintic.rs:3140."""
        rc = lib().orc_fs_gram_orthonormalise(self.section_values.reshape(-1), None if self.section_derivs is None else self.section_derivs.ctypes.data,
                                              self.weights, self.n_points, self.n_basis)
        if rc != 0:
            raise ValueError("FS Gram matrix not positive-definite")
        self.h_block = identity_h(self.n_basis)

    def donaldson_step(self) -> float:
        """quintic.rs:428 -> donaldson_step_workspace (quintic.rs:1734)."""
        r = C.c_double(0.0)
        lib().orc_donaldson_step(self.section_values.reshape(-1), self.weights, self.n_points, self.n_basis,
                                 self.h_block.reshape(-1), C.byref(r))
        return r.value

    def donaldson_step_unfixed(self) -> float:
        """The reference's Donaldson step as it was before its 2026-04-29 fix (quintic.rs:1722-1726 describes
        it): the trace-renormalised lower-index T(h) stored into h_block without inversion, residual
        ||T(h) - h||_F.  Not the drop-in; kept only to reproduce run records made with it
        (output/p5_3_multi_seed_ensemble.json)."""
        t = t_operator(self.section_values, self.weights, self.h_block)
        r = float(np.linalg.norm(t - self.h_block))
        self.h_block = np.ascontiguousarray(t)
        return r

    def donaldson_solve(self, max_iter: int, tol: float, unfixed: bool = False) -> int:
        """quintic.rs:433 (with `unfixed`, the earlier step of donaldson_step_unfixed)."""
        self.donaldson_residuals = []
        for _ in range(max_iter):
            r = self.donaldson_step_unfixed() if unfixed else self.donaldson_step()
            self.donaldson_residuals.append(r)
            if r < tol:
                break
        return len(self.donaldson_residuals)

    def sigma(self, return_eta: bool = False):
        """quintic.rs:423 -> compute_sigma_from_workspace (quintic.rs:1301)."""
        eta = np.empty(self.n_points)
        v = lib().orc_sigma(self.section_values.reshape(-1), self.section_derivs.reshape(-1), self.points.reshape(-1),
                            self.log_omega_sq, self.weights, self.n_points, self.n_basis, self.psi.real,
                            self.psi.imag, self.h_block.reshape(-1), eta.ctypes.data)
        return (v, eta) if return_eta else v

    def sigma_squared_and_gradient(self):
        """sigma_squared_and_gradient (quintic.rs:2714): (sigma_L2^2, grad[2N^2], sigma_L1)."""
        n = self.n_basis
        g = np.empty(2 * n * n)
        l2 = C.c_double()
        l1 = C.c_double()
        lib().orc_sigma_grad(self.section_values.reshape(-1), self.section_derivs.reshape(-1), self.points.reshape(-1),
                             self.log_omega_sq, self.weights, self.n_points, n, self.psi.real, self.psi.imag,
                             self.h_block.reshape(-1), C.byref(l2), g, C.byref(l1))
        return l2.value, g, l1.value

    def laplacian_rows(self, test_degree: int = 2):
        """Per-point Galerkin rows at the current h: f [P][nf], e [P][3][nf] (complex) and c_p = w_p eta_p."""
        nd = len(monomials(test_degree))
        nf = nd * nd
        P = self.n_points
        F = np.empty((P, nf), np.complex128)
        E = np.empty((P, 3, nf), np.complex128)
        c = np.empty(P, np.float64)
        got = lib().orc_laplacian_rows(self.section_values.reshape(-1), self.section_derivs.reshape(-1),
                                       self.points.reshape(-1), self.weights, self.log_omega_sq, P, self.n_basis,
                                       self.psi.real, self.psi.imag, self.h_block.reshape(-1), test_degree,
                                       F.view(np.float64).reshape(-1), E.view(np.float64).reshape(-1), c)
        if got != nf:
            raise ValueError("unsupported test degree")
        return F, E, c

    def laplacian_matrices(self, test_degree: int = 2):
        """Galerkin mass and stiffness matrices (complex nf x nf, normalised by sum c) at the current h."""
        return laplacian_gram(*self.laplacian_rows(test_degree))

    def laplacian_eigs(self, n_eigs: int = 40, test_degree: int = 2, reg: float = 1e-12):
        return laplacian_eigs(*self.laplacian_matrices(test_degree), n_eigs=n_eigs, reg=reg)

    def yukawa(self, coeffs: np.ndarray, test_degree: int = 2) -> np.ndarray:
        c = np.ascontiguousarray(coeffs, dtype=np.complex128)
        nm = c.shape[0]
        y = np.empty(nm ** 3, np.complex128)
        got = lib().orc_yukawa(self.points.reshape(-1), self.weights, self.n_points, self.psi.real, self.psi.imag,
                               test_degree, c.view(np.float64).reshape(-1), nm, y.view(np.float64).reshape(-1))
        if got < 0:
            raise ValueError("unsupported test degree or mode count")
        return y.reshape(nm, nm, nm)

    def sigma_refine_analytic(self, n_iter: int, lr: float, beta1=0.9, beta2=0.999, eps=1e-8):
        """QuinticSolver::sigma_refine_analytic (quintic.rs:453)."""
        hist = np.empty(max(n_iter, 1))
        done = lib().orc_adam_refine(self.section_values.reshape(-1), self.section_derivs.reshape(-1),
                                     self.points.reshape(-1), self.log_omega_sq, self.weights, self.n_points,
                                     self.n_basis, self.psi.real, self.psi.imag, self.h_block.reshape(-1), n_iter, lr,
                                     beta1, beta2, eps, hist)
        return list(hist[:done])


def _unpack_h(hb: np.ndarray, n: int):
    """h_block -> (h_re, h_im) (quintic.rs:4081-4085 packing)."""
    return hb[0::2, 0::2].copy(), -hb[0::2, 1::2].copy()


def _pack_renorm_h(hre: np.ndarray, him: np.ndarray, n: int) -> np.ndarray:
    """pack_h_block_workspace + renormalise_h_trace_workspace (quintic.rs:2148-2160, 3169-3182)."""
    hb = np.empty((2 * n, 2 * n))
    hb[0::2, 0::2] = hre
    hb[0::2, 1::2] = -him
    hb[1::2, 0::2] = him
    hb[1::2, 1::2] = hre
    tr = 0.0
    for a in range(n):
        tr += hb[2 * a, 2 * a]
    if tr > 1e-10:
        hb *= n / tr
    return hb


def _apply_lbfgs_step(h_save: np.ndarray, d: np.ndarray, step: float, n: int) -> np.ndarray:
    """apply_lbfgs_step (quintic.rs:2003-2047) from h_save."""
    hre, him = _unpack_h(h_save, n)
    nn = n * n
    hre = hre + step * d[:nn].reshape(n, n)
    iu = np.triu_indices(n, 1)
    avg = 0.5 * (hre[iu] + hre.T[iu])
    hre[iu] = avg
    hre.T[iu] = avg
    upd = step * d[nn:].reshape(n, n)[iu]
    him[iu] += upd
    him.T[iu] -= upd
    him[np.diag_indices(n)] = 0.0
    return _pack_renorm_h(hre, him, n)


def _seq_dot(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.dot(a, b))


def lbfgs_refine(solver, n_iter: int, m_history: int):
    """QuinticSolver::sigma_refine_lbfgs_gpu_legacy (quintic.rs:678-890) on the oracle: the optimizer of the
    reference step for step, the objective sigma_squared_and_gradient (quintic.rs:2714).  Returns the
    sigma_L1 history (start and every accepted step) and leaves the lowest-sigma h in the solver."""
    n = solver.n_basis
    n_dof = 2 * n * n
    f, g, sigma = solver.sigma_squared_and_gradient()
    hist = []
    if not np.isfinite(sigma):
        return hist
    hist.append(sigma)
    best_sigma, best_h = sigma, solver.h_block.copy()
    s_hist, y_hist, rho_hist = [], [], []
    for _ in range(n_iter):
        q = g.copy()
        m = len(s_hist)
        alphas = [0.0] * m
        for k in range(m - 1, -1, -1):
            a = rho_hist[k] * _seq_dot(s_hist[k], q)
            alphas[k] = a
            q -= a * y_hist[k]
        gamma = 1.0
        if m > 0:
            sy, yy = rho_hist[-1], _seq_dot(y_hist[-1], y_hist[-1])
            gamma = 1.0 / (sy * yy) if (yy > 1e-30 and np.isfinite(sy)) else 1.0
        q *= gamma
        for k in range(m):
            b = rho_hist[k] * _seq_dot(y_hist[k], q)
            q += s_hist[k] * (alphas[k] - b)
        d = -q
        gd = _seq_dot(g, d)
        used = m > 0
        if not np.isfinite(gd) or gd >= 0.0:
            s_hist, y_hist, rho_hist = [], [], []
            d = -g
            gd = _seq_dot(g, d)
            used = False
            if gd >= 0.0:
                break
        gn = float(np.sqrt(_seq_dot(g, g)))
        h_save = solver.h_block.copy()

        def search(step0):
            t = step0
            for _ls in range(30):
                solver.h_block = _apply_lbfgs_step(h_save, d, t, n)
                ft, gt, st = solver.sigma_squared_and_gradient()
                if np.isfinite(ft) and ft <= f + 1e-4 * t * gd:
                    return t, ft, gt, st
                t *= 0.5
            return None

        res = search(1.0 if used else (1.0 / gn if gn > 1e-30 else 1.0))
        if res is None and used:
            s_hist, y_hist, rho_hist = [], [], []
            d = -g
            gd = _seq_dot(g, d)
            res = search(1.0 / gn if gn > 1e-30 else 1.0)
        if res is None:
            solver.h_block = h_save
            break
        step, f_new, g_new, s_new = res
        sk, yk = step * d, g_new - g
        sy = _seq_dot(sk, yk)
        if sy > 1e-12:
            s_hist.append(sk)
            y_hist.append(yk)
            rho_hist.append(1.0 / sy)
            if len(s_hist) > m_history:
                s_hist.pop(0)
                y_hist.pop(0)
                rho_hist.pop(0)
        if np.isfinite(s_new) and s_new < best_sigma:
            best_sigma, best_h = s_new, solver.h_block.copy()
        f, g = f_new, g_new
        hist.append(s_new)
    solver.h_block = best_h
    return hist


def lbfgs_refine_restarts(solver, n_restarts: int, n_iter: int, m_history: int, perturb_scale: float, seed: int):
    """QuinticSolver::sigma_refine_lbfgs_with_restarts_gpu (quintic.rs:1100-1139) on the oracle, with
    perturb_h_block_hermitian (quintic.rs:1195-1223) drawing from LCG(seed)."""
    n = solver.n_basis
    lbfgs_refine(solver, n_iter, m_history)
    best = solver.sigma()
    best_h = solver.h_block.copy()
    hist = [best]
    u = lcg_uniforms(seed, n_restarts * n * n + 1)
    pos = 0
    for _ in range(n_restarts):
        hre, him = _unpack_h(best_h, n)
        for a in range(n):
            hre[a, a] += perturb_scale * (u[pos] * 2.0 - 1.0)
            pos += 1
            for b in range(a + 1, n):
                dr = perturb_scale * (u[pos] * 2.0 - 1.0)
                di = perturb_scale * (u[pos + 1] * 2.0 - 1.0)
                pos += 2
                hre[a, b] += dr
                hre[b, a] += dr
                him[a, b] += di
                him[b, a] -= di
        solver.h_block = _pack_renorm_h(hre, him, n)
        lbfgs_refine(solver, n_iter, m_history)
        trial = solver.sigma()
        hist.append(trial)
        if np.isfinite(trial) and trial < best:
            best, best_h = trial, solver.h_block.copy()
    solver.h_block = best_h
    return best, hist


def laplacian_gram(F: np.ndarray, E: np.ndarray, c: np.ndarray):
    """M = sum c conj(f) f^T / sum c and K = sum c e^H e / sum c, accumulated point by point in FP64."""
    F = np.ascontiguousarray(F, np.complex128)
    E = np.ascontiguousarray(E, np.complex128)
    c = np.ascontiguousarray(c, np.float64)
    P, nf = F.shape
    M = np.empty((nf, nf), np.complex128)
    K = np.empty((nf, nf), np.complex128)
    lib().orc_laplacian_gram(F.view(np.float64).reshape(-1), E.view(np.float64).reshape(-1), c, P, nf,
                             M.view(np.float64).reshape(-1), K.view(np.float64).reshape(-1))
    return M, K


def laplacian_eigs(M: np.ndarray, K: np.ndarray, n_eigs: int = 40, reg: float = 1e-12) -> np.ndarray:
    """Lowest n_eigs of K v = lambda (M + reg |M|_F I) v by magnitude (metric_laplacian.rs:350-392:
    Frobenius-scaled Tikhonov shift of the mass matrix, eigenvalues sorted by |lambda|)."""
    import scipy.linalg

    n = M.shape[0]
    Mr = M + reg * np.linalg.norm(M) * np.eye(n)
    ev = scipy.linalg.eigh(K, Mr, eigvals_only=True)
    return np.sort(np.abs(ev))[:n_eigs]


# ---------------------------------------------------------------------------------------------
# Tian-Yau (oracle/cicy_oracle.cpp): the reference's solve_ty_metric path (route34/ty_metric.rs)
# ---------------------------------------------------------------------------------------------
def ty_rng_u64(seed: int, n: int) -> np.ndarray:
    """First n u64 of ChaCha8Rng::seed_from_u64(seed) (rand_chacha 0.9)."""
    out = np.empty(n, dtype=np.uint64)
    lib().orc_ty_rng_u64(int(seed), int(n), out.ctypes.data)
    return out


def ty_normals(seed: int, n: int) -> np.ndarray:
    """First n StandardNormal draws (rand_distr 0.5 ziggurat) from ChaCha8Rng::seed_from_u64(seed)."""
    out = np.empty(n)
    lib().orc_ty_normals(int(seed), int(n), out)
    return out


def ty_sample(n: int, seed: int, gpu_stream: bool = False, z3: bool = True):
    """CicySampler::sample_batch (cicy_sampler.rs:600) [+ apply_z3_quotient].  gpu_stream draws the
    line inputs as sample_batch_gpu does (max(4n, 64) lines, one Newton attempt each).
    Returns (coords [P,16], omega [P] complex, weight [P], zw [P,2])."""
    coords = np.empty((n, 16))
    om = np.empty((n, 2))
    w = np.empty(n)
    zw = np.empty((n, 2), dtype=np.int32)
    P = lib().orc_ty_sample(int(seed), int(n), int(gpu_stream), int(z3), coords, om, w, zw)
    return coords[:P].copy(), (om[:P, 0] + 1j * om[:P, 1]), w[:P].copy(), zw[:P].copy()


def ty_post_process(x: np.ndarray):
    """post_process_solved_point (cicy_sampler.rs:452) of one line solution x [16]; None on rejection."""
    coords = np.empty((1, 16))
    om = np.empty((1, 2))
    w = np.empty(1)
    zw = np.empty((1, 2), dtype=np.int32)
    if not lib().orc_ty_post_process(np.ascontiguousarray(x, dtype=np.float64), coords, om, w, zw):
        return None
    return coords[0], complex(om[0, 0], om[0, 1]), float(w[0]), zw[0]


def ty_groebner_lms() -> np.ndarray:
    """Leading monomials of the reduced deg-lex Groebner basis of the Tian-Yau ideal (groebner.rs:556)."""
    out = np.zeros(4096 * 8, dtype=np.int32)
    n = lib().orc_ty_groebner_lms(out, 4096)
    return out[: n * 8].reshape(n, 8)


def ty_basis(k: int) -> np.ndarray:
    """build_ty_invariant_reduced_basis (ty_metric.rs:870): [N, 8] exponents."""
    cap = 20000
    out = np.zeros(cap * 8, dtype=np.int32)
    n = lib().orc_ty_basis(int(k), out, cap)
    return out[: n * 8].reshape(n, 8)


def ty_sections(coords: np.ndarray, basis: np.ndarray, derivs: bool = True):
    """Section values [P, 2N] and derivatives [P, 8, 2N] (ty_metric.rs:930-1000)."""
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    basis = np.ascontiguousarray(basis, dtype=np.int32)
    P, N = coords.shape[0], basis.shape[0]
    vals = np.empty((P, 2 * N))
    ders = np.empty((P, 8, 2 * N)) if derivs else None
    lib().orc_ty_sections(coords, P, basis, N, vals, ders.ctypes.data if derivs else None)
    return (vals, ders) if derivs else vals


def ty_frames(coords: np.ndarray, zw: np.ndarray) -> np.ndarray:
    """ty_affine_chart_frame (ty_metric.rs:1929) per point: [P, 3, 8] complex."""
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    P = coords.shape[0]
    out = np.empty((P, 3, 16))
    lib().orc_ty_frames(coords, np.ascontiguousarray(zw, dtype=np.int32), P, out)
    return out[..., 0::2] + 1j * out[..., 1::2]


def ty_donaldson_step(vals: np.ndarray, w: np.ndarray, h: np.ndarray, alpha: float = 1.0):
    """donaldson_iteration (ty_metric.rs:1062): h (N x N complex, upper index) -> (h_new, residual)."""
    P, N = vals.shape[0], vals.shape[1] // 2
    hr = np.ascontiguousarray(h.real, dtype=np.float64).copy()
    hi = np.ascontiguousarray(h.imag, dtype=np.float64).copy()
    r = lib().orc_ty_donaldson_step(np.ascontiguousarray(vals), np.ascontiguousarray(w, dtype=np.float64),
                                    P, N, hr, hi, float(alpha))
    return hr + 1j * hi, r


def ty_sigma(coords: np.ndarray, omega_sq: np.ndarray, w: np.ndarray, k: int, h: np.ndarray):
    """compute_sigma (ty_metric.rs:1402) on the points for metric h: (sigma, eta [P])."""
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    P = coords.shape[0]
    eta = np.empty(P)
    s = lib().orc_ty_sigma(coords, np.ascontiguousarray(omega_sq, dtype=np.float64),
                           np.ascontiguousarray(w, dtype=np.float64), P, int(k),
                           np.ascontiguousarray(h.real, dtype=np.float64),
                           np.ascontiguousarray(h.imag, dtype=np.float64), eta.ctypes.data)
    return s, eta


def ty_solve(k: int, n_sample: int, max_iter: int, tol: float, seed: int):
    """solve_ty_metric (ty_metric.rs:461) with the spec defaults of cy3_metric_unified.rs:249-261.
    Returns a dict with n_points, n_basis, iterations_run, sigma_fs_identity, sigma_final,
    final_donaldson_residual, sigma_history, donaldson_history and h (N x N complex)."""
    rec = np.zeros(6)
    cap = max(8, 8 * max_iter + 8)
    sh = np.zeros(cap)
    rh = np.zeros(cap)
    hcap = 4096 * 4096
    n_est = int(ty_basis(k).shape[0])
    hr = np.zeros(n_est * n_est)
    hi = np.zeros(n_est * n_est)
    n = lib().orc_ty_solve(int(k), int(n_sample), int(max_iter), float(tol), int(seed), rec, sh, rh, cap,
                           hr.ctypes.data, hi.ctypes.data, hr.size)
    if n < 0:
        raise RuntimeError(f"orc_ty_solve failed ({n})")
    N = int(rec[1])
    return dict(n_points=int(rec[0]), n_basis=N, iterations_run=int(rec[2]), sigma_fs_identity=rec[3],
                sigma_final=rec[4], final_donaldson_residual=rec[5], sigma_history=sh[:n].copy(),
                donaldson_history=rh[:n].copy(), h=(hr + 1j * hi).reshape(N, N))


# ---------------------------------------------------------------------------------------------
# Schoen (oracle/cicy_oracle.cpp): solve_schoen_metric (route34/schoen_metric.rs:766)
# ---------------------------------------------------------------------------------------------
def schoen_sample(n: int, seed: int, gpu_stream: bool = False, quotient: bool = True):
    """SchoenSampler::sample_points (schoen_sampler.rs:482) [+ apply_z3xz3_quotient]; gpu_stream: one Newton
    attempt per line, the device sampler's layout.  Returns (coords [P,16], omega [P] complex, weight [P],
    patch [P,3])."""
    coords = np.empty((n, 16))
    om = np.empty((n, 2))
    w = np.empty(n)
    pa = np.empty((n, 3), dtype=np.int32)
    P = lib().orc_schoen_sample(int(seed), int(n), int(gpu_stream), int(quotient), coords, om, w, pa)
    return coords[:P].copy(), (om[:P, 0] + 1j * om[:P, 1]), w[:P].copy(), pa[:P].copy()


def schoen_groebner_lms() -> np.ndarray:
    out = np.zeros(4096 * 8, dtype=np.int32)
    n = lib().orc_schoen_groebner_lms(out, 4096)
    return out[: n * 8].reshape(n, 8)


def schoen_basis(dx: int, dy: int, dt: int) -> np.ndarray:
    """build_schoen_invariant_reduced_basis (schoen_metric.rs:1185): [N, 8] exponents."""
    cap = 20000
    out = np.zeros(cap * 8, dtype=np.int32)
    n = lib().orc_schoen_basis(int(dx), int(dy), int(dt), out, cap)
    return out[: n * 8].reshape(n, 8)


def schoen_frames(coords: np.ndarray) -> np.ndarray:
    """schoen_affine_chart_frame (schoen_metric.rs:2202) per point: [P, 3, 8] complex."""
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    P = coords.shape[0]
    out = np.empty((P, 3, 16))
    lib().orc_schoen_frames(coords, P, out)
    return out[..., 0::2] + 1j * out[..., 1::2]


def schoen_sigma(coords, omega_sq, w, d, h):
    """compute_sigma (schoen_metric.rs:1685) for bidegree d = (dx, dy, dt): (sigma, eta [P])."""
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    P = coords.shape[0]
    eta = np.empty(P)
    s = lib().orc_schoen_sigma(coords, np.ascontiguousarray(omega_sq, dtype=np.float64),
                               np.ascontiguousarray(w, dtype=np.float64), P, int(d[0]), int(d[1]), int(d[2]),
                               np.ascontiguousarray(h.real, dtype=np.float64),
                               np.ascontiguousarray(h.imag, dtype=np.float64), eta.ctypes.data)
    return s, eta


def schoen_solve(d, n_sample: int, max_iter: int, tol: float, seed: int):
    """solve_schoen_metric (schoen_metric.rs:766) with the spec defaults (cy3_metric_unified.rs:289-320)."""
    rec = np.zeros(6)
    cap = max(8, 8 * max_iter + 8)
    sh = np.zeros(cap)
    rh = np.zeros(cap)
    n_est = int(schoen_basis(*d).shape[0])
    hr = np.zeros(n_est * n_est)
    hi = np.zeros(n_est * n_est)
    n = lib().orc_schoen_solve(int(d[0]), int(d[1]), int(d[2]), int(n_sample), int(max_iter), float(tol), int(seed),
                               rec, sh, rh, cap, hr.ctypes.data, hi.ctypes.data, hr.size)
    if n < 0:
        raise RuntimeError(f"orc_schoen_solve failed ({n})")
    N = int(rec[1])
    return dict(n_points=int(rec[0]), n_basis=N, iterations_run=int(rec[2]), sigma_fs_identity=rec[3],
                sigma_final=rec[4], final_donaldson_residual=rec[5], sigma_history=sh[:n].copy(),
                donaldson_history=rh[:n].copy(), h=(hr + 1j * hi).reshape(N, N))


def cicy_adam_refine(geom: str, d, coords, omega_sq, w, h, max_iters=50, lr=1e-3, fd_step=1e-3, tol=1e-6):
    """adam_refine_sigma_ty (ty_metric.rs:1488) / the Schoen twin: finite-difference Adam on sigma^2.
    geom "ty" (d = (k,)) or "schoen" (d = (d_x, d_y, d_t)); returns (h, sigma history)."""
    dd = np.zeros(3, dtype=np.int32)
    dd[: len(d)] = d
    hr = np.ascontiguousarray(h.real, dtype=np.float64).copy()
    hi = np.ascontiguousarray(h.imag, dtype=np.float64).copy()
    cap = max_iters + 2
    hist = np.zeros(cap)
    n = lib().orc_cicy_adam_refine(0 if geom == "ty" else 1, dd, np.ascontiguousarray(coords, dtype=np.float64),
                                   np.ascontiguousarray(omega_sq, dtype=np.float64),
                                   np.ascontiguousarray(w, dtype=np.float64), coords.shape[0], hr, hi,
                                   int(max_iters), float(lr), float(fd_step), float(tol), hist, cap)
    return hr + 1j * hi, hist[:n].copy()
