"""cy3q_sigma_noalloc: sigma computed without any device allocation by the library.

The entry point exists for callers that must not have a library allocate device memory (a process
that reserved its HBM in one arena at start-up, a fixed per-process memory budget on a shared GPU,
or a loop that cannot afford the device-wide synchronisation a cudaMalloc / cudaFree may cause).
Such a caller owns every device buffer; the library keeps its intermediates in one fixed device
array.  Here the test plays that caller: it allocates the inputs and the eta output itself (with
torch) and checks, on two calls in a row, that the result equals the allocating path (cy3q_sigma
through a solver handle) and the FP64 oracle to the parity tolerance of the FP64 tests (1e-10 relative),
and that the second call changes neither the device's free memory, nor the reserved and used bytes of
the default stream-ordered memory pool, nor torch's allocated bytes.

This file is collected last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.fixture(scope="module")
def cy():
    from papers_b200 import build as b

    b.build()
    import papers_b200

    return papers_b200


def _device_memory(dev):
    """Free device bytes, the default memory pool's reserved and used bytes, and torch's allocated bytes."""
    import torch

    free, _ = torch.cuda.mem_get_info(dev)
    pool = (None, None)
    try:
        from cuda.bindings import runtime as rt
    except ImportError:  # older cuda-python layout
        try:
            from cuda import cudart as rt
        except ImportError:
            rt = None
    if rt is not None:
        err, p = rt.cudaDeviceGetDefaultMemPool(dev.index)
        if int(err) == 0:
            vals = []
            for attr in (rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent,
                         rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent):
                e2, v = rt.cudaMemPoolGetAttribute(p, attr)
                vals.append(int(v) if int(e2) == 0 else None)
            pool = tuple(vals)
    return free, pool, torch.cuda.memory_allocated(dev)


def _call(L, k, reduced, psi, dp, dw, dlo, P, dh, deta, stream):
    sig = C.c_double(float("nan"))
    st = L.cy3q_sigma_noalloc(0, k, int(reduced), psi.real, psi.imag, dp.data_ptr(), dw.data_ptr(), dlo.data_ptr(),
                              P, dh.data_ptr(), deta.data_ptr(), C.byref(sig), stream)
    return st, sig.value


@pytest.mark.parametrize("k,psi,reduced", [(4, 0.1 + 0.2j, False), (6, 0.5, True)])
def test_sigma_noalloc_matches_sigma_twice(cy, orc, k, psi, reduced):
    import torch

    from papers_b200 import cy3q

    L = cy3q.lib()
    P = 12000
    o = orc.OracleSolver.new_with_psi_sz(k, P, 31, psi, reduced=reduced)
    g = cy.QuinticSolver.from_points(k, o.points, o.weights, o.log_omega_sq, psi=psi, reduced_basis=reduced)
    for _ in range(3):
        g.donaldson_step()
    s_ref = g.sigma()
    eta_ref = g.eta()
    h = g.h_block
    dev = torch.device("cuda", 0)
    dp = torch.from_numpy(np.ascontiguousarray(o.points)).to(dev)
    dw = torch.from_numpy(o.weights.copy()).to(dev)
    dlo = torch.from_numpy(o.log_omega_sq.copy()).to(dev)
    dh = torch.from_numpy(np.ascontiguousarray(h)).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    detas = [torch.full((P,), float("nan"), dtype=torch.float64, device=dev) for _ in range(2)]
    torch.cuda.synchronize()
    mem, out = [], []
    for call in range(2):
        out.append(_call(L, k, reduced, complex(psi), dp, dw, dlo, P, dh, detas[call], stream))
        torch.cuda.synchronize()
        mem.append(_device_memory(dev))
    o.h_block = np.ascontiguousarray(h)
    s_orc = o.sigma()
    assert s_ref == pytest.approx(s_orc, rel=TOL)
    for call, (st, sig) in enumerate(out):
        assert st == 0, cy3q._err(None)
        assert sig == pytest.approx(s_ref, rel=TOL), call
        assert sig == pytest.approx(s_orc, rel=TOL), call
        eta = detas[call].cpu().numpy()
        m = np.isfinite(eta_ref)
        assert np.array_equal(m, np.isfinite(eta)), call
        np.testing.assert_allclose(eta[m], eta_ref[m], rtol=TOL)
    # the contract itself: the second call (after the first has loaded the kernels) allocated no device
    # memory, neither from the driver nor from the stream-ordered pool nor from torch's allocator
    assert mem[1] == mem[0], mem


def test_sigma_noalloc_rejects_basis_beyond_limit(cy):
    import torch

    from papers_b200 import cy3q

    L = cy3q.lib()
    dev = torch.device("cuda", 0)
    buf = torch.zeros(64, dtype=torch.float64, device=dev)
    # k = 7 (full basis): N = 330 > 224 sections
    st, _ = _call(L, 7, False, 0j, buf, buf, buf, 4, buf, buf, None)
    assert st == cy3q.ERR_SHAPE
    assert "at most 224" in cy3q._err(None)
