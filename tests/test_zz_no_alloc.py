"""The allocation-free operator apply (sil_mag2d_apply_noalloc).

Callers that may not allocate device memory while applying the operator --
a matrix-free operator called in every iteration of another library's Krylov
loop, or code under a host framework's memory pool or cap -- use this entry
point; its scratch is a fixed device array inside the library.  The test
calls it through the C ABI and checks it against sil_mag2d_apply and against
the oracle's operator on two calls in a row (the shared array keeps the
previous call's contents, which must not leak into the next result), and
that oversized grids are refused.
This file sorts last so a run that stops at the first failure has already
run every other test."""
import ctypes

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative, the operator-parity tolerance of the other GPU tests


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_apply_matches_allocating_apply(torch):
    from similie_b200 import _native
    import similie_b200.magnetostatics as mag
    L = _native.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(2024)
    for n in (257, 96):  # two calls in a row, the second smaller than the first
        p = mag.synthetic_problem(rng, n)
        mu = torch.from_numpy(p.node_mu()).cuda()
        a = torch.from_numpy(rng.standard_normal(n * n)).cuda()
        y_ref = torch.full_like(a, float("nan"))
        y_new = torch.full_like(a, float("nan"))
        assert L.sil_mag2d_apply(stream, n, n, _ptr(mu), _ptr(a), _ptr(y_ref)) == 0
        assert L.sil_mag2d_apply_noalloc(stream, n, n, _ptr(mu), _ptr(a), _ptr(y_new)) == 0, L.sil_last_error()
        torch.cuda.synchronize()
        ref = y_ref.cpu().numpy()
        got = y_new.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got - ref)) <= TOL * np.max(np.abs(ref))
        oref = O.mag2d_apply(n, n, p.node_mu(), a.cpu().numpy())
        assert np.max(np.abs(got - oref)) <= TOL * np.max(np.abs(oref))


def test_noalloc_apply_rejects_oversized_grid(torch):
    from similie_b200 import _native
    L = _native.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = L.sil_mag2d_apply_noalloc(stream, 2048, 2048, _ptr(dummy), _ptr(dummy), _ptr(dummy))
    assert rc == 1
    assert b"exceeds" in L.sil_last_error()
