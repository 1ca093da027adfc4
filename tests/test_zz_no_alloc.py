"""The allocation-free eigensolver entry point, called through the C ABI.

rcwa_eig_noalloc serves callers that cannot allocate device memory (code
recording a CUDA graph, allocator-free real-time loops, hosts with a fixed
memory budget): its scratch is a fixed device array inside the library.  This
test checks, on two calls in a row that share that array, that its results
match the allocating rcwa_eig on the same input, that the input is left
unchanged, and that sizes beyond the fixed limit are rejected.

Kept in its own file so pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-11   # same algorithm and launch shapes as rcwa_eig: agreement to rounding


def _run_noalloc(lib, A, torch):
    b, n, _ = A.shape
    Af = np.ascontiguousarray(A.transpose(0, 2, 1))          # column-major per matrix
    A_d = torch.from_numpy(Af.view(np.float64).copy()).cuda()
    lam_d = torch.full((b * n * 2,), float("nan"), dtype=torch.float64, device="cuda")
    W_d = torch.full((b * n * n * 2,), float("nan"), dtype=torch.float64, device="cuda")
    st_d = torch.full((b,), 7, dtype=torch.int32, device="cuda")  # must be cleared by the call
    torch.cuda.synchronize()
    rc = lib.rcwa_eig_noalloc(n, b, A_d.data_ptr(), lam_d.data_ptr(), W_d.data_ptr(),
                              st_d.data_ptr(), None)
    assert rc == 0, lib.rcwa_last_error()
    torch.cuda.synchronize()
    assert np.array_equal(A_d.cpu().numpy().reshape(-1), Af.view(np.float64).reshape(-1)), "input modified"
    lam = lam_d.cpu().numpy().view(np.complex128).reshape(b, n)
    W = W_d.cpu().numpy().view(np.complex128).reshape(b, n, n).transpose(0, 2, 1)
    st = st_d.cpu().numpy()
    return lam, W, st


def test_eig_noalloc_matches_rcwa_eig_twice():
    torch = pytest.importorskip("torch")
    from rcwa_b200 import lib as L
    lib = L.load()
    ctx = L.Context(0)
    rng = np.random.default_rng(2024)
    n, b = 98, 4
    for call in range(2):     # two calls in a row on the shared scratch array
        A = rng.standard_normal((b, n, n)) + 1j * rng.standard_normal((b, n, n))
        lam_ref, W_ref, st_ref = ctx.eig(A)
        lam, W, st = _run_noalloc(lib, A, torch)
        assert not st.any() and not st_ref.any()
        scale = np.abs(lam_ref).max()
        assert np.abs(lam - lam_ref).max() <= TOL * scale, call
        assert np.abs(W - W_ref).max() <= TOL, call
        # and the pairs are eigenpairs of A
        for k in range(b):
            res = np.abs(A[k] @ W[k] - W[k] * lam[k][None, :]).max()
            assert res <= 1e-10 * np.abs(A[k]).max() * n
    ctx.close()


def test_eig_noalloc_rejects_oversize():
    from rcwa_b200 import lib as L
    lib = L.load()
    dummy = ctypes.c_void_p(16)   # never dereferenced: the size check comes first
    rc = lib.rcwa_eig_noalloc(129, 1, dummy, dummy, dummy, dummy, None)
    assert rc == L.RCWA_ERR_INVALID
    assert b"scratch" in lib.rcwa_last_error()
    rc = lib.rcwa_eig_noalloc(128, 64, dummy, dummy, dummy, dummy, None)
    assert rc == L.RCWA_ERR_INVALID
    # the documented largest batches: one more matrix no longer fits
    for n, bmax in ((32, 56), (64, 22), (98, 11), (128, 7)):
        rc = lib.rcwa_eig_noalloc(n, bmax + 1, dummy, dummy, dummy, dummy, None)
        assert rc == L.RCWA_ERR_INVALID, (n, bmax)


def test_eig_noalloc_largest_documented_batch():
    """n = 128 with the documented largest batch (7) runs and matches rcwa_eig."""
    torch = pytest.importorskip("torch")
    from rcwa_b200 import lib as L
    lib = L.load()
    ctx = L.Context(0)
    rng = np.random.default_rng(7)
    A = rng.standard_normal((7, 128, 128)) + 1j * rng.standard_normal((7, 128, 128))
    lam_ref, W_ref, st_ref = ctx.eig(A)
    lam, W, st = _run_noalloc(lib, A, torch)
    assert not st.any() and not st_ref.any()
    assert np.abs(lam - lam_ref).max() <= TOL * np.abs(lam_ref).max()
    assert np.abs(W - W_ref).max() <= TOL
    ctx.close()
