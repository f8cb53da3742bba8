"""sps_la_svd_noalloc: the allocation-free SVD entry point, through the C ABI.

Some callers cannot call cudaMalloc (code entered while another component
owns the device allocator, memory-capped embeddings, callers that must not
grow their allocator's pool).  This entry point takes the caller's device
buffers and keeps its scratch in a fixed file-scope device array.  The test
checks it against the allocating entry point sps_la_svd on two calls in a
row (the shared array keeps the previous call's contents), within the SVD
tolerance of the linear-algebra tests.  It passes alone or after the other
tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _call(lib, torch, a_np):
    m, n = a_np.shape
    k = min(m, n)
    dev = torch.device("cuda:0")
    a = torch.from_numpy(np.asfortranarray(a_np).T.copy()).to(dev)      # row-major (n, m) == column-major (m, n)
    u = torch.zeros((k, m), dtype=torch.float64, device=dev)            # column-major (m, k)
    s = torch.zeros(k, dtype=torch.float64, device=dev)
    vt = torch.zeros((n, k), dtype=torch.float64, device=dev)           # column-major (k, n)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.sps_la_svd_noalloc(0, C.c_void_p(stream), m, n, C.c_void_p(a.data_ptr()), C.c_void_p(u.data_ptr()),
                                C.c_void_p(s.data_ptr()), C.c_void_p(vt.data_ptr()))
    assert rc == 0, rc
    return u.cpu().numpy().T, s.cpu().numpy(), vt.cpu().numpy().T


@pytest.mark.parametrize("m,n", [(120, 90), (64, 128), (256, 128), (31, 31)])
def test_noalloc_svd_matches_allocating_entry_point(sps, m, n):
    import torch
    lib = sps._lib.load()
    eng = sps.Engine(2, 2)
    rng = np.random.default_rng(11 * m + n)
    for call in range(2):
        a = rng.standard_normal((m, n)) * np.exp(-0.05 * np.arange(n))[None, :]
        u, s, vt = _call(lib, torch, a)
        u0, s0, vt0, _, _ = eng.la_svd(a)
        np.testing.assert_allclose(s, s0, rtol=TOL, atol=TOL * s0[0])
        np.testing.assert_allclose((u * s) @ vt, a, atol=TOL * s0[0])
        # singular vectors agree with the allocating entry point up to sign
        np.testing.assert_allclose(np.abs(np.sum(u * u0, axis=0)), 1.0, atol=1e-9)
        k = min(m, n)
        np.testing.assert_allclose(u.T @ u, np.eye(k), atol=TOL)


@pytest.mark.parametrize("m,n,r", [(100, 60, 20), (40, 90, 7), (50, 50, 0)])
def test_noalloc_svd_rank_deficient(sps, m, n, r):
    """Rank r < min(m, n) (r = 0: the zero matrix): the singular values match
    numpy.linalg.svd, zero values stay zero, and both factors are still
    orthonormal (the columns of the zero values are completed), on two calls
    in a row."""
    import torch
    lib = sps._lib.load()
    rng = np.random.default_rng(7 * m + n + r)
    k = min(m, n)
    for call in range(2):
        a = rng.standard_normal((m, r)) @ rng.standard_normal((r, n)) if r else np.zeros((m, n))
        u, s, vt = _call(lib, torch, a)
        s_np = np.linalg.svd(a, compute_uv=False)
        scale = max(1.0, s_np[0])
        np.testing.assert_allclose(s, s_np, atol=1e-12 * scale)
        np.testing.assert_allclose((u * s) @ vt, a, atol=1e-12 * scale)
        np.testing.assert_allclose(u.T @ u, np.eye(k), atol=1e-12)
        np.testing.assert_allclose(vt @ vt.T, np.eye(k), atol=1e-12)


def test_noalloc_rejects_nonfinite_input(sps):
    """NaN or Inf in the input returns SPS_ERR_NUMERIC (3), and the next call
    on a finite matrix is unaffected."""
    import torch
    lib = sps._lib.load()
    a = np.random.default_rng(3).standard_normal((30, 20))
    for bad in (np.nan, np.inf):
        b = a.copy()
        b[4, 7] = bad
        dev = torch.device("cuda:0")
        t = torch.from_numpy(np.asfortranarray(b).T.copy()).to(dev)
        out = [torch.zeros(n, dtype=torch.float64, device=dev) for n in (30 * 20, 20, 20 * 20)]
        rc = lib.sps_la_svd_noalloc(0, None, 30, 20, C.c_void_p(t.data_ptr()), C.c_void_p(out[0].data_ptr()),
                                    C.c_void_p(out[1].data_ptr()), C.c_void_p(out[2].data_ptr()))
        assert rc == 3, rc
    u, s, vt = _call(lib, torch, a)
    np.testing.assert_allclose(s, np.linalg.svd(a, compute_uv=False), rtol=1e-12)


def test_noalloc_rejects_sizes_beyond_the_array(sps):
    lib = sps._lib.load()
    assert lib.sps_la_svd_noalloc(0, None, 300, 10, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1),
                                  C.c_void_p(1)) == 1
    assert lib.sps_la_svd_noalloc(0, None, 200, 200, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1),
                                  C.c_void_p(1)) == 1
