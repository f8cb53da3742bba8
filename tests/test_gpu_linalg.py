"""The engine's dense factorization kernels against NumPy/LAPACK (FP64).

Householder QR (single-CTA and blocked multi-CTA) and one-sided Jacobi SVD
(single-CTA, cooperative element-pair and block variants) must reproduce the
factorizations to roundoff: A = QR with orthonormal Q, and the singular
values of LAPACK gesdd with orthonormal singular vectors.  The subspace
iteration for the leading singular triplets must reproduce LAPACK's leading
values and its rank-k truncation to roundoff.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng(sps):
    return sps.Engine(2, 2)


def graded(m, n, decay, seed):
    rng = np.random.default_rng(seed)
    u, _ = np.linalg.qr(rng.standard_normal((m, min(m, n))))
    v, _ = np.linalg.qr(rng.standard_normal((n, min(m, n))))
    s = np.exp(-decay * np.arange(min(m, n)))
    return (u * s) @ v.T


@pytest.mark.parametrize("m,n", [(40, 30), (30, 40), (200, 190), (700, 650), (648, 648), (900, 200)])
@pytest.mark.parametrize("decay", [0.0, 0.05])
def test_svd_matches_lapack(eng, m, n, decay):
    a = graded(m, n, decay, m + n) if decay else np.random.default_rng(m * n).standard_normal((m, n))
    u, s, vt, sweeps, ms = eng.la_svd(a)
    ref = np.linalg.svd(a, compute_uv=False)
    np.testing.assert_allclose(s, ref, rtol=1e-12, atol=1e-13 * ref[0])
    k = min(m, n)
    np.testing.assert_allclose(u.T @ u, np.eye(k), atol=1e-12)
    np.testing.assert_allclose(vt @ vt.T, np.eye(k), atol=1e-12)
    np.testing.assert_allclose((u * s) @ vt, a, atol=1e-12 * ref[0])


@pytest.mark.parametrize("m,n", [(50, 20), (20, 50), (2048, 128), (5000, 300), (23328, 96)])
def test_qr_matches_lapack(eng, m, n):
    a = np.random.default_rng(m + 7 * n).standard_normal((m, n))
    q, r, ms = eng.la_qr(a)
    k = min(m, n)
    np.testing.assert_allclose(q @ r, a, atol=1e-12 * np.abs(a).max() * np.sqrt(n))
    np.testing.assert_allclose(q.T @ q, np.eye(k), atol=1e-12)
    assert np.allclose(np.triu(r), r)
    rr = np.linalg.qr(a, mode="r")
    np.testing.assert_allclose(np.abs(np.diag(r)), np.abs(np.diag(rr)), rtol=1e-10)


@pytest.mark.parametrize("m,n", [(60, 40), (200, 200), (648, 648), (900, 300), (1300, 180)])
def test_left_jacobi_matches_lapack(eng, m, n):
    """The U-only Jacobi of the truncated boundary SVD (block and element-pair variants)."""
    a = graded(m, n, 0.03, 3 * m + n)
    u, s, sweeps, ms = eng.la_svd_left(a)
    ref_u, ref_s, _ = np.linalg.svd(a, full_matrices=False)
    np.testing.assert_allclose(s, ref_s, rtol=1e-11, atol=1e-13 * ref_s[0])
    np.testing.assert_allclose(u.T @ u, np.eye(n), atol=1e-10)
    top = min(n, 36)
    np.testing.assert_allclose(np.abs(np.sum(u[:, :top] * ref_u[:, :top], axis=0)), 1.0, atol=1e-9)


@pytest.mark.parametrize("m,n,k,decay", [(648, 648, 18, 0.1), (648, 648, 36, 0.1), (648, 648, 18, 0.03),
                                         (1296, 648, 18, 0.08), (500, 900, 30, 0.06), (128, 128, 8, 0.2),
                                         (2048, 2048, 32, 0.05), (333, 517, 12, 0.08), (646, 650, 18, 0.1),
                                         (101, 97, 4, 0.3)])
def test_topk_matches_lapack(eng, m, n, k, decay):
    """Leading singular triplets by block subspace iteration (truncated boundary SVD)."""
    a = graded(m, n, decay, 5 * m + n + k)
    u, s, v, iters, ms = eng.la_svd_topk(a, k)
    ref_u, ref_s, ref_vt = np.linalg.svd(a, full_matrices=False)
    np.testing.assert_allclose(s, ref_s[:k], rtol=1e-12, atol=1e-13 * ref_s[0])
    np.testing.assert_allclose(u.T @ u, np.eye(k), atol=1e-12)
    np.testing.assert_allclose(v.T @ v, np.eye(k), atol=1e-12)
    # the rank-k truncation is LAPACK's
    mine = u @ (u.T @ a)
    ref = ref_u[:, :k] @ (ref_u[:, :k].T @ a)
    assert np.linalg.norm(mine - ref) <= 1e-12 * ref_s[0]
    np.testing.assert_allclose(a @ v, u * s, atol=1e-12 * ref_s[0])
    assert 1 <= iters <= 48


@pytest.mark.parametrize("m,n,k,decay", [(648, 648, 18, 0.1), (1296, 1296, 36, 0.06), (646, 650, 18, 0.1),
                                         (333, 517, 12, 0.08), (518, 341, 20, 0.05), (2048, 2048, 32, 0.05)])
def test_topk_gram_mode_matches_lapack(eng, m, n, k, decay):
    """The zip-up splits' mode: iterate on a a^T (formed by the symmetric GEMM, split-K below about 1800
    rows, mirrored in the epilogue above), extract and test residuals on a (1e-10 relative)."""
    a = graded(m, n, decay, 11 * m + n + k)
    u, s, v, iters, ms = eng.la_svd_topk(a, k, gram=True, rtol=1e-10)
    ref_u, ref_s, _ = np.linalg.svd(a, full_matrices=False)
    np.testing.assert_allclose(s, ref_s[:k], rtol=1e-10, atol=2e-10 * ref_s[0])
    np.testing.assert_allclose(u.T @ u, np.eye(k), atol=1e-10)
    np.testing.assert_allclose(v.T @ v, np.eye(k), atol=1e-10)
    assert np.linalg.norm(a @ v - u * s, axis=0).max() <= 1e-10 * ref_s[0] * (1 + 1e-6)
    mine = u @ (u.T @ a)
    ref = ref_u[:, :k] @ (ref_u[:, :k].T @ a)
    assert np.linalg.norm(mine - ref) <= 5e-8 * ref_s[0]


@pytest.mark.parametrize("m,n,k,decay", [(648, 648, 18, 0.55), (630, 648, 18, 0.6), (1296, 1296, 36, 0.3),
                                         (648, 648, 18, 0.8)])
@pytest.mark.parametrize("gram", [True, False])
def test_topk_fast_decay_matches_lapack(eng, m, n, k, decay, gram):
    """Spectra that fall by 1e-5 to 1e-6 over the kept k values, as the boundary blocks of a purified
    state do: the oversampling columns of the iterate reach the rounding level (on a a^T already
    after two iterations), the plain Cholesky QR of the extraction meets non-positive pivots and is
    redone with the shift plus two deflating passes.  The iteration steps repeat their shifted pass
    when it leaves a column short of unit norm, so that wanted directions down to about 1e-9 of the
    largest stay in the iterate.  The kept triplets still match LAPACK."""
    a = graded(m, n, decay, 3 * m + n + k)
    u, s, v, iters, ms = eng.la_svd_topk(a, k, gram=gram, rtol=1e-10)
    ref_u, ref_s, _ = np.linalg.svd(a, full_matrices=False)
    np.testing.assert_allclose(s, ref_s[:k], rtol=1e-9, atol=1e-12 * ref_s[0])
    np.testing.assert_allclose(u.T @ u, np.eye(k), atol=1e-10)
    np.testing.assert_allclose(v.T @ v, np.eye(k), atol=1e-10)
    assert np.linalg.norm(a @ v - u * s, axis=0).max() <= 1e-10 * ref_s[0] * (1 + 1e-6)
    mine = u @ (u.T @ a)
    ref = ref_u[:, :k] @ (ref_u[:, :k].T @ a)
    assert np.linalg.norm(mine - ref) <= 1e-9 * ref_s[0]


def test_topk_rank_below_k_is_reported(eng):
    """A block of rank 10 asked for 18 triplets: the plain Cholesky QR of the extraction meets pivots
    at the rounding level and the deflating passes leave 10 columns.  On a a^T the call stops and
    runs again on a, where the extraction converges with eight zero values: status 4, which this
    entry point reports as non-convergence (the engine instead completes the eight vectors)."""
    rng = np.random.default_rng(4)
    a = rng.standard_normal((648, 10)) @ rng.standard_normal((10, 648))
    for gram in (True, False):
        with pytest.raises(Exception) as ei:
            eng.la_svd_topk(a, 18, gram=gram, rtol=1e-10)
        assert getattr(ei.value, "code", None) == 5


@pytest.mark.parametrize("ta", [False, True])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (37, 19, 5), (130, 70, 17), (648, 18, 648), (2000, 648, 648),
                                   (648, 648, 23328), (300, 200, 0)])
def test_gemm_matches_numpy(eng, ta, m, n, k):
    """The FP64 tensor-core GEMM (tiled, split-K, both operand layouts) to roundoff."""
    rng = np.random.default_rng(m + 3 * n + 7 * k + ta)
    a = rng.standard_normal((k, m) if ta else (m, k))
    b = rng.standard_normal((k, n))
    c0 = rng.standard_normal((m, n))
    c, ms = eng.la_gemm(a, b, c0, alpha=0.75, beta=-0.5, transpose_a=ta)
    ref = 0.75 * ((a.T if ta else a) @ b) - 0.5 * c0
    np.testing.assert_allclose(c, ref, atol=4e-13 * max(1, k) ** 0.5, rtol=1e-13)
