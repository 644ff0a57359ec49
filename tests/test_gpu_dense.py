"""The ring LU's dense kernels through the C ABI: the strided-batched complex GEMM (both
variants, edge sizes, alpha / beta, batch strides) against NumPy's complex products, the two
variants bit for bit against each other, and the FP64 throughput probes."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def crandn(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def zgemm(cuda, M, N, K, alpha, A, B, beta, C, variant):
    """C_z <- alpha A_z B_z + beta C_z on the device (A, B, C: (batch, rows, cols) complex,
    stored column-major per batch entry with leading dimension = rows)."""
    from pyeulerale_b200 import _lib

    def dev(a):
        # column-major per batch entry: (batch, cols, rows) row-major == (batch, rows, cols) F
        return cuda.from_numpy(np.ascontiguousarray(a.transpose(0, 2, 1)).view(np.float64)).cuda()

    dA, dB, dC = dev(A), dev(B), dev(C)
    batch = A.shape[0]
    _lib.call("eb_zgemm_strided_batched", M, N, K, alpha, dA.data_ptr(), M, M * K,
              dB.data_ptr(), K, K * N, beta, dC.data_ptr(), M, M * N, batch, variant, None)
    cuda.cuda.synchronize()
    out = dC.cpu().numpy().view(np.complex128).reshape(batch, N, M)
    return out.transpose(0, 2, 1)


@pytest.mark.parametrize("M,N,K", [(64, 64, 16), (512, 512, 512), (512, 64, 64), (100, 37, 29),
                                   (7, 5, 3), (130, 129, 131)])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.0, 1.0)])
def test_zgemm_matches_numpy_and_variants_agree(cuda, M, N, K, alpha, beta):
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    batch = 3
    A, B, C = crandn(rng, (batch, M, K)), crandn(rng, (batch, K, N)), crandn(rng, (batch, M, N))
    want = alpha * np.einsum("zmk,zkn->zmn", A, B) + beta * C
    got = [zgemm(cuda, M, N, K, alpha, A, B, beta, C, v) for v in (0, 1, 2)]
    scale = np.sqrt(K) * np.max(np.abs(want))
    for g in got:
        assert np.max(np.abs(g - want)) <= 1e-14 * scale
    np.testing.assert_array_equal(got[0], got[1])
    np.testing.assert_array_equal(got[0], got[2])
    np.testing.assert_array_equal(zgemm(cuda, M, N, K, alpha, A, B, beta, C, -1), got[1])


def test_zgemm_beta_zero_ignores_c(cuda):
    """beta == 0 does not read C (NaN there stays out of the result)."""
    rng = np.random.default_rng(5)
    A, B = crandn(rng, (2, 40, 24)), crandn(rng, (2, 24, 72))
    C = np.full((2, 40, 72), np.nan + 0j)
    for v in (0, 1, 2):
        got = zgemm(cuda, 40, 72, 24, 1.0, A, B, 0.0, C, v)
        assert np.all(np.isfinite(got))


def test_zgemm_bad_arguments_rejected(cuda):
    from pyeulerale_b200 import _lib

    t = cuda.zeros(64, dtype=cuda.float64, device="cuda")
    p = t.data_ptr()
    for args in [(4, 4, 4, 1.0, p, 3, 16, p, 4, 16, 0.0, p, 4, 16, 1, 0),   # lda < M
                 (4, 4, 4, 1.0, p, 4, 16, p, 4, 16, 0.0, p, 4, 16, 1, 3),   # variant
                 (-1, 4, 4, 1.0, p, 4, 16, p, 4, 16, 0.0, p, 4, 16, 1, 0)]:  # size
        with pytest.raises(_lib.EulerB200Error) as err:
            _lib.call("eb_zgemm_strided_batched", *args, None)
        assert err.value.code == _lib.EB_ERR_ARG


def test_fp64_probes_run(cuda):
    from pyeulerale_b200 import _lib

    sink = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    _lib.call("eb_fp64_fma_probe", 10, 2, sink.data_ptr(), None)
    _lib.call("eb_fp64_mma_probe", 10, 2, sink.data_ptr(), None)
    cuda.cuda.synchronize()
    assert sink.item() == 0.0
