// Dense complex double products of the ring-block LU (dense.cu): the library's own strided-batched
// GEMM on the FP64 tensor cores and matrix-vector products, in place of a BLAS library.
#pragma once

#include <cuComplex.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace eb {
namespace dense {

// GEMM kernel variants (identical results): register-staged double buffer, cp.async ring of
// three slices on 64 x 64 tiles, cp.async ring of two slices on 64 x 32 tiles (four CTAs per SM).
constexpr int kStaged = 0, kAsync = 1, kAsyncNarrow = 2;
constexpr int kDefaultVariant = kAsyncNarrow;  // 32.5 against 26.3 TFLOP/s on 512^3 x 16

// C_z = alpha A_z B_z + beta C_z for z < batch, column-major, A_z = A + z stride_a (elements)
// etc.; alpha, beta real; beta == 0 does not read C. variant < 0 takes the default (or the one
// EB_ZGEMM=v<k> names). Returns an EB_* status.
int zgemm_nn_batched(int M, int N, int K, double alpha, const cuDoubleComplex* A, int lda,
                     int64_t stride_a, const cuDoubleComplex* B, int ldb, int64_t stride_b,
                     double beta, cuDoubleComplex* C, int ldc, int64_t stride_c, int batch,
                     cudaStream_t st, int variant = -1);

// y_z = alpha op(A_z) x_z + beta y_z for z < batch, A_z square n x n column-major (lda),
// op(A) = A (conj_trans = 0) or A^H (conj_trans = 1); alpha, beta real; beta == 0 does not
// read y. x and y contiguous; strides in elements.
int zgemv_batched(int conj_trans, int n, double alpha, const cuDoubleComplex* A, int lda,
                  int64_t stride_a, const cuDoubleComplex* x, int64_t stride_x, double beta,
                  cuDoubleComplex* y, int64_t stride_y, int batch, cudaStream_t st);

// C_z = alpha A_z B_z + beta C_z with A_z n x n and B_z, C_z n x nr (nr <= 8 right-hand
// sides), column-major; batch entry z uses A + zmap[z] stride_a (etc.; zmap == nullptr: z), and
// entries z >= *n_batch (device int; n_batch == nullptr: all) do nothing. beta == 0 does not
// read C. With bd != nullptr, C_z also takes - Bd_z V_z: Bd_z = n / 4 real column-major 4 x 4
// blocks at (const char*) bd + zmap[z] bd_stride, V_z (n x nr, leading dimension ldc) at
// V + zmap[z] stride_v. Returns an EB_* status.
int zgemm_skinny_batched(int n, int nr, double alpha, const cuDoubleComplex* A, int lda,
                         int64_t stride_a, const cuDoubleComplex* B, int ldb, int64_t stride_b,
                         double beta, cuDoubleComplex* C, int ldc, int64_t stride_c, int batch,
                         const int* zmap, const int* n_batch, cudaStream_t st,
                         const void* bd = nullptr, int64_t bd_stride = 0,
                         const cuDoubleComplex* V = nullptr, int64_t stride_v = 0);

}  // namespace dense
}  // namespace eb
