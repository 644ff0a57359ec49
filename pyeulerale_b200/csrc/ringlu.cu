// Direct resolvent: block LU of (dR/dU - shift I) over the grid's rings.
//
// A ring is one radial layer m (all N angular cells, 4N unknowns). The nine-point stencil
// couples ring m only to rings m-2..m+2, so in ring ordering the shifted Jacobian is block
// pentadiagonal with 4N x 4N super-blocks: the diagonal block is periodic block-pentadiagonal
// in the angular index (slots c, b, bb, f, ff) and the off-diagonal blocks start block
// diagonal (slots i, ii, o, oo). Block Gaussian elimination over the rings (pivoting inside
// each diagonal super-block only) factors it exactly:
//   A = Lt Ut,  Lt = I + sum L_a[m] (block (m, m-a)),  Ut = blockdiag(D_m) + sum C_b[m] (m, m+b).
// This replaces the reference's SuperLU factorisation (src/py_euler_ale/core.py:512-599)
// and is the robust path for shifts near zero, where Krylov methods with local
// preconditioners stagnate. One factorisation serves both the forward solve and the
// Hermitian-adjoint solve A^H x = b (the reference's solve_odes_wrt_states_adj solves
// (J - conj(s) I)^T x = b, which is A^H for A = J - s I).
//
// Dense super-block work uses cuSOLVER (getrf / getrs) and cuBLAS (gemm / trsm / gemv); the
// assembly from the nine-slot Jacobian, the layout permutations, the pivot application and
// the residual / refinement loop are kernels of this library. All device memory comes from
// the caller's workspace.

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/euler_b200.h"
#include "physics.cuh"

namespace eb {

int fail(int code, const char* msg);
int check_launch(const char* what);
int validate(const eb_batch* b);

namespace rl {

struct Handles {
  int device = -1;
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t solver = nullptr;
};

thread_local Handles g_handles;

int handles(cudaStream_t st, Handles*& h) {
  int dev = 0;
  cudaGetDevice(&dev);
  h = &g_handles;
  if (h->device != dev) {
    if (h->blas) cublasDestroy(h->blas);
    if (h->solver) cusolverDnDestroy(h->solver);
    h->blas = nullptr;
    h->solver = nullptr;
    if (cublasCreate(&h->blas) != CUBLAS_STATUS_SUCCESS) return fail(EB_ERR_CUDA, "cublasCreate failed");
    if (cusolverDnCreate(&h->solver) != CUSOLVER_STATUS_SUCCESS)
      return fail(EB_ERR_CUDA, "cusolverDnCreate failed");
    h->device = dev;
  }
  cublasSetStream(h->blas, st);
  cusolverDnSetStream(h->solver, st);
  return EB_OK;
}

inline size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

struct Layout {
  int M, N, K;
  size_t blk;  // bytes of one K x K complex block
  size_t off_D, off_L1, off_L2, off_C1, off_C2, off_piv, off_info, off_y, off_x, off_r, off_work;
  size_t total;
};

Layout plan(int M, int N, int lwork) {
  Layout L;
  L.M = M;
  L.N = N;
  L.K = 4 * N;
  L.blk = (size_t)L.K * L.K * sizeof(cuDoubleComplex);
  size_t o = 0;
  auto take = [&](size_t bytes) {
    size_t at = o;
    o = align_up(o + bytes);
    return at;
  };
  L.off_D = take(L.blk * M);
  L.off_L1 = take(L.blk * M);
  L.off_L2 = take(L.blk * M);
  L.off_C1 = take(L.blk * M);
  L.off_C2 = take(L.blk * M);
  L.off_piv = take(sizeof(int) * (size_t)L.K * M);
  L.off_info = take(sizeof(int) * M);
  const size_t vec = sizeof(cuDoubleComplex) * (size_t)L.K * M;
  L.off_y = take(vec);
  L.off_x = take(vec);
  L.off_r = take(vec);
  L.off_work = take(sizeof(cuDoubleComplex) * (size_t)(lwork > 0 ? lwork : 1));
  L.total = o;
  return L;
}

// Scatters the 4x4 blocks of the nine-slot Jacobian into the ring super-blocks
// (column-major K x K) and subtracts the shift on the diagonal.
__global__ void k_assemble(int M, int N, const double* J, double sr, double si,
                           cuDoubleComplex* D, cuDoubleComplex* B1, cuDoubleComplex* B2,
                           cuDoubleComplex* C1, cuDoubleComplex* C2) {
  const int64_t cells = (int64_t)M * N;
  const int K = 4 * N;
  const int64_t blk = (int64_t)K * K;
  const int64_t slot_stride = 16 * cells;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < cells * 9;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(g / cells);
    const int64_t c = g % cells;
    const int m = (int)(c % M), n = (int)(c / M);
    if (!slot_active(s, m, M)) continue;
    const double* J16 = J + slot_stride * s + 16 * c;
    const int nn = wrap(n + slot_dn(s), N);
    cuDoubleComplex* T;
    switch (s) {
      case kI: T = B1 + blk * m; break;
      case kII: T = B2 + blk * m; break;
      case kO: T = C1 + blk * m; break;
      case kOO: T = C2 + blk * m; break;
      default: T = D + blk * m; break;
    }
    for (int i = 0; i < 4; ++i)
      for (int r = 0; r < 4; ++r) {
        double v = J16[r + 4 * i];
        double w = 0.0;
        if (s == kC && r == i) {
          v -= sr;
          w = -si;
        }
        T[(int64_t)(4 * nn + i) * K + (4 * n + r)] = make_cuDoubleComplex(v, w);
      }
  }
}

// X <- X P^T for the row pivots of getrf (column interchanges in reverse order), one thread
// per row of X.
__global__ void k_col_pivots(int K, const int* ipiv, cuDoubleComplex* X) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= K) return;
  for (int k = K - 1; k >= 0; --k) {
    const int p = ipiv[k] - 1;
    if (p != k) {
      const cuDoubleComplex t = X[(int64_t)k * K + row];
      X[(int64_t)k * K + row] = X[(int64_t)p * K + row];
      X[(int64_t)p * K + row] = t;
    }
  }
}

// Reference layout (4, M, N) <-> ring layout [m][n][v].
__global__ void k_to_rings(int M, int N, const double* in, cuDoubleComplex* out) {
  const int64_t cells = (int64_t)M * N;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cells;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(c % M), n = (int)(c / M);
    for (int v = 0; v < 4; ++v)
      out[(int64_t)m * 4 * N + 4 * n + v] = make_cuDoubleComplex(in[8 * c + 2 * v], in[8 * c + 2 * v + 1]);
  }
}
__global__ void k_from_rings(int M, int N, const cuDoubleComplex* in, double* out, int add) {
  const int64_t cells = (int64_t)M * N;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cells;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(c % M), n = (int)(c / M);
    for (int v = 0; v < 4; ++v) {
      const cuDoubleComplex z = in[(int64_t)m * 4 * N + 4 * n + v];
      if (add) {
        out[8 * c + 2 * v] += z.x;
        out[8 * c + 2 * v + 1] += z.y;
      } else {
        out[8 * c + 2 * v] = z.x;
        out[8 * c + 2 * v + 1] = z.y;
      }
    }
  }
}

// r = b - A x with A = J - s I (adj: A^H = J^T - conj(s) I), reference layout; also
// accumulates |r|^2 and |b|^2 into acc[0], acc[1] (caller zeroes acc).
__global__ void __launch_bounds__(128) k_residual_op(int M, int N, const double* J, double sr,
                                                     double si, int adj, const double* x,
                                                     const double* b, double* r, double* acc) {
  const int64_t cells = (int64_t)M * N;
  const int64_t slot_stride = 16 * cells;
  double rr = 0.0, bb = 0.0;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cells;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(c % M), n = (int)(c / M);
    double ar[4] = {0, 0, 0, 0}, ai[4] = {0, 0, 0, 0};
    for (int s = 0; s < 9; ++s) {
      if (!adj) {
        if (!slot_active(s, m, M)) continue;
        const double* blk = J + slot_stride * s + 16 * c;
        const int64_t j = (m + slot_dm(s)) + (int64_t)M * wrap(n + slot_dn(s), N);
        for (int i = 0; i < 4; ++i) {
          const double xr = x[8 * j + 2 * i], xi = x[8 * j + 2 * i + 1];
          for (int q = 0; q < 4; ++q) {
            ar[q] += blk[q + 4 * i] * xr;
            ai[q] += blk[q + 4 * i] * xi;
          }
        }
      } else {
        const int mc = m - slot_dm(s);
        if (mc < 0 || mc >= M || !slot_active(s, mc, M)) continue;
        const int64_t src = mc + (int64_t)M * wrap(n - slot_dn(s), N);
        const double* blk = J + slot_stride * s + 16 * src;
        for (int q = 0; q < 4; ++q) {
          const double xr = x[8 * src + 2 * q], xi = x[8 * src + 2 * q + 1];
          for (int i = 0; i < 4; ++i) {
            ar[i] += blk[q + 4 * i] * xr;
            ai[i] += blk[q + 4 * i] * xi;
          }
        }
      }
    }
    const double ssr = sr, ssi = adj ? -si : si;
    for (int q = 0; q < 4; ++q) {
      const double xr = x[8 * c + 2 * q], xi = x[8 * c + 2 * q + 1];
      const double vr = ar[q] - (ssr * xr - ssi * xi);
      const double vi = ai[q] - (ssr * xi + ssi * xr);
      const double br = b[8 * c + 2 * q], bi = b[8 * c + 2 * q + 1];
      r[8 * c + 2 * q] = br - vr;
      r[8 * c + 2 * q + 1] = bi - vi;
      rr += (br - vr) * (br - vr) + (bi - vi) * (bi - vi);
      bb += br * br + bi * bi;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    rr += __shfl_xor_sync(0xffffffffu, rr, o);
    bb += __shfl_xor_sync(0xffffffffu, bb, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(acc, rr);
    atomicAdd(acc + 1, bb);
  }
}

struct Factor {
  Layout L;
  char* base;
  cuDoubleComplex* blk(size_t off, int m) const {
    return reinterpret_cast<cuDoubleComplex*>(base + off + L.blk * (size_t)m);
  }
  int* piv(int m) const { return reinterpret_cast<int*>(base + L.off_piv) + (size_t)L.K * m; }
};

// Ring-ordered triangular solves with the stored factors, in place on ring vector y.
int ring_solve(Handles* h, const Factor& F, cuDoubleComplex* y, bool adjoint) {
  const int M = F.L.M, K = F.L.K;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
  const cuDoubleComplex mone = make_cuDoubleComplex(-1.0, 0.0);
  int* info = reinterpret_cast<int*>(F.base + F.L.off_info);
  auto vec = [&](int m) { return y + (size_t)K * m; };
  if (!adjoint) {
    for (int m = 1; m < M; ++m) {  // Lt z = b
      cublasZgemv(h->blas, CUBLAS_OP_N, K, K, &mone, F.blk(F.L.off_L1, m), K, vec(m - 1), 1, &one, vec(m), 1);
      if (m >= 2)
        cublasZgemv(h->blas, CUBLAS_OP_N, K, K, &mone, F.blk(F.L.off_L2, m), K, vec(m - 2), 1, &one, vec(m), 1);
    }
    for (int m = M - 1; m >= 0; --m) {  // Ut x = z
      if (m + 1 < M)
        cublasZgemv(h->blas, CUBLAS_OP_N, K, K, &mone, F.blk(F.L.off_C1, m), K, vec(m + 1), 1, &one, vec(m), 1);
      if (m + 2 < M)
        cublasZgemv(h->blas, CUBLAS_OP_N, K, K, &mone, F.blk(F.L.off_C2, m), K, vec(m + 2), 1, &one, vec(m), 1);
      cusolverDnZgetrs(h->solver, CUBLAS_OP_N, K, 1, F.blk(F.L.off_D, m), K, F.piv(m), vec(m), K, info + m);
    }
  } else {
    for (int m = 0; m < M; ++m) {  // Ut^H z = b
      if (m >= 1)
        cublasZgemv(h->blas, CUBLAS_OP_C, K, K, &mone, F.blk(F.L.off_C1, m - 1), K, vec(m - 1), 1, &one, vec(m), 1);
      if (m >= 2)
        cublasZgemv(h->blas, CUBLAS_OP_C, K, K, &mone, F.blk(F.L.off_C2, m - 2), K, vec(m - 2), 1, &one, vec(m), 1);
      cusolverDnZgetrs(h->solver, CUBLAS_OP_C, K, 1, F.blk(F.L.off_D, m), K, F.piv(m), vec(m), K, info + m);
    }
    for (int m = M - 1; m >= 0; --m) {  // Lt^H x = z
      if (m + 1 < M)
        cublasZgemv(h->blas, CUBLAS_OP_C, K, K, &mone, F.blk(F.L.off_L1, m + 1), K, vec(m + 1), 1, &one, vec(m), 1);
      if (m + 2 < M)
        cublasZgemv(h->blas, CUBLAS_OP_C, K, K, &mone, F.blk(F.L.off_L2, m + 2), K, vec(m + 2), 1, &one, vec(m), 1);
    }
  }
  return check_launch("ring solve");
}

inline int grid_for(int64_t n, int threads) {
  int64_t blocks = (n + threads - 1) / threads;
  if (blocks > 148 * 16) blocks = 148 * 16;
  return (int)(blocks < 1 ? 1 : blocks);
}

}  // namespace rl
}  // namespace eb

using namespace eb;
using namespace eb::rl;

extern "C" {

int64_t eb_ringlu_workspace_bytes(int M, int N) {
  if (M < 4 || N < 5) return -1;
  Handles* h = nullptr;
  if (handles(nullptr, h) != EB_OK) return -1;
  const int K = 4 * N;
  int lwork = 0;
  if (cusolverDnZgetrf_bufferSize(h->solver, K, K, nullptr, K, &lwork) != CUSOLVER_STATUS_SUCCESS)
    return -1;
  return (int64_t)plan(M, N, lwork).total;
}

int eb_ringlu_factor(const eb_batch* b, const double* J, double shift_re, double shift_im,
                     void* workspace, int64_t workspace_bytes, void* stream) {
  int rc = validate(b);
  if (rc != EB_OK) return rc;
  if (b->n_inst != 1 || b->d_table) return fail(EB_ERR_ARG, "ringlu: single instance only");
  if (!J || !workspace) return fail(EB_ERR_ARG, "ringlu: null argument");
  const int M = b->single.M, N = b->single.N, K = 4 * N;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  Handles* h = nullptr;
  if ((rc = handles(st, h)) != EB_OK) return rc;
  int lwork = 0;
  cusolverDnZgetrf_bufferSize(h->solver, K, K, nullptr, K, &lwork);
  const Layout L = plan(M, N, lwork);
  if ((int64_t)L.total > workspace_bytes) return fail(EB_ERR_ARG, "ringlu: workspace too small");
  Factor F{L, static_cast<char*>(workspace)};
  cudaMemsetAsync(F.base, 0, L.off_piv, st);  // the five block arrays
  k_assemble<<<grid_for((int64_t)M * N * 9, 256), 256, 0, st>>>(
      M, N, J, shift_re, shift_im, F.blk(L.off_D, 0), F.blk(L.off_L1, 0), F.blk(L.off_L2, 0),
      F.blk(L.off_C1, 0), F.blk(L.off_C2, 0));
  if ((rc = check_launch("ringlu assemble")) != EB_OK) return rc;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
  const cuDoubleComplex mone = make_cuDoubleComplex(-1.0, 0.0);
  int* info = reinterpret_cast<int*>(F.base + L.off_info);
  cuDoubleComplex* work = reinterpret_cast<cuDoubleComplex*>(F.base + L.off_work);
  for (int m = 0; m < M; ++m) {
    cuDoubleComplex* D = F.blk(L.off_D, m);
    if (cusolverDnZgetrf(h->solver, K, K, D, K, work, F.piv(m), info + m) != CUSOLVER_STATUS_SUCCESS)
      return fail(EB_ERR_CUDA, "ringlu: getrf failed");
    // L_a[m+a] = B_a[m+a] D_m^-1 = B U^-1 L^-1 P^T
    for (int a = 1; a <= 2; ++a) {
      if (m + a >= M) continue;
      cuDoubleComplex* X = F.blk(a == 1 ? L.off_L1 : L.off_L2, m + a);
      cublasZtrsm(h->blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N,
                  CUBLAS_DIAG_NON_UNIT, K, K, &one, D, K, X, K);
      cublasZtrsm(h->blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                  CUBLAS_DIAG_UNIT, K, K, &one, D, K, X, K);
      k_col_pivots<<<(K + 127) / 128, 128, 0, st>>>(K, F.piv(m), X);
    }
    // Schur complements of the next two rings
    if (m + 1 < M)
      cublasZgemm(h->blas, CUBLAS_OP_N, CUBLAS_OP_N, K, K, K, &mone, F.blk(L.off_L1, m + 1), K,
                  F.blk(L.off_C1, m), K, &one, F.blk(L.off_D, m + 1), K);
    if (m + 2 < M) {
      cublasZgemm(h->blas, CUBLAS_OP_N, CUBLAS_OP_N, K, K, K, &mone, F.blk(L.off_L2, m + 2), K,
                  F.blk(L.off_C2, m), K, &one, F.blk(L.off_D, m + 2), K);
      cublasZgemm(h->blas, CUBLAS_OP_N, CUBLAS_OP_N, K, K, K, &mone, F.blk(L.off_L2, m + 2), K,
                  F.blk(L.off_C1, m), K, &one, F.blk(L.off_L1, m + 2), K);
      cublasZgemm(h->blas, CUBLAS_OP_N, CUBLAS_OP_N, K, K, K, &mone, F.blk(L.off_L1, m + 1), K,
                  F.blk(L.off_C2, m), K, &one, F.blk(L.off_C1, m + 1), K);
    }
  }
  if ((rc = check_launch("ringlu factor")) != EB_OK) return rc;
  std::vector<int> hinfo(M);
  if (cudaMemcpyAsync(hinfo.data(), info, sizeof(int) * M, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return check_launch("ringlu info");
  for (int m = 0; m < M; ++m)
    if (hinfo[m] != 0) return fail(EB_ERR_NAN, "ringlu: singular ring block");
  return EB_OK;
}

int eb_ringlu_solve(const eb_batch* b, const double* J, double shift_re, double shift_im,
                    int adjoint, const void* workspace, int64_t workspace_bytes,
                    const double* rhs, double* x, double tol, int max_refine,
                    double* rel_residual, void* stream) {
  int rc = validate(b);
  if (rc != EB_OK) return rc;
  if (b->n_inst != 1 || b->d_table) return fail(EB_ERR_ARG, "ringlu: single instance only");
  if (!J || !workspace || !rhs || !x) return fail(EB_ERR_ARG, "ringlu: null argument");
  const int M = b->single.M, N = b->single.N, K = 4 * N;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  Handles* h = nullptr;
  if ((rc = handles(st, h)) != EB_OK) return rc;
  int lwork = 0;
  cusolverDnZgetrf_bufferSize(h->solver, K, K, nullptr, K, &lwork);
  const Layout L = plan(M, N, lwork);
  if ((int64_t)L.total > workspace_bytes) return fail(EB_ERR_ARG, "ringlu: workspace too small");
  Factor F{L, static_cast<char*>(const_cast<void*>(workspace))};
  cuDoubleComplex* y = reinterpret_cast<cuDoubleComplex*>(F.base + L.off_y);
  double* r = reinterpret_cast<double*>(F.base + L.off_r);
  double* acc = reinterpret_cast<double*>(F.base + L.off_x);  // two doubles of scratch
  const int gc = grid_for((int64_t)M * N, 128);
  // x = A^-1 b, then refine x += A^-1 (b - A x) until the relative residual reaches tol
  k_to_rings<<<gc, 128, 0, st>>>(M, N, rhs, y);
  if ((rc = ring_solve(h, F, y, adjoint != 0)) != EB_OK) return rc;
  k_from_rings<<<gc, 128, 0, st>>>(M, N, y, x, 0);
  double rel = INFINITY;
  for (int it = 0;; ++it) {
    cudaMemsetAsync(acc, 0, 2 * sizeof(double), st);
    k_residual_op<<<gc, 128, 0, st>>>(M, N, J, shift_re, shift_im, adjoint, x, rhs, r, acc);
    double hacc[2];
    if (cudaMemcpyAsync(hacc, acc, sizeof(hacc), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return check_launch("ringlu residual");
    rel = hacc[1] > 0 ? std::sqrt(hacc[0] / hacc[1]) : std::sqrt(hacc[0]);
    if (!std::isfinite(rel)) {
      if (rel_residual) *rel_residual = rel;
      return fail(EB_ERR_NAN, "ringlu: non-finite residual");
    }
    if (rel <= tol || it >= max_refine) break;
    k_to_rings<<<gc, 128, 0, st>>>(M, N, r, y);
    if ((rc = ring_solve(h, F, y, adjoint != 0)) != EB_OK) return rc;
    k_from_rings<<<gc, 128, 0, st>>>(M, N, y, x, 1);
  }
  if (rel_residual) *rel_residual = rel;
  if (rel > tol) return fail(EB_ERR_NOCONV, "ringlu: refinement did not reach the tolerance");
  return check_launch("ringlu solve");
}

}  // extern "C"
