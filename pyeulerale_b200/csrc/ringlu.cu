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
#include <deque>
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

// One cuBLAS / cuSOLVER handle pair per concurrent stream slot (a handle's internal workspace
// must not be shared by work that overlaps on the device). A deque keeps the pointers stable.
thread_local std::deque<Handles> g_handles;

int handles(int slot, cudaStream_t st, Handles*& h) {
  int dev = 0;
  cudaGetDevice(&dev);
  while ((int)g_handles.size() <= slot) g_handles.emplace_back();
  h = &g_handles[slot];
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

// X <- X P^T for the row pivots of getrf (the column interchanges applied in reverse order).
// Each CTA first composes the interchanges into one permutation in shared memory, then moves
// a tile of `rows` rows of X through shared memory in permuted column order.
__global__ void k_col_pivots(int K, int rows, const int* ipiv, cuDoubleComplex* X) {
  extern __shared__ __align__(16) unsigned char pv_smem[];
  cuDoubleComplex* tile = reinterpret_cast<cuDoubleComplex*>(pv_smem);
  int* idx = reinterpret_cast<int*>(tile + (size_t)rows * K);
  for (int j = threadIdx.x; j < K; j += blockDim.x) idx[j] = j;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = K - 1; k >= 0; --k) {
      const int p = ipiv[k] - 1;
      if (p != k) {
        const int t = idx[k];
        idx[k] = idx[p];
        idx[p] = t;
      }
    }
  }
  const int r0 = blockIdx.x * rows;
  const int nr = min(rows, K - r0);
  for (int e = threadIdx.x; e < nr * K; e += blockDim.x) {
    const int rr = e % nr, col = e / nr;
    tile[(size_t)rr * K + col] = X[(int64_t)col * K + r0 + rr];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nr * K; e += blockDim.x) {
    const int rr = e % nr, col = e / nr;
    X[(int64_t)col * K + r0 + rr] = tile[(size_t)rr * K + idx[col]];
  }
}

// Rows per CTA of k_col_pivots: up to 8, within 200 KB of shared memory.
inline int pivot_rows(int K) {
  const size_t budget = 200 * 1024 - sizeof(int) * (size_t)K;
  const size_t per_row = sizeof(cuDoubleComplex) * (size_t)K;
  const int r = per_row > budget ? 0 : (int)(budget / per_row);
  return r > 8 ? 8 : r;
}
inline size_t pivot_smem(int K, int rows) {
  return (size_t)rows * K * sizeof(cuDoubleComplex) + sizeof(int) * (size_t)K;
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
  if (M < 4 || N < 5 || pivot_rows(4 * N) < 1) return -1;
  Handles* h = nullptr;
  if (handles(0, nullptr, h) != EB_OK) return -1;
  const int K = 4 * N;
  int lwork = 0;
  if (cusolverDnZgetrf_bufferSize(h->solver, K, K, nullptr, K, &lwork) != CUSOLVER_STATUS_SUCCESS)
    return -1;
  return (int64_t)plan(M, N, lwork).total;
}

}  // extern "C"

namespace eb {
namespace rl {

// One ring of the block elimination for one factorisation (all work on stream st).
int factor_ring(Handles* h, const Factor& f, int m, cudaStream_t st) {
  const Layout& L = f.L;
  const int M = L.M, K = L.K;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
  const cuDoubleComplex mone = make_cuDoubleComplex(-1.0, 0.0);
  int* info = reinterpret_cast<int*>(f.base + L.off_info);
  cuDoubleComplex* work = reinterpret_cast<cuDoubleComplex*>(f.base + L.off_work);
  cuDoubleComplex* D = f.blk(L.off_D, m);
  if (cusolverDnZgetrf(h->solver, K, K, D, K, work, f.piv(m), info + m) != CUSOLVER_STATUS_SUCCESS)
    return fail(EB_ERR_CUDA, "ringlu: getrf failed");
  // L_a[m+a] = B_a[m+a] D_m^-1 = B U^-1 L^-1 P^T
  for (int a = 1; a <= 2; ++a) {
    if (m + a >= M) continue;
    cuDoubleComplex* X = f.blk(a == 1 ? L.off_L1 : L.off_L2, m + a);
    cublasZtrsm(h->blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N,
                CUBLAS_DIAG_NON_UNIT, K, K, &one, D, K, X, K);
    cublasZtrsm(h->blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                CUBLAS_DIAG_UNIT, K, K, &one, D, K, X, K);
    const int rows = pivot_rows(K);
    k_col_pivots<<<(K + rows - 1) / rows, 256, pivot_smem(K, rows), st>>>(K, rows, f.piv(m), X);
  }
  // Schur complements of the next two rings
  if (m + 1 < M)
    cublasZgemm(h->blas, CUBLAS_OP_N, CUBLAS_OP_N, K, K, K, &mone, f.blk(L.off_L1, m + 1), K,
                f.blk(L.off_C1, m), K, &one, f.blk(L.off_D, m + 1), K);
  if (m + 2 < M) {
    cublasZgemm(h->blas, CUBLAS_OP_N, CUBLAS_OP_N, K, K, K, &mone, f.blk(L.off_L2, m + 2), K,
                f.blk(L.off_C2, m), K, &one, f.blk(L.off_D, m + 2), K);
    cublasZgemm(h->blas, CUBLAS_OP_N, CUBLAS_OP_N, K, K, K, &mone, f.blk(L.off_L2, m + 2), K,
                f.blk(L.off_C1, m), K, &one, f.blk(L.off_L1, m + 2), K);
    cublasZgemm(h->blas, CUBLAS_OP_N, CUBLAS_OP_N, K, K, K, &mone, f.blk(L.off_L1, m + 1), K,
                f.blk(L.off_C2, m), K, &one, f.blk(L.off_C1, m + 1), K);
  }
  return EB_OK;
}

int check_info(const Factor& f, cudaStream_t st) {
  const int M = f.L.M;
  std::vector<int> hinfo(M);
  if (cudaMemcpyAsync(hinfo.data(), f.base + f.L.off_info, sizeof(int) * M,
                      cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return check_launch("ringlu info");
  for (int m = 0; m < M; ++m)
    if (hinfo[m] != 0) return fail(EB_ERR_NAN, "ringlu: singular ring block");
  return EB_OK;
}

}  // namespace rl
}  // namespace eb

extern "C" {

int eb_ringlu_factor_many(const eb_batch* b, const double* J, int n_shifts,
                          const double* shifts, void* const* workspaces, int64_t workspace_bytes,
                          void* const* streams) {
  int rc = validate(b);
  if (rc != EB_OK) return rc;
  if (b->n_inst != 1 || b->d_table) return fail(EB_ERR_ARG, "ringlu: single instance only");
  if (!J || !workspaces || !shifts || n_shifts < 1) return fail(EB_ERR_ARG, "ringlu: null argument");
  const int M = b->single.M, N = b->single.N, K = 4 * N;
  auto stream_of = [&](int s) {
    return streams ? reinterpret_cast<cudaStream_t>(streams[s]) : (cudaStream_t) nullptr;
  };
  std::vector<Handles*> h(n_shifts);
  for (int s = 0; s < n_shifts; ++s)
    if ((rc = handles(s, stream_of(s), h[s])) != EB_OK) return rc;
  int lwork = 0;
  cusolverDnZgetrf_bufferSize(h[0]->solver, K, K, nullptr, K, &lwork);
  const Layout L = plan(M, N, lwork);
  if ((int64_t)L.total > workspace_bytes) return fail(EB_ERR_ARG, "ringlu: workspace too small");
  if (cudaFuncSetAttribute(k_col_pivots, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)pivot_smem(K, pivot_rows(K))) != cudaSuccess)
    return check_launch("ringlu pivot attribute");
  std::vector<Factor> F(n_shifts);
  for (int s = 0; s < n_shifts; ++s) {
    if (!workspaces[s]) return fail(EB_ERR_ARG, "ringlu: null workspace");
    F[s] = Factor{L, static_cast<char*>(workspaces[s])};
    cudaStream_t st = stream_of(s);
    cudaMemsetAsync(F[s].base, 0, L.off_piv, st);  // the five block arrays
    k_assemble<<<grid_for((int64_t)M * N * 9, 256), 256, 0, st>>>(
        M, N, J, shifts[2 * s], shifts[2 * s + 1], F[s].blk(L.off_D, 0), F[s].blk(L.off_L1, 0),
        F[s].blk(L.off_L2, 0), F[s].blk(L.off_C1, 0), F[s].blk(L.off_C2, 0));
  }
  if ((rc = check_launch("ringlu assemble")) != EB_OK) return rc;
  // Ring by ring; within a ring every shift's independent work goes to its own stream, so
  // the latency-bound dense steps of different shifts overlap on the GPU.
  for (int m = 0; m < M; ++m)
    for (int s = 0; s < n_shifts; ++s)
      if ((rc = factor_ring(h[s], F[s], m, stream_of(s))) != EB_OK) return rc;
  if ((rc = check_launch("ringlu factor")) != EB_OK) return rc;
  for (int s = 0; s < n_shifts; ++s)
    if ((rc = check_info(F[s], stream_of(s))) != EB_OK) return rc;
  return EB_OK;
}

int eb_ringlu_factor(const eb_batch* b, const double* J, double shift_re, double shift_im,
                     void* workspace, int64_t workspace_bytes, void* stream) {
  const double shift[2] = {shift_re, shift_im};
  void* ws[1] = {workspace};
  void* st[1] = {stream};
  return eb_ringlu_factor_many(b, J, 1, shift, ws, workspace_bytes, st);
}

int eb_ringlu_solve_many(const eb_batch* b, const double* J, int n_shifts, const double* shifts,
                         int adjoint, void* const* workspaces, int64_t workspace_bytes,
                         const double* const* rhs, double* const* x, double tol, int max_refine,
                         double* rel_residuals, void* const* streams) {
  int rc = validate(b);
  if (rc != EB_OK) return rc;
  if (b->n_inst != 1 || b->d_table) return fail(EB_ERR_ARG, "ringlu: single instance only");
  if (!J || !workspaces || !shifts || !rhs || !x || n_shifts < 1)
    return fail(EB_ERR_ARG, "ringlu: null argument");
  for (int s = 0; s < n_shifts; ++s)
    if (!workspaces[s] || !rhs[s] || !x[s]) return fail(EB_ERR_ARG, "ringlu: null argument");
  const int M = b->single.M, N = b->single.N, K = 4 * N;
  auto stream_of = [&](int s) {
    return streams ? reinterpret_cast<cudaStream_t>(streams[s]) : (cudaStream_t) nullptr;
  };
  std::vector<Handles*> h(n_shifts);
  for (int s = 0; s < n_shifts; ++s)
    if ((rc = handles(s, stream_of(s), h[s])) != EB_OK) return rc;
  int lwork = 0;
  cusolverDnZgetrf_bufferSize(h[0]->solver, K, K, nullptr, K, &lwork);
  const Layout L = plan(M, N, lwork);
  if ((int64_t)L.total > workspace_bytes) return fail(EB_ERR_ARG, "ringlu: workspace too small");
  const int gc = grid_for((int64_t)M * N, 128);
  std::vector<Factor> F(n_shifts);
  std::vector<double> rel(n_shifts, INFINITY);
  std::vector<char> active(n_shifts, 1);
  for (int s = 0; s < n_shifts; ++s) F[s] = Factor{L, static_cast<char*>(workspaces[s])};
  auto y_of = [&](int s) { return reinterpret_cast<cuDoubleComplex*>(F[s].base + L.off_y); };
  auto r_of = [&](int s) { return reinterpret_cast<double*>(F[s].base + L.off_r); };
  // two doubles of scratch for the norms (the x ring vector is not used by the solve)
  auto acc_of = [&](int s) { return reinterpret_cast<double*>(F[s].base + L.off_x); };
  // x = A^-1 b, then refine x += A^-1 (b - A x) until the relative residual reaches tol. Every
  // pass issues the work of all unfinished shifts on their streams before reading any norm.
  for (int it = 0;; ++it) {
    int n_active = 0;
    for (int s = 0; s < n_shifts; ++s) {
      if (!active[s]) continue;
      ++n_active;
      cudaStream_t st = stream_of(s);
      k_to_rings<<<gc, 128, 0, st>>>(M, N, it == 0 ? rhs[s] : r_of(s), y_of(s));
      if ((rc = ring_solve(h[s], F[s], y_of(s), adjoint != 0)) != EB_OK) return rc;
      k_from_rings<<<gc, 128, 0, st>>>(M, N, y_of(s), x[s], it == 0 ? 0 : 1);
      cudaMemsetAsync(acc_of(s), 0, 2 * sizeof(double), st);
      k_residual_op<<<gc, 128, 0, st>>>(M, N, J, shifts[2 * s], shifts[2 * s + 1], adjoint, x[s],
                                        rhs[s], r_of(s), acc_of(s));
    }
    if (n_active == 0) break;
    if ((rc = check_launch("ringlu solve")) != EB_OK) return rc;
    for (int s = 0; s < n_shifts; ++s) {
      if (!active[s]) continue;
      double hacc[2];
      if (cudaMemcpyAsync(hacc, acc_of(s), sizeof(hacc), cudaMemcpyDeviceToHost, stream_of(s)) !=
              cudaSuccess ||
          cudaStreamSynchronize(stream_of(s)) != cudaSuccess)
        return check_launch("ringlu residual");
      rel[s] = hacc[1] > 0 ? std::sqrt(hacc[0] / hacc[1]) : std::sqrt(hacc[0]);
      if (!std::isfinite(rel[s])) {
        if (rel_residuals)
          for (int q = 0; q < n_shifts; ++q) rel_residuals[q] = rel[q];
        return fail(EB_ERR_NAN, "ringlu: non-finite residual");
      }
      if (rel[s] <= tol || it >= max_refine) active[s] = 0;
    }
  }
  if (rel_residuals)
    for (int s = 0; s < n_shifts; ++s) rel_residuals[s] = rel[s];
  for (int s = 0; s < n_shifts; ++s)
    if (rel[s] > tol) return fail(EB_ERR_NOCONV, "ringlu: refinement did not reach the tolerance");
  return EB_OK;
}

int eb_ringlu_solve(const eb_batch* b, const double* J, double shift_re, double shift_im,
                    int adjoint, const void* workspace, int64_t workspace_bytes,
                    const double* rhs, double* x, double tol, int max_refine,
                    double* rel_residual, void* stream) {
  const double shift[2] = {shift_re, shift_im};
  void* ws[1] = {const_cast<void*>(workspace)};
  const double* in[1] = {rhs};
  double* out[1] = {x};
  void* st[1] = {stream};
  return eb_ringlu_solve_many(b, J, 1, shift, adjoint, ws, workspace_bytes, in, out, tol,
                              max_refine, rel_residual, st);
}

}  // extern "C"
