// Dense complex double products of the ring-block LU (ringlu.cu): strided-batched
// C = alpha A B + beta C (column-major, no transposes) on the FP64 tensor-core instruction
// mma.sync.m8n8k4.f64, and strided-batched matrix-vector products y = alpha op(A) x + beta y with
// op(A) = A or A^H. alpha and beta are real (the LU uses +-1 and 0 / 1).
//
// GEMM: a CTA computes a kBM x kBN tile of C for one batch entry with four warps, each a 32 x 32
// sub-tile as 4 x 4 products of 8 x 8 (m8n8k4 fragments; real and imaginary parts in separate
// accumulators: re += Ar Br - Ai Bi, im += Ar Bi + Ai Br, four real MMAs per complex product).
// The kBK-deep slices of A and B go through shared memory as separate real / imaginary planes,
// two slices in flight (the next slice's global loads are issued before the current slice's
// MMAs). Edges (sizes not multiples of the tile) load zeros and store under bounds checks.
// A second variant (kAsync) moves the slices with cp.async into a three-stage ring of shared
// buffers that keep each complex element's two parts together (one 16-byte fragment load gives
// both), with no register staging; it issues the same MMAs in the same order, so the two
// variants give identical results.

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>

#include "../../include/euler_b200.h"
#include "dense.cuh"

namespace eb {

int check_launch(const char* what);
int fail(int code, const char* msg);

namespace dense {
namespace {

constexpr int kBM = 64, kBN = 64, kBK = 16;
constexpr int kGemmThreads = 128;
// Shared-memory pitches (doubles) of the A planes [k][m] and B planes [n][k], 4 modulo 16, so
// that a warp's fragment loads (4 k x 8 m, and 8 n x 4 k) fall on distinct banks within each
// half-warp.
constexpr int kPadM = kBM + 4;
constexpr int kPadK = kBK + 4;

struct GemmSmem {
  double ar[2][kBK][kPadM], ai[2][kBK][kPadM];
  double br[2][kBN][kPadK], bi[2][kBN][kPadK];
};

// D = A B + C for one 8 x 8 x 4 FP64 tile (a: A[lane / 4][lane % 4], b: B[lane % 4][lane / 4],
// c / d: C[lane / 4][2 (lane % 4) + {0, 1}]).
// (Not volatile: the instruction has no effect beyond its outputs, so the compiler may
// interleave independent MMAs to cover their latency.)
__device__ __forceinline__ void mma884(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

// A 16-byte read-only load that the compiler keeps in program order with the other such loads,
// so that a thread's unrolled loads of a matrix are all in flight before the first is used (left
// to itself the compiler may sink each load next to its use, one DRAM latency per column).
__device__ __forceinline__ double2 ldg_inflight(const double2* p) {
  double2 v;
  asm volatile("ld.global.nc.v2.f64 {%0, %1}, [%2];\n" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}

// Global -> registers for one kBK slice: each thread holds kBM * kBK / kGemmThreads complex
// elements of A and kBK * kBN / kGemmThreads of B (zero outside the matrices).
constexpr int kAPer = kBM * kBK / kGemmThreads;  // 8
constexpr int kBPer = kBK * kBN / kGemmThreads;  // 8

__device__ __forceinline__ void load_slice(const double2* A, int lda, const double2* B, int ldb,
                                           int M, int N, int K, int m0, int n0, int k0,
                                           double2 (&ra)[kAPer], double2 (&rb)[kBPer]) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int q = 0; q < kAPer; ++q) {  // A: consecutive threads along m (columns are contiguous)
    const int e = tid + kGemmThreads * q, m = e % kBM, k = e / kBM;
    const int gm = m0 + m, gk = k0 + k;
    ra[q] = (gm < M && gk < K) ? A[gm + (int64_t)lda * gk] : make_double2(0.0, 0.0);
  }
#pragma unroll
  for (int q = 0; q < kBPer; ++q) {  // B: consecutive threads along k
    const int e = tid + kGemmThreads * q, k = e % kBK, n = e / kBK;
    const int gk = k0 + k, gn = n0 + n;
    rb[q] = (gk < K && gn < N) ? B[gk + (int64_t)ldb * gn] : make_double2(0.0, 0.0);
  }
}

__device__ __forceinline__ void store_slice(GemmSmem& S, int buf, const double2 (&ra)[kAPer],
                                            const double2 (&rb)[kBPer]) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int q = 0; q < kAPer; ++q) {
    const int e = tid + kGemmThreads * q, m = e % kBM, k = e / kBM;
    S.ar[buf][k][m] = ra[q].x;
    S.ai[buf][k][m] = ra[q].y;
  }
#pragma unroll
  for (int q = 0; q < kBPer; ++q) {
    const int e = tid + kGemmThreads * q, k = e % kBK, n = e / kBK;
    S.br[buf][n][k] = rb[q].x;
    S.bi[buf][n][k] = rb[q].y;
  }
}

__global__ void __launch_bounds__(kGemmThreads)
    k_zgemm_nn(int M, int N, int K, double alpha, const double2* A, int lda, int64_t sa,
               const double2* B, int ldb, int64_t sb, double beta, double2* C, int ldc,
               int64_t sc) {
  extern __shared__ __align__(16) unsigned char zg_smem[];
  GemmSmem& S = *reinterpret_cast<GemmSmem*>(zg_smem);
  const int64_t z = blockIdx.z;
  A += sa * z;
  B += sb * z;
  C += sc * z;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;  // the warp's 32 x 32 sub-tile
  const int fr = lane >> 2, fc = lane & 3;                 // fragment row / column indices
  double re[4][4][2], im[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) re[i][j][0] = re[i][j][1] = im[i][j][0] = im[i][j][1] = 0.0;
  double2 ra[kAPer], rb[kBPer];
  load_slice(A, lda, B, ldb, M, N, K, m0, n0, 0, ra, rb);
  store_slice(S, 0, ra, rb);
  __syncthreads();
  const int slices = (K + kBK - 1) / kBK;
  for (int s = 0; s < slices; ++s) {
    const int buf = s & 1;
    if (s + 1 < slices) load_slice(A, lda, B, ldb, M, N, K, m0, n0, (s + 1) * kBK, ra, rb);
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 4) {
      double a_r[4], a_i[4], a_n[4], b_r[4], b_i[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        a_r[i] = S.ar[buf][kk + fc][wm + 8 * i + fr];
        a_i[i] = S.ai[buf][kk + fc][wm + 8 * i + fr];
        a_n[i] = -a_i[i];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        b_r[j] = S.br[buf][wn + 8 * j + fr][kk + fc];
        b_i[j] = S.bi[buf][wn + 8 * j + fr][kk + fc];
      }
      // two rounds over the 4 x 4 tiles, so that an accumulator's two MMAs of a k-step are
      // 32 independent MMAs apart (same order of the terms per accumulator)
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          mma884(re[i][j], a_r[i], b_r[j]);
          mma884(im[i][j], a_r[i], b_i[j]);
        }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          mma884(re[i][j], a_n[i], b_i[j]);
          mma884(im[i][j], a_i[i], b_r[j]);
        }
    }
    if (s + 1 < slices) {
      store_slice(S, buf ^ 1, ra, rb);
      __syncthreads();
    }
  }
  // epilogue: C = alpha acc + beta C (beta == 0: C is not read)
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gm = m0 + wm + 8 * i + fr, gn = n0 + wn + 8 * j + 2 * fc + h;
        if (gm < M && gn < N) {
          double2* c = C + gm + (int64_t)ldc * gn;
          double2 v = make_double2(alpha * re[i][j][h], alpha * im[i][j][h]);
          if (beta != 0.0) {
            const double2 o = *c;
            v.x = fma(beta, o.x, v.x);
            v.y = fma(beta, o.y, v.y);
          }
          *c = v;
        }
      }
}

// ---- cp.async variants --------------------------------------------------------------------
// pitches in complex elements: A rows [k][m] 2 modulo 8, B rows [n][k] 4 modulo 8, so that the
// 16-byte fragment loads of each quarter-warp fall on distinct banks
constexpr int kPitchA = kBM + 2;
constexpr int kPitchB = kBK + 4;

// BN: tile columns (64: warps of 32 x 32; 32: warps of 32 x 16, half the registers and shared
// memory, four CTAs per SM, twice the tiles); Stages: slices in flight.
template <int BN, int Stages>
struct AsyncSmem {
  double2 a[Stages][kBK][kPitchA];
  double2 b[Stages][BN][kPitchB];
};

// 16-byte global -> shared copy; valid == false fills zeros (src is then not read).
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(src), "r"(n)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int Pending>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(Pending) : "memory");
}

template <int BN, int Stages>
__global__ void __launch_bounds__(kGemmThreads)
    k_zgemm_nn_async(int M, int N, int K, double alpha, const double2* A, int lda, int64_t sa,
                     const double2* B, int ldb, int64_t sb, double beta, double2* C, int ldc,
                     int64_t sc) {
  constexpr int NJ = BN / 16;                        // 8-column fragments per warp
  constexpr int kBPerT = kBK * BN / kGemmThreads;   // B elements per thread and slice
  extern __shared__ __align__(16) unsigned char zg_smem[];
  AsyncSmem<BN, Stages>& S = *reinterpret_cast<AsyncSmem<BN, Stages>*>(zg_smem);
  const int64_t z = blockIdx.z;
  A += sa * z;
  B += sb * z;
  C += sc * z;
  const int tid = threadIdx.x;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
  const int lane = tid & 31, warp = tid >> 5;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * (BN / 2);
  const int fr = lane >> 2, fc = lane & 3;
  double re[4][NJ][2], im[4][NJ][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j) re[i][j][0] = re[i][j][1] = im[i][j][0] = im[i][j][1] = 0.0;
  const int slices = (K + kBK - 1) / kBK;
  // slice s into buffer s % Stages (one commit group per call, empty past the last slice)
  auto issue = [&](int s) {
    if (s < slices) {
      const int buf = s % Stages, k0 = s * kBK;
#pragma unroll
      for (int q = 0; q < kAPer; ++q) {  // A: consecutive threads along m
        const int e = tid + kGemmThreads * q, m = e % kBM, k = e / kBM;
        const int gm = m0 + m, gk = k0 + k;
        const bool ok = gm < M && gk < K;
        cp_async16(&S.a[buf][k][m], ok ? A + gm + (int64_t)lda * gk : A, ok);
      }
#pragma unroll
      for (int q = 0; q < kBPerT; ++q) {  // B: consecutive threads along k
        const int e = tid + kGemmThreads * q, k = e % kBK, n = e / kBK;
        const int gk = k0 + k, gn = n0 + n;
        const bool ok = gk < K && gn < N;
        cp_async16(&S.b[buf][n][k], ok ? B + gk + (int64_t)ldb * gn : B, ok);
      }
    }
    cp_async_commit();
  };
#pragma unroll
  for (int s = 0; s < Stages - 1; ++s) issue(s);
  for (int s = 0; s < slices; ++s) {
    cp_async_wait<Stages - 2>();  // slice s has landed (this thread's copies)
    __syncthreads();              // ... everyone's; and slice s - 1's buffer is free
    issue(s + Stages - 1);
    const int buf = s % Stages;
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 4) {
      double2 a[4], b[NJ];
      double a_n[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        a[i] = S.a[buf][kk + fc][wm + 8 * i + fr];
        a_n[i] = -a[i].y;
      }
#pragma unroll
      for (int j = 0; j < NJ; ++j) b[j] = S.b[buf][wn + 8 * j + fr][kk + fc];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
          mma884(re[i][j], a[i].x, b[j].x);
          mma884(im[i][j], a[i].x, b[j].y);
        }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
          mma884(re[i][j], a_n[i], b[j].y);
          mma884(im[i][j], a[i].y, b[j].x);
        }
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gm = m0 + wm + 8 * i + fr, gn = n0 + wn + 8 * j + 2 * fc + h;
        if (gm < M && gn < N) {
          double2* c = C + gm + (int64_t)ldc * gn;
          double2 v = make_double2(alpha * re[i][j][h], alpha * im[i][j][h]);
          if (beta != 0.0) {
            const double2 o = *c;
            v.x = fma(beta, o.x, v.x);
            v.y = fma(beta, o.y, v.y);
          }
          *c = v;
        }
      }
}

}  // namespace

int zgemm_nn_batched(int M, int N, int K, double alpha, const cuDoubleComplex* A, int lda,
                     int64_t stride_a, const cuDoubleComplex* B, int ldb, int64_t stride_b,
                     double beta, cuDoubleComplex* C, int ldc, int64_t stride_c, int batch,
                     cudaStream_t st, int variant) {
  if (M <= 0 || N <= 0 || batch <= 0) return 0;
  if (variant < 0) {  // the default, or EB_ZGEMM=v<k> (measurements of the variants in place)
    const char* e = std::getenv("EB_ZGEMM");
    variant = (e && e[0] == 'v' && e[1] >= '0' && e[1] <= '2') ? e[1] - '0' : kDefaultVariant;
  }
  auto kernel = variant == kAsync      ? k_zgemm_nn_async<64, 3>
                : variant == kAsyncNarrow ? k_zgemm_nn_async<32, 2>
                                          : k_zgemm_nn;
  const int smem = variant == kAsync        ? (int)sizeof(AsyncSmem<64, 3>)
                   : variant == kAsyncNarrow ? (int)sizeof(AsyncSmem<32, 2>)
                                             : (int)sizeof(GemmSmem);
  const int bn = variant == kAsyncNarrow ? 32 : kBN;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
      cudaSuccess)
    return check_launch("zgemm attribute");
  const dim3 grid((M + kBM - 1) / kBM, (N + bn - 1) / bn, batch);
  kernel<<<grid, kGemmThreads, smem, st>>>(
      M, N, K, alpha, reinterpret_cast<const double2*>(A), lda, stride_a,
      reinterpret_cast<const double2*>(B), ldb, stride_b, beta, reinterpret_cast<double2*>(C),
      ldc, stride_c);
  return check_launch("zgemm");
}

namespace {

// y = alpha A x + beta y: a CTA of 256 threads takes 32 rows; thread (r, g) sums the columns
// j = g (mod 8) of row r (a warp reads 32 consecutive rows of one column), the eight partial sums
// of a row are added in a fixed order through shared memory.
__global__ void __launch_bounds__(256) k_zgemv_n(int n, double alpha, const double2* A, int lda,
                                                 int64_t sa, const double2* x, int64_t sx,
                                                 double beta, double2* y, int64_t sy) {
  __shared__ double2 part[8][32];
  const int64_t z = blockIdx.y;
  A += sa * z;
  x += sx * z;
  y += sy * z;
  const int r = threadIdx.x & 31, g = threadIdx.x >> 5;
  const int i = blockIdx.x * 32 + r;
  double sr = 0.0, si = 0.0;
  if (i < n) {
    constexpr int kUnroll = 8;  // column loads in flight per thread (ldg_inflight)
    int j = g;
    for (; j + 8 * (kUnroll - 1) < n; j += 8 * kUnroll) {
      double2 a[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) a[u] = ldg_inflight(A + i + (int64_t)lda * (j + 8 * u));
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        const double2 v = x[j + 8 * u];
        sr = fma(a[u].x, v.x, fma(-a[u].y, v.y, sr));
        si = fma(a[u].x, v.y, fma(a[u].y, v.x, si));
      }
    }
    for (; j < n; j += 8) {
      const double2 a = A[i + (int64_t)lda * j], v = x[j];
      sr = fma(a.x, v.x, fma(-a.y, v.y, sr));
      si = fma(a.x, v.y, fma(a.y, v.x, si));
    }
  }
  part[g][r] = make_double2(sr, si);
  __syncthreads();
  if (g == 0 && i < n) {
    double tr = 0.0, ti = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      tr += part[k][r].x;
      ti += part[k][r].y;
    }
    double2 out = make_double2(alpha * tr, alpha * ti);
    if (beta != 0.0) {
      out.x = fma(beta, y[i].x, out.x);
      out.y = fma(beta, y[i].y, out.y);
    }
    y[i] = out;
  }
}

// y = alpha A^H x + beta y: one warp per output j (column j of A, read by the lanes in
// consecutive rows), a fixed shuffle tree adds the lanes' partial sums.
__global__ void __launch_bounds__(256) k_zgemv_c(int n, double alpha, const double2* A, int lda,
                                                 int64_t sa, const double2* x, int64_t sx,
                                                 double beta, double2* y, int64_t sy) {
  const int64_t z = blockIdx.y;
  A += sa * z;
  x += sx * z;
  y += sy * z;
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (j >= n) return;
  const double2* col = A + (int64_t)lda * j;
  double sr = 0.0, si = 0.0;
  constexpr int kUnroll = 8;  // row loads in flight per lane (ldg_inflight)
  int i = lane;
  for (; i + 32 * (kUnroll - 1) < n; i += 32 * kUnroll) {  // conj(a) v
    double2 a[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) a[u] = ldg_inflight(col + i + 32 * u);
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const double2 v = x[i + 32 * u];
      sr = fma(a[u].x, v.x, fma(a[u].y, v.y, sr));
      si = fma(a[u].x, v.y, fma(-a[u].y, v.x, si));
    }
  }
  for (; i < n; i += 32) {
    const double2 a = col[i], v = x[i];
    sr = fma(a.x, v.x, fma(a.y, v.y, sr));
    si = fma(a.x, v.y, fma(-a.y, v.x, si));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sr += __shfl_xor_sync(0xffffffffu, sr, o);
    si += __shfl_xor_sync(0xffffffffu, si, o);
  }
  if (lane == 0) {
    double2 out = make_double2(alpha * sr, alpha * si);
    if (beta != 0.0) {
      out.x = fma(beta, y[j].x, out.x);
      out.y = fma(beta, y[j].y, out.y);
    }
    y[j] = out;
  }
}

// C = alpha A B + beta C with A n x n and B, C n x nr (nr <= kMaxRhs right-hand sides): the
// multi-right-hand-side form of k_zgemv_n (one read of A serves all nr columns). A cluster of
// kSkCluster CTAs takes 32 rows: CTA c of the cluster sums the columns of its contiguous share,
// thread (r, g) of its 256 the columns j = g (mod 8) of that share for row r and every
// right-hand side, with eight column loads in flight; the eight warps' partial sums are added
// in a fixed order in shared memory, and the cluster's leader adds the CTAs' partial sums in
// rank order through distributed shared memory and writes C. Spreading a product over the
// cluster puts eight SMs' loads in flight where one CTA per 32 rows left each SM streaming
// its 256 KB share alone. Batch entry z (grid z) uses A + zmap[z] sa etc. (zmap == nullptr: z
// itself); entries z >= *n_batch exit (the whole cluster alike). With bd != nullptr the
// epilogue also subtracts Bd V, Bd being n / 4 real 4 x 4 blocks (column-major) at
// bd + zmap[z] bd_stride bytes and V (n x nr, leading dimension ldc) at V + zmap[z] sv: the ring
// LU's block-diagonal coupling, fused into the product that precedes it.
constexpr int kMaxRhs = 8;
constexpr int kSkCluster = 8;

__global__ void __cluster_dims__(1, kSkCluster, 1) __launch_bounds__(256)
    k_zgemm_skinny(int n, int nr, double alpha, const double2* A, int lda, int64_t sa,
                   const double2* B, int ldb, int64_t sb, double beta, double2* C, int ldc,
                   int64_t sc, const int* zmap, const int* n_batch, const char* bd,
                   int64_t bd_stride, const double2* V, int64_t sv) {
  extern __shared__ __align__(16) unsigned char sk_smem[];
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  if (n_batch && (int)blockIdx.z >= *n_batch) return;  // uniform over the cluster
  const int64_t z = zmap ? zmap[blockIdx.z] : blockIdx.z;
  A += sa * z;
  B += sb * z;
  C += sc * z;
  const double* Bd = bd ? reinterpret_cast<const double*>(bd + bd_stride * z) : nullptr;
  if (V) V += sv * z;
  const int rank = (int)cluster.block_rank();
  const int share = (((n + kSkCluster - 1) / kSkCluster) + 7) / 8 * 8;  // columns per CTA
  const int j0 = rank * share, j1 = min(n, j0 + share);
  const int cols = max(j1 - j0, 0);
  double2* Bs = reinterpret_cast<double2*>(sk_smem);  // cols x nr (this CTA's rows of B)
  double2* part = Bs + (size_t)share * nr;            // 8 x 32 x nr, then the CTA's 32 x nr
  const int total = cols * nr;
  for (int e0 = 0; e0 < total; e0 += 8 * 256) {  // eight loads in flight per thread
    double2 b[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = e0 + 256 * u + (int)threadIdx.x;
      if (e < total) {
        const int q = e / cols, j = e - q * cols;
        b[u] = ldg_inflight(B + j0 + j + (int64_t)ldb * q);
      }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = e0 + 256 * u + (int)threadIdx.x;
      if (e < total) Bs[e] = b[u];
    }
  }
  __syncthreads();
  const int r = threadIdx.x & 31, g = threadIdx.x >> 5;
  const int i = blockIdx.x * 32 + r;
  double sr[kMaxRhs], si[kMaxRhs];
#pragma unroll
  for (int q = 0; q < kMaxRhs; ++q) sr[q] = si[q] = 0.0;
  if (i < n) {
    constexpr int kUnroll = 8;
    int j = g;
    for (; j + 8 * (kUnroll - 1) < cols; j += 8 * kUnroll) {
      double2 a[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u)
        a[u] = ldg_inflight(A + i + (int64_t)lda * (j0 + j + 8 * u));
#pragma unroll
      for (int u = 0; u < kUnroll; ++u)
#pragma unroll
        for (int q = 0; q < kMaxRhs; ++q) {
          if (q < nr) {
            const double2 v = Bs[j + 8 * u + cols * q];
            sr[q] = fma(a[u].x, v.x, fma(-a[u].y, v.y, sr[q]));
            si[q] = fma(a[u].x, v.y, fma(a[u].y, v.x, si[q]));
          }
        }
    }
    for (; j < cols; j += 8) {
      const double2 a = A[i + (int64_t)lda * (j0 + j)];
#pragma unroll
      for (int q = 0; q < kMaxRhs; ++q) {
        if (q < nr) {
          const double2 v = Bs[j + cols * q];
          sr[q] = fma(a.x, v.x, fma(-a.y, v.y, sr[q]));
          si[q] = fma(a.x, v.y, fma(a.y, v.x, si[q]));
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kMaxRhs; ++q)
    if (q < nr) part[(q * 8 + g) * 32 + r] = make_double2(sr[q], si[q]);
  __syncthreads();
  // the CTA's partial sums (warps in order) into part[q * 32 + r] (after the 8 x 32 x nr block)
  double2* mine = part + 8 * 32 * nr;
  for (int e = threadIdx.x; e < 32 * nr; e += 256) {
    const int q = e >> 5, rr = e & 31;
    double tr = 0.0, ti = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      tr += part[(q * 8 + k) * 32 + rr].x;
      ti += part[(q * 8 + k) * 32 + rr].y;
    }
    mine[e] = make_double2(tr, ti);
  }
  cluster.sync();  // every CTA's partial sums are visible to the leader
  if (rank == 0) {
    for (int e = threadIdx.x; e < 32 * nr; e += 256) {
      const int q = e >> 5, rr = e & 31;
      const int row = blockIdx.x * 32 + rr;
      double tr = 0.0, ti = 0.0;
      for (int c = 0; c < kSkCluster; ++c) {
        const double2* other = cluster.map_shared_rank(mine, c);
        const double2 v = other[e];
        tr += v.x;
        ti += v.y;
      }
      if (row < n) {
        double2* out = C + row + (int64_t)ldc * q;
        double2 o = make_double2(alpha * tr, alpha * ti);
        if (beta != 0.0) {
          o.x = fma(beta, out->x, o.x);
          o.y = fma(beta, out->y, o.y);
        }
        if (Bd) {  // - Bd V for row = 4 blk + rr4
          const int blk = row >> 2, rr4 = row & 3;
          const double* b = Bd + 16 * blk;
          const double2* v = V + (int64_t)ldc * q + 4 * blk;
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const double bk = b[rr4 + 4 * k];
            o.x = fma(-bk, v[k].x, o.x);
            o.y = fma(-bk, v[k].y, o.y);
          }
        }
        *out = o;
      }
    }
  }
  cluster.sync();  // the leader has read every CTA's shared memory before any exits
}

}  // namespace

int zgemv_batched(int conj_trans, int n, double alpha, const cuDoubleComplex* A, int lda,
                  int64_t stride_a, const cuDoubleComplex* x, int64_t stride_x, double beta,
                  cuDoubleComplex* y, int64_t stride_y, int batch, cudaStream_t st) {
  if (n <= 0 || batch <= 0) return 0;
  const double2* a = reinterpret_cast<const double2*>(A);
  const double2* v = reinterpret_cast<const double2*>(x);
  double2* w = reinterpret_cast<double2*>(y);
  if (conj_trans)
    k_zgemv_c<<<dim3((n + 7) / 8, batch), 256, 0, st>>>(n, alpha, a, lda, stride_a, v, stride_x,
                                                        beta, w, stride_y);
  else
    k_zgemv_n<<<dim3((n + 31) / 32, batch), 256, 0, st>>>(n, alpha, a, lda, stride_a, v,
                                                          stride_x, beta, w, stride_y);
  return check_launch("zgemv");
}

int zgemm_skinny_batched(int n, int nr, double alpha, const cuDoubleComplex* A, int lda,
                         int64_t stride_a, const cuDoubleComplex* B, int ldb, int64_t stride_b,
                         double beta, cuDoubleComplex* C, int ldc, int64_t stride_c, int batch,
                         const int* zmap, const int* n_batch, cudaStream_t st, const void* bd,
                         int64_t bd_stride, const cuDoubleComplex* V, int64_t stride_v) {
  if (bd && n % 4 != 0) return fail(EB_ERR_ARG, "zgemm_skinny: block diagonal needs n % 4 == 0");
  if (n <= 0 || batch <= 0 || nr <= 0) return 0;
  if (nr > kMaxRhs) return fail(EB_ERR_ARG, "zgemm_skinny: too many right-hand sides");
  const int share = (((n + kSkCluster - 1) / kSkCluster) + 7) / 8 * 8;
  const size_t smem = sizeof(double2) * ((size_t)share * nr + 9 * 32 * (size_t)nr);
  if (smem > 200 * 1024) return fail(EB_ERR_ARG, "zgemm_skinny: right-hand sides too large");
  if (cudaFuncSetAttribute(k_zgemm_skinny, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return check_launch("zgemm_skinny attribute");
  k_zgemm_skinny<<<dim3((n + 31) / 32, kSkCluster, batch), 256, smem, st>>>(
      n, nr, alpha, reinterpret_cast<const double2*>(A), lda, stride_a,
      reinterpret_cast<const double2*>(B), ldb, stride_b, beta, reinterpret_cast<double2*>(C),
      ldc, stride_c, zmap, n_batch, static_cast<const char*>(bd), bd_stride,
      reinterpret_cast<const double2*>(V), stride_v);
  return check_launch("zgemm_skinny");
}

}  // namespace dense
}  // namespace eb

extern "C" int eb_zgemm_strided_batched(int M, int N, int K, double alpha, const double* A,
                                        int lda, int64_t stride_a, const double* B, int ldb,
                                        int64_t stride_b, double beta, double* C, int ldc,
                                        int64_t stride_c, int batch, int variant, void* stream) {
  if (M < 0 || N < 0 || K < 0 || batch < 0 || lda < (M > 1 ? M : 1) ||
      ldb < (K > 1 ? K : 1) || ldc < (M > 1 ? M : 1) || variant < -1 || variant > 2 ||
      (M > 0 && N > 0 && batch > 0 && (!A || !B || !C)))
    return eb::fail(EB_ERR_ARG, "zgemm: bad sizes, leading dimensions, variant or pointers");
  return eb::dense::zgemm_nn_batched(
      M, N, K, alpha, reinterpret_cast<const cuDoubleComplex*>(A), lda, stride_a,
      reinterpret_cast<const cuDoubleComplex*>(B), ldb, stride_b, beta,
      reinterpret_cast<cuDoubleComplex*>(C), ldc, stride_c, batch,
      reinterpret_cast<cudaStream_t>(stream), variant);
}
