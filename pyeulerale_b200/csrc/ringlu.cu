// Direct resolvent: block LU of (dR/dU - shift I) over the grid's rings, for many shifts at once.
//
// A ring is one radial layer m (all N angular cells, K = 4N unknowns). The nine-point stencil
// couples ring m only to rings m-2..m+2, so in ring ordering the shifted Jacobian is block
// pentadiagonal with K x K super-blocks: the diagonal block D_m is periodic block-pentadiagonal
// in the angular index (slots c, b, bb, f, ff), the off-diagonal blocks B1_m (slot i), B2_m
// (slot ii), C1_m (slot o) and C2_m (slot oo) start block diagonal. Block Gaussian elimination
// over the rings (pivoting inside each diagonal super-block) factors it exactly:
//   A = Lt Ut,  Lt = I + sum L_a[m] (block (m, m-a)),  Ut = blockdiag(D_m) + sum C_b[m] (m, m+b),
// with, at ring m,
//   Dinv_m = D_m^-1                      (Gauss-Jordan inversion with partial pivoting)
//   L1[m+1] = B1'[m+1] Dinv_m,  L2[m+2] = B2[m+2] Dinv_m
//   D[m+1] -= L1[m+1] C1'[m],   B1'[m+2] -= L2[m+2] C1'[m]
//   D[m+2] -= L2[m+2] C2[m],    C1'[m+1] -= L1[m+1] C2[m]
// (primes: blocks already updated by earlier rings). B2 and C2 are never updated, so they stay
// block diagonal and the products with them are block-row / block-column scalings instead of
// dense GEMMs: a ring costs one inversion and three dense complex GEMMs of order K.
// Storage per ring: Dinv_m, L1[m] and C1'[m] as dense super-blocks, B2 and C2 as their N real
// 4 x 4 diagonal blocks. L2[m+2] is only needed while ring m is eliminated (one scratch block):
// the solves apply it as B2[m+2] (Dinv_m y), one dense product with the stored inverse.
// This replaces the reference's SuperLU factorisation (src/py_euler_ale/core.py:512-599) and is
// the robust path for shifts near zero, where Krylov methods with local preconditioners
// stagnate. One factorisation serves both the forward solve and the Hermitian-adjoint solve
// A^H x = b (the reference's solve_odes_wrt_states_adj solves (J - conj(s) I)^T x = b, which
// is A^H for A = J - s I).
//
// Batching: the shifts of one call share the instance and the Jacobian; shift s has its own
// workspace at base + s * stride. Every step of the elimination is one launch for all shifts
// (grid dimension = shift), the dense GEMMs and GEMVs are the library's own strided-batched
// kernels (dense.cu: complex GEMM on the FP64 tensor cores, GEMV), so the
// launch count per ring does not grow with the number of shifts. All device memory comes from
// the caller's workspace.
//
// Gauss-Jordan inversion (blocked, nb columns per panel, implicit row pivoting): the panel
// kernel runs the nb elimination steps on the panel columns in shared memory (pivot = largest
// modulus among the rows not yet chosen; in-place storage of the transformation); the update
// kernel applies the panel's transformation to all other columns as a rank-nb update
// A[:, c] += G R[:, c], R = the panel's pivot rows, G = panel columns minus the unit vectors of
// the pivot rows. After K steps the working array W holds T P (T = product of the elementary
// transformations), and the inverse is Dinv[j, p_k] = W[p_j, k] (one permuting copy).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/euler_b200.h"
#include "dense.cuh"
#include "physics.cuh"

namespace eb {

int fail(int code, const char* msg);
int check_launch(const char* what);
int validate(const eb_batch* b);

namespace rl {

// For the lanes after the first, a stream of this library and its fork / join events.
struct Handle {
  int device = -1;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  cudaEvent_t start = nullptr;
};

// Lane 0: the caller's stream; 1: the second half of a multi-shift call; 2 and 3: the side
// streams on which the Gauss-Jordan block updates of lanes 0 and 1 run ahead of the next block.
constexpr int kLanes = 4;
thread_local Handle g_handle[kLanes];

// The stream of a lane (lane 0: the caller's stream st), created on first use per device.
int lane_stream(cudaStream_t st, cudaStream_t& out, int lane = 0) {
  if (lane == 0) {
    out = st;
    return EB_OK;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  Handle& h = g_handle[lane];
  if (h.device != dev) {
    h.stream = nullptr;  // streams and events of another device are left to that device
    h.done = nullptr;
    h.start = nullptr;
    if (cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h.done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h.start, cudaEventDisableTiming) != cudaSuccess)
      return check_launch("ringlu lane stream");
    h.device = dev;
  }
  out = h.stream;
  return EB_OK;
}

inline size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

// Panel width of the Gauss-Jordan inversion: the largest of 16, 8, 4 that divides K (= 4N) and
// keeps a thread's panel rows (K / 512 rounded up, at most 2) within 16 complex registers.
inline int panel_width(int K) {
  if (K > 1024) return 0;
  const int rows = (K + 511) / 512;
  for (int nb = 16; nb >= 4; nb /= 2)
    if (K % nb == 0 && rows * nb <= 16) return nb;
  return 0;
}

// Width of the Gauss-Jordan column blocks whose trailing update is one ZGEMM (when it divides
// K and a stream's group has at least kGjBlockMinShifts shifts; otherwise every panel updates
// the whole block itself). On the 129x129 grid (K = 512) the blocked form takes 0.175 instead
// of 0.200 ms per ring and shift with 16 shifts per group (0.180 without the look-ahead of
// invert_ring), breaks even at 4 and stays 8 % slower with one shift even with the look-ahead:
// the single shift's thin ZGEMMs and extra launches cost more than its streaming passes.
constexpr int kGjBlock = 64;
constexpr int kGjBlockMinShifts = 8;

struct Layout {
  int M, N, K;
  size_t blk;   // bytes of one K x K complex block
  size_t bdr;   // bytes of one ring's block diagonal (N real 4 x 4 blocks)
  size_t off_D, off_L1, off_C1, off_B2, off_C2, off_T, off_L2, off_Rp, off_perm, off_info,
      off_acc, off_shift;
  size_t off_y, off_x, off_r, off_w;
  size_t total;
};

Layout plan(int M, int N) {
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
  L.bdr = sizeof(double) * 16 * (size_t)N;
  L.off_D = take(L.blk * M);
  L.off_L1 = take(L.blk * M);
  L.off_C1 = take(L.blk * M);
  L.off_B2 = take(L.bdr * M);
  L.off_C2 = take(L.bdr * M);
  L.off_T = take(L.blk);
  L.off_L2 = take(L.blk);
  L.off_Rp = take(sizeof(cuDoubleComplex) * (size_t)kGjBlock * L.K);
  L.off_perm = take(sizeof(int) * (size_t)L.K);
  L.off_info = take(sizeof(int) * 4);
  L.off_acc = take(sizeof(double) * 2);
  L.off_shift = take(sizeof(double) * 2);
  const size_t vec = sizeof(cuDoubleComplex) * (size_t)L.K * M;
  L.off_y = take(vec);
  L.off_x = take(vec);
  L.off_r = take(vec);
  L.off_w = take(vec);
  L.total = o;
  return L;
}

// Scatters the 4x4 blocks of the nine-slot Jacobian into the ring super-blocks
// (column-major K x K) and subtracts the shift on the diagonal; the ii / oo blocks (B2, C2)
// go to the rings' block diagonals (ring m, cell n: 16 doubles at 16 (m N + n), column-major).
__global__ void k_assemble(int M, int N, const double* J, const double* shift,
                           cuDoubleComplex* D, cuDoubleComplex* B1, double* B2,
                           cuDoubleComplex* C1, double* C2) {
  const double sr = shift[0], si = shift[1];
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
    if (s == kII || s == kOO) {
      double* bd = (s == kII ? B2 : C2) + 16 * ((int64_t)m * N + n);
      for (int e = 0; e < 16; ++e) bd[e] = J16[e];
      continue;
    }
    const int nn = wrap(n + slot_dn(s), N);
    cuDoubleComplex* T;
    switch (s) {
      case kI: T = B1 + blk * m; break;
      case kO: T = C1 + blk * m; break;
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

__device__ __forceinline__ cuDoubleComplex cmul(cuDoubleComplex a, cuDoubleComplex b) {
  return make_cuDoubleComplex(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// acc + a b
__device__ __forceinline__ cuDoubleComplex cfma(cuDoubleComplex a, cuDoubleComplex b,
                                                cuDoubleComplex acc) {
  return make_cuDoubleComplex(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
}
// acc - a b
__device__ __forceinline__ cuDoubleComplex cfms(cuDoubleComplex a, cuDoubleComplex b,
                                                cuDoubleComplex acc) {
  return make_cuDoubleComplex(fma(-a.x, b.x, fma(a.y, b.y, acc.x)), fma(-a.x, b.y, fma(-a.y, b.x, acc.y)));
}

// Per-shift pointer into the workspace.
template <class T>
__device__ __forceinline__ T* at(char* ws0, int64_t stride, size_t off) {
  return reinterpret_cast<T*>(ws0 + stride * blockIdx.y + off);
}

// Gauss-Jordan panel: elimination steps j0 .. j0+NB-1 on the panel columns of the K x K block
// `in` (byte offset off_in of each shift's workspace), result written to the same columns of
// `out` (grid: 1 x n_shifts, 512 threads). Thread t keeps rows t + 512 r (r < ROWS) of the panel
// in registers. A step: every warp finds its best row among the rows not chosen yet (largest
// modulus, ties to the smaller row) and stages it in shared memory; after one barrier every
// warp reduces the warp candidates itself, so all threads know the pivot row p and its values,
// and eliminate the pivot column from their rows (row p: scaled by the pivot's inverse), which
// also yields their candidates for the next step. The staging buffers alternate between steps,
// so one barrier per step suffices. Records the pivot row of each step in perm and flags a zero
// or non-finite pivot in info[0].
// Maximum of a 64-bit key over the warp as two 32-bit warp reductions: the high words, then
// the low words of the lanes that hold the maximal high word (the exact 64-bit maximum).
__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long key) {
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned H = __reduce_max_sync(0xffffffffu, hi);
  const unsigned L = __reduce_max_sync(0xffffffffu, hi == H ? lo : 0u);
  return ((unsigned long long)H << 32) | L;
}

constexpr int kPanelThreads = 512;
constexpr int kMaxK = 1024;
template <int NB, int ROWS>
__global__ void __launch_bounds__(kPanelThreads, 1)
    k_gj_panel(int K, int j0, char* ws0, int64_t stride, size_t off_in, size_t off_out,
               size_t off_perm, size_t off_info) {
  constexpr int kWarps = kPanelThreads / 32;
  __shared__ cuDoubleComplex cand[2][kWarps][NB];
  __shared__ cuDoubleComplex cand_inv[2][kWarps];  // 1 / (the candidate's pivot value)
  __shared__ unsigned long long cand_key[2][kWarps];
  __shared__ unsigned char chosen[kMaxK];
  const cuDoubleComplex* in = at<cuDoubleComplex>(ws0, stride, off_in);
  cuDoubleComplex* out = at<cuDoubleComplex>(ws0, stride, off_out);
  int* perm = at<int>(ws0, stride, off_perm);
  int* info = at<int>(ws0, stride, off_info);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (*info != 0) return;  // an earlier panel met a singular pivot
  for (int i = tid; i < K; i += kPanelThreads) chosen[i] = 0;
  __syncthreads();
  for (int j = tid; j < j0; j += kPanelThreads) {
    const int pj = perm[j];
    if (pj >= 0 && pj < K) chosen[pj] = 1;
  }
  cuDoubleComplex a[ROWS][NB];
#pragma unroll
  for (int r = 0; r < ROWS; ++r) {
    const int i = tid + r * kPanelThreads;
#pragma unroll
    for (int k = 0; k < NB; ++k)
      a[r][k] = i < K ? in[(size_t)K * (j0 + k) + i] : make_cuDoubleComplex(0.0, 0.0);
  }
  __syncthreads();
  double best = -1.0;
  int bi = kMaxK;
#pragma unroll
  for (int r = 0; r < ROWS; ++r) {
    const int i = tid + r * kPanelThreads;
    if (i < K && !chosen[i]) {
      const double v = a[r][0].x * a[r][0].x + a[r][0].y * a[r][0].y;
      if (v > best) {
        best = v;
        bi = i;
      }
    }
  }
#pragma unroll 1
  for (int jj = 0; jj < NB; ++jj) {
    const int par = jj & 1;
    // Arg-max as a max of 64-bit keys: the bits of |a|^2 (>= 0, so ordered like the values)
    // with the low 10 mantissa bits replaced by 1023 - row, so equal (to 2^-42 relative) moduli
    // go to the smaller row; 0 is "no candidate".
    unsigned long long key =
        bi < kMaxK ? (((unsigned long long)__double_as_longlong(best) & ~0x3FFull) |
                      (unsigned long long)(kMaxK - 1 - bi))
                   : 0ull;
    const unsigned long long mine = key;
    // the reciprocal of this thread's candidate pivot, formed while the arg-max runs (the
    // winner stages it with its row, which takes the division off the step's critical path)
    cuDoubleComplex cinv = make_cuDoubleComplex(0.0, 0.0);
    if (bi < kMaxK) {
      cuDoubleComplex c0 = a[0][0];
#pragma unroll
      for (int r = 1; r < ROWS; ++r)
        if (bi == tid + r * kPanelThreads) c0 = a[r][0];
      const double d = 1.0 / (c0.x * c0.x + c0.y * c0.y);
      cinv = make_cuDoubleComplex(c0.x * d, -c0.y * d);
    }
    key = warp_max_u64(key);
    if (key != 0ull && mine == key) {  // this thread owns the warp's best row: stage it
      const int wi = kMaxK - 1 - (int)(key & 0x3FFull);
#pragma unroll
      for (int r = 0; r < ROWS; ++r)
        if (wi == tid + r * kPanelThreads) {
#pragma unroll
          for (int k = 0; k < NB; ++k) cand[par][warp][k] = a[r][k];
        }
      cand_inv[par][warp] = cinv;
    }
    if (lane == 0) cand_key[par][warp] = key;
    __syncthreads();
    const unsigned long long kb = warp_max_u64(lane < kWarps ? cand_key[par][lane] : 0ull);
    const int p = kMaxK - 1 - (int)(kb & 0x3FFull);
    const int w = (p % kPanelThreads) / 32;  // the warp of the thread that owns row p
    const double v = __longlong_as_double((long long)(kb & ~0x3FFull));
    if (!(kb != 0ull && v > 0.0 && v <= 1.7e308 && p < K)) {  // the same decision in every thread
      if (tid == 0) atomicExch(info, 1);
      return;
    }
    if (tid == 0) {
      perm[j0 + jj] = p;
      chosen[p] = 1;
    }
    // Each row is kept rotated by jj columns: the pivot column of this step is a[.][0] and the
    // next one a[.][1]; after the elimination the row rotates by one more column, so after NB
    // steps it is back in order. The staged pivot row is rotated the same way.
    const cuDoubleComplex* prow = cand[par][w];
    const cuDoubleComplex inv = cand_inv[par][w];
    best = -1.0;
    bi = kMaxK;
#pragma unroll
    for (int r = 0; r < ROWS; ++r) {
      const int i = tid + r * kPanelThreads;
      if (i == p) {
#pragma unroll
        for (int k = 1; k < NB; ++k) a[r][k] = cmul(a[r][k], inv);
        a[r][0] = inv;
      } else {
        const cuDoubleComplex fi = cmul(a[r][0], inv);
#pragma unroll
        for (int k = 1; k < NB; ++k) a[r][k] = cfms(fi, prow[k], a[r][k]);
        a[r][0] = make_cuDoubleComplex(-fi.x, -fi.y);
      }
      if (jj + 1 < NB && i < K && i != p && !chosen[i]) {
        const double cv = a[r][1].x * a[r][1].x + a[r][1].y * a[r][1].y;
        if (cv > best) {
          best = cv;
          bi = i;
        }
      }
      const cuDoubleComplex first = a[r][0];
#pragma unroll
      for (int k = 0; k + 1 < NB; ++k) a[r][k] = a[r][k + 1];
      a[r][NB - 1] = first;
    }
  }
#pragma unroll
  for (int r = 0; r < ROWS; ++r) {
    const int i = tid + r * kPanelThreads;
    if (i < K) {
#pragma unroll
      for (int k = 0; k < NB; ++k) out[(size_t)K * (j0 + k) + i] = a[r][k];
    }
  }
}

// Gauss-Jordan update, out of place: out[:, c] = in[:, c] + G R[:, c] for every column c of
// [c_lo, c_hi) outside the panel, where R[k, c] = in[perm[j0 + k], c] and G[:, k] =
// out[:, j0 + k] - e_{perm[j0 + k]} (the panel columns that k_gj_panel wrote). One CTA per
// 64-row x 32-column tile; a thread prefetches its 8 inputs before the rank-NB products.
// Grid: tiles x shifts.
constexpr int kUpdRowsT = 64;
constexpr int kUpdColsT = 32;
template <int NB>
__global__ void __launch_bounds__(256, 3) k_gj_update(int K, int j0, int c_lo, int c_hi,
                                                   char* ws0, int64_t stride, size_t off_in,
                                                   size_t off_out, size_t off_perm,
                                                   size_t off_info) {
  constexpr int kPer = kUpdRowsT * kUpdColsT / 256;  // outputs per thread
  constexpr int kGI = (NB * kUpdRowsT + 255) / 256, kRI = (NB * kUpdColsT + 255) / 256;
  __shared__ cuDoubleComplex G[NB][kUpdRowsT];
  __shared__ cuDoubleComplex R[NB][kUpdColsT];
  const int ctiles = (c_hi - c_lo + kUpdColsT - 1) / kUpdColsT;
  const int c0 = c_lo + (blockIdx.x % ctiles) * kUpdColsT;
  const int r0 = (blockIdx.x / ctiles) * kUpdRowsT;
  const cuDoubleComplex* in = at<cuDoubleComplex>(ws0, stride, off_in);
  cuDoubleComplex* out = at<cuDoubleComplex>(ws0, stride, off_out);
  const int* perm = at<int>(ws0, stride, off_perm);
  const int tid = threadIdx.x;
  const int r = tid % kUpdRowsT, row = r0 + r, cb = tid / kUpdRowsT;
  // All of this thread's loads first: its inputs (columns cb, cb + 4, ...), its elements of the
  // G tile (panel columns) and of the R tile (pivot rows, addressed through perm, which is
  // checked before use); then the shared-memory stores and one barrier that also agrees on
  // whether the panel was singular.
  cuDoubleComplex acc[kPer], gv[kGI], rv[kRI];
#pragma unroll
  for (int q = 0; q < kPer; ++q) {
    const int col = c0 + cb + 4 * q;
    acc[q] = row < K && col < c_hi ? in[(size_t)K * col + row] : make_cuDoubleComplex(0.0, 0.0);
  }
  int bad = *at<int>(ws0, stride, off_info) != 0;
  int pg[kGI];
#pragma unroll
  for (int q = 0; q < kGI; ++q) {
    const int e = tid + 256 * q, k = e / kUpdRowsT, rr = r0 + e % kUpdRowsT;
    gv[q] = make_cuDoubleComplex(0.0, 0.0);
    pg[q] = -1;
    if (e < NB * kUpdRowsT) {
      pg[q] = perm[j0 + k];
      if (rr < K) gv[q] = out[(size_t)K * (j0 + k) + rr];
    }
  }
#pragma unroll
  for (int q = 0; q < kRI; ++q) {
    const int e = tid + 256 * q, k = e / kUpdColsT, col = c0 + e % kUpdColsT;
    rv[q] = make_cuDoubleComplex(0.0, 0.0);
    if (e < NB * kUpdColsT) {
      const int pr = perm[j0 + k];
      if (pr < 0 || pr >= K) bad = 1;
      else if (col < c_hi) rv[q] = in[(size_t)K * col + pr];
    }
  }
#pragma unroll
  for (int q = 0; q < kGI; ++q) {
    const int e = tid + 256 * q, k = e / kUpdRowsT, x = e % kUpdRowsT;
    if (e < NB * kUpdRowsT) {
      if (r0 + x == pg[q]) gv[q].x -= 1.0;
      G[k][x] = gv[q];
    }
  }
#pragma unroll
  for (int q = 0; q < kRI; ++q) {
    const int e = tid + 256 * q;
    if (e < NB * kUpdColsT) R[e / kUpdColsT][e % kUpdColsT] = rv[q];
  }
  if (__syncthreads_or(bad)) return;  // singular block: pivots incomplete, the caller fails
  if (row >= K) return;
  // k outside the columns: one G value live at a time (few registers, more resident CTAs);
  // every output still sums k = 0 .. NB-1 in order
#pragma unroll
  for (int k = 0; k < NB; ++k) {
    const cuDoubleComplex g = G[k][r];
#pragma unroll
    for (int q = 0; q < kPer; ++q) acc[q] = cfma(g, R[k][cb + 4 * q], acc[q]);
  }
#pragma unroll
  for (int q = 0; q < kPer; ++q) {
    const int col = c0 + cb + 4 * q;
    if (col < c_hi && !(col >= j0 && col < j0 + NB)) out[(size_t)K * col + row] = acc[q];
  }
}

// Two-level Gauss-Jordan: after the panel steps of a block of BW columns [b0, b0 + BW) (pivot
// rows P = perm[b0 .. b0 + BW - 1]), every column c outside the block becomes
// W[:, c] + (W[:, block] - E_P) W[P, c]. This kernel moves the pivot rows W[P, c] of those
// columns into R (BW x K, column-major) and zeroes them in W, which turns the update into
// W[:, c] += W[:, block] R[:, c], one strided-batched ZGEMM per column range. Grid: K columns
// x shifts; skipped when a panel met a singular pivot (the factorisation then fails anyway).
__global__ void __launch_bounds__(64) k_gj_take_pivot_rows(int K, int b0, int BW, char* ws0,
                                                          int64_t stride, size_t off_W,
                                                          size_t off_R, size_t off_perm,
                                                          size_t off_info) {
  const int c = blockIdx.x;
  if (c >= b0 && c < b0 + BW) return;
  if (*at<int>(ws0, stride, off_info) != 0) return;
  cuDoubleComplex* W = at<cuDoubleComplex>(ws0, stride, off_W);
  cuDoubleComplex* R = at<cuDoubleComplex>(ws0, stride, off_R);
  const int* perm = at<int>(ws0, stride, off_perm);
  for (int k = threadIdx.x; k < BW; k += blockDim.x) {
    const int p = perm[b0 + k];
    if (p < 0 || p >= K) continue;
    R[(size_t)BW * c + k] = W[(size_t)K * c + p];
    W[(size_t)K * c + p] = make_cuDoubleComplex(0.0, 0.0);
  }
}

// Dinv[j, perm[k]] = W[perm[j], k]: the inverse from the Gauss-Jordan working array (W at
// off_W, result at off_out; grid: column groups x shifts).
__global__ void __launch_bounds__(256) k_gj_permute(int K, char* ws0, int64_t stride, size_t off_W,
                                                    size_t off_out, size_t off_perm, size_t off_info) {
  extern __shared__ int pm[];
  __shared__ int bad;
  const cuDoubleComplex* W = at<cuDoubleComplex>(ws0, stride, off_W);
  cuDoubleComplex* out = at<cuDoubleComplex>(ws0, stride, off_out);
  const int* perm = at<int>(ws0, stride, off_perm);
  if (threadIdx.x == 0) bad = *at<int>(ws0, stride, off_info);
  __syncthreads();
  for (int i = threadIdx.x; i < K; i += blockDim.x) {
    pm[i] = perm[i];
    if (pm[i] < 0 || pm[i] >= K) atomicExch(&bad, 1);
  }
  __syncthreads();
  if (bad) return;  // singular block: pivots incomplete, the caller fails
  for (int k = blockIdx.x; k < K; k += gridDim.x) {
    const cuDoubleComplex* w = W + (size_t)K * k;
    cuDoubleComplex* o = out + (size_t)K * pm[k];
    for (int j = threadIdx.x; j < K; j += blockDim.x) o[j] = w[pm[j]];
  }
}

// Block-diagonal left product: X = Bd S, Bd the N real 4 x 4 blocks at off_bd (one ring's
// block diagonal), S the K x K block at off_S, X the K x K block at off_X.
// Grid: N row blocks x shifts.
__global__ void __launch_bounds__(256) k_bd_left(int K, char* ws0, int64_t stride, size_t off_bd,
                                                 size_t off_S, size_t off_X) {
  __shared__ double bd[16];
  const double* B = at<const double>(ws0, stride, off_bd);
  const cuDoubleComplex* S = at<cuDoubleComplex>(ws0, stride, off_S);
  cuDoubleComplex* X = at<cuDoubleComplex>(ws0, stride, off_X);
  const int n = blockIdx.x;
  if (threadIdx.x < 16) bd[threadIdx.x] = B[16 * n + threadIdx.x];
  __syncthreads();
  for (int c = threadIdx.x; c < K; c += blockDim.x) {
    const cuDoubleComplex* s = S + (size_t)K * c + 4 * n;
    const cuDoubleComplex s0 = s[0], s1 = s[1], s2 = s[2], s3 = s[3];
    cuDoubleComplex* x = X + (size_t)K * c + 4 * n;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const double b0 = bd[r], b1 = bd[r + 4], b2 = bd[r + 8], b3 = bd[r + 12];
      x[r] = make_cuDoubleComplex(fma(b3, s3.x, fma(b2, s2.x, fma(b1, s1.x, b0 * s0.x))),
                                  fma(b3, s3.y, fma(b2, s2.y, fma(b1, s1.y, b0 * s0.y))));
    }
  }
}

// Block-diagonal right products: Y -= X Bd for two (X, Y) pairs selected by blockIdx.z, Bd the
// N real 4 x 4 blocks at off_bd. Grid: N column blocks x shifts x 2.
__global__ void __launch_bounds__(256) k_bd_right(int K, char* ws0, int64_t stride, size_t off_bd,
                                                  size_t off_X0, size_t off_Y0, size_t off_X1,
                                                  size_t off_Y1) {
  __shared__ double bd[16];
  const double* B = at<const double>(ws0, stride, off_bd);
  const cuDoubleComplex* X = at<cuDoubleComplex>(ws0, stride, blockIdx.z ? off_X1 : off_X0);
  cuDoubleComplex* Y = at<cuDoubleComplex>(ws0, stride, blockIdx.z ? off_Y1 : off_Y0);
  const int n = blockIdx.x;
  if (threadIdx.x < 16) bd[threadIdx.x] = B[16 * n + threadIdx.x];
  __syncthreads();
  for (int r = threadIdx.x; r < K; r += blockDim.x) {
    cuDoubleComplex x[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) x[q] = X[(size_t)K * (4 * n + q) + r];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      cuDoubleComplex* y = Y + (size_t)K * (4 * n + c) + r;
      cuDoubleComplex acc = *y;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double b = bd[q + 4 * c];
        acc.x = fma(-x[q].x, b, acc.x);
        acc.y = fma(-x[q].y, b, acc.y);
      }
      *y = acc;
    }
  }
}

// Block-diagonal vector product of the solves: out -= Bd v (trans = 0) or out -= Bd^T v
// (trans = 1; the blocks are real, so Bd^H = Bd^T), or out = -(...) when `assign` is set. Bd:
// N real 4 x 4 blocks at off_bd; v, out: K complex at off_v, off_out. Grid: blocks x shifts.
__global__ void __launch_bounds__(128) k_bd_vec(int N, char* ws0, int64_t stride, size_t off_bd,
                                                size_t off_v, size_t off_out, int trans,
                                                int assign) {
  const double* B = at<const double>(ws0, stride, off_bd);
  const cuDoubleComplex* v = at<cuDoubleComplex>(ws0, stride, off_v);
  cuDoubleComplex* out = at<cuDoubleComplex>(ws0, stride, off_out);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 4 * N; e += gridDim.x * blockDim.x) {
    const int n = e >> 2, r = e & 3;
    const double* b = B + 16 * n;
    const cuDoubleComplex* vn = v + 4 * n;
    cuDoubleComplex acc = assign ? make_cuDoubleComplex(0.0, 0.0) : out[e];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double bi = trans ? b[i + 4 * r] : b[r + 4 * i];
      acc.x = fma(-bi, vn[i].x, acc.x);
      acc.y = fma(-bi, vn[i].y, acc.y);
    }
    out[e] = acc;
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

inline int grid_for(int64_t n, int threads) {
  int64_t blocks = (n + threads - 1) / threads;
  if (blocks > 148 * 16) blocks = 148 * 16;
  return (int)(blocks < 1 ? 1 : blocks);
}

// The shifts of one call: workspace of shift s at base + s * stride.
struct Group {
  Layout L;
  char* base;
  int64_t stride;  // bytes
  int S;
  int64_t es() const { return stride / (int64_t)sizeof(cuDoubleComplex); }
  cuDoubleComplex* blk(size_t off, int m) const {
    return reinterpret_cast<cuDoubleComplex*>(base + off + L.blk * (size_t)m);
  }
  size_t boff(size_t off, int m) const { return off + L.blk * (size_t)m; }
};

int check_group(const eb_batch* b, int n_shifts, const void* ws, int64_t stride, Layout& L) {
  int rc = validate(b);
  if (rc != EB_OK) return rc;
  if (b->n_inst != 1 || b->d_table) return fail(EB_ERR_ARG, "ringlu: single instance only");
  if (n_shifts < 1 || n_shifts > 65535 || !ws) return fail(EB_ERR_ARG, "ringlu: bad shifts or workspace");
  const int M = b->single.M, N = b->single.N;
  if (M < 4 || N < 5 || panel_width(4 * N) == 0) return fail(EB_ERR_ARG, "ringlu: unsupported grid size");
  L = plan(M, N);
  if (stride < (int64_t)L.total || stride % 256 != 0)
    return fail(EB_ERR_ARG, "ringlu: workspace stride too small or not a multiple of 256");
  if (reinterpret_cast<uintptr_t>(ws) % 256 != 0) return fail(EB_ERR_ARG, "ringlu: workspace not 256-byte aligned");
  return EB_OK;
}

// Panel steps j0 .. j0 + NB - 1 (in -> out) and their update of the columns [c_lo, c_hi).
template <int NB, int ROWS>
void gj_pass(const Group& g, int j0, int c_lo, int c_hi, size_t off_in, size_t off_out,
             cudaStream_t st) {
  const int K = g.L.K;
  const int tiles = ((c_hi - c_lo + kUpdColsT - 1) / kUpdColsT) * ((K + kUpdRowsT - 1) / kUpdRowsT);
  k_gj_panel<NB, ROWS><<<dim3(1, g.S), kPanelThreads, 0, st>>>(K, j0, g.base, g.stride, off_in, off_out,
                                                               g.L.off_perm, g.L.off_info);
  k_gj_update<NB><<<dim3(tiles, g.S), 256, 0, st>>>(K, j0, c_lo, c_hi, g.base, g.stride, off_in,
                                                    off_out, g.L.off_perm, g.L.off_info);
}

void gj_pass_any(const Group& g, int nb, int rows, int j0, int c_lo, int c_hi, size_t in,
                 size_t out, cudaStream_t st) {
  if (rows == 1) {
    if (nb == 16) gj_pass<16, 1>(g, j0, c_lo, c_hi, in, out, st);
    else if (nb == 8) gj_pass<8, 1>(g, j0, c_lo, c_hi, in, out, st);
    else gj_pass<4, 1>(g, j0, c_lo, c_hi, in, out, st);
  } else {
    if (nb == 8) gj_pass<8, 2>(g, j0, c_lo, c_hi, in, out, st);
    else gj_pass<4, 2>(g, j0, c_lo, c_hi, in, out, st);
  }
}

// D_m <- D_m^-1 for every shift by Gauss-Jordan with implicit row pivoting (ping-pong between
// D_m and the scratch block T). In the blocked form the columns go in blocks of kGjBlock:
// the panels of a block update only the block's columns (an even number of passes, so the
// block ends in D_m), and the rest of D_m takes the block's combined rank-kGjBlock update as
// strided-batched ZGEMMs (tensor-core DMMA) instead of kGjBlock / nb streaming passes.
int invert_ring(const Group& g, int m, cudaStream_t st, int side_lane) {
  const Layout& L = g.L;
  const int K = L.K, nb = panel_width(K), rows = (K + kPanelThreads - 1) / kPanelThreads;
  const size_t buf[2] = {g.boff(L.off_D, m), L.off_T};
  const int passes = K / nb;
  const bool blocked = K % kGjBlock == 0 && (kGjBlock / nb) % 2 == 0 && g.S >= kGjBlockMinShifts;
  if (!blocked) {
    for (int p = 0; p < passes; ++p)
      gj_pass_any(g, nb, rows, p * nb, 0, K, buf[p & 1], buf[(p + 1) & 1], st);
  } else {
    // Look-ahead: the block's update of the next block's columns runs on st, right before the
    // next block's panels; its update of every other column runs on the side stream, under
    // those panels. st waits for the side stream before it moves the next pivot rows (which
    // reads and zeroes rows of those columns and overwrites R) and at the end.
    cudaStream_t hs = nullptr;
    int rc = lane_stream(st, hs, side_lane);
    if (rc != EB_OK) return rc;
    Handle& side = g_handle[side_lane];
    const int64_t es = g.es();
    cuDoubleComplex* W = g.blk(L.off_D, m);
    cuDoubleComplex* Rp = reinterpret_cast<cuDoubleComplex*>(g.base + L.off_Rp);
    auto update = [&](cudaStream_t hh, int c_lo, int c_hi, int b0) {
      if (c_hi <= c_lo) return EB_OK;
      return dense::zgemm_nn_batched(K, c_hi - c_lo, kGjBlock, 1.0, W + (size_t)K * b0, K, es,
                                     Rp + (size_t)kGjBlock * c_lo, kGjBlock, es, 1.0,
                                     W + (size_t)K * c_lo, K, es, g.S, hh);
    };
    bool side_busy = false;
    for (int b0 = 0; b0 < K; b0 += kGjBlock) {
      for (int q = 0; q < kGjBlock / nb; ++q)
        gj_pass_any(g, nb, rows, b0 + q * nb, b0, b0 + kGjBlock, buf[q & 1], buf[(q + 1) & 1], st);
      if (K == kGjBlock) break;
      if (side_busy && cudaStreamWaitEvent(st, side.done, 0) != cudaSuccess)
        return check_launch("ringlu side join");
      k_gj_take_pivot_rows<<<dim3(K, g.S), 64, 0, st>>>(K, b0, kGjBlock, g.base, g.stride, buf[0],
                                                        L.off_Rp, L.off_perm, L.off_info);
      const int n0 = b0 + kGjBlock, n1 = std::min(K, b0 + 2 * kGjBlock);  // the next block
      if ((rc = update(st, n0, n1, b0)) != EB_OK) return rc;
      if (cudaEventRecord(side.start, st) != cudaSuccess ||
          cudaStreamWaitEvent(side.stream, side.start, 0) != cudaSuccess)
        return check_launch("ringlu side fork");
      if ((rc = update(hs, 0, b0, b0)) != EB_OK) return rc;
      if ((rc = update(hs, n1, K, b0)) != EB_OK) return rc;
      if (cudaEventRecord(side.done, side.stream) != cudaSuccess) return check_launch("ringlu side");
      side_busy = true;
    }
    if (side_busy && cudaStreamWaitEvent(st, side.done, 0) != cudaSuccess)
      return check_launch("ringlu side join");
  }
  const size_t W = blocked ? buf[0] : buf[passes & 1];
  const size_t other = blocked ? buf[1] : buf[(passes + 1) & 1];
  k_gj_permute<<<dim3(std::min(K, 1024), g.S), 256, sizeof(int) * K, st>>>(K, g.base, g.stride, W, other,
                                                                          L.off_perm, L.off_info);
  if (other != buf[0] &&
      cudaMemcpy2DAsync(g.base + buf[0], g.stride, g.base + other, g.stride, L.blk, g.S,
                        cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return check_launch("ringlu inverse copy");
  return EB_OK;
}

// One ring of the block elimination for every shift of the group.
int factor_ring(const Group& g, int m, cudaStream_t st, int side_lane) {
  const Layout& L = g.L;
  const int M = L.M, K = L.K, N = L.N;
  const int64_t es = g.es();
  int rc = invert_ring(g, m, st, side_lane);
  if (rc != EB_OK) return rc;
  if (m + 1 < M) {
    // T = L1[m+1] = B1'[m+1] Dinv_m;  D[m+1] -= T C1'[m]
    if ((rc = dense::zgemm_nn_batched(K, K, K, 1.0, g.blk(L.off_L1, m + 1), K, es,
                                      g.blk(L.off_D, m), K, es, 0.0, g.blk(L.off_T, 0), K, es,
                                      g.S, st)) != EB_OK)
      return rc;
    if ((rc = dense::zgemm_nn_batched(K, K, K, -1.0, g.blk(L.off_T, 0), K, es,
                                      g.blk(L.off_C1, m), K, es, 1.0, g.blk(L.off_D, m + 1), K,
                                      es, g.S, st)) != EB_OK)
      return rc;
  }
  if (m + 2 < M) {
    // L2[m+2] = B2[m+2] Dinv_m (scratch);  B1'[m+2] -= L2[m+2] C1'[m]
    k_bd_left<<<dim3(N, g.S), 256, 0, st>>>(K, g.base, g.stride, L.off_B2 + L.bdr * (m + 2),
                                            g.boff(L.off_D, m), L.off_L2);
    if ((rc = dense::zgemm_nn_batched(K, K, K, -1.0, g.blk(L.off_L2, 0), K, es,
                                      g.blk(L.off_C1, m), K, es, 1.0, g.blk(L.off_L1, m + 2), K,
                                      es, g.S, st)) != EB_OK)
      return rc;
    // D[m+2] -= L2[m+2] C2[m];  C1'[m+1] -= L1[m+1] C2[m]
    k_bd_right<<<dim3(N, g.S, 2), 256, 0, st>>>(K, g.base, g.stride, L.off_C2 + L.bdr * m,
                                                L.off_L2, g.boff(L.off_D, m + 2),
                                                L.off_T, g.boff(L.off_C1, m + 1));
  }
  if (m + 1 < M &&
      cudaMemcpy2DAsync(g.blk(L.off_L1, m + 1), g.stride, g.blk(L.off_T, 0), g.stride, L.blk, g.S,
                        cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return check_launch("ringlu L1 copy");
  return EB_OK;
}

// Ring-ordered triangular solves with the stored factors for every shift: y (ring layout)
// holds the right-hand sides on entry; the solutions are left in x (w: scratch vectors).
// A = Lt Ut with L2[m] = B2[m] Dinv_{m-2}, so the forward sweep keeps w[m] = Dinv_m y[m] of the
// finished rings and subtracts B2[m] w[m-2]; the adjoint sweep applies L2[m+2]^H as
// Dinv_m^H (B2[m+2]^T x[m+2]).
int ring_solve(const Group& g, bool adjoint, cudaStream_t stream) {
  const Layout& L = g.L;
  const int M = L.M, K = L.K, N = L.N;
  const int64_t es = g.es();
  cuDoubleComplex* y = reinterpret_cast<cuDoubleComplex*>(g.base + L.off_y);
  cuDoubleComplex* x = reinterpret_cast<cuDoubleComplex*>(g.base + L.off_x);
  cuDoubleComplex* w = reinterpret_cast<cuDoubleComplex*>(g.base + L.off_w);
  auto yv = [&](int m) { return y + (size_t)K * m; };
  auto xv = [&](int m) { return x + (size_t)K * m; };
  auto wv = [&](int m) { return w + (size_t)K * m; };
  const size_t vb = sizeof(cuDoubleComplex) * (size_t)K;  // bytes of one ring vector
  const int kN = 0, kH = 1;  // op(A) = A, A^H
  auto gemv = [&](int op, double alpha, const cuDoubleComplex* A, const cuDoubleComplex* v,
                  double beta, cuDoubleComplex* out) {
    return dense::zgemv_batched(op, K, alpha, A, K, es, v, es, beta, out, es, g.S, stream);
  };
  const dim3 bdg((4 * N + 127) / 128, g.S);
  // out -= Bd v (trans: Bd^T v), ring vectors given by workspace offsets; assign: out = -Bd v
  auto bdvec = [&](size_t off_bd, size_t off_v, size_t off_out, int trans, int assign) {
    k_bd_vec<<<bdg, 128, 0, stream>>>(N, g.base, g.stride, off_bd, off_v, off_out, trans, assign);
  };
  int st = EB_OK;
  auto run = [&](int s) {
    if (s != EB_OK) st = s;
  };
  if (!adjoint) {
    for (int m = 0; m < M; ++m) {  // Lt z = b (z in y), w[m] = Dinv_m z[m]
      if (m >= 1) run(gemv(kN, -1.0, g.blk(L.off_L1, m), yv(m - 1), 1.0, yv(m)));
      if (m >= 2) bdvec(L.off_B2 + L.bdr * m, L.off_w + vb * (m - 2), L.off_y + vb * m, 0, 0);
      if (m + 2 < M) run(gemv(kN, 1.0, g.blk(L.off_D, m), yv(m), 0.0, wv(m)));
    }
    for (int m = M - 1; m >= 0; --m) {  // Ut x = z
      if (m + 1 < M) run(gemv(kN, -1.0, g.blk(L.off_C1, m), xv(m + 1), 1.0, yv(m)));
      if (m + 2 < M) bdvec(L.off_C2 + L.bdr * m, L.off_x + vb * (m + 2), L.off_y + vb * m, 0, 0);
      run(gemv(kN, 1.0, g.blk(L.off_D, m), yv(m), 0.0, xv(m)));
    }
  } else {
    for (int m = 0; m < M; ++m) {  // Ut^H z = b (z in x)
      if (m >= 1) run(gemv(kH, -1.0, g.blk(L.off_C1, m - 1), xv(m - 1), 1.0, yv(m)));
      if (m >= 2) bdvec(L.off_C2 + L.bdr * (m - 2), L.off_x + vb * (m - 2), L.off_y + vb * m, 1, 0);
      run(gemv(kH, 1.0, g.blk(L.off_D, m), yv(m), 0.0, xv(m)));
    }
    for (int m = M - 1; m >= 0; --m) {  // Lt^H x = z
      if (m + 1 < M) run(gemv(kH, -1.0, g.blk(L.off_L1, m + 1), xv(m + 1), 1.0, xv(m)));
      if (m + 2 < M) {  // x[m] -= Dinv_m^H (B2[m+2]^T x[m+2]), with w[m] = -B2[m+2]^T x[m+2]
        bdvec(L.off_B2 + L.bdr * (m + 2), L.off_x + vb * (m + 2), L.off_w + vb * m, 1, 1);
        run(gemv(kH, 1.0, g.blk(L.off_D, m), wv(m), 1.0, xv(m)));
      }
    }
  }
  if (st != EB_OK) return st;
  return check_launch("ring solve");
}

// ---- many right-hand sides per factorisation (the anchored GMRES preconditioner) ----------
//
// A set of factorised shifts ("anchors", workspace of anchor a at base + a * stride) and nr
// right-hand sides per anchor. The right-hand sides of anchor a are ring vectors stored as M ring
// blocks of K x nr (column-major, leading dimension K) at Y + a * mstride (likewise X, W). The
// launches cover the anchors zmap[0 .. *n_active - 1] (device arrays), so anchors whose systems
// have all converged drop out without a change of launch shape.

// System vectors (reference layout, system s at in + s * vstride doubles) -> column sys_col[s]
// of anchor sys_anchor[s]'s ring blocks.
__global__ void k_sys_to_multi(int M, int N, int nr, int n_sys, const int* sys_anchor,
                               const int* sys_col, const double* in, int64_t vstride,
                               cuDoubleComplex* Y, int64_t mstride) {
  const int s = blockIdx.y;
  if (s >= n_sys) return;
  const int K = 4 * N;
  const int64_t cells = (int64_t)M * N;
  const double* v = in + (int64_t)s * vstride;
  cuDoubleComplex* y = Y + (int64_t)sys_anchor[s] * mstride + (int64_t)sys_col[s] * K;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cells;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(c % M), n = (int)(c / M);
    const double2* a = reinterpret_cast<const double2*>(v + 8 * c);
    cuDoubleComplex* o = y + (int64_t)m * K * nr + 4 * n;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double2 z = a[k];
      o[k] = make_cuDoubleComplex(z.x, z.y);
    }
  }
}

// The inverse of k_sys_to_multi for the systems with active[s] (accumulate: out += ...).
__global__ void k_multi_to_sys(int M, int N, int nr, int n_sys, const int* sys_anchor,
                               const int* sys_col, const int* active,
                               const cuDoubleComplex* X, int64_t mstride, double* out,
                               int64_t vstride, int accumulate) {
  const int s = blockIdx.y;
  if (s >= n_sys || !active[s]) return;
  const int K = 4 * N;
  const int64_t cells = (int64_t)M * N;
  double* v = out + (int64_t)s * vstride;
  const cuDoubleComplex* x = X + (int64_t)sys_anchor[s] * mstride + (int64_t)sys_col[s] * K;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < cells;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(c % M), n = (int)(c / M);
    const cuDoubleComplex* i = x + (int64_t)m * K * nr + 4 * n;
    double2* o = reinterpret_cast<double2*>(v + 8 * c);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      double2 z = make_double2(i[k].x, i[k].y);
      if (accumulate) {
        const double2 w = o[k];
        z = make_double2(w.x + z.x, w.y + z.y);
      }
      o[k] = z;
    }
  }
}

// X = A^-1 Y column by column for the anchors in zmap (A = the anchor's shifted Jacobian): the
// forward sweep of ring_solve with every matrix-vector product over nr right-hand sides. Y is
// overwritten; W is scratch.
int ring_solve_multi(const Group& g, int nr, cuDoubleComplex* Y, cuDoubleComplex* X,
                     cuDoubleComplex* W, int64_t mstride, const int* zmap, const int* n_active,
                     cudaStream_t st) {
  const Layout& L = g.L;
  const int M = L.M, K = L.K;
  const int64_t es = g.es();
  auto blk = [&](cuDoubleComplex* base, int m) { return base + (size_t)K * nr * m; };
  int rc = EB_OK;
  // C = alpha A B + beta C [- Bd V: the block-diagonal coupling at off_bd, fused into the
  // product's epilogue]
  auto gemm = [&](double alpha, const cuDoubleComplex* A, const cuDoubleComplex* B, double beta,
                  cuDoubleComplex* C, size_t off_bd = 0, const cuDoubleComplex* V = nullptr) {
    if (rc == EB_OK)
      rc = dense::zgemm_skinny_batched(K, nr, alpha, A, K, es, B, K, mstride, beta, C, K,
                                       mstride, g.S, zmap, n_active, st,
                                       V ? g.base + off_bd : nullptr, g.stride, V, mstride);
  };
  for (int m = 0; m < M; ++m) {  // Lt z = b (z in Y), W[m] = Dinv_m z[m]
    if (m >= 2)
      gemm(-1.0, g.blk(L.off_L1, m), blk(Y, m - 1), 1.0, blk(Y, m), L.off_B2 + L.bdr * m,
           blk(W, m - 2));
    else if (m == 1)
      gemm(-1.0, g.blk(L.off_L1, m), blk(Y, m - 1), 1.0, blk(Y, m));
    if (m + 2 < M) gemm(1.0, g.blk(L.off_D, m), blk(Y, m), 0.0, blk(W, m));
  }
  for (int m = M - 1; m >= 0; --m) {  // Ut x = z
    if (m + 2 < M)
      gemm(-1.0, g.blk(L.off_C1, m), blk(X, m + 1), 1.0, blk(Y, m), L.off_C2 + L.bdr * m,
           blk(X, m + 2));
    else if (m + 1 < M)
      gemm(-1.0, g.blk(L.off_C1, m), blk(X, m + 1), 1.0, blk(Y, m));
    gemm(1.0, g.blk(L.off_D, m), blk(Y, m), 0.0, blk(X, m));
  }
  if (rc != EB_OK) return rc;
  return check_launch("ring solve multi");
}

// out = A_{anchor(s)}^-1 in for the systems of one instance (the anchored GMRES preconditioner):
// gather into the anchors' ring blocks, the forward sweeps, scatter to the active systems.
bool graphs_enabled();
int ptc_stream(cudaStream_t& out);

// The sweep's launch sequence depends only on the buffers, the factors and the sizes (the active
// anchors are read on the device), so the first apply of a solve captures it into a CUDA graph
// (*graph) that every later apply replays: one launch instead of 4 (M - 1). The caller
// destroys the graph when the solve ends. With EB_RINGLU_GRAPHS=0, or if the capture fails, the
// sweep is launched directly.
int sweep_graph(const Group& g, int nr, cuDoubleComplex* Y, cuDoubleComplex* X,
                cuDoubleComplex* W, int64_t mstride, const int* zmap, const int* n_active,
                void** graph, cudaStream_t st) {
  if (!graph || !graphs_enabled())
    return ring_solve_multi(g, nr, Y, X, W, mstride, zmap, n_active, st);
  if (!*graph) {
    cudaStream_t cs = nullptr;
    int rc = ptc_stream(cs);
    if (rc != EB_OK) return rc;
    cudaGraph_t gr = nullptr;
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed) == cudaSuccess) {
      const int rc_cap = ring_solve_multi(g, nr, Y, X, W, mstride, zmap, n_active, cs);
      const cudaError_t e = cudaStreamEndCapture(cs, &gr);
      cudaGraphExec_t ex = nullptr;
      if (rc_cap == EB_OK && e == cudaSuccess && gr &&
          cudaGraphInstantiate(&ex, gr, 0) == cudaSuccess)
        *graph = ex;
      if (gr) cudaGraphDestroy(gr);
    }
    cudaGetLastError();  // a failed capture leaves no error behind: the direct launches follow
  }
  if (!*graph) return ring_solve_multi(g, nr, Y, X, W, mstride, zmap, n_active, st);
  if (cudaGraphLaunch(static_cast<cudaGraphExec_t>(*graph), st) != cudaSuccess)
    return check_launch("anchored sweep graph");
  return EB_OK;
}

int anchored_apply(int M, int N, const void* ringlu_ws, int64_t ringlu_stride, int n_anchors,
                   int nr, int n_sys, const int* d_sys_anchor, const int* d_sys_col,
                   const int* d_active, const int* d_zmap, const int* d_n_active,
                   cuDoubleComplex* Y, cuDoubleComplex* X, cuDoubleComplex* W, int64_t mstride,
                   const double* in, double* out, int64_t vstride, int accumulate,
                   void** graph, cudaStream_t st) {
  const Group g{plan(M, N), static_cast<char*>(const_cast<void*>(ringlu_ws)), ringlu_stride,
                n_anchors};
  const int gc = grid_for((int64_t)M * N, 128) / 4 + 1;
  k_sys_to_multi<<<dim3(gc, n_sys), 128, 0, st>>>(M, N, nr, n_sys, d_sys_anchor, d_sys_col, in,
                                                  vstride, Y, mstride);
  int rc = sweep_graph(g, nr, Y, X, W, mstride, d_zmap, d_n_active, graph, st);
  if (rc != EB_OK) return rc;
  k_multi_to_sys<<<dim3(gc, n_sys), 128, 0, st>>>(M, N, nr, n_sys, d_sys_anchor, d_sys_col,
                                                  d_active, X, mstride, out, vstride,
                                                  accumulate);
  return check_launch("anchored preconditioner");
}

}  // namespace rl
}  // namespace eb

using namespace eb;
using namespace eb::rl;

extern "C" {

int64_t eb_ringlu_workspace_bytes(int M, int N) {
  if (M < 4 || N < 5 || panel_width(4 * N) == 0) return -1;
  return (int64_t)plan(M, N).total;
}

}  // extern "C"

namespace eb {
namespace rl {

// Everything a factorisation launches, on stream st (and the second lane's stream): zeroing,
// assembly from J[s] and the shift stored in each workspace, and the ring eliminations. The
// sequence depends only on the workspace, the Jacobian pointers and the sizes, so it can be
// captured once in a CUDA graph and replayed for any shifts.
int issue_factor(const Group& g, const double* const* J, cudaStream_t st) {
  const Layout& L = g.L;
  const int M = L.M, N = L.N, n_shifts = g.S;
  int rc = EB_OK;
  for (int s = 0; s < n_shifts; ++s) {
    char* w = g.base + (int64_t)s * g.stride;
    cudaMemsetAsync(w, 0, L.off_T, st);  // the stored super-blocks and block diagonals
    cudaMemsetAsync(w + L.off_info, 0, sizeof(int) * 4, st);
    k_assemble<<<grid_for((int64_t)M * N * 9, 256), 256, 0, st>>>(
        M, N, J[s], reinterpret_cast<const double*>(w + L.off_shift),
        reinterpret_cast<cuDoubleComplex*>(w + L.off_D), reinterpret_cast<cuDoubleComplex*>(w + L.off_L1),
        reinterpret_cast<double*>(w + L.off_B2), reinterpret_cast<cuDoubleComplex*>(w + L.off_C1),
        reinterpret_cast<double*>(w + L.off_C2));
  }
  if ((rc = check_launch("ringlu assemble")) != EB_OK) return rc;
  if (n_shifts == 1) {
    for (int m = 0; m < M; ++m)
      if ((rc = factor_ring(g, m, st, 2)) != EB_OK) return rc;
    return EB_OK;
  }
  // Two halves of the shifts on two streams, ring by ring: one half's latency-bound
  // Gauss-Jordan panels overlap the other half's GEMMs on the rest of the GPU.
  cudaStream_t s2 = nullptr;
  if ((rc = lane_stream(st, s2, 1)) != EB_OK) return rc;
  const Handle& lane = g_handle[1];
  const int s1 = (n_shifts + 1) / 2;
  const Group g1{L, g.base, g.stride, s1};
  const Group g2{L, g.base + (int64_t)s1 * g.stride, g.stride, n_shifts - s1};
  cudaEventRecord(lane.start, st);
  cudaStreamWaitEvent(lane.stream, lane.start, 0);
  for (int m = 0; m < M; ++m) {
    if ((rc = factor_ring(g1, m, st, 2)) != EB_OK) return rc;
    if ((rc = factor_ring(g2, m, s2, 3)) != EB_OK) return rc;
  }
  cudaEventRecord(lane.done, lane.stream);
  cudaStreamWaitEvent(st, lane.done, 0);
  return EB_OK;
}

// Captured factorisations: the first call with a given (device, workspace, stride, sizes,
// Jacobian pointers) runs eagerly (kernel attributes are set outside any capture), the second
// captures the launch sequence into a CUDA graph, later ones replay it. A few graphs are kept
// per thread (least recently used first out). EB_RINGLU_GRAPHS=0 turns capture off.
struct GraphKey {
  int device, M, N, S;
  const char* base;
  int64_t stride;
  std::vector<const double*> J;
  bool operator==(const GraphKey& o) const {
    return device == o.device && M == o.M && N == o.N && S == o.S && base == o.base &&
           stride == o.stride && J == o.J;
  }
};
struct GraphEntry {
  GraphKey key;
  cudaGraphExec_t exec = nullptr;  // null: seen once, not captured yet
  uint64_t used = 0;
  bool eager_only = false;         // capture failed once: run eagerly from now on
};
thread_local std::vector<GraphEntry> g_graphs;
thread_local uint64_t g_graph_clock = 0;
constexpr size_t kMaxGraphs = 8;

bool graphs_enabled() {
  const char* v = std::getenv("EB_RINGLU_GRAPHS");
  return !(v && v[0] == '0');
}

int run_factor(const Group& g, const double* const* J, cudaStream_t st) {
  if (!graphs_enabled()) return issue_factor(g, J, st);
  int dev = 0;
  cudaGetDevice(&dev);
  GraphKey key{dev, g.L.M, g.L.N, g.S, g.base, g.stride, std::vector<const double*>(J, J + g.S)};
  GraphEntry* e = nullptr;
  for (auto& x : g_graphs)
    if (x.key == key) e = &x;
  if (!e) {  // first sight: eager, remember the key
    if (g_graphs.size() >= kMaxGraphs) {
      auto lru = std::min_element(g_graphs.begin(), g_graphs.end(),
                                  [](const GraphEntry& a, const GraphEntry& b) { return a.used < b.used; });
      if (lru->exec) cudaGraphExecDestroy(lru->exec);
      g_graphs.erase(lru);
    }
    g_graphs.push_back(GraphEntry{key, nullptr, ++g_graph_clock, false});
    return issue_factor(g, J, st);
  }
  e->used = ++g_graph_clock;
  if (e->eager_only) return issue_factor(g, J, st);
  if (!e->exec) {
    cudaGraph_t graph = nullptr;
    cudaError_t err = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    int rc = EB_OK;
    if (err == cudaSuccess) {
      rc = issue_factor(g, J, st);
      err = cudaStreamEndCapture(st, &graph);
    }
    if (rc == EB_OK && err == cudaSuccess && graph)
      err = cudaGraphInstantiate(&e->exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (rc != EB_OK || err != cudaSuccess || !e->exec) {  // not capturable here: stay eager
      cudaGetLastError();
      e->exec = nullptr;
      e->eager_only = true;
      return issue_factor(g, J, st);
    }
  }
  if (cudaGraphLaunch(e->exec, st) != cudaSuccess) return check_launch("ringlu graph launch");
  return EB_OK;
}

}  // namespace rl
}  // namespace eb

extern "C" {

int eb_ringlu_factor_many(const eb_batch* b, const double* const* J, int n_shifts,
                          const double* shifts, void* workspace, int64_t workspace_stride,
                          void* stream) {
  Layout L;
  int rc = check_group(b, n_shifts, workspace, workspace_stride, L);
  if (rc != EB_OK) return rc;
  if (!J || !shifts) return fail(EB_ERR_ARG, "ringlu: null argument");
  for (int s = 0; s < n_shifts; ++s)
    if (!J[s]) return fail(EB_ERR_ARG, "ringlu: null Jacobian");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const Group g{L, static_cast<char*>(workspace), workspace_stride, n_shifts};
  for (int s = 0; s < n_shifts; ++s)
    if (cudaMemcpyAsync(g.base + (int64_t)s * g.stride + L.off_shift, shifts + 2 * s,
                        2 * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess)
      return check_launch("ringlu shifts");
  if ((rc = run_factor(g, J, st)) != EB_OK) return rc;
  if ((rc = check_launch("ringlu factor")) != EB_OK) return rc;
  std::vector<int> info(n_shifts);
  for (int s = 0; s < n_shifts; ++s)
    if (cudaMemcpyAsync(&info[s], g.base + (int64_t)s * g.stride + L.off_info, sizeof(int),
                        cudaMemcpyDeviceToHost, st) != cudaSuccess)
      return check_launch("ringlu info");
  if (cudaStreamSynchronize(st) != cudaSuccess) return check_launch("ringlu info");
  for (int s = 0; s < n_shifts; ++s)
    if (info[s] != 0) return fail(EB_ERR_NAN, "ringlu: singular or non-finite ring block");
  return EB_OK;
}

int eb_ringlu_factor(const eb_batch* b, const double* J, double shift_re, double shift_im,
                     void* workspace, int64_t workspace_bytes, void* stream) {
  const double shift[2] = {shift_re, shift_im};
  const double* js[1] = {J};
  return eb_ringlu_factor_many(b, js, 1, shift, workspace, workspace_bytes & ~(int64_t)255, stream);
}

int eb_ringlu_solve_many(const eb_batch* b, const double* const* J, int n_shifts,
                         const double* shifts, int adjoint, const void* workspace,
                         int64_t workspace_stride, const double* const* rhs, double* const* x,
                         double tol, int max_refine, double* rel_residuals, void* stream) {
  Layout L;
  int rc = check_group(b, n_shifts, workspace, workspace_stride, L);
  if (rc != EB_OK) return rc;
  if (!J || !shifts || !rhs || !x) return fail(EB_ERR_ARG, "ringlu: null argument");
  for (int s = 0; s < n_shifts; ++s) {
    if (!J[s] || !rhs[s] || !x[s]) return fail(EB_ERR_ARG, "ringlu: null argument");
    if ((reinterpret_cast<uintptr_t>(rhs[s]) | reinterpret_cast<uintptr_t>(x[s])) & 15)
      return fail(EB_ERR_ARG, "ringlu: rhs and x must be 16-byte aligned");
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const Group g{L, static_cast<char*>(const_cast<void*>(workspace)), workspace_stride, n_shifts};
  const int M = L.M, N = L.N;
  const int gc = grid_for((int64_t)M * N, 128);
  auto ws = [&](int s) { return g.base + (int64_t)s * g.stride; };
  std::vector<double> rel(n_shifts, INFINITY);
  std::vector<double> acc(2 * (size_t)n_shifts);
  // x = A^-1 b, then refine x += A^-1 (b - A x) until every relative residual reaches tol
  for (int it = 0;; ++it) {
    for (int s = 0; s < n_shifts; ++s)
      k_to_rings<<<gc, 128, 0, st>>>(M, N, it == 0 ? rhs[s] : reinterpret_cast<double*>(ws(s) + L.off_r),
                                     reinterpret_cast<cuDoubleComplex*>(ws(s) + L.off_y));
    if ((rc = ring_solve(g, adjoint != 0, st)) != EB_OK) return rc;
    for (int s = 0; s < n_shifts; ++s) {
      double* a = reinterpret_cast<double*>(ws(s) + L.off_acc);
      k_from_rings<<<gc, 128, 0, st>>>(M, N, reinterpret_cast<cuDoubleComplex*>(ws(s) + L.off_x), x[s],
                                       it == 0 ? 0 : 1);
      cudaMemsetAsync(a, 0, 2 * sizeof(double), st);
      k_residual_op<<<gc, 128, 0, st>>>(M, N, J[s], shifts[2 * s], shifts[2 * s + 1], adjoint, x[s], rhs[s],
                                        reinterpret_cast<double*>(ws(s) + L.off_r), a);
      if (cudaMemcpyAsync(&acc[2 * s], a, 2 * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return check_launch("ringlu residual");
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return check_launch("ringlu residual");
    bool done = true, finite = true;
    for (int s = 0; s < n_shifts; ++s) {
      rel[s] = acc[2 * s + 1] > 0 ? std::sqrt(acc[2 * s] / acc[2 * s + 1]) : std::sqrt(acc[2 * s]);
      finite = finite && std::isfinite(rel[s]);
      done = done && rel[s] <= tol;
    }
    if (!finite) {
      if (rel_residuals)
        for (int s = 0; s < n_shifts; ++s) rel_residuals[s] = rel[s];
      return fail(EB_ERR_NAN, "ringlu: non-finite residual");
    }
    if (done || it >= max_refine) break;
  }
  if (rel_residuals)
    for (int s = 0; s < n_shifts; ++s) rel_residuals[s] = rel[s];
  for (int s = 0; s < n_shifts; ++s)
    if (rel[s] > tol) return fail(EB_ERR_NOCONV, "ringlu: refinement did not reach the tolerance");
  return check_launch("ringlu solve");
}

int eb_ringlu_solve(const eb_batch* b, const double* J, double shift_re, double shift_im,
                    int adjoint, const void* workspace, int64_t workspace_bytes,
                    const double* rhs, double* x, double tol, int max_refine,
                    double* rel_residual, void* stream) {
  const double shift[2] = {shift_re, shift_im};
  const double* js[1] = {J};
  const double* in[1] = {rhs};
  double* out[1] = {x};
  return eb_ringlu_solve_many(b, js, 1, shift, adjoint, workspace, workspace_bytes & ~(int64_t)255,
                              in, out, tol, max_refine, rel_residual, stream);
}

}  // extern "C"

// ---- PTC/SER steady state on the device ------------------------------------------------------
//
// The pseudo-transient continuation with switched evolution relaxation of the reference's
// example driver (examples/response/run.py:84-123): per step the residual R of the current state,
// its infinity norm relative to the initial state's (rel), the shift rel / ser (the inverse of
// the time step ser / rel), the states Jacobian, and the update U += Re((J - shift I)^-1 (-R));
// the loop stops at rel <= rtol (or a non-finite rel) or after max_steps steps. Here a step is a
// fixed launch sequence whose control values (norm, rel, shift, the stop flag) live in device
// memory: the first step runs eagerly, the sequence is then captured once in a CUDA graph and
// replayed, and the host reads only the stop flag of the previous step (so at most one replay
// runs past the last step; its update and history entry are skipped on the device). The solve is
// the ring-block LU with one refinement step against the device residual.

namespace eb {
namespace rl {

struct PtcCtl {
  unsigned long long norm_bits;  // max |R| of the step (bits of a non-negative double)
  double norm0;                  // max |R| of the initial state
  int run;                       // the loop had not stopped when this step began
  int done;                      // stopped: rel <= rtol, rel not finite, or a singular block
  int steps;                     // relative norms recorded
  int status;                    // EB_OK or EB_ERR_NAN
};

struct PtcLayout {
  Layout lu;
  size_t off_lu, off_x, off_r, off_ctl, off_hist, total;
};

PtcLayout ptc_plan(int M, int N, int max_steps) {
  PtcLayout P;
  P.lu = plan(M, N);
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o = align_up(o + bytes);
    return at;
  };
  P.off_lu = take(P.lu.total);
  P.off_x = take(sizeof(double) * 8 * (size_t)M * N);
  P.off_r = take(sizeof(double) * 8 * (size_t)M * N);
  P.off_ctl = take(sizeof(PtcCtl));
  P.off_hist = take(sizeof(double) * 2 * (size_t)max_steps);
  P.total = o;
  return P;
}

__global__ void k_ptc_begin(PtcCtl* c) {
  c->run = !c->done;
  c->norm_bits = 0ull;
}

// max |v| over v, as the maximum of the bit patterns of |v| (ordered like the values for
// non-negative doubles; a NaN compares above every finite value and infinity)
__global__ void __launch_bounds__(256) k_ptc_absmax(int64_t n, const double* v, PtcCtl* c) {
  unsigned long long m = 0ull;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    m = max(m, (unsigned long long)__double_as_longlong(fabs(v[i])));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(&c->norm_bits, m);
}

__global__ void k_ptc_init(PtcCtl* c) {
  c->norm0 = __longlong_as_double((long long)c->norm_bits);
  c->run = 1;
  c->done = 0;
  c->steps = 0;
  c->status = EB_OK;
}

// rel = |R| / |R_0|, the history entry (|R|, rel), the stop test and the shift of the step
// (time step ser * rel^-1, shift = time step^-1, the example driver's arithmetic).
__global__ void k_ptc_control(PtcCtl* c, double ser, double rtol, double* hist, double* shift) {
  if (!c->run) return;
  const double norm = __longlong_as_double((long long)c->norm_bits);
  const double rel = norm / c->norm0;
  hist[2 * c->steps] = norm;
  hist[2 * c->steps + 1] = rel;
  c->steps += 1;
  if (rel <= rtol || isnan(rel)) {
    c->done = 1;
    c->status = isnan(rel) ? EB_ERR_NAN : EB_OK;
    return;
  }
  const double time_step = ser * (1.0 / rel);
  shift[0] = 1.0 / time_step;
  shift[1] = 0.0;
}

// y (ring layout, complex) = -R
__global__ void k_ptc_rhs(int M, int N, const double* R, const PtcCtl* c, cuDoubleComplex* y) {
  if (c->done) return;
  const int64_t cells = (int64_t)M * N;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < cells;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(g % M), n = (int)(g / M);
    for (int v = 0; v < 4; ++v)
      y[(int64_t)m * 4 * N + 4 * n + v] = make_cuDoubleComplex(-R[4 * g + v], 0.0);
  }
}

// r = -R - (J - s I) x for the solution x of the first solve (x copied to the reference layout
// into xs): the residual the refinement step solves for.
__global__ void __launch_bounds__(128) k_ptc_refine_rhs(int M, int N, const double* J,
                                                        const double* shift,
                                                        const cuDoubleComplex* x_ring,
                                                        const double* R, const PtcCtl* c,
                                                        double* xs, double* r) {
  if (c->done) return;
  const int64_t cells = (int64_t)M * N, slot_stride = 16 * cells;
  const double sr = shift[0], si = shift[1];
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < cells;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(g % M), n = (int)(g / M);
    double ar[4] = {0, 0, 0, 0}, ai[4] = {0, 0, 0, 0};
    for (int s = 0; s < 9; ++s) {
      if (!slot_active(s, m, M)) continue;
      const double* blk = J + slot_stride * s + 16 * g;
      const int mm = m + slot_dm(s), nn = wrap(n + slot_dn(s), N);
      const cuDoubleComplex* xj = x_ring + (int64_t)mm * 4 * N + 4 * nn;
      for (int i = 0; i < 4; ++i)
        for (int q = 0; q < 4; ++q) {
          ar[q] += blk[q + 4 * i] * xj[i].x;
          ai[q] += blk[q + 4 * i] * xj[i].y;
        }
    }
    const cuDoubleComplex* xc = x_ring + (int64_t)m * 4 * N + 4 * n;
    for (int q = 0; q < 4; ++q) {
      const double xr = xc[q].x, xi = xc[q].y;
      xs[8 * g + 2 * q] = xr;
      xs[8 * g + 2 * q + 1] = xi;
      r[8 * g + 2 * q] = -R[4 * g + q] - (ar[q] - (sr * xr - si * xi));
      r[8 * g + 2 * q + 1] = -(ai[q] - (sr * xi + si * xr));
    }
  }
}

// U += Re(xs + correction); a singular ring block (LU info) stops the loop instead
__global__ void k_ptc_update(int M, int N, const cuDoubleComplex* x_ring, const double* xs,
                             const int* lu_info, PtcCtl* c, double* U) {
  if (c->done) return;
  if (*lu_info != 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      c->done = 1;
      c->status = EB_ERR_NAN;
    }
    return;
  }
  const int64_t cells = (int64_t)M * N;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < cells;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(g % M), n = (int)(g / M);
    for (int v = 0; v < 4; ++v)
      U[4 * g + v] += xs[8 * g + 2 * v] + x_ring[(int64_t)m * 4 * N + 4 * n + v].x;
  }
}

// One PTC step's launch sequence on st (all control values on the device).
int issue_ptc_step(const eb_batch* b, const PtcLayout& P, char* ws, const double* X,
                   const double* V, double* U, double* R, double* J, double ser, double rtol,
                   cudaStream_t st) {
  const int M = P.lu.M, N = P.lu.N;
  const int64_t cells = (int64_t)M * N;
  PtcCtl* ctl = reinterpret_cast<PtcCtl*>(ws + P.off_ctl);
  char* lw = ws + P.off_lu;
  const Group g{P.lu, lw, (int64_t)P.lu.total, 1};
  double* shift = reinterpret_cast<double*>(lw + P.lu.off_shift);
  cuDoubleComplex* y = reinterpret_cast<cuDoubleComplex*>(lw + P.lu.off_y);
  cuDoubleComplex* x = reinterpret_cast<cuDoubleComplex*>(lw + P.lu.off_x);
  double* xs = reinterpret_cast<double*>(ws + P.off_x);
  double* r = reinterpret_cast<double*>(ws + P.off_r);
  const int gc = grid_for(cells, 128);
  int rc;
  k_ptc_begin<<<1, 1, 0, st>>>(ctl);
  if ((rc = eb_compute_odes(b, X, V, U, R, st)) != EB_OK) return rc;
  k_ptc_absmax<<<grid_for(4 * cells, 256), 256, 0, st>>>(4 * cells, R, ctl);
  k_ptc_control<<<1, 1, 0, st>>>(ctl, ser, rtol, reinterpret_cast<double*>(ws + P.off_hist),
                                 shift);
  if ((rc = eb_compute_odes_wrt_states(b, X, V, U, J, st)) != EB_OK) return rc;
  const double* js[1] = {J};
  if ((rc = issue_factor(g, js, st)) != EB_OK) return rc;
  k_ptc_rhs<<<gc, 128, 0, st>>>(M, N, R, ctl, y);
  if ((rc = ring_solve(g, false, st)) != EB_OK) return rc;
  k_ptc_refine_rhs<<<gc, 128, 0, st>>>(M, N, J, shift, x, R, ctl, xs, r);
  k_to_rings<<<gc, 128, 0, st>>>(M, N, r, y);
  if ((rc = ring_solve(g, false, st)) != EB_OK) return rc;
  k_ptc_update<<<gc, 128, 0, st>>>(M, N, x, xs, reinterpret_cast<int*>(lw + P.lu.off_info), ctl,
                                   U);
  return check_launch("ptc step");
}

// The stream the PTC loop runs on, one per thread and device: a CUDA graph cannot be captured
// from the legacy default stream, which is what many callers pass.
int ptc_stream(cudaStream_t& out) {
  struct Own {
    int device = -1;
    cudaStream_t stream = nullptr;
  };
  thread_local Own own;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return check_launch("ptc device");
  if (own.device != dev) {
    own.stream = nullptr;  // a stream of another device is left to that device
    if (cudaStreamCreateWithFlags(&own.stream, cudaStreamNonBlocking) != cudaSuccess)
      return check_launch("ptc stream");
    own.device = dev;
  }
  out = own.stream;
  return EB_OK;
}

}  // namespace rl
}  // namespace eb

extern "C" {

int64_t eb_ptc_workspace_bytes(int M, int N, int max_steps) {
  if (M < 4 || N < 5 || panel_width(4 * N) == 0 || max_steps < 1) return -1;
  return (int64_t)ptc_plan(M, N, max_steps).total;
}

int eb_ptc_run(const eb_batch* b, const double* X, const double* V, double* U, double* R,
               double* J, double ser, double rtol, int max_steps, void* workspace,
               int64_t workspace_bytes, double* history, int* n_steps, void* stream) {
  int rc = validate(b);
  if (rc != EB_OK) return rc;
  if (b->n_inst != 1 || b->d_table) return fail(EB_ERR_ARG, "ptc: single instance only");
  if (!X || !U || !R || !J || !workspace || !history || !n_steps)
    return fail(EB_ERR_ARG, "ptc: null argument");
  if ((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(V) |
       reinterpret_cast<uintptr_t>(U) | reinterpret_cast<uintptr_t>(R) |
       reinterpret_cast<uintptr_t>(J)) & 15)
    return fail(EB_ERR_ARG, "ptc: arrays must be 16-byte aligned");
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
    return fail(EB_ERR_ARG, "ptc: workspace not 256-byte aligned");
  if (max_steps < 1 || !(ser > 0) || !(rtol >= 0)) return fail(EB_ERR_ARG, "ptc: bad options");
  const int M = b->single.M, N = b->single.N;
  if (M < 4 || N < 5 || panel_width(4 * N) == 0) return fail(EB_ERR_ARG, "ptc: unsupported grid size");
  const PtcLayout P = ptc_plan(M, N, max_steps);
  if (workspace_bytes < (int64_t)P.total) return fail(EB_ERR_ARG, "ptc: workspace too small");
  // the loop runs on a stream of its own, after the work queued on the caller's stream (and
  // the caller's stream waits for the loop before anything queued on it later)
  const cudaStream_t caller = reinterpret_cast<cudaStream_t>(stream);
  cudaStream_t st = nullptr;
  if ((rc = ptc_stream(st)) != EB_OK) return rc;
  char* ws = static_cast<char*>(workspace);
  PtcCtl* ctl = reinterpret_cast<PtcCtl*>(ws + P.off_ctl);
  const int64_t cells = (int64_t)M * N;
  *n_steps = 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaGraphExec_t exec = nullptr;
  auto cleanup = [&]() {
    if (exec) cudaGraphExecDestroy(exec);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
  };
  for (auto& e : ev)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      cleanup();
      return check_launch("ptc events");
    }
  if (cudaEventRecord(ev[0], caller) != cudaSuccess || cudaStreamWaitEvent(st, ev[0], 0) != cudaSuccess) {
    cleanup();
    return check_launch("ptc stream order");
  }
  // the initial state's residual norm
  k_ptc_begin<<<1, 1, 0, st>>>(ctl);
  if ((rc = eb_compute_odes(b, X, V, U, R, st)) == EB_OK) {
    k_ptc_absmax<<<grid_for(4 * cells, 256), 256, 0, st>>>(4 * cells, R, ctl);
    k_ptc_init<<<1, 1, 0, st>>>(ctl);
    rc = check_launch("ptc init");
  }
  // two stop flags in pinned host memory (allocated once per thread), so that reading one back
  // does not wait for the step queued after it
  thread_local int* done_h = nullptr;
  if (rc == EB_OK && !done_h &&
      cudaHostAlloc(reinterpret_cast<void**>(&done_h), 2 * sizeof(int), cudaHostAllocDefault) !=
          cudaSuccess) {
    done_h = nullptr;
    rc = check_launch("ptc flag buffer");
  }
  if (rc != EB_OK) {
    cudaStreamSynchronize(st);
    cleanup();
    return rc;
  }
  done_h[0] = done_h[1] = 0;
  for (int k = 0; k < max_steps; ++k) {
    if (k == 0) {  // eagerly (the autotuner times its variants outside any capture)
      rc = issue_ptc_step(b, P, ws, X, V, U, R, J, ser, rtol, st);
    } else {
      if (!exec) {
        cudaGraph_t graph = nullptr;
        cudaError_t err = cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed);
        if (err == cudaSuccess) {
          rc = issue_ptc_step(b, P, ws, X, V, U, R, J, ser, rtol, st);
          err = cudaStreamEndCapture(st, &graph);
        }
        if (rc == EB_OK && err == cudaSuccess) err = cudaGraphInstantiate(&exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (rc != EB_OK || err != cudaSuccess) {
          cudaGetLastError();  // a failed capture must not leave its error to later calls
          cudaStreamSynchronize(st);
          cleanup();
          if (rc != EB_OK) return rc;
          return fail(EB_ERR_CUDA, (std::string("ptc: graph capture failed: ") +
                                    cudaGetErrorString(err)).c_str());
        }
      }
      rc = cudaGraphLaunch(exec, st) == cudaSuccess ? EB_OK : check_launch("ptc graph launch");
    }
    if (rc != EB_OK) {
      cleanup();
      return rc;
    }
    // the stop flag of this step, read back once the next step is queued
    if (cudaMemcpyAsync(&done_h[k & 1], &ctl->done, sizeof(int), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaEventRecord(ev[k & 1], st) != cudaSuccess) {
      cleanup();
      return check_launch("ptc flag");
    }
    if (k >= 1) {
      if (cudaEventSynchronize(ev[(k - 1) & 1]) != cudaSuccess) {
        cleanup();
        return check_launch("ptc flag");
      }
      if (done_h[(k - 1) & 1]) break;
    }
  }
  PtcCtl hc;
  const cudaError_t e1 = cudaMemcpyAsync(&hc, ctl, sizeof(PtcCtl), cudaMemcpyDeviceToHost, st);
  const cudaError_t e2 = cudaStreamSynchronize(st);
  cudaEventRecord(ev[0], st);
  cudaStreamWaitEvent(caller, ev[0], 0);
  cleanup();
  if (e1 != cudaSuccess || e2 != cudaSuccess) return check_launch("ptc result");
  const int n = std::min(hc.steps, max_steps);
  if (n > 0 && cudaMemcpy(history, ws + P.off_hist, sizeof(double) * 2 * n,
                          cudaMemcpyDeviceToHost) != cudaSuccess)
    return check_launch("ptc history");
  *n_steps = n;
  if (hc.status != EB_OK)
    return fail(hc.status, "ptc: non-finite residual or singular ring block");
  return EB_OK;
}

}  // extern "C"
