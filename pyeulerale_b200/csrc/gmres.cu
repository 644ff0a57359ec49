// Resolvent solves (dR/dU - shift I) x = b and (dR/dU - shift I)^H x = b on the device.
//
// Replaces the reference's SuperLU factorisation per call (src/py_euler_ale/core.py:512-599)
// with restarted complex GMRES, right-preconditioned by the inverse 4x4 diagonal blocks
// (block Jacobi), on the structured nine-slot Jacobian (the d(odes)/d(states) layout of
// src/spatial_discretization.f90:676 -- no index arrays needed).
//
// Many systems are solved together: a "system" is (instance, shift, right-hand side), so the
// frequency response's shifts sharing one Jacobian and the instances of a mixed batch are all
// systems of one call. Each system has its own Krylov basis and coefficients; its vectors are
// stored contiguously (system-major), and all per-iteration work is one launch over all
// systems. Reductions are deterministic two-pass (per-CTA partials, then per-system sums).
// Arnoldi uses classical Gram-Schmidt with one re-orthogonalisation pass (CGS2).
//
// The driver loop (eb_gmres_solve) is native C++; the caller passes all device memory as
// one workspace (eb_gmres_workspace_bytes), so a solve performs no allocation.

#include <cuComplex.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <functional>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/euler_b200.h"
#include "physics.cuh"

namespace eb {

int fail(int code, const char* msg);
int check_launch(const char* what);
int validate(const eb_batch* b);
extern thread_local std::string g_last_error;

namespace rl {
int anchored_apply(int M, int N, const void* ringlu_ws, int64_t ringlu_stride, int n_anchors,
                   int nr, int n_sys, const int* d_sys_anchor, const int* d_sys_col,
                   const int* d_active, const int* d_zmap, const int* d_n_active,
                   cuDoubleComplex* Y, cuDoubleComplex* X, cuDoubleComplex* W, int64_t mstride,
                   const double* in, double* out, int64_t vstride, int accumulate,
                   void** graph, cudaStream_t st);
}  // namespace rl

namespace gm {

constexpr int kChunkCells = 256;  // cells per reduction chunk (1024 complex entries)

struct Sys {
  int64_t cell_begin;   // first cell of the system in system space
  int64_t n_cells;      // cells of the system
  int64_t chunk_begin;  // first reduction chunk of the system
  int64_t jac_cell;     // first cell of the system's instance in the Jacobian / batch arrays
  int32_t M, N;         // grid of the instance
  double sr, si;        // shift applied to the operator (already conjugated for the adjoint)
};

struct cplx {
  double r, i;
};
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return {a.r + b.r, a.i + b.i}; }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return {a.r - b.r, a.i - b.i}; }
__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r};
}
__device__ __forceinline__ cplx cconjmul(cplx a, cplx b) {  // conj(a) * b
  return {a.r * b.r + a.i * b.i, a.r * b.i - a.i * b.r};
}
__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
  // Smith's algorithm
  if (fabs(b.r) >= fabs(b.i)) {
    const double t = b.i / b.r, d = b.r + b.i * t;
    return {(a.r + a.i * t) / d, (a.i - a.r * t) / d};
  }
  const double t = b.r / b.i, d = b.r * t + b.i;
  return {(a.r * t + a.i) / d, (a.i * t - a.r) / d};
}
__device__ __forceinline__ cplx ld(const double* p) {
  const double2 v = *reinterpret_cast<const double2*>(p);
  return {v.x, v.y};
}
__device__ __forceinline__ void st(double* p, cplx c) {
  *reinterpret_cast<double2*>(p) = make_double2(c.r, c.i);
}

__device__ __forceinline__ int find_sys(const Sys* sys, int n_sys, int64_t cell) {
  int lo = 0, hi = n_sys - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (sys[mid].cell_begin <= cell) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// x_c <- D_c^-1 x_c with D_c = J_cc - shift I (adjoint: J_cc^T - conj(shift) I): Gaussian
// elimination with partial pivoting on the 4x4 complex block, in registers.
__device__ __forceinline__ void block_solve(const double* Jcc, bool adj, double sr, double si,
                                            cplx x[4]) {
  cplx A[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double v = adj ? Jcc[c + 4 * r] : Jcc[r + 4 * c];
      A[r][c] = {v - (r == c ? sr : 0.0), (r == c ? -si : 0.0)};
    }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    int p = k;
    double best = fabs(A[k][k].r) + fabs(A[k][k].i);
#pragma unroll
    for (int r = k + 1; r < 4; ++r) {
      const double v = fabs(A[r][k].r) + fabs(A[r][k].i);
      if (v > best) {
        best = v;
        p = r;
      }
    }
    if (p != k) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const cplx t = A[k][c];
        A[k][c] = A[p][c];
        A[p][c] = t;
      }
      const cplx t = x[k];
      x[k] = x[p];
      x[p] = t;
    }
#pragma unroll
    for (int r = k + 1; r < 4; ++r) {
      const cplx f = cdiv(A[r][k], A[k][k]);
#pragma unroll
      for (int c = k + 1; c < 4; ++c) A[r][c] = csub(A[r][c], cmul(f, A[k][c]));
      x[r] = csub(x[r], cmul(f, x[k]));
    }
  }
#pragma unroll
  for (int k = 3; k >= 0; --k) {
    cplx s = x[k];
#pragma unroll
    for (int c = k + 1; c < 4; ++c) s = csub(s, cmul(A[k][c], x[c]));
    x[k] = cdiv(s, A[k][k]);
  }
}

// out = D^-1 in (accumulate: out += D^-1 in), per active system.
__global__ void k_prec(const Sys* sys, int n_sys, int64_t n_cells, const int* active,
                       const double* J, int adj, const double* in, double* out, int accumulate) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_cells;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int s = find_sys(sys, n_sys, g);
    if (!active[s]) continue;
    const Sys S = sys[s];
    const int64_t c = g - S.cell_begin;
    cplx x[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) x[k] = ld(in + 8 * g + 2 * k);
    block_solve(J + 144 * S.jac_cell + 16 * c, adj != 0, S.sr, S.si, x);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (accumulate) x[k] = cadd(x[k], ld(out + 8 * g + 2 * k));
      st(out + 8 * g + 2 * k, x[k]);
    }
  }
}

// y = (J - shift I) x (adj: (J^T - shift I) x; the shift is pre-conjugated). With `b` given,
// y = b - (J - shift I) x (residual).
__global__ void __launch_bounds__(128) k_op(const Sys* sys, int n_sys, int64_t n_cells,
                                            const int* active, const double* J, int adj,
                                            const double* x, const double* b, double* y) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_cells;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int s = find_sys(sys, n_sys, g);
    if (!active[s]) continue;
    const Sys S = sys[s];
    const int M = S.M, N = S.N;
    const int64_t c = g - S.cell_begin;
    const int m = (int)(c % M), n = (int)(c / M);
    const int64_t slot_stride = 16 * (int64_t)M * N;
    const double* Ji = J + 144 * S.jac_cell;
    const double* xs = x + 8 * S.cell_begin;
    cplx acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
    if (!adj) {
#pragma unroll
      for (int sl = 0; sl < 9; ++sl) {
        if (!slot_active(sl, m, M)) continue;
        const double* blk = Ji + slot_stride * sl + 16 * c;
        const int64_t j = (m + slot_dm(sl)) + (int64_t)M * wrap(n + slot_dn(sl), N);
        cplx xv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) xv[i] = ld(xs + 8 * j + 2 * i);
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const double a = blk[r + 4 * i];
            acc[r].r += a * xv[i].r;
            acc[r].i += a * xv[i].i;
          }
      }
    } else {
#pragma unroll
      for (int sl = 0; sl < 9; ++sl) {
        const int mc = m - slot_dm(sl);
        if (mc < 0 || mc >= M || !slot_active(sl, mc, M)) continue;
        const int64_t src = mc + (int64_t)M * wrap(n - slot_dn(sl), N);
        const double* blk = Ji + slot_stride * sl + 16 * src;
        cplx xv[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) xv[r] = ld(xs + 8 * src + 2 * r);
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const double a = blk[r + 4 * i];
            acc[i].r += a * xv[r].r;
            acc[i].i += a * xv[r].i;
          }
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const cplx xc = ld(xs + 8 * c + 2 * k);
      cplx v = csub(acc[k], cmul({S.sr, S.si}, xc));
      if (b) v = csub(ld(b + 8 * g + 2 * k), v);
      st(y + 8 * g + 2 * k, v);
    }
  }
}

// Partial sums over one chunk of cells: part[chunk][k] = sum conj(V_k) w for k < nk (dots)
// or part[chunk][0] = sum |w|^2 (nk = 0).
__global__ void __launch_bounds__(256) k_partial(const Sys* sys, int n_sys, int64_t n_chunks,
                                                 const int* active, const double* V,
                                                 int64_t vstride, int nk, const double* w,
                                                 double* part, int part_stride) {
  __shared__ double2 ws[kChunkCells * 4];
  const int64_t ch = blockIdx.x;
  if (ch >= n_chunks) return;
  int s = 0;
  {
    int lo = 0, hi = n_sys - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (sys[mid].chunk_begin <= ch) lo = mid; else hi = mid - 1;
    }
    s = lo;
  }
  if (!active[s]) return;
  const Sys S = sys[s];
  const int64_t c0 = S.cell_begin + (ch - S.chunk_begin) * kChunkCells;
  const int64_t c1 = min(c0 + kChunkCells, S.cell_begin + S.n_cells);
  const int ne = (int)(4 * (c1 - c0));
  for (int e = threadIdx.x; e < ne; e += blockDim.x)
    ws[e] = *reinterpret_cast<const double2*>(w + 2 * (4 * c0 + e));
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  if (nk == 0) {
    double acc = 0.0;
    for (int e = threadIdx.x; e < ne; e += blockDim.x) acc += ws[e].x * ws[e].x + ws[e].y * ws[e].y;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ double red[32];
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int q = 0; q < nw; ++q) t += red[q];
      part[ch * part_stride] = t;
    }
    return;
  }
  for (int k = warp; k < nk; k += nw) {
    const double* vk = V + (int64_t)k * vstride + 2 * 4 * c0;
    double ar = 0.0, ai = 0.0;
    for (int e = lane; e < ne; e += 32) {
      const double2 v = *reinterpret_cast<const double2*>(vk + 2 * e);
      ar += v.x * ws[e].x + v.y * ws[e].y;
      ai += v.x * ws[e].y - v.y * ws[e].x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ar += __shfl_xor_sync(0xffffffffu, ar, o);
      ai += __shfl_xor_sync(0xffffffffu, ai, o);
    }
    if (lane == 0) {
      part[ch * part_stride + 2 * k] = ar;
      part[ch * part_stride + 2 * k + 1] = ai;
    }
  }
}

// Sums the chunk partials of every system: out[s][k] (complex) or out[s] (norm^2, nk == 0).
__global__ void k_reduce(const Sys* sys, int n_sys, const int* active, int nk,
                         const double* part, int part_stride, double* out, int out_stride) {
  const int s = blockIdx.x;
  if (s >= n_sys || !active[s]) return;
  const Sys S = sys[s];
  const int64_t nch = (S.n_cells + kChunkCells - 1) / kChunkCells;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int items = nk == 0 ? 1 : nk;
  for (int k = warp; k < items; k += nw) {
    double ar = 0.0, ai = 0.0;
    for (int64_t q = lane; q < nch; q += 32) {
      const double* p = part + (S.chunk_begin + q) * part_stride;
      if (nk == 0) {
        ar += p[0];
      } else {
        ar += p[2 * k];
        ai += p[2 * k + 1];
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ar += __shfl_xor_sync(0xffffffffu, ar, o);
      ai += __shfl_xor_sync(0xffffffffu, ai, o);
    }
    if (lane == 0) {
      if (nk == 0) {
        out[s * out_stride] = ar;
      } else {
        out[s * out_stride + 2 * k] = ar;
        out[s * out_stride + 2 * k + 1] = ai;
      }
    }
  }
}

// w -= sum_k h[s][k] V_k (CGS projection); h accumulated into H[:, j] (add = 1 second pass).
__global__ void k_project(const Sys* sys, int n_sys, int64_t n_cells, const int* active,
                          const double* V, int64_t vstride, int nk, const double* h,
                          int h_stride, double* w) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_cells;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int s = find_sys(sys, n_sys, g);
    if (!active[s]) continue;
    const double* hs = h + s * h_stride;
    cplx acc[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[e] = ld(w + 8 * g + 2 * e);
    for (int k = 0; k < nk; ++k) {
      const cplx hk = {hs[2 * k], hs[2 * k + 1]};
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[e] = csub(acc[e], cmul(hk, ld(V + k * vstride + 8 * g + 2 * e)));
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) st(w + 8 * g + 2 * e, acc[e]);
  }
}

// Per-system Arnoldi bookkeeping after the projections of column j:
// H[:, j] = h1 + h2, beta = ||w||, Givens update of the least-squares residual.
struct State {
  double bnorm;   // ||b||
  double beta;    // current residual norm (start of cycle)
  double est;     // implicit residual estimate |g_{j+1}|
  double inv;     // 1 / H[j+1, j] used to normalise the new basis vector (0 on breakdown)
  int jlen;       // columns in the current cycle
  int iters;      // total Arnoldi steps
  int breakdown;  // happy breakdown in this cycle
  int pad;
};

__global__ void k_givens(int n_sys, const int* active, int j, int m, const double* h1,
                         const double* h2, int h_stride, const double* wn2, double* H,
                         double* cs, double* g, State* st_) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_sys || !active[s]) return;
  State& S = st_[s];
  if (S.breakdown) return;
  double* Hs = H + (int64_t)s * 2 * (m + 1) * m;  // column-major (m+1) x m complex
  double* col = Hs + 2 * (int64_t)(m + 1) * j;
  for (int k = 0; k <= j; ++k) {
    col[2 * k] = h1[s * h_stride + 2 * k] + h2[s * h_stride + 2 * k];
    col[2 * k + 1] = h1[s * h_stride + 2 * k + 1] + h2[s * h_stride + 2 * k + 1];
  }
  const double beta = sqrt(wn2[s]);
  col[2 * (j + 1)] = beta;
  col[2 * (j + 1) + 1] = 0.0;
  // apply the previous rotations: [c  s; -conj(s) c] with real c
  double* css = cs + (int64_t)s * 3 * m;  // (c, s_re, s_im) per rotation
  for (int k = 0; k < j; ++k) {
    const double c = css[3 * k], sr = css[3 * k + 1], si = css[3 * k + 2];
    const double ar = col[2 * k], ai = col[2 * k + 1];
    const double br = col[2 * (k + 1)], bi = col[2 * (k + 1) + 1];
    // a' = c a + s b ; b' = -conj(s) a + c b
    col[2 * k] = c * ar + (sr * br - si * bi);
    col[2 * k + 1] = c * ai + (sr * bi + si * br);
    col[2 * (k + 1)] = -(sr * ar + si * ai) + c * br;
    col[2 * (k + 1) + 1] = -(sr * ai - si * ar) + c * bi;
  }
  // new rotation zeroing col[j+1] (real, = beta)
  const double ar = col[2 * j], ai = col[2 * j + 1];
  const double amag = hypot(ar, ai);
  double c, sr, si, rr, ri;
  if (beta == 0.0) {
    c = 1.0; sr = 0.0; si = 0.0; rr = ar; ri = ai;
  } else if (amag == 0.0) {
    c = 0.0; sr = 1.0; si = 0.0; rr = beta; ri = 0.0;
  } else {
    const double nrm = hypot(amag, beta);
    c = amag / nrm;
    // s = (a/|a|) * conj(b) / nrm, b = beta real
    sr = (ar / amag) * beta / nrm;
    si = (ai / amag) * beta / nrm;
    rr = (ar / amag) * nrm;
    ri = (ai / amag) * nrm;
  }
  css[3 * j] = c;
  css[3 * j + 1] = sr;
  css[3 * j + 2] = si;
  col[2 * j] = rr;
  col[2 * j + 1] = ri;
  col[2 * (j + 1)] = 0.0;
  col[2 * (j + 1) + 1] = 0.0;
  double* gs = g + (int64_t)s * 2 * (m + 1);
  const double gr = gs[2 * j], gi = gs[2 * j + 1];
  gs[2 * j] = c * gr;
  gs[2 * j + 1] = c * gi;
  gs[2 * (j + 1)] = -(sr * gr + si * gi);
  gs[2 * (j + 1) + 1] = -(sr * gi - si * gr);
  S.est = hypot(gs[2 * (j + 1)], gs[2 * (j + 1) + 1]);
  S.jlen = j + 1;
  S.iters += 1;
  const double tiny = 1e-300;
  if (beta <= tiny * (S.beta > 0 ? S.beta : 1.0) || !(beta == beta)) {
    S.breakdown = 1;
    S.inv = 0.0;
  } else {
    S.inv = 1.0 / beta;
  }
}

// V_{j+1} = w * inv (w is stored in place as V_{j+1}).
__global__ void k_scale(const Sys* sys, int n_sys, int64_t n_cells, const int* active,
                        const State* st_, double* w) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_cells;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int s = find_sys(sys, n_sys, g);
    if (!active[s]) continue;
    const double f = st_[s].inv;
#pragma unroll
    for (int e = 0; e < 8; ++e) w[8 * g + e] *= f;
  }
}

// Start of a cycle: beta = ||r||, V_0 = r / beta, g = (beta, 0, ...), reset the cycle.
__global__ void k_cycle_start(int n_sys, const int* active, int m, const double* rn2,
                              double* g, State* st_) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_sys || !active[s]) return;
  State& S = st_[s];
  S.beta = sqrt(rn2[s]);
  S.est = S.beta;
  S.jlen = 0;
  S.breakdown = 0;
  S.inv = S.beta > 0 ? 1.0 / S.beta : 0.0;
  double* gs = g + (int64_t)s * 2 * (m + 1);
  for (int k = 0; k <= m; ++k) {
    gs[2 * k] = 0.0;
    gs[2 * k + 1] = 0.0;
  }
  gs[0] = S.beta;
}

// Back substitution H y = g for the columns of the cycle (upper triangular after rotations).
__global__ void k_backsolve(int n_sys, const int* active, int m, const double* H,
                            const double* g, double* y, const State* st_) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_sys || !active[s]) return;
  const int n = st_[s].jlen;
  const double* Hs = H + (int64_t)s * 2 * (m + 1) * m;
  const double* gs = g + (int64_t)s * 2 * (m + 1);
  double* ys = y + (int64_t)s * 2 * m;
  for (int k = n - 1; k >= 0; --k) {
    double sr = gs[2 * k], si = gs[2 * k + 1];
    for (int c = k + 1; c < n; ++c) {
      const double hr = Hs[2 * ((int64_t)(m + 1) * c + k)], hi = Hs[2 * ((int64_t)(m + 1) * c + k) + 1];
      sr -= hr * ys[2 * c] - hi * ys[2 * c + 1];
      si -= hr * ys[2 * c + 1] + hi * ys[2 * c];
    }
    const double dr = Hs[2 * ((int64_t)(m + 1) * k + k)], di = Hs[2 * ((int64_t)(m + 1) * k + k) + 1];
    const double den = dr * dr + di * di;
    ys[2 * k] = den > 0 ? (sr * dr + si * di) / den : 0.0;
    ys[2 * k + 1] = den > 0 ? (si * dr - sr * di) / den : 0.0;
  }
  for (int k = n; k < m; ++k) {
    ys[2 * k] = 0.0;
    ys[2 * k + 1] = 0.0;
  }
}

// z = sum_k y_k V_k for the columns of the cycle.
__global__ void k_combine(const Sys* sys, int n_sys, int64_t n_cells, const int* active,
                          const double* V, int64_t vstride, int m, const double* y,
                          const State* st_, double* z) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_cells;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int s = find_sys(sys, n_sys, g);
    if (!active[s]) continue;
    const int n = st_[s].jlen;
    const double* ys = y + (int64_t)s * 2 * m;
    cplx acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
    for (int k = 0; k < n; ++k) {
      const cplx yk = {ys[2 * k], ys[2 * k + 1]};
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[e] = cadd(acc[e], cmul(yk, ld(V + k * vstride + 8 * g + 2 * e)));
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) st(z + 8 * g + 2 * e, acc[e]);
  }
}

// ---- workspace --------------------------------------------------------------------------

struct Layout {
  int64_t n_cells = 0, n_chunks = 0;
  int m = 0, S = 0;
  size_t off_sys, off_active, off_arn, off_state, off_V, off_z, off_t, off_H, off_cs, off_g, off_y,
      off_h1, off_h2, off_n2, off_part, total;
};

inline size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

Layout plan(int S, int64_t n_cells, int64_t n_chunks, int m) {
  Layout L;
  L.n_cells = n_cells;
  L.n_chunks = n_chunks;
  L.m = m;
  L.S = S;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    size_t at = o;
    o = align_up(o + bytes);
    return at;
  };
  const size_t vec = (size_t)n_cells * 8 * sizeof(double);
  L.off_sys = take(sizeof(Sys) * S);
  L.off_active = take(sizeof(int) * S);
  L.off_arn = take(sizeof(int) * S);
  L.off_state = take(sizeof(State) * S);
  L.off_V = take(vec * (m + 1));
  L.off_z = take(vec);
  L.off_t = take(vec);
  L.off_H = take(sizeof(double) * 2 * (m + 1) * m * S);
  L.off_cs = take(sizeof(double) * 3 * m * S);
  L.off_g = take(sizeof(double) * 2 * (m + 1) * S);
  L.off_y = take(sizeof(double) * 2 * m * S);
  L.off_h1 = take(sizeof(double) * 2 * (m + 1) * S);
  L.off_h2 = take(sizeof(double) * 2 * (m + 1) * S);
  L.off_n2 = take(sizeof(double) * 2 * S);
  L.off_part = take(sizeof(double) * 2 * (m + 1) * n_chunks);
  L.total = o;
  return L;
}

inline int grid_for(int64_t n, int threads) {
  int64_t blocks = (n + threads - 1) / threads;
  const int64_t cap = 148 * 32;
  if (blocks > cap) blocks = cap;
  return (int)(blocks < 1 ? 1 : blocks);
}

bool build_systems(const eb_batch* b, const eb_instance* host_table, int n_sys,
                   const int32_t* sys_inst, const double* shifts, int adjoint,
                   std::vector<Sys>& out, int64_t& n_cells, int64_t& n_chunks) {
  out.resize(n_sys);
  n_cells = 0;
  n_chunks = 0;
  for (int s = 0; s < n_sys; ++s) {
    const int i = sys_inst ? sys_inst[s] : 0;
    if (i < 0 || i >= b->n_inst) return false;
    const eb_instance& in = host_table ? host_table[i] : b->single;
    Sys& S = out[s];
    S.cell_begin = n_cells;
    S.n_cells = (int64_t)in.M * in.N;
    S.chunk_begin = n_chunks;
    S.jac_cell = in.cell_offset;
    S.M = in.M;
    S.N = in.N;
    S.sr = shifts[2 * s];
    S.si = adjoint ? -shifts[2 * s + 1] : shifts[2 * s + 1];
    n_cells += S.n_cells;
    n_chunks += (S.n_cells + kChunkCells - 1) / kChunkCells;
  }
  return true;
}

}  // namespace gm
}  // namespace eb

using namespace eb;
using namespace eb::gm;

extern "C" {

int64_t eb_gmres_workspace_bytes(const eb_batch* b, const eb_instance* host_table, int n_sys,
                                 const int32_t* sys_inst, int restart) {
  if (!b || n_sys < 1 || restart < 1) return -1;
  std::vector<double> zero(2 * (size_t)n_sys, 0.0);
  std::vector<Sys> sys;
  int64_t n_cells, n_chunks;
  if (!build_systems(b, host_table, n_sys, sys_inst, zero.data(), 0, sys, n_cells, n_chunks))
    return -1;
  return (int64_t)plan(n_sys, n_cells, n_chunks, restart).total;
}

}  // extern "C"

namespace eb {
namespace gm {

// The anchored preconditioner's state (see eb_gmres_solve_anchored): the anchors' ring-LU
// factors, the systems' anchor and column, and the anchors' multi-right-hand-side ring blocks.
struct Anchored {
  int M, N;
  const void* ringlu_ws;
  int64_t ringlu_stride;
  int n_anchors, nr;
  const int* d_sys_anchor;
  const int* d_sys_col;
  int* d_zmap;
  int* d_n_active;
  cuDoubleComplex *Y, *X, *W;
  int64_t mstride;
  std::vector<int> sys_anchor;  // host copy
  std::vector<int> zmap;        // host staging of the active anchors
  void* graph = nullptr;        // the captured sweep (a cudaGraphExec_t), destroyed at the end
};

// The restarted GMRES of eb_gmres_solve with the block-Jacobi preconditioner (ap == nullptr) or
// the anchored ring-LU preconditioner.
int gmres_core(const eb_batch* b, const eb_instance* host_table, const double* J, int n_sys,
               const int32_t* sys_inst, const double* shifts, int adjoint, const double* rhs,
               double* x, const eb_gmres_options* opt, void* workspace, int64_t workspace_bytes,
               eb_gmres_info* info, void* stream, Anchored* ap) {
  if ((reinterpret_cast<uintptr_t>(J) | reinterpret_cast<uintptr_t>(rhs) |
       reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(workspace)) & 15)
    return fail(EB_ERR_ARG, "gmres: arrays must be 16-byte aligned");
  int rc = validate(b);
  if (rc != EB_OK) return rc;
  if (!J || !rhs || !x || !opt || !workspace || !info || !shifts || n_sys < 1)
    return fail(EB_ERR_ARG, "gmres: null argument");
  if (b->n_inst > 1 && !host_table) return fail(EB_ERR_ARG, "gmres: batch needs host_table");
  const int m = opt->restart;
  if (m < 1 || opt->max_iterations < 1 || opt->check_every < 1 || !(opt->tol > 0))
    return fail(EB_ERR_ARG, "gmres: bad options (restart, max_iterations and check_every >= 1, tol > 0)");
  std::vector<Sys> sys;
  int64_t n_cells, n_chunks;
  if (!build_systems(b, host_table, n_sys, sys_inst, shifts, adjoint, sys, n_cells, n_chunks))
    return fail(EB_ERR_ARG, "gmres: system instance index out of range");
  const Layout L = plan(n_sys, n_cells, n_chunks, m);
  if ((int64_t)L.total > workspace_bytes) return fail(EB_ERR_ARG, "gmres: workspace too small");
  cudaStream_t st_ = reinterpret_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  Sys* d_sys = reinterpret_cast<Sys*>(ws + L.off_sys);
  int* d_active = reinterpret_cast<int*>(ws + L.off_active);
  // Arnoldi-active systems: the cycle's active systems whose residual estimate has not yet
  // reached the tolerance; a system that has stops its Arnoldi steps (its basis and
  // Hessenberg columns so far give its update at the end of the cycle)
  int* d_arn = reinterpret_cast<int*>(ws + L.off_arn);
  State* d_state = reinterpret_cast<State*>(ws + L.off_state);
  double* V = reinterpret_cast<double*>(ws + L.off_V);
  double* z = reinterpret_cast<double*>(ws + L.off_z);
  double* t = reinterpret_cast<double*>(ws + L.off_t);
  double* H = reinterpret_cast<double*>(ws + L.off_H);
  double* cs = reinterpret_cast<double*>(ws + L.off_cs);
  double* g = reinterpret_cast<double*>(ws + L.off_g);
  double* y = reinterpret_cast<double*>(ws + L.off_y);
  double* h1 = reinterpret_cast<double*>(ws + L.off_h1);
  double* h2 = reinterpret_cast<double*>(ws + L.off_h2);
  double* n2 = reinterpret_cast<double*>(ws + L.off_n2);
  double* part = reinterpret_cast<double*>(ws + L.off_part);
  const int64_t vstride = n_cells * 8;
  const int part_stride = 2 * (m + 1);
  const int hs = 2 * (m + 1);

  std::vector<int> active(n_sys, 1);
  std::vector<State> hst(n_sys);
  std::memset(hst.data(), 0, sizeof(State) * n_sys);
  if (cudaMemcpyAsync(d_sys, sys.data(), sizeof(Sys) * n_sys, cudaMemcpyHostToDevice, st_) != cudaSuccess ||
      cudaMemcpyAsync(d_active, active.data(), sizeof(int) * n_sys, cudaMemcpyHostToDevice, st_) != cudaSuccess ||
      cudaMemcpyAsync(d_state, hst.data(), sizeof(State) * n_sys, cudaMemcpyHostToDevice, st_) != cudaSuccess)
    return check_launch("gmres setup copy");

  const int gc = grid_for(n_cells, 128);
  const int gs = (n_sys + 127) / 128;
  auto norms2 = [&](const int* flags, const double* w, double* out) {
    k_partial<<<(unsigned)n_chunks, 256, 0, st_>>>(d_sys, n_sys, n_chunks, flags, nullptr, 0, 0,
                                                   w, part, part_stride);
    k_reduce<<<n_sys, 256, 0, st_>>>(d_sys, n_sys, flags, 0, part, part_stride, out, 1);
  };

  // out = P^-1 in (accumulate: out += P^-1 in) for the systems with flags[s]
  auto prec = [&](const int* flags, const double* in, double* out, int accumulate) {
    if (!ap) {
      k_prec<<<gc, 128, 0, st_>>>(d_sys, n_sys, n_cells, flags, J, adjoint, in, out,
                                  accumulate);
      return EB_OK;
    }
    return rl::anchored_apply(ap->M, ap->N, ap->ringlu_ws, ap->ringlu_stride, ap->n_anchors,
                              ap->nr, n_sys, ap->d_sys_anchor, ap->d_sys_col, flags,
                              ap->d_zmap, ap->d_n_active, ap->Y, ap->X, ap->W, ap->mstride, in,
                              out, (int64_t)ap->M * ap->N * 8, accumulate, &ap->graph, st_);
  };
  // the anchored preconditioner works on the anchors that have a system with flags[s]
  auto prec_active = [&](const std::vector<int>& flags) {
    if (!ap) return EB_OK;
    std::vector<char> any(ap->n_anchors, 0);
    for (int s = 0; s < n_sys; ++s)
      if (flags[s]) any[ap->sys_anchor[s]] = 1;
    ap->zmap.clear();
    for (int a = 0; a < ap->n_anchors; ++a)
      if (any[a]) ap->zmap.push_back(a);
    const int n_act = (int)ap->zmap.size();
    ap->zmap.push_back(n_act);  // the count goes to d_n_active
    if (cudaMemcpyAsync(ap->d_zmap, ap->zmap.data(), sizeof(int) * n_act, cudaMemcpyHostToDevice,
                        st_) != cudaSuccess ||
        cudaMemcpyAsync(ap->d_n_active, &ap->zmap[n_act], sizeof(int), cudaMemcpyHostToDevice,
                        st_) != cudaSuccess ||
        cudaStreamSynchronize(st_) != cudaSuccess)
      return check_launch("gmres anchors");
    return EB_OK;
  };

  // ||b|| (kept in n2[S + s]) and the initial residual r = b - A x0 with x0 = 0.
  norms2(d_active, rhs, n2 + n_sys);
  if (!opt->use_initial_guess) cudaMemsetAsync(x, 0, sizeof(double) * 8 * n_cells, st_);
  k_op<<<gc, 128, 0, st_>>>(d_sys, n_sys, n_cells, d_active, J, adjoint, x, rhs, V);
  norms2(d_active, V, n2);

  std::vector<double> hn2(2 * n_sys);
  std::vector<int> arn(n_sys, 0);
  int total_iters = 0;
  int status = EB_OK;
  int cycles = 0;
  for (;;) {
    // convergence test on the true residual
    if (cudaMemcpyAsync(hn2.data(), n2, sizeof(double) * 2 * n_sys, cudaMemcpyDeviceToHost, st_) != cudaSuccess ||
        cudaStreamSynchronize(st_) != cudaSuccess)
      return check_launch("gmres residual read");
    int n_active = 0;
    bool bad = false;
    for (int s = 0; s < n_sys; ++s) {
      const double r = std::sqrt(hn2[s]), bn = std::sqrt(hn2[n_sys + s]);
      info[s].rel_residual = bn > 0 ? r / bn : r;
      if (!std::isfinite(r)) {
        bad = true;
        active[s] = 0;
      } else if (active[s] && r <= opt->tol * bn) {
        active[s] = 0;
      }
      n_active += active[s];
    }
    if (bad) status = EB_ERR_NAN;
    if (n_active == 0) break;
    if (total_iters >= opt->max_iterations) {
      status = status == EB_OK ? EB_ERR_NOCONV : status;
      break;
    }
    cudaMemcpyAsync(d_active, active.data(), sizeof(int) * n_sys, cudaMemcpyHostToDevice, st_);
    arn = active;
    cudaMemcpyAsync(d_arn, arn.data(), sizeof(int) * n_sys, cudaMemcpyHostToDevice, st_);
    if ((rc = prec_active(arn)) != EB_OK) return rc;
    ++cycles;
    k_cycle_start<<<gs, 128, 0, st_>>>(n_sys, d_active, m, n2, g, d_state);
    k_scale<<<gc, 128, 0, st_>>>(d_sys, n_sys, n_cells, d_active, d_state, V);
    int j = 0;
    for (; j < m && total_iters < opt->max_iterations; ++j, ++total_iters) {
      double* vj = V + (int64_t)j * vstride;
      double* w = V + (int64_t)(j + 1) * vstride;
      if ((rc = prec(d_arn, vj, z, 0)) != EB_OK) return rc;
      k_op<<<gc, 128, 0, st_>>>(d_sys, n_sys, n_cells, d_arn, J, adjoint, z, nullptr, w);
      for (int pass = 0; pass < 2; ++pass) {
        double* h = pass == 0 ? h1 : h2;
        k_partial<<<(unsigned)n_chunks, 256, 0, st_>>>(d_sys, n_sys, n_chunks, d_arn, V,
                                                       vstride, j + 1, w, part, part_stride);
        k_reduce<<<n_sys, 256, 0, st_>>>(d_sys, n_sys, d_arn, j + 1, part, part_stride, h, hs);
        k_project<<<gc, 128, 0, st_>>>(d_sys, n_sys, n_cells, d_arn, V, vstride, j + 1, h, hs, w);
      }
      norms2(d_arn, w, n2);
      k_givens<<<gs, 128, 0, st_>>>(n_sys, d_arn, j, m, h1, h2, hs, n2, H, cs, g, d_state);
      k_scale<<<gc, 128, 0, st_>>>(d_sys, n_sys, n_cells, d_arn, d_state, w);
      if (((j + 1) % opt->check_every) == 0 || j + 1 == m) {
        if (cudaMemcpyAsync(hst.data(), d_state, sizeof(State) * n_sys, cudaMemcpyDeviceToHost, st_) != cudaSuccess ||
            cudaStreamSynchronize(st_) != cudaSuccess)
          return check_launch("gmres state read");
        // systems whose estimate has reached the tolerance (or that broke down) stop here
        bool all_done = true, changed = false;
        for (int s = 0; s < n_sys; ++s) {
          if (!arn[s]) continue;
          const double bn = std::sqrt(hn2[n_sys + s]);
          if (hst[s].breakdown || hst[s].est <= 0.5 * opt->tol * bn) {
            arn[s] = 0;
            changed = true;
          } else {
            all_done = false;
          }
        }
        if (all_done) {
          ++j;
          ++total_iters;
          break;
        }
        if (changed) {
          cudaMemcpyAsync(d_arn, arn.data(), sizeof(int) * n_sys, cudaMemcpyHostToDevice, st_);
          if ((rc = prec_active(arn)) != EB_OK) return rc;
        }
      }
    }
    // x += P^-1 (V y) for every system of the cycle (each with its own number of steps), then
    // the true residual
    if (ap && (rc = prec_active(active)) != EB_OK) return rc;
    k_backsolve<<<gs, 128, 0, st_>>>(n_sys, d_active, m, H, g, y, d_state);
    k_combine<<<gc, 128, 0, st_>>>(d_sys, n_sys, n_cells, d_active, V, vstride, m, y, d_state, t);
    if ((rc = prec(d_active, t, x, 1)) != EB_OK) return rc;
    k_op<<<gc, 128, 0, st_>>>(d_sys, n_sys, n_cells, d_active, J, adjoint, x, rhs, V);
    norms2(d_active, V, n2);
    rc = check_launch("gmres cycle");
    if (rc != EB_OK) return rc;
  }
  if (cudaMemcpyAsync(hst.data(), d_state, sizeof(State) * n_sys, cudaMemcpyDeviceToHost, st_) != cudaSuccess ||
      cudaStreamSynchronize(st_) != cudaSuccess)
    return check_launch("gmres final read");
  for (int s = 0; s < n_sys; ++s) {
    info[s].iterations = hst[s].iters;
    info[s].cycles = cycles;
    info[s].converged = info[s].rel_residual <= opt->tol ? 1 : 0;
  }
  if (status != EB_OK) {
    return fail(status, status == EB_ERR_NAN ? "gmres: non-finite residual"
                                             : "gmres: iteration limit reached");
  }
  return EB_OK;
}

// Bytes of the anchored preconditioner's auxiliary buffer (anchor map and count, systems'
// anchors and columns, three ring-block sets of n_anchors x M x 4N x nr complex).
struct AuxLayout {
  size_t off_zmap, off_nact, off_sa, off_sc, off_Y, off_X, off_W, total;
  int64_t mstride;
};
AuxLayout aux_plan(int M, int N, int n_sys, int n_anchors, int nr) {
  AuxLayout A;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o = (o + bytes + 255) & ~(size_t)255;
    return at;
  };
  A.mstride = (int64_t)M * 4 * N * nr;
  A.off_zmap = take(sizeof(int) * (size_t)n_anchors);
  A.off_nact = take(sizeof(int));
  A.off_sa = take(sizeof(int) * (size_t)n_sys);
  A.off_sc = take(sizeof(int) * (size_t)n_sys);
  const size_t blocks = sizeof(cuDoubleComplex) * (size_t)A.mstride * n_anchors;
  A.off_Y = take(blocks);
  A.off_X = take(blocks);
  A.off_W = take(blocks);
  A.total = o;
  return A;
}

}  // namespace gm
}  // namespace eb

extern "C" {

int eb_gmres_solve(const eb_batch* b, const eb_instance* host_table, const double* J, int n_sys,
                   const int32_t* sys_inst, const double* shifts, int adjoint,
                   const double* rhs, double* x, const eb_gmres_options* opt, void* workspace,
                   int64_t workspace_bytes, eb_gmres_info* info, void* stream) {
  return eb::gm::gmres_core(b, host_table, J, n_sys, sys_inst, shifts, adjoint, rhs, x, opt,
                            workspace, workspace_bytes, info, stream, nullptr);
}

int64_t eb_gmres_anchored_aux_bytes(int M, int N, int n_sys, int n_anchors,
                                    const int32_t* sys_anchor) {
  if (M < 1 || N < 1 || n_sys < 1 || n_anchors < 1 || !sys_anchor) return -1;
  std::vector<int> count(n_anchors, 0);
  int nr = 0;
  for (int s = 0; s < n_sys; ++s) {
    if (sys_anchor[s] < 0 || sys_anchor[s] >= n_anchors) return -1;
    nr = std::max(nr, ++count[sys_anchor[s]]);
  }
  if (nr > 8) return -1;
  return (int64_t)eb::gm::aux_plan(M, N, n_sys, n_anchors, nr).total;
}

int eb_gmres_solve_anchored(const eb_batch* b, const double* J, int n_sys, const double* shifts,
                            const double* rhs, double* x, const eb_gmres_options* opt,
                            int n_anchors, const int32_t* sys_anchor, const void* ringlu_workspace,
                            int64_t ringlu_stride, void* workspace, int64_t workspace_bytes,
                            void* aux, int64_t aux_bytes, eb_gmres_info* info, void* stream) {
  using namespace eb::gm;
  int rc = validate(b);
  if (rc != EB_OK) return rc;
  if (b->n_inst != 1 || b->d_table)
    return fail(EB_ERR_ARG, "gmres anchored: single instance only");
  if (!sys_anchor || !ringlu_workspace || !aux || n_anchors < 1 || n_sys < 1)
    return fail(EB_ERR_ARG, "gmres anchored: null argument");
  const int M = b->single.M, N = b->single.N;
  const int64_t ws_need = eb_ringlu_workspace_bytes(M, N);
  if (ws_need < 0 || ringlu_stride < ws_need || ringlu_stride % 256 != 0 ||
      reinterpret_cast<uintptr_t>(ringlu_workspace) % 256 != 0)
    return fail(EB_ERR_ARG, "gmres anchored: bad ring-LU workspace or stride");
  std::vector<int> count(n_anchors, 0), col(n_sys, 0), sa(n_sys, 0);
  int nr = 0;
  for (int s = 0; s < n_sys; ++s) {
    if (sys_anchor[s] < 0 || sys_anchor[s] >= n_anchors)
      return fail(EB_ERR_ARG, "gmres anchored: anchor index out of range");
    sa[s] = sys_anchor[s];
    col[s] = count[sa[s]]++;
    nr = std::max(nr, count[sa[s]]);
  }
  if (nr > 8) return fail(EB_ERR_ARG, "gmres anchored: more than 8 systems on one anchor");
  const AuxLayout A = aux_plan(M, N, n_sys, n_anchors, nr);
  if ((int64_t)A.total > aux_bytes || reinterpret_cast<uintptr_t>(aux) % 256 != 0)
    return fail(EB_ERR_ARG, "gmres anchored: auxiliary buffer too small or not 256-byte aligned");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  char* ab = static_cast<char*>(aux);
  Anchored ap;
  ap.M = M;
  ap.N = N;
  ap.ringlu_ws = ringlu_workspace;
  ap.ringlu_stride = ringlu_stride;
  ap.n_anchors = n_anchors;
  ap.nr = nr;
  ap.d_sys_anchor = reinterpret_cast<const int*>(ab + A.off_sa);
  ap.d_sys_col = reinterpret_cast<const int*>(ab + A.off_sc);
  ap.d_zmap = reinterpret_cast<int*>(ab + A.off_zmap);
  ap.d_n_active = reinterpret_cast<int*>(ab + A.off_nact);
  ap.Y = reinterpret_cast<cuDoubleComplex*>(ab + A.off_Y);
  ap.X = reinterpret_cast<cuDoubleComplex*>(ab + A.off_X);
  ap.W = reinterpret_cast<cuDoubleComplex*>(ab + A.off_W);
  ap.mstride = A.mstride;
  ap.sys_anchor = sa;
  // columns an anchor does not use stay zero through the sweeps
  if (cudaMemsetAsync(ab + A.off_Y, 0, A.total - A.off_Y, st) != cudaSuccess ||
      cudaMemcpyAsync(ab + A.off_sa, sa.data(), sizeof(int) * n_sys, cudaMemcpyHostToDevice,
                      st) != cudaSuccess ||
      cudaMemcpyAsync(ab + A.off_sc, col.data(), sizeof(int) * n_sys, cudaMemcpyHostToDevice,
                      st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return check_launch("gmres anchored setup");
  rc = gmres_core(b, nullptr, J, n_sys, nullptr, shifts, 0, rhs, x, opt, workspace,
                  workspace_bytes, info, stream, &ap);
  if (ap.graph) cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(ap.graph));
  return rc;
}

}  // extern "C"

// ---- scratch-free variant ----------------------------------------------------------------
//
// Some callers cannot allocate device memory themselves: host programs whose device memory is
// owned by another runtime's pool (a second allocator would break its budget), or solver loops
// that run under a no-allocation-after-start-up rule. For them eb_gmres_solve_noalloc runs the
// same solve with its workspace in this fixed device array. Every GPU that loads the library
// holds the array until the process exits; all calls share it.

namespace eb {
namespace gm {

constexpr size_t kStaticScratchBytes = (size_t)48 << 20;  // 48 MiB
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_static_mutex;
void* g_static_ptr[128] = {};

// Device address of the static scratch on the current device, looked up once per device.
int static_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128)
    return fail(EB_ERR_CUDA, "gmres_noalloc: no current device");
  std::lock_guard<std::mutex> lock(g_static_mutex);
  if (!g_static_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p) {
      g_last_error = std::string("gmres_noalloc: cudaGetSymbolAddress failed: ") +
                     cudaGetErrorString(e);
      return EB_ERR_CUDA;
    }
    g_static_ptr[dev] = p;
  }
  *out = g_static_ptr[dev];
  return EB_OK;
}

}  // namespace gm
}  // namespace eb

extern "C" int eb_gmres_solve_noalloc(const eb_batch* b, const eb_instance* host_table,
                                      const double* J, int n_sys, const int32_t* sys_inst,
                                      const double* shifts, int adjoint, const double* rhs,
                                      double* x, const eb_gmres_options* opt,
                                      eb_gmres_info* info, void* stream) {
  if (!b || !opt || n_sys < 1) return fail(EB_ERR_ARG, "gmres_noalloc: null argument");
  if ((reinterpret_cast<uintptr_t>(J) | reinterpret_cast<uintptr_t>(rhs) |
       reinterpret_cast<uintptr_t>(x)) & 15)
    return fail(EB_ERR_ARG, "gmres_noalloc: arrays must be 16-byte aligned");
  if (opt->restart < 1 || opt->max_iterations < 1 || opt->check_every < 1 || !(opt->tol > 0))
    return fail(EB_ERR_ARG, "gmres_noalloc: bad options (restart, max_iterations and check_every >= 1, tol > 0)");
  const int64_t need = eb_gmres_workspace_bytes(b, host_table, n_sys, sys_inst, opt->restart);
  if (need < 0) return fail(EB_ERR_ARG, "gmres_noalloc: invalid systems");
  if (need > (int64_t)kStaticScratchBytes) {
    g_last_error = "gmres_noalloc: the systems need " + std::to_string(need) +
                   " bytes of workspace, more than the 48 MiB static scratch; use "
                   "eb_gmres_solve with a caller-provided workspace";
    return EB_ERR_ARG;
  }
  void* scratch = nullptr;
  const int rc = static_scratch(&scratch);
  if (rc != EB_OK) return rc;
  return eb_gmres_solve(b, host_table, J, n_sys, sys_inst, shifts, adjoint, rhs, x, opt, scratch,
                        (int64_t)kStaticScratchBytes, info, stream);
}
