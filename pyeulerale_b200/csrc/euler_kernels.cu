// FP64 stencil kernels and their C ABI (include/euler_b200.h).
//
// One CUDA thread per cell (or per wall face / vertex), grid-stride over the packed cells of
// all instances. Cells of an instance are numbered m + M*n like the reference's Fortran
// arrays, so consecutive threads touch consecutive 32-byte states and every stencil load of
// a warp is a contiguous segment. The instance owning a global cell is found by binary
// search over the instance table (a single instance is passed by value, no table).
//
// Derivatives are forward-mode duals (scalar.cuh) through the same physics source
// (physics.cuh) that produces the residual; they replace the reference's complex-step
// procedures (src/spatial_discretization.f90:552-1256).

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>

#include <algorithm>

#include "common.cuh"

namespace eb {

int launch_residual_tiled(const eb_batch* b, const double* X, const double* V, const double* U,
                          double* R, cudaStream_t stream, int max_tiles);
int launch_tangent_tiled(const eb_batch* b, const double* X, const double* V, const double* U,
                         const double* dU, const double* dX, const double* dV, const double* dMa,
                         double* dR, double* R, cudaStream_t stream, int max_tiles);
int residual_tiles(int M, int N);

thread_local std::string g_last_error;

int fail(int code, const char* msg) {
  g_last_error = msg;
  return code;
}

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return EB_ERR_CUDA;
  }
  return EB_OK;
}

int validate(const eb_batch* b) {
  if (!b) return fail(EB_ERR_ARG, "null batch");
  if (b->n_inst < 1) return fail(EB_ERR_ARG, "batch has no instances");
  if (b->n_inst > 1 && b->d_table == nullptr)
    return fail(EB_ERR_ARG, "batch of several instances needs a device table");
  if (b->n_inst == 1 && b->d_table == nullptr) {
    const eb_instance& s = b->single;
    if (s.M < 4 || s.N < 5) return fail(EB_ERR_ARG, "grid needs M >= 4 and N >= 5 cells");
    if (b->n_cells != (int64_t)s.M * s.N) return fail(EB_ERR_ARG, "n_cells != M*N");
    if (b->n_verts != (int64_t)(s.M + 1) * (s.N + 1)) return fail(EB_ERR_ARG, "n_verts mismatch");
    if (b->n_wall != s.N) return fail(EB_ERR_ARG, "n_wall != N");
  }
  if (b->n_cells <= 0) return fail(EB_ERR_ARG, "n_cells <= 0");
  return EB_OK;
}

// Grid of a per-instance kernel: y = instance (no search of the instance table per thread), x
// covers the largest instance's items (`per_item` threads for each of its cells, or vertices),
// capped so that the whole grid stays within a few waves of 148 SMs. A batch of several
// instances needs max_dim (the largest M or N) and at most 65535 instances.
int per_instance_grid(const eb_batch* b, bool vertices, int per_item, int threads, dim3& grid) {
  int64_t M = b->single.M, N = b->single.N;
  if (b->n_inst > 1 || b->d_table) {
    if (b->max_dim < 5) return fail(EB_ERR_ARG, "batch max_dim must be the largest M or N");
    if (b->n_inst > 65535) return fail(EB_ERR_ARG, "at most 65535 instances per batch");
    M = N = b->max_dim;
  }
  const int64_t items = vertices ? (M + 1) * (N + 1) : M * N;
  int64_t x = (per_item * items + threads - 1) / threads;
  const int64_t cap = std::max<int64_t>(1, (int64_t)148 * 64 * 8 / b->n_inst);
  grid = dim3((unsigned)std::max<int64_t>(1, std::min(x, cap)), (unsigned)b->n_inst);
  return EB_OK;
}

// ---- kernels -----------------------------------------------------------------------------

__global__ void k_free_stream(Table t, int64_t n_cells, double* U) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_cells;
       g += (int64_t)gridDim.x * blockDim.x) {
    const Instance in = t.cell(g);
    const S4<double> fs = free_stream(in.mach, in);
    double2* o = reinterpret_cast<double2*>(U + 4 * g);
    o[0] = make_double2(fs.v[0], fs.v[1]);
    o[1] = make_double2(fs.v[2], fs.v[3]);
  }
}

// Pressure coefficient ((gamma-1)(E - |j|^2/2/rho) - 1) / q, q = gamma Ma^2 / 2, of every cell
// (compute_pressure_coefficients, core.py:1423-1449, in the reference's operation order).
__global__ void k_pressure_coef(Table t, int64_t n_cells, const double* U, double* cp) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_cells;
       g += (int64_t)gridDim.x * blockDim.x) {
    const Instance in = t.cell(g);
    const double q = in.mach * in.mach * kGamma / 2;
    const double2 a = __ldg(reinterpret_cast<const double2*>(U + 4 * g));
    const double2 b = __ldg(reinterpret_cast<const double2*>(U + 4 * g + 2));
    cp[g] = (kGm1 * (b.y - (a.y * a.y + b.x * b.x) / 2. / a.x) - 1.) / q;
  }
}

// Its tangent along complex dU (apply_pressure_coefficients_wrt_states_fwd, core.py:1451-1488):
// (gamma-1)(dE + |j|^2/rho^2/2 drho - (jx djx + jz djz)/rho) / q.
__global__ void k_pressure_coef_fwd(Table t, int64_t n_cells, const double* U, const double* dU,
                                    double* dcp) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_cells;
       g += (int64_t)gridDim.x * blockDim.x) {
    const Instance in = t.cell(g);
    const double q = in.mach * in.mach * kGamma / 2;
    const double rho = U[4 * g], jx = U[4 * g + 1], jz = U[4 * g + 2];
    const double c1 = (jx * jx + jz * jz) / (rho * rho) / 2.;
    const double* d = dU + 8 * g;
#pragma unroll
    for (int part = 0; part < 2; ++part) {  // real, imaginary
      const double drho = d[part], djx = d[2 + part], djz = d[4 + part], de = d[6 + part];
      dcp[2 * g + part] = kGm1 * (de + c1 * drho - (jx * djx + jz * djz) / rho) / q;
    }
  }
}

__global__ void __launch_bounds__(128) k_residual(Table t, int64_t n_cells, const double* X,
                                                  const double* V, const double* U, double* R) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_cells;
       g += (int64_t)gridDim.x * blockDim.x) {
    const Instance in = t.cell(g);
    Plain p;
    load_plain(in, g - in.cell_offset, X, V, U, p);
    Cell<double, double, double, double> c;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      c.x[k] = p.x[k];
      c.w[k] = p.w[k];
    }
#pragma unroll
    for (int s = 0; s < 9; ++s) c.u[s] = p.u[s];
    c.mach = in.mach;
    c.flag = p.flag;
    const S4<double> o = make_ode(c, in);
    double2* out = reinterpret_cast<double2*>(R + 4 * g);
    out[0] = make_double2(o.v[0], o.v[1]);
    out[1] = make_double2(o.v[2], o.v[3]);
  }
}

// Wall forces and force coefficients: one CTA per instance, warp-shuffle reductions of the
// three coefficient sums (core.py:1277-1364; c_d omits the chord, as the reference does).
__global__ void __launch_bounds__(256) k_forces(Table t, const double* X, const double* U,
                                                double* F, double* coef) {
  const Instance in = t.dev ? t.dev[blockIdx.x] : t.single;
  const int M = in.M, N = in.N;
  const double* Xi = X + 2 * in.vert_offset;
  const double* Ui = U + 4 * in.cell_offset;
  double sx = 0.0, sz = 0.0, sm = 0.0;
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    const P2<double> a = ld2(Xi + 2 * ((int64_t)(M + 1) * n));
    const P2<double> b = ld2(Xi + 2 * ((int64_t)(M + 1) * (n + 1)));
    const double p = pressure(ld4(Ui + 4 * ((int64_t)M * n)));
    const P2<double> nv = normal(a, b);
    const double fx = p * nv.x, fz = p * nv.z;
    F[2 * (in.wall_offset + n)] = fx;
    F[2 * (in.wall_offset + n) + 1] = fz;
    const double px = (a.x + b.x) / 2.0 - in.xc, pz = (a.z + b.z) / 2.0 - in.zc;
    sx += fx;
    sz += fz;
    sm += pz * fx - px * fz;
  }
  if (!coef) return;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
    sz += __shfl_xor_sync(0xffffffffu, sz, o);
    sm += __shfl_xor_sync(0xffffffffu, sm, o);
  }
  __shared__ double red[3][8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    red[0][warp] = sx;
    red[1][warp] = sz;
    red[2][warp] = sm;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ax = 0.0, az = 0.0, am = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      ax += red[0][w];
      az += red[1][w];
      am += red[2][w];
    }
    const double q = in.mach * in.mach * kGamma / 2.0;  // dynamic pressure, core.py:144-146
    const int i = t.dev ? blockIdx.x : 0;
    coef[3 * i + 0] = ax / q;
    coef[3 * i + 1] = az / (q * in.chord);
    coef[3 * i + 2] = am / (q * in.chord * in.chord);
  }
}

// ---- Jacobian products -------------------------------------------------------------------

// apply_odes_wrt_states_fwd, f90:825-864: y_c = sum_s J_s(c) x_nb(c,s), with four threads per
// output cell. Thread i takes column i of each of the cell's 4x4 blocks (32 contiguous bytes;
// the four threads of a cell read a block's 128 bytes together, the eight cells of a warp 1 KB)
// and component i of the neighbour's state, and accumulates all four rows; two shuffle steps
// add the four columns' sums and thread i writes row i. Each column's products are summed over
// the slots before the columns are added (the reference sums each block's product row by row),
// a reordering at the rounding level. The loop runs per warp so that every lane reaches the
// shuffles.
__global__ void __launch_bounds__(256) k_apply_states_fwd4(Table t, const double* J,
                                                           const double* x, double* y) {
  const int i = threadIdx.x & 3;
  const Instance in = t.dev ? t.dev[blockIdx.y] : t.single;  // grid y = instance
  const int M = in.M, N = in.N;
  const int64_t cells = (int64_t)M * N;
  const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t wq = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; wq * 8 < cells;
       wq += n_warps) {
    const int64_t local = 8 * wq + ((threadIdx.x & 31) >> 2);
    const bool live = local < cells;
    const int64_t g = in.cell_offset + local;
    double ar[4] = {0.0, 0.0, 0.0, 0.0}, ai[4] = {0.0, 0.0, 0.0, 0.0};
    if (live) {
      const int m = (int)(local % M), n = (int)(local / M);
      const int64_t slot_stride = 16 * (int64_t)M * N;
      const double* Jc = J + 144 * in.cell_offset + 16 * local + 4 * i;
      const double* xi = x + 8 * in.cell_offset + 2 * i;
#pragma unroll
      for (int s = 0; s < 9; ++s) {
        if (!slot_active(s, m, M)) continue;
        const int64_t j = (m + slot_dm(s)) + (int64_t)M * wrap(n + slot_dn(s), N);
        const double2 b01 = __ldg(reinterpret_cast<const double2*>(Jc + slot_stride * s));
        const double2 b23 = __ldg(reinterpret_cast<const double2*>(Jc + slot_stride * s + 2));
        const C2 xv = ldc(xi + 8 * j);
        const double bl[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          ar[r] = fma(bl[r], xv.re, ar[r]);
          ai[r] = fma(bl[r], xv.im, ai[r]);
        }
      }
    }
#pragma unroll
    for (int o = 1; o <= 2; o <<= 1)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        ar[r] += __shfl_xor_sync(0xffffffffu, ar[r], o);
        ai[r] += __shfl_xor_sync(0xffffffffu, ai[r], o);
      }
    if (live) {
      const C2 out = i == 0 ? C2{ar[0], ai[0]}
                   : i == 1 ? C2{ar[1], ai[1]}
                   : i == 2 ? C2{ar[2], ai[2]} : C2{ar[3], ai[3]};
      stc(y + 8 * g + 2 * i, out);
    }
  }
}

// apply_odes_wrt_states_rev, f90:875-918, as a gather over the transposed stencil: the
// output state j collects J_s(c)^T w_c from every cell c whose slot s reads j. Four threads
// per output state: thread i computes component i from column i of each 4x4 block (32
// contiguous bytes; the four threads of a state read the block's 128 bytes together). Few
// registers per thread let many warps keep DRAM loads in flight (one thread per state, with
// the whole block in registers, reached 64 % of the HBM copy bandwidth, this 84 %).
__global__ void __launch_bounds__(256) k_apply_states_rev4(Table t, const double* J,
                                                           const double* w, double* y) {
  const Instance in = t.dev ? t.dev[blockIdx.y] : t.single;  // grid y = instance
  const int M = in.M, N = in.N;
  const int64_t cells = (int64_t)M * N;
  for (int64_t lq = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; lq < 4 * cells;
       lq += (int64_t)gridDim.x * blockDim.x) {
    const int64_t local = lq >> 2;
    const int64_t g = in.cell_offset + local;
    const int i = (int)(lq & 3);
    const int m = (int)(local % M), n = (int)(local / M);
    const int64_t slot_stride = 16 * (int64_t)M * N;
    const double* Ji = J + 144 * in.cell_offset;
    const double* wi = w + 8 * in.cell_offset;
    C2 acc = {0, 0};
#pragma unroll
    for (int s = 0; s < 9; ++s) {
      const int mc = m - slot_dm(s);
      if (mc < 0 || mc >= M || !slot_active(s, mc, M)) continue;
      const int64_t c = mc + (int64_t)M * wrap(n - slot_dn(s), N);
      const double* col = Ji + slot_stride * s + 16 * c + 4 * i;
      const double2 b01 = __ldg(reinterpret_cast<const double2*>(col));
      const double2 b23 = __ldg(reinterpret_cast<const double2*>(col + 2));
      const double bl[4] = {b01.x, b01.y, b23.x, b23.y};
      double tr = 0.0, ti = 0.0;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const C2 wv = ldc(wi + 8 * c + 2 * r);
        tr += wv.re * bl[r];
        ti += wv.im * bl[r];
      }
      acc.re += tr;
      acc.im += ti;
    }
    stc(y + 8 * g + 2 * i, acc);
  }
}

// apply_odes_wrt_vertices_fwd, f90:1005-1032.
__global__ void __launch_bounds__(128) k_apply_vertices_fwd(Table t, const double* J,
                                                            const double* x, double* y) {
  const Instance in = t.dev ? t.dev[blockIdx.y] : t.single;  // grid y = instance
  const int M = in.M, N = in.N;
  const int64_t cells = (int64_t)M * N;
  for (int64_t local = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; local < cells;
       local += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = in.cell_offset + local;
    const int m = (int)(local % M), n = (int)(local / M);
    const int64_t slot_stride = 8 * (int64_t)M * N;
    const double* Jc = J + 32 * in.cell_offset + 8 * local;
    const double* xi = x + 4 * in.vert_offset;
    const int64_t v[4] = {m + (int64_t)(M + 1) * n, m + (int64_t)(M + 1) * (n + 1),
                          m + 1 + (int64_t)(M + 1) * (n + 1), m + 1 + (int64_t)(M + 1) * n};
    C2 acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      // the 4x2 block (64 contiguous bytes) in four 16-byte loads
      const double2* b2 = reinterpret_cast<const double2*>(Jc + slot_stride * k);
      const double2 q0 = __ldg(b2), q1 = __ldg(b2 + 1), q2 = __ldg(b2 + 2), q3 = __ldg(b2 + 3);
      const double blk[8] = {q0.x, q0.y, q1.x, q1.y, q2.x, q2.y, q3.x, q3.y};
      const C2 a = ldc(xi + 4 * v[k]), b = ldc(xi + 4 * v[k] + 2);
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        acc[r].re += blk[r] * a.re + blk[r + 4] * b.re;
        acc[r].im += blk[r] * a.im + blk[r + 4] * b.im;
      }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) stc(y + 8 * g + 2 * r, acc[r]);
  }
}

// apply_odes_wrt_vertices_rev, f90:1044-1072, gathered per vertex (no wrap: the closing
// vertex column n = N is distinct from n = 0, as in the reference).
__global__ void __launch_bounds__(256) k_apply_vertices_rev(Table t, const double* J,
                                                            const double* w, double* y) {
  // Two threads per vertex: thread d computes component d from column d of each 4x2 block
  // (32 contiguous bytes), which keeps the registers per thread low and many loads in flight.
  const Instance in = t.dev ? t.dev[blockIdx.y] : t.single;  // grid y = instance
  const int M = in.M, N = in.N;
  const int64_t verts = (int64_t)(M + 1) * (N + 1);
  for (int64_t lq = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; lq < 2 * verts;
       lq += (int64_t)gridDim.x * blockDim.x) {
    const int64_t local = lq >> 1;
    const int64_t g = in.vert_offset + local;
    const int d = (int)(lq & 1);
    const int m = (int)(local % (M + 1)), n = (int)(local / (M + 1));
    const int64_t slot_stride = 8 * (int64_t)M * N;
    const double* Ji = J + 32 * in.cell_offset;
    const double* wi = w + 8 * in.cell_offset;
    // (corner, cell offset): the vertex is corner BI of (m, n), FI of (m, n-1),
    // FO of (m-1, n-1) and BO of (m-1, n).
    const int cm[4] = {m, m, m - 1, m - 1};
    const int cn[4] = {n, n - 1, n - 1, n};
    C2 acc = {0, 0};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (cm[k] < 0 || cm[k] >= M || cn[k] < 0 || cn[k] >= N) continue;
      const int64_t c = cm[k] + (int64_t)M * cn[k];
      const double* col = Ji + slot_stride * k + 8 * c + 4 * d;
      const double2 b01 = __ldg(reinterpret_cast<const double2*>(col));
      const double2 b23 = __ldg(reinterpret_cast<const double2*>(col + 2));
      const double bl[4] = {b01.x, b01.y, b23.x, b23.y};
      double tr = 0.0, ti = 0.0;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const C2 wv = ldc(wi + 8 * c + 2 * r);
        tr += wv.re * bl[r];
        ti += wv.im * bl[r];
      }
      acc.re += tr;
      acc.im += ti;
    }
    stc(y + 4 * g + 2 * d, acc);
  }
}

// apply_odes_wrt_mach_fwd, f90:604-621.
__global__ void k_apply_mach_fwd(Table t, const double* J, const double* dm, double* y) {
  const Instance in = t.dev ? t.dev[blockIdx.y] : t.single;  // grid y = instance
  const C2 d = ldc(dm + 2 * blockIdx.y);
  const int64_t cells = (int64_t)in.M * in.N;
  for (int64_t local = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; local < cells;
       local += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = in.cell_offset + local;
    const double2 j01 = __ldg(reinterpret_cast<const double2*>(J + 4 * g));
    const double2 j23 = __ldg(reinterpret_cast<const double2*>(J + 4 * g + 2));
    const double jv[4] = {j01.x, j01.y, j23.x, j23.y};
#pragma unroll
    for (int r = 0; r < 4; ++r) stc(y + 8 * g + 2 * r, C2{jv[r] * d.re, jv[r] * d.im});
  }
}

// apply_odes_wrt_mach_rev, f90:632-650: one CTA per instance, warp-shuffle reduction.
__global__ void __launch_bounds__(512) k_apply_mach_rev(Table t, const double* J,
                                                        const double* w, double* dm) {
  const Instance in = t.dev ? t.dev[blockIdx.x] : t.single;
  const int64_t cells = (int64_t)in.M * in.N;
  double sr = 0.0, si = 0.0;
  // 16-byte loads, and the cell loop unrolled so that several cells' loads are in flight
#pragma unroll 4
  for (int64_t c = threadIdx.x; c < cells; c += blockDim.x) {
    const int64_t g = in.cell_offset + c;
    const double2 j01 = __ldg(reinterpret_cast<const double2*>(J + 4 * g));
    const double2 j23 = __ldg(reinterpret_cast<const double2*>(J + 4 * g + 2));
    const double jr[4] = {j01.x, j01.y, j23.x, j23.y};
    double tr = 0.0, ti = 0.0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const double2 wv = __ldg(reinterpret_cast<const double2*>(w + 8 * g + 2 * r));
      tr += wv.x * jr[r];
      ti += wv.y * jr[r];
    }
    sr += tr;
    si += ti;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sr += __shfl_xor_sync(0xffffffffu, sr, o);
    si += __shfl_xor_sync(0xffffffffu, si, o);
  }
  __shared__ double red[2][16];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    red[0][warp] = sr;
    red[1][warp] = si;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      a += red[0][k];
      b += red[1][k];
    }
    const int i = t.dev ? blockIdx.x : 0;
    dm[2 * i] = a;
    dm[2 * i + 1] = b;
  }
}

// apply_forces_wrt_states_fwd, f90:1333-1348.
__global__ void k_apply_forces_states_fwd(Table t, int64_t n_wall, const double* J,
                                          const double* x, double* y) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_wall;
       g += (int64_t)gridDim.x * blockDim.x) {
    const Instance in = t.wall(g);
    const int n = (int)(g - in.wall_offset);
    const double* xv = x + 8 * (in.cell_offset + (int64_t)in.M * n);
    const double* jb = J + 8 * g;
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      double tr = 0.0, ti = 0.0;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        tr += jb[d + 2 * i] * xv[2 * i];
        ti += jb[d + 2 * i] * xv[2 * i + 1];
      }
      stc(y + 4 * g + 2 * d, C2{tr, ti});
    }
  }
}

// apply_forces_wrt_states_rev, f90:1359-1375: only the wall row is non-zero.
__global__ void k_apply_forces_states_rev(Table t, int64_t n_cells, const double* J,
                                          const double* w, double* y) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_cells;
       g += (int64_t)gridDim.x * blockDim.x) {
    const Instance in = t.cell(g);
    const int64_t local = g - in.cell_offset;
    const int m = (int)(local % in.M), n = (int)(local / in.M);
    if (m != 0) {
#pragma unroll
      for (int i = 0; i < 4; ++i) stc(y + 8 * g + 2 * i, C2{0.0, 0.0});
      continue;
    }
    const int64_t f = in.wall_offset + n;
    const double* jb = J + 8 * f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      double tr = 0.0, ti = 0.0;
#pragma unroll
      for (int d = 0; d < 2; ++d) {
        tr += w[4 * f + 2 * d] * jb[d + 2 * i];
        ti += w[4 * f + 2 * d + 1] * jb[d + 2 * i];
      }
      stc(y + 8 * g + 2 * i, C2{tr, ti});
    }
  }
}

// apply_forces_wrt_vertices_fwd, f90:1267-1288.
__global__ void k_apply_forces_vertices_fwd(Table t, int64_t n_wall, const double* J,
                                            const double* x, double* y) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_wall;
       g += (int64_t)gridDim.x * blockDim.x) {
    const Instance in = t.wall(g);
    const int n = (int)(g - in.wall_offset), M = in.M, N = in.N;
    const double* xa = x + 4 * (in.vert_offset + (int64_t)(M + 1) * n);
    const double* xb = x + 4 * (in.vert_offset + (int64_t)(M + 1) * (n + 1));
    const double* J0 = J + 8 * in.wall_offset + 4 * n;
    const double* J1 = J + 8 * in.wall_offset + 4 * (n + (int64_t)N);
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      const double t0r = J0[d] * xa[0] + J0[d + 2] * xa[2];
      const double t0i = J0[d] * xa[1] + J0[d + 2] * xa[3];
      const double t1r = J1[d] * xb[0] + J1[d + 2] * xb[2];
      const double t1i = J1[d] * xb[1] + J1[d + 2] * xb[3];
      stc(y + 4 * g + 2 * d, C2{t0r + t1r, t0i + t1i});
    }
  }
}

// apply_forces_wrt_vertices_rev, f90:1299-1322, gathered per vertex.
__global__ void k_apply_forces_vertices_rev(Table t, int64_t n_verts, const double* J,
                                            const double* w, double* y) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_verts;
       g += (int64_t)gridDim.x * blockDim.x) {
    const Instance in = t.vert(g);
    const int M = in.M, N = in.N;
    const int64_t local = g - in.vert_offset;
    const int m = (int)(local % (M + 1)), n = (int)(local / (M + 1));
    C2 acc[2] = {{0, 0}, {0, 0}};
    if (m == 0) {
      // vertex n is `bi` of wall face n (k = 0) and `fi` of wall face n-1 (k = 1)
      for (int k = 0; k < 2; ++k) {
        const int f = n - k;
        if (f < 0 || f >= N) continue;
        const double* jb = J + 8 * in.wall_offset + 4 * (f + (int64_t)N * k);
        const double* wv = w + 4 * (in.wall_offset + f);
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          acc[e].re += wv[0] * jb[2 * e] + wv[2] * jb[2 * e + 1];
          acc[e].im += wv[1] * jb[2 * e] + wv[3] * jb[2 * e + 1];
        }
      }
    }
    stc(y + 4 * g, acc[0]);
    stc(y + 4 * g + 2, acc[1]);
  }
}

// convert_odes_wrt_states, f90:765-814, one thread per block row. For N >= 5 and M >= 4 the
// nine stencil columns of a row are distinct, so the row holds 5 + [m>=1] + [m>=2] +
// [m<=M-2] + [m<=M-3] blocks, emitted in ascending column order with 1-based indices.
// Eight threads per block row: each finds the row's sorted columns (the same few register
// operations in all eight) and copies its 16-byte pair of every block, so a block moves as one
// coalesced 128-byte access; thread 0 of the row writes the indices and the row pointer.
__global__ void __launch_bounds__(256) k_convert_bsr(int M, int N, const double* J, double* data,
                                                     int32_t* indices, int32_t* indptr) {
  const int64_t rows = (int64_t)M * N;
  const int64_t line = 9 * (int64_t)M - 6;  // blocks per angular line
  const int l = threadIdx.x & 7;
  for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 3; r < rows;
       r += ((int64_t)gridDim.x * blockDim.x) >> 3) {
    const int m = (int)(r % M), n = (int)(r / M);
    // blocks in the rows m' < m of this line
    int64_t before = 5 * (int64_t)m + (m > 1 ? m - 1 : 0) + (m > 2 ? m - 2 : 0) +
                     (m < M - 1 ? m : M - 1) + (m < M - 2 ? m : M - 2);
    int64_t ptr = (int64_t)n * line + before;
    int64_t col[9];
    int slot[9];
    int cnt = 0;
    for (int s = 0; s < 9; ++s) {
      const int mm = m + slot_dm(s);
      if (mm < 0 || mm >= M) continue;
      col[cnt] = mm + (int64_t)M * wrap(n + slot_dn(s), N);
      slot[cnt] = s;
      ++cnt;
    }
    for (int a = 1; a < cnt; ++a) {  // insertion sort by column
      const int64_t c = col[a];
      const int sl = slot[a];
      int b = a - 1;
      while (b >= 0 && col[b] > c) {
        col[b + 1] = col[b];
        slot[b + 1] = slot[b];
        --b;
      }
      col[b + 1] = c;
      slot[b + 1] = sl;
    }
    if (l == 0) {
      indptr[r] = (int32_t)(ptr + 1);
      if (r == rows - 1) indptr[rows] = (int32_t)(ptr + cnt + 1);
    }
    const int64_t slot_stride = 16 * rows;
    for (int a = 0; a < cnt; ++a) {
      const double2* blk = reinterpret_cast<const double2*>(J + slot_stride * slot[a] + 16 * r);
      reinterpret_cast<double2*>(data + 16 * (ptr + a))[l] = __ldg(blk + l);
      if (l == 0) indices[ptr + a] = (int32_t)(col[a] + 1);
    }
  }
}

// y = (A - shift I) x for a BSR matrix with 1-based indices (complex x, y). Eight threads per
// block row: thread l of a row loads the 16-byte pair (2l, 2l + 1) of each 4x4 block (column
// l / 2, rows 2 (l % 2) and 2 (l % 2) + 1, the blocks being column-major), so the eight threads
// read a block's 128 bytes in one coalesced access, and multiplies it by component l / 2 of
// the block column's x; shuffles over the four threads with the same row pair add the columns,
// and threads 0 and 1 of the row write rows 0-1 and 2-3. The loop runs per warp (four rows)
// so that every lane reaches the shuffles.
__global__ void __launch_bounds__(256) k_bsr_spmv(int64_t rows, const double* data,
                                                  const int32_t* indices, const int32_t* indptr,
                                                  double sr, double si, const double* x,
                                                  double* y) {
  const int l = threadIdx.x & 7;
  const int col = l >> 1, q0 = 2 * (l & 1);
  const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t wq = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; wq * 4 < rows;
       wq += n_warps) {
    const int64_t r = 4 * wq + ((threadIdx.x & 31) >> 3);
    const bool live = r < rows;
    double a0r = 0.0, a0i = 0.0, a1r = 0.0, a1i = 0.0;
    const int32_t p0 = live ? indptr[r] - 1 : 0, p1 = live ? indptr[r + 1] - 1 : 0;
    // The first kRowBlocks blocks of the row (all of them for the nine-point stencil pattern):
    // every index, block and x load is issued before the products, so the row costs one
    // dependent load chain instead of one per block.
    constexpr int kRowBlocks = 9;
    double2 b[kRowBlocks], xv[kRowBlocks];
#pragma unroll
    for (int k = 0; k < kRowBlocks; ++k) {
      const int32_t p = p0 + k;
      const bool ok = p < p1;
      const int64_t c = ok ? __ldg(indices + p) - 1 : 0;
      b[k] = ok ? __ldg(reinterpret_cast<const double2*>(data + 16 * (int64_t)p) + l)
                : make_double2(0.0, 0.0);
      xv[k] = ok ? __ldg(reinterpret_cast<const double2*>(x + 8 * c + 2 * col))
                 : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int k = 0; k < kRowBlocks; ++k) {
      a0r = fma(b[k].x, xv[k].x, a0r);
      a0i = fma(b[k].x, xv[k].y, a0i);
      a1r = fma(b[k].y, xv[k].x, a1r);
      a1i = fma(b[k].y, xv[k].y, a1i);
    }
    for (int32_t p = p0 + kRowBlocks; p < p1; ++p) {  // longer rows of a general BSR matrix
      const double2 bp = __ldg(reinterpret_cast<const double2*>(data + 16 * (int64_t)p) + l);
      const int64_t c = __ldg(indices + p) - 1;
      const double2 xp = __ldg(reinterpret_cast<const double2*>(x + 8 * c + 2 * col));
      a0r = fma(bp.x, xp.x, a0r);
      a0i = fma(bp.x, xp.y, a0i);
      a1r = fma(bp.y, xp.x, a1r);
      a1i = fma(bp.y, xp.y, a1i);
    }
#pragma unroll
    for (int o = 2; o <= 4; o <<= 1) {
      a0r += __shfl_xor_sync(0xffffffffu, a0r, o);
      a0i += __shfl_xor_sync(0xffffffffu, a0i, o);
      a1r += __shfl_xor_sync(0xffffffffu, a1r, o);
      a1i += __shfl_xor_sync(0xffffffffu, a1i, o);
    }
    if (live && col == 0) {
      const double2* xr = reinterpret_cast<const double2*>(x + 8 * r + 2 * q0);
      const double2 x0 = xr[0], x1 = xr[1];
      double2* yr = reinterpret_cast<double2*>(y + 8 * r + 2 * q0);
      yr[0] = make_double2(a0r - (sr * x0.x - si * x0.y), a0i - (sr * x0.y + si * x0.x));
      yr[1] = make_double2(a1r - (sr * x1.x - si * x1.y), a1i - (sr * x1.y + si * x1.x));
    }
  }
}

}  // namespace eb

// =========================================================================================
// C ABI
// =========================================================================================
using namespace eb;

extern "C" {

const char* eb_last_error(void) { return g_last_error.c_str(); }
const char* eb_version(void) { return "euler_b200 1.0 (sm_100a, FP64)"; }

int eb_set_free_stream_state(const eb_batch* b, double* U, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(U);
  if (!U) return fail(EB_ERR_ARG, "null states");
  const Table t = make_table(b);
  k_free_stream<<<grid_for(b->n_cells, 256), 256, 0, EB_STREAM(stream)>>>(t, b->n_cells, U);
  return check_launch("set_free_stream_state");
}

int eb_compute_odes(const eb_batch* b, const double* X, const double* V, const double* U,
                    double* R, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, V, U, R);
  if (!X || !U || !R) return fail(EB_ERR_ARG, "null array");
  int dim = b->max_dim;
  if (b->n_inst == 1 && b->d_table == nullptr) dim = std::max(b->single.M, b->single.N);
  if (dim < 5) return fail(EB_ERR_ARG, "batch max_dim must be the largest M or N");
  return launch_residual_tiled(b, X, V, U, R, EB_STREAM(stream), residual_tiles(dim, dim));
}

// The untiled per-cell residual (one thread per cell, every stencil state from global memory).
// Kept as the plain variant for comparison; the tiled kernel serves eb_compute_odes.
int eb_compute_odes_untiled(const eb_batch* b, const double* X, const double* V, const double* U,
                            double* R, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, V, U, R);
  if (!X || !U || !R) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  k_residual<<<grid_for(b->n_cells, 128), 128, 0, EB_STREAM(stream)>>>(t, b->n_cells, X, V, U, R);
  return check_launch("compute_odes_untiled");
}

int eb_compute_forces(const eb_batch* b, const double* X, const double* U, double* F,
                      double* coef, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, U, F);
  if (!X || !U || !F) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  k_forces<<<b->n_inst, 256, 0, EB_STREAM(stream)>>>(t, X, U, F, coef);
  return check_launch("compute_forces");
}

int eb_compute_pressure_coefficients(const eb_batch* b, const double* U, double* cp,
                                     void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(U);
  if (!U || !cp) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  k_pressure_coef<<<grid_for(b->n_cells, 256), 256, 0, EB_STREAM(stream)>>>(t, b->n_cells, U, cp);
  return check_launch("compute_pressure_coefficients");
}

int eb_apply_pressure_coefficients_wrt_states_fwd(const eb_batch* b, const double* U,
                                                  const double* d_states, double* d_cp,
                                                  void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(U, d_states);
  if (!U || !d_states || !d_cp) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  k_pressure_coef_fwd<<<grid_for(b->n_cells, 256), 256, 0, EB_STREAM(stream)>>>(t, b->n_cells, U,
                                                                                 d_states, d_cp);
  return check_launch("apply_pressure_coefficients_wrt_states_fwd");
}

int eb_apply_odes_wrt_mach_fwd(const eb_batch* b, const double* J, const double* d_mach,
                               double* d_odes, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(J, d_mach, d_odes);
  if (!J || !d_mach || !d_odes) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  dim3 grid;
  if (int rc = per_instance_grid(b, false, 1, 256, grid)) return rc;
  k_apply_mach_fwd<<<grid, 256, 0, EB_STREAM(stream)>>>(t, J, d_mach, d_odes);
  return check_launch("apply_odes_wrt_mach_fwd");
}

int eb_apply_odes_wrt_mach_rev(const eb_batch* b, const double* J, const double* d_odes,
                               double* d_mach, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(J, d_odes, d_mach);
  if (!J || !d_mach || !d_odes) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  k_apply_mach_rev<<<b->n_inst, 512, 0, EB_STREAM(stream)>>>(t, J, d_odes, d_mach);
  return check_launch("apply_odes_wrt_mach_rev");
}

int eb_apply_odes_wrt_states_fwd(const eb_batch* b, const double* J, const double* d_states,
                                 double* d_odes, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(J, d_states, d_odes);
  if (!J || !d_states || !d_odes) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  dim3 grid;
  if (int rc = per_instance_grid(b, false, 4, 256, grid)) return rc;
  k_apply_states_fwd4<<<grid, 256, 0, EB_STREAM(stream)>>>(t, J, d_states, d_odes);
  return check_launch("apply_odes_wrt_states_fwd");
}

int eb_apply_odes_wrt_states_rev(const eb_batch* b, const double* J, const double* d_odes,
                                 double* d_states, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(J, d_odes, d_states);
  if (!J || !d_states || !d_odes) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  dim3 grid;
  if (int rc = per_instance_grid(b, false, 4, 256, grid)) return rc;
  k_apply_states_rev4<<<grid, 256, 0, EB_STREAM(stream)>>>(t, J, d_odes, d_states);
  return check_launch("apply_odes_wrt_states_rev");
}

int eb_apply_odes_wrt_vertices_fwd(const eb_batch* b, const double* J,
                                   const double* d_vertices, double* d_odes, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(J, d_vertices, d_odes);
  if (!J || !d_vertices || !d_odes) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  dim3 grid;
  if (int rc = per_instance_grid(b, false, 1, 128, grid)) return rc;
  k_apply_vertices_fwd<<<grid, 128, 0, EB_STREAM(stream)>>>(t, J, d_vertices, d_odes);
  return check_launch("apply_odes_wrt_vertices_fwd");
}

int eb_apply_odes_wrt_vertices_rev(const eb_batch* b, const double* J, const double* d_odes,
                                   double* d_vertices, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(J, d_odes, d_vertices);
  if (!J || !d_vertices || !d_odes) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  dim3 grid;
  if (int rc = per_instance_grid(b, true, 2, 256, grid)) return rc;
  k_apply_vertices_rev<<<grid, 256, 0, EB_STREAM(stream)>>>(t, J, d_odes, d_vertices);
  return check_launch("apply_odes_wrt_vertices_rev");
}

int eb_apply_forces_wrt_states_fwd(const eb_batch* b, const double* J, const double* d_states,
                                   double* d_forces, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(J, d_states, d_forces);
  if (!J || !d_states || !d_forces) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  k_apply_forces_states_fwd<<<grid_for(b->n_wall, 128), 128, 0, EB_STREAM(stream)>>>(
      t, b->n_wall, J, d_states, d_forces);
  return check_launch("apply_forces_wrt_states_fwd");
}

int eb_apply_forces_wrt_states_rev(const eb_batch* b, const double* J, const double* d_forces,
                                   double* d_states, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(J, d_forces, d_states);
  if (!J || !d_states || !d_forces) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  k_apply_forces_states_rev<<<grid_for(b->n_cells, 256), 256, 0, EB_STREAM(stream)>>>(
      t, b->n_cells, J, d_forces, d_states);
  return check_launch("apply_forces_wrt_states_rev");
}

int eb_apply_forces_wrt_vertices_fwd(const eb_batch* b, const double* J,
                                     const double* d_vertices, double* d_forces, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(J, d_vertices, d_forces);
  if (!J || !d_vertices || !d_forces) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  k_apply_forces_vertices_fwd<<<grid_for(b->n_wall, 128), 128, 0, EB_STREAM(stream)>>>(
      t, b->n_wall, J, d_vertices, d_forces);
  return check_launch("apply_forces_wrt_vertices_fwd");
}

int eb_apply_forces_wrt_vertices_rev(const eb_batch* b, const double* J,
                                     const double* d_forces, double* d_vertices, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(J, d_forces, d_vertices);
  if (!J || !d_vertices || !d_forces) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  k_apply_forces_vertices_rev<<<grid_for(b->n_verts, 256), 256, 0, EB_STREAM(stream)>>>(
      t, b->n_verts, J, d_forces, d_vertices);
  return check_launch("apply_forces_wrt_vertices_rev");
}

int eb_apply_odes_tangent(const eb_batch* b, const double* X, const double* V, const double* U,
                          const double* dU, const double* dX, const double* dV,
                          const double* dMa, double* dR, double* R, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, V, U, dU, dX, dV, dMa, dR, R);
  if (!X || !U || !dR) return fail(EB_ERR_ARG, "null array");
  int dim = b->max_dim;
  if (b->n_inst == 1 && b->d_table == nullptr) dim = std::max(b->single.M, b->single.N);
  if (dim < 5) return fail(EB_ERR_ARG, "batch max_dim must be the largest M or N");
  return launch_tangent_tiled(b, X, V, U, dU, dX, dV, dMa, dR, R, EB_STREAM(stream),
                              residual_tiles(dim, dim));
}

int eb_convert_odes_wrt_states(const eb_batch* b, const double* J, double* data,
                               int32_t* indices, int32_t* index_pointers, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(J, data);
  if (b->n_inst != 1 || b->d_table) return fail(EB_ERR_ARG, "convert takes a single instance");
  if (!J || !data || !indices || !index_pointers) return fail(EB_ERR_ARG, "null array");
  const int M = b->single.M, N = b->single.N;
  k_convert_bsr<<<grid_for(8 * (int64_t)M * N, 256), 256, 0, EB_STREAM(stream)>>>(
      M, N, J, data, indices, index_pointers);
  return check_launch("convert_odes_wrt_states");
}

int eb_bsr_shifted_spmv(int64_t n_rows, const double* data, const int32_t* indices,
                        const int32_t* index_pointers, double shift_re, double shift_im,
                        const double* x, double* y, void* stream) {
  if (n_rows <= 0 || !data || !indices || !index_pointers || !x || !y)
    return fail(EB_ERR_ARG, "bad BSR arguments");
  if (((uintptr_t)data | (uintptr_t)x | (uintptr_t)y) & 15)
    return fail(EB_ERR_ARG, "BSR data, x and y must be 16-byte aligned");
  k_bsr_spmv<<<grid_for(8 * n_rows, 256), 256, 0, EB_STREAM(stream)>>>(
      n_rows, data, indices, index_pointers, shift_re, shift_im, x, y);
  return check_launch("bsr_shifted_spmv");
}

}  // extern "C"
