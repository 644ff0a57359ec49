// Tiled FP64 residual kernel: R(Ma, U, X, V) for packed instances (eb_compute_odes), and the
// same kernel in one-component dual numbers for the matrix-free forward tangent
// (eb_apply_odes_tangent).
//
// One CTA computes a tile of kTM x kTN cells (radial x angular) of one instance:
//  1. it stages the tile's states with a two-cell halo (the reach of the nine-point cross
//     stencil, periodic in the angular index) and the tile's vertices and vertex velocities in
//     shared memory, with coalesced 16-byte loads (consecutive threads = consecutive radial
//     cells = consecutive 32-byte states);
//  2. per staged state it computes once what every face needs: 1/rho, the pressure and the
//     speed of sound (the reference recomputes these for each use, f90:128-171);
//  3. per state it computes the two pressure sensors |p_a - 2 p_b + p_c| / (p_a + 2 p_b + p_c)
//     centred on the state along the angular and the radial direction (each face's JST sensor
//     is the max_c of the sensors centred on its two cells, f90:208-211; the wall and
//     far-field rows use their ghost states as the missing neighbour);
//  4. each face is evaluated once for its two cells: the reference evaluates it twice, once in
//     each cell's orientation, and the two evaluations share the central and ALE parts and the
//     differences (negated), which are formed once; the asymmetric max_c decisions
//     (f90:111-120) are taken per orientation. Faces whose two evaluations use different
//     stencils (next to the wall and the far field, f90:401-436) are evaluated per cell. Each
//     cell then writes -(F_b + F_f + F_i + F_o) / area (f90:370-436).
// Results agree with the reference to the rounding of the reordered arithmetic (<= 1e-12
// relative); every branch (boundary cases, max_c tolerance) follows the reference.
//
// The kernel is a template on its scalar type T. T = double is the residual. T = Dual<double,
// 1> is the tangent along a complex direction (dU, dX, dV, dMa): CTA 2 t + h of a tile t
// carries part h (0: real, 1: imaginary) of the direction as the dual component, with abs_c /
// max_c (f90:97-120) taking their branches from the values as the reference's complex step
// does.

#include "common.cuh"
#include "tile_faces.cuh"

namespace eb {

constexpr int kTM = 32;                       // radial cells per tile (warp-contiguous)
constexpr int kTN = 8;                        // angular cells per tile
constexpr int kThreads = kTM * kTN;           // one thread per cell
constexpr int kSR = kTM + 4;                  // staged rows (radial halo 2)
constexpr int kSC = kTN + 4;                  // staged columns (angular halo 2)
constexpr int kStaged = kSR * kSC;
constexpr int kVR = kTM + 1, kVC = kTN + 1;   // staged vertices
constexpr int kVerts = kVR * kVC;

using D1 = Dual<double, 1>;

template <class T>
struct TileSmem {
  T rho[kStaged], j1[kStaged], j2[kStaged], e[kStaged];
  T p[kStaged], ir[kStaged], cs[kStaged];
  T s_ang[kTM * (kTN + 2)];   // angular sensor centred on (r, c), c in [-1, kTN]
  T s_rad[(kTM + 2) * kTN];   // radial sensor centred on (r, c), r in [-1, kTM]
  T x[kVerts], z[kVerts], vx[kVerts], vz[kVerts];
  T ff[4][kTN][kTM];          // flux through face f of each cell (from its f neighbour's face)
  T fo[4][kTN][kTM];          // flux through face o of each cell (from its o neighbour's face)
};

__device__ __forceinline__ int sidx(int r, int c) { return (c + 2) * kSR + (r + 2); }
__device__ __forceinline__ int vidx(int r, int c) { return c * kVR + r; }

template <class T>
__device__ __forceinline__ St<T> staged(const TileSmem<T>& S, int i) {
  return St<T>{S.rho[i], S.j1[i], S.j2[i], S.e[i], S.p[i], S.ir[i], S.cs[i]};
}

// Phases 2-4 of a tile whose states (with derived quantities) and vertices are staged in S:
// sensors, faces, and the residual (or its tangent part) of the tile's cells. Every thread of
// the CTA calls it.
template <class T>
__device__ __forceinline__ void tile_compute(TileSmem<T>& S, const Instance& in, const T& mach,
                                             int m0, int n0, double* R, double* dR, int h) {
  const int M = in.M, N = in.N;
  const int tid = threadIdx.x;
  // 2. sensors centred on each needed state: every thread evaluates one angular and one radial
  // sensor, and the kAngX + kRadX left over go to warps 2-4, so that no warp evaluates more
  // than three (the phase ends at a barrier: its slowest warp sets its time)
  constexpr int kAng = kTM * (kTN + 2), kRad = (kTM + 2) * kTN;
  constexpr int kAngX = kAng - kThreads, kRadX = kRad - kThreads, kX0 = 64;
  static_assert(kAngX >= 0 && kRadX >= 0 && kX0 + kAngX + kRadX <= kThreads, "sensor split");
  auto angular_sensor = [&](int e) {
    const int r = e % kTM, c = e / kTM - 1;
    S.s_ang[e] = sensor(S.p[sidx(r, c - 1)], S.p[sidx(r, c)], S.p[sidx(r, c + 1)]);
  };
  auto radial_sensor = [&](int e) {
    const int r = e % (kTM + 2) - 1, c = e / (kTM + 2);
    const int m = m0 + r;
    T s = lift<T>(0.0);
    if (m == 0) {  // inner neighbour: the wall ghost of this wall cell (face o, flag 1)
      const T nx = S.z[vidx(r, c + 1)] - S.z[vidx(r, c)];
      const T nz = S.x[vidx(r, c)] - S.x[vidx(r, c + 1)];
      const T gx = (S.vx[vidx(r, c)] + S.vx[vidx(r, c + 1)]) / 2.0;
      const T gz = (S.vz[vidx(r, c)] + S.vz[vidx(r, c + 1)]) / 2.0;
      const St<T> gh = wall_ghost_st(staged(S, sidx(r, c)), nx, nz, gx, gz);
      s = sensor(gh.p, S.p[sidx(r, c)], S.p[sidx(r + 1, c)]);
    } else if (m == M - 1) {  // outer neighbour: the far-field ghost (face i, flag 5)
      const St<T> gh = farfield_ghost_st(staged(S, sidx(r, c)), mach, in);
      s = sensor(gh.p, S.p[sidx(r, c)], S.p[sidx(r - 1, c)]);
    } else if (m > 0 && m < M - 1) {
      s = sensor(S.p[sidx(r - 1, c)], S.p[sidx(r, c)], S.p[sidx(r + 1, c)]);
    }
    S.s_rad[e] = s;
  };
  angular_sensor(tid);
  radial_sensor(tid);
  if (tid >= kX0 && tid < kX0 + kAngX) angular_sensor(kThreads + tid - kX0);
  else if (tid >= kX0 + kAngX && tid < kX0 + kAngX + kRadX)
    radial_sensor(kThreads + tid - kX0 - kAngX);
  __syncthreads();

  // 3. faces. Thread (r, c) evaluates the angular face between cells (r, c-1) and (r, c) and the
  // radial face between cells (r-1, c) and (r, c), each once for both adjacent cells where the
  // reference's two evaluations have the same stencil; its own cell's fluxes (faces b and i)
  // stay in registers, the neighbours' (faces f and o) go to shared memory. The tile's last
  // face column / row is evaluated by threads 0..31 / 32..39 in addition.
  const int r = tid % kTM, c = tid / kTM;
  const int m = m0 + r, n = n0 + c;
  const bool own = m < M && n < N;
  Flux<T> Fb, Fi;
#pragma unroll
  for (int k = 0; k < 4; ++k) Fb.f[k] = Fi.f[k] = lift<T>(0.0);
  auto exists = [&](int rr, int cc) { return rr >= 0 && cc >= 0 && m0 + rr < M && n0 + cc < N; };
  auto angular_face = [&](int fr, int fc, bool want_b, bool want_f, Flux<T>& Fb_out) {
    // l = (fr, fc), r = (fr, fc - 1): face b of (fr, fc) and face f of (fr, fc - 1)
    const T nbx = S.z[vidx(fr, fc)] - S.z[vidx(fr + 1, fc)];
    const T nbz = S.x[vidx(fr + 1, fc)] - S.x[vidx(fr, fc)];
    const T vn = (S.vx[vidx(fr + 1, fc)] + S.vx[vidx(fr, fc)]) / 2.0 * nbx +
                 (S.vz[vidx(fr + 1, fc)] + S.vz[vidx(fr, fc)]) / 2.0 * nbz;
    const T len = sqrt_(nbx * nbx + nbz * nbz);
    Flux<T> F, Fp;
    jst_pair(staged(S, sidx(fr, fc + 1)), staged(S, sidx(fr, fc)), staged(S, sidx(fr, fc - 1)),
             staged(S, sidx(fr, fc - 2)), nbx, nbz, len, vn, S.s_ang[fc * kTM + fr + kTM],
             S.s_ang[(fc - 1) * kTM + fr + kTM], in, F, Fp);
    if (want_b) Fb_out = F;
    if (want_f)
#pragma unroll
      for (int k = 0; k < 4; ++k) S.ff[k][fc - 1][fr] = Fp.f[k];
  };
  auto radial_face = [&](int fr, int fc, bool want_i, bool want_o, Flux<T>& Fi_out) {
    // l = (fr, fc), r = (fr - 1, fc): face i of (fr, fc) and face o of (fr - 1, fc)
    const int fm = m0 + fr;
    const T nix = S.z[vidx(fr, fc + 1)] - S.z[vidx(fr, fc)];
    const T niz = S.x[vidx(fr, fc)] - S.x[vidx(fr, fc + 1)];
    const T gx = (S.vx[vidx(fr, fc)] + S.vx[vidx(fr, fc + 1)]) / 2.0;
    const T gz = (S.vz[vidx(fr, fc)] + S.vz[vidx(fr, fc + 1)]) / 2.0;
    const T vn = gx * nix + gz * niz;
    Flux<T> F, Fp;
#pragma unroll
    for (int k = 0; k < 4; ++k) F.f[k] = Fp.f[k] = lift<T>(0.0);
    if (fm == 0) {  // wall face of cell 0 (flag 1): central flux with the wall ghost
      const St<T> C = staged(S, sidx(fr, fc));
      F = central(C, wall_ghost_st(C, nix, niz, gx, gz), nix, niz, vn);
    } else if (fm == M) {  // far-field face of cell M-1 (flag 5): central flux with the ghost
      const St<T> C = staged(S, sidx(fr - 1, fc));
      Fp = central(C, farfield_ghost_st(C, mach, in), -nix, -niz, -vn);
    } else {
      const T len = sqrt_(nix * nix + niz * niz);
      const St<T> L = staged(S, sidx(fr, fc)), Rs = staged(S, sidx(fr - 1, fc));
      const T sl = S.s_rad[fc * (kTM + 2) + fr + 1], sr = S.s_rad[fc * (kTM + 2) + fr];
      if (fm == 1) {
        // face i of cell 1 (flag 2): central; face o of cell 0 (flag 1): JST whose outer
        // neighbour is the wall ghost of cell 0
        F = central(L, Rs, nix, niz, vn);
        if (want_o) {
          const T wx = S.z[vidx(fr - 1, fc + 1)] - S.z[vidx(fr - 1, fc)];
          const T wz = S.x[vidx(fr - 1, fc)] - S.x[vidx(fr - 1, fc + 1)];
          const T wgx = (S.vx[vidx(fr - 1, fc)] + S.vx[vidx(fr - 1, fc + 1)]) / 2.0;
          const T wgz = (S.vz[vidx(fr - 1, fc)] + S.vz[vidx(fr - 1, fc + 1)]) / 2.0;
          Fp = jst(wall_ghost_st(Rs, wx, wz, wgx, wgz), Rs, L, staged(S, sidx(fr + 1, fc)), -nix,
                   -niz, len, -vn, sr, sl, in);
        }
      } else if (fm == M - 1) {
        // face i of cell M-1 (flag 5): JST whose outer neighbour is the far-field ghost;
        // face o of cell M-2 (flag 4): central
        F = jst(farfield_ghost_st(L, mach, in), L, Rs, staged(S, sidx(fr - 2, fc)), nix, niz,
                len, vn, sl, sr, in);
        Fp = central(Rs, L, -nix, -niz, -vn);
      } else {
        jst_pair(staged(S, sidx(fr + 1, fc)), L, Rs, staged(S, sidx(fr - 2, fc)), nix, niz, len,
                 vn, sl, sr, in, F, Fp);
      }
    }
    if (want_i) Fi_out = F;
    if (want_o)
#pragma unroll
      for (int k = 0; k < 4; ++k) S.fo[k][fc][fr - 1] = Fp.f[k];
  };
  if (m < M && (own || exists(r, c - 1))) angular_face(r, c, own, exists(r, c - 1), Fb);
  if (m <= M && n < N) radial_face(r, c, own, exists(r - 1, c), Fi);
  if (tid < kTM) {
    if (exists(tid, kTN - 1)) {
      Flux<T> unused;
      angular_face(tid, kTN, false, true, unused);
    }
  } else if (tid < kTM + kTN) {
    if (exists(kTM - 1, tid - kTM)) {
      Flux<T> unused;
      radial_face(kTM, tid - kTM, false, true, unused);
    }
  }
  __syncthreads();
  if (!own) return;
  const T bix = S.x[vidx(r, c)], biz = S.z[vidx(r, c)];
  const T fix = S.x[vidx(r, c + 1)], fiz = S.z[vidx(r, c + 1)];
  const T fox = S.x[vidx(r + 1, c + 1)], foz = S.z[vidx(r + 1, c + 1)];
  const T box = S.x[vidx(r + 1, c)], boz = S.z[vidx(r + 1, c)];
  const T area = abs_c((fox - bix) * (boz - fiz) - (foz - biz) * (box - fix)) / 2.0;
  const T ia = 1.0 / area;
  T res[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) res[k] = -(((Fb.f[k] + S.ff[k][c][r]) + Fi.f[k]) + S.fo[k][c][r]) * ia;
  const int64_t g = in.cell_offset + m + (int64_t)M * n;
  if constexpr (std::is_same<T, double>::value) {
    double* out = R + 4 * g;
    reinterpret_cast<double2*>(out)[0] = make_double2(res[0], res[1]);
    reinterpret_cast<double2*>(out)[1] = make_double2(res[2], res[3]);
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) dR[8 * g + 2 * k + h] = res[k].d[0];
    if (R && h == 0) {
      double* out = R + 4 * g;
      reinterpret_cast<double2*>(out)[0] = make_double2(res[0].v, res[1].v);
      reinterpret_cast<double2*>(out)[1] = make_double2(res[2].v, res[3].v);
    }
  }
}

// Scalar of type T from a value and (for the dual) part h of an interleaved complex tangent.
template <class T>
__device__ __forceinline__ T with_part(double v, const double* d, int64_t at, int h) {
  if constexpr (std::is_same<T, double>::value) {
    return v;
  } else {
    T r;
    r.v = v;
    r.d[0] = d ? __ldg(d + at + h) : 0.0;
    return r;
  }
}

// Residual: three CTAs per SM (80 registers, with a few spills); on the 256-instance 129x129
// batch this runs 11 % faster than two CTAs at 120 registers and 4 % faster than four at 64.
// Tangent (twice the shared memory): two CTAs per SM.
template <class T>
constexpr int kMinBlocks = std::is_same<T, double>::value ? 3 : 2;

template <class T>
__global__ void __launch_bounds__(kThreads, kMinBlocks<T>)
k_residual_tiled(Table t, const double* X, const double* V, const double* U, const double* dX,
                 const double* dV, const double* dU, const double* dMa, double* R, double* dR) {
  extern __shared__ __align__(16) unsigned char tile_smem[];
  TileSmem<T>& S = *reinterpret_cast<TileSmem<T>*>(tile_smem);
  const Instance in = t.dev ? t.dev[blockIdx.y] : t.single;
  const int M = in.M, N = in.N;
  // the dual kernel's two parts of a tile are neighbouring CTAs (x = 2 tile + part), so the
  // second finds the tile's inputs in L2 and completes the output sectors the first began
  constexpr bool kDual = !std::is_same<T, double>::value;
  const int h = kDual ? (int)(blockIdx.x & 1) : 0;
  const int tile = kDual ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
  const int tiles_m = (M + kTM - 1) / kTM;
  const int tiles = tiles_m * ((N + kTN - 1) / kTN);
  if (tile >= tiles) return;
  const int m0 = (tile % tiles_m) * kTM, n0 = (tile / tiles_m) * kTN;
  const double* Ui = U + 4 * in.cell_offset;
  const double* Xi = X + 2 * in.vert_offset;
  const double* Vi = V ? V + 2 * in.vert_offset : nullptr;
  const double* dUi = dU ? dU + 8 * in.cell_offset : nullptr;
  const double* dXi = dX ? dX + 4 * in.vert_offset : nullptr;
  const double* dVi = dV ? dV + 4 * in.vert_offset : nullptr;
  const T mach = with_part<T>(in.mach, dMa, 2 * (int64_t)blockIdx.y, h);
  const int tid = threadIdx.x;

  // 1. stage states (cross-shaped halo) and derived quantities, vertices and grid velocities.
  // A thread first issues all of its global loads (at most two staged states and two vertex
  // pairs: kStaged = 432 and kVerts = 297 are below 2 * kThreads), then derives and stores, so
  // its loads are in flight together instead of one round after another. The second-round
  // states go to the highest threads and the second-round vertices to the lowest, so that no
  // warp derives a second state and also stages a second vertex.
  static_assert(kStaged <= 2 * kThreads && kVerts <= 2 * kThreads, "two staging rounds");
  auto state_item = [&](int k) { return k == 0 ? tid : tid + kStaged - kThreads; };
  auto state_valid = [&](int k, int e) { return (k == 0 || e >= kThreads) && e < kStaged; };
  double2 sa[2], sb[2], xv[2], vv[2];
  int64_t sj[2], vj[2];
  bool sval[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int e = state_item(k);
    const int r = e % kSR - 2, c = e / kSR - 2;
    const bool corner = (r < 0 || r >= kTM) && (c < 0 || c >= kTN);
    const int m = m0 + r;
    sval[k] = state_valid(k, e) && !corner && m >= 0 && m < M;
    sa[k] = make_double2(1.0, 0.0);
    sb[k] = make_double2(0.0, 1.0);
    sj[k] = 0;
    if (sval[k]) {
      int n = n0 + c;  // periodic in the angular index: n0 + c lies in [-2, N + kTN + 1]
      while (n < 0) n += N;
      while (n >= N) n -= N;
      sj[k] = m + (int64_t)M * n;
      const double* q = Ui + 4 * sj[k];
      sa[k] = __ldg(reinterpret_cast<const double2*>(q));
      sb[k] = __ldg(reinterpret_cast<const double2*>(q + 2));
    }
    const int ev = tid + k * kThreads;
    xv[k] = make_double2(0.0, 0.0);
    vv[k] = make_double2(0.0, 0.0);
    vj[k] = 0;
    if (ev < kVerts) {
      const int vm = min(m0 + ev % kVR, M), vn = min(n0 + ev / kVR, N);
      vj[k] = vm + (int64_t)(M + 1) * vn;
      xv[k] = __ldg(reinterpret_cast<const double2*>(Xi + 2 * vj[k]));
      if (Vi) vv[k] = __ldg(reinterpret_cast<const double2*>(Vi + 2 * vj[k]));
    }
  }
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int e = state_item(k);
    if (state_valid(k, e)) {
      if (sval[k]) {
        const double* dq = dUi ? dUi + 8 * sj[k] : nullptr;
        const St<T> st = derive<T>(with_part<T>(sa[k].x, dq, 0, h), with_part<T>(sa[k].y, dq, 2, h),
                                   with_part<T>(sb[k].x, dq, 4, h), with_part<T>(sb[k].y, dq, 6, h));
        S.rho[e] = st.rho; S.j1[e] = st.j1; S.j2[e] = st.j2; S.e[e] = st.e;
        S.p[e] = st.p; S.ir[e] = st.ir; S.cs[e] = st.cs;
      } else {  // outside the grid or an unused corner: finite placeholders
        S.rho[e] = lift<T>(1.0); S.j1[e] = lift<T>(0.0); S.j2[e] = lift<T>(0.0);
        S.e[e] = lift<T>(1.0); S.p[e] = lift<T>(1.0); S.ir[e] = lift<T>(1.0);
        S.cs[e] = lift<T>(1.0);
      }
    }
    const int ev = tid + k * kThreads;
    if (ev < kVerts) {
      S.x[ev] = with_part<T>(xv[k].x, dXi, 4 * vj[k], h);
      S.z[ev] = with_part<T>(xv[k].y, dXi, 4 * vj[k] + 2, h);
      S.vx[ev] = with_part<T>(vv[k].x, dVi, 4 * vj[k], h);
      S.vz[ev] = with_part<T>(vv[k].y, dVi, 4 * vj[k] + 2, h);
    }
  }
  __syncthreads();

  tile_compute<T>(S, in, mach, m0, n0, R, dR, h);
}

int launch_residual_tiled(const eb_batch* b, const double* X, const double* V, const double* U,
                          double* R, cudaStream_t stream, int max_tiles) {
  const Table t = make_table(b);
  dim3 grid(max_tiles, b->n_inst);
  if (cudaFuncSetAttribute(k_residual_tiled<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sizeof(TileSmem<double>)) != cudaSuccess)
    return check_launch("compute_odes attribute");
  k_residual_tiled<double><<<grid, kThreads, sizeof(TileSmem<double>), stream>>>(
      t, X, V, U, nullptr, nullptr, nullptr, nullptr, R, nullptr);
  return check_launch("compute_odes");
}

int launch_tangent_tiled(const eb_batch* b, const double* X, const double* V, const double* U,
                         const double* dU, const double* dX, const double* dV, const double* dMa,
                         double* dR, double* R, cudaStream_t stream, int max_tiles) {
  const Table t = make_table(b);
  dim3 grid(2 * max_tiles, b->n_inst);
  if (cudaFuncSetAttribute(k_residual_tiled<D1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sizeof(TileSmem<D1>)) != cudaSuccess)
    return check_launch("apply_odes_tangent attribute");
  k_residual_tiled<D1><<<grid, kThreads, sizeof(TileSmem<D1>), stream>>>(t, X, V, U, dX, dV, dU,
                                                                         dMa, R, dR);
  return check_launch("apply_odes_tangent");
}

int residual_tiles(int M, int N) { return ((M + kTM - 1) / kTM) * ((N + kTN - 1) / kTN); }

}  // namespace eb
