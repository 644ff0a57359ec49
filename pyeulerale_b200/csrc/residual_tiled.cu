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
// Threads map to the cells of the tile's part inside the grid (tm x tn cells, tm = min(kTM, M -
// m0), tn = min(kTN, N - n0)), so that a tile at the grid's outer rows or last columns (129 = 4 x
// 32 + 1 rows leaves a one-row tile) occupies as many warps as it has cells instead of running
// every warp for one valid lane; the full tiles take a path with the extents as constants.
// Results agree with the reference to the rounding of the reordered arithmetic (<= 1e-12
// relative); every branch (boundary cases, max_c tolerance) follows the reference.
//
// The kernel is a template on its scalar type T. T = double is the residual. T = Dual<double,
// 1> is the tangent along a complex direction (dU, dX, dV, dMa): CTA 2 t + h of a tile t
// carries part h (0: real, 1: imaginary) of the direction as the dual component, with abs_c /
// max_c (f90:97-120) taking their branches from the values as the reference's complex step
// does.

#include "autotune.cuh"
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
// Full: the tile lies inside the grid (tm = kTM, tn = kTN as constants). Pre: a thread loads its
// own cell's state and corners once for both of its faces and its area (more registers live
// across the faces) instead of per use; the same arithmetic either way.
template <class T, bool Full, bool Pre>
__device__ __forceinline__ void tile_compute(TileSmem<T>& S, const Instance& in, const T& mach,
                                             int m0, int n0, int tm_in, int tn_in, double* R,
                                             double* dR, int h) {
  const int M = in.M;
  const int tm = Full ? kTM : tm_in, tn = Full ? kTN : tn_in;
  const int tid = threadIdx.x;
  // 2. sensors centred on each needed state: every thread evaluates one angular and one radial
  // sensor, and the ones left over (na + nr - 2 kThreads in a full tile) go to warps 2-4, so
  // that no warp evaluates more than three (the phase ends at a barrier: its slowest warp sets
  // its time)
  const int na = tm * (tn + 2), nr = (tm + 2) * tn;
  const int ax = max(na - kThreads, 0), rx = max(nr - kThreads, 0);
  constexpr int kX0 = 64;
  static_assert(kX0 + (kTM * (kTN + 2) - kThreads) + ((kTM + 2) * kTN - kThreads) <= kThreads,
                "sensor split");
  auto angular_sensor = [&](int e) {
    const int r = e % tm, c = e / tm - 1;
    S.s_ang[(c + 1) * kTM + r] =
        sensor(S.p[sidx(r, c - 1)], S.p[sidx(r, c)], S.p[sidx(r, c + 1)]);
  };
  auto radial_sensor = [&](int e) {
    const int r = e % (tm + 2) - 1, c = e / (tm + 2);
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
    S.s_rad[c * (kTM + 2) + r + 1] = s;
  };
  if (tid < na) angular_sensor(tid);
  if (tid < nr) radial_sensor(tid);
  if (tid >= kX0 && tid < kX0 + ax) angular_sensor(kThreads + tid - kX0);
  else if (tid >= kX0 + ax && tid < kX0 + ax + rx) radial_sensor(kThreads + tid - kX0 - ax);
  __syncthreads();

  // 3. faces. Thread (r, c) evaluates the angular face between cells (r, c-1) and (r, c) and the
  // radial face between cells (r-1, c) and (r, c), each once for both adjacent cells where the
  // reference's two evaluations have the same stencil; its own cell's fluxes (faces b and i)
  // stay in registers, the neighbours' (faces f and o) go to shared memory. The faces past the
  // tile's last column / row (face f of column tn - 1, face o of row tm - 1: interior faces, or
  // the far-field faces of a tile that ends at the grid's outer row) are evaluated by threads
  // 0 .. tm - 1 / tm .. tm + tn - 1 in addition.
  const int r = tid % tm, c = tid / tm;
  const int m = m0 + r;
  const bool own = tid < tm * tn;
  Flux<T> Fb, Fi;
#pragma unroll
  for (int k = 0; k < 4; ++k) Fb.f[k] = Fi.f[k] = lift<T>(0.0);
  // The state of cell (fr, fc) and the vertices (fr, fc), (fr + 1, fc) [angular] or
  // (fr, fc + 1) [radial] come as arguments: a thread loads its own cell's state and corners
  // once for both of its faces and its area.
  struct Vtx {
    T x, z, vx, vz;
  };
  auto vtx = [&](int vr, int vc) {
    const int i = vidx(vr, vc);
    return Vtx{S.x[i], S.z[i], S.vx[i], S.vz[i]};
  };
  auto angular_face = [&](int fr, int fc, bool want_b, bool want_f, Flux<T>& Fb_out,
                          const St<T>& L, const Vtx& v0, const Vtx& v1) {
    // l = (fr, fc), r = (fr, fc - 1): face b of (fr, fc) and face f of (fr, fc - 1);
    // v0 = vertex (fr, fc), v1 = vertex (fr + 1, fc)
    const T nbx = v0.z - v1.z;
    const T nbz = v1.x - v0.x;
    const T vn = (v1.vx + v0.vx) / 2.0 * nbx + (v1.vz + v0.vz) / 2.0 * nbz;
    const T len = sqrt_(nbx * nbx + nbz * nbz);
    Flux<T> F, Fp;
    jst_pair(staged(S, sidx(fr, fc + 1)), L, staged(S, sidx(fr, fc - 1)),
             staged(S, sidx(fr, fc - 2)), nbx, nbz, len, vn, S.s_ang[fc * kTM + fr + kTM],
             S.s_ang[(fc - 1) * kTM + fr + kTM], in, F, Fp);
    if (want_b) Fb_out = F;
    if (want_f)
#pragma unroll
      for (int k = 0; k < 4; ++k) S.ff[k][fc - 1][fr] = Fp.f[k];
  };
  auto radial_face = [&](int fr, int fc, bool want_i, bool want_o, Flux<T>& Fi_out,
                         const St<T>& Lin, const Vtx& v0, const Vtx& v2) {
    // l = (fr, fc), r = (fr - 1, fc): face i of (fr, fc) and face o of (fr - 1, fc);
    // v0 = vertex (fr, fc), v2 = vertex (fr, fc + 1)
    const int fm = m0 + fr;
    const T nix = v2.z - v0.z;
    const T niz = v0.x - v2.x;
    const T gx = (v0.vx + v2.vx) / 2.0;
    const T gz = (v0.vz + v2.vz) / 2.0;
    const T vn = gx * nix + gz * niz;
    // The stencil line (o, c, i, ii) = rows fr + 1, fr, fr - 1, fr - 2, with a ghost state in
    // place of the missing neighbour at the wall and far-field rows (make_ode's five cases,
    // f90:401-436), so that every case is one jst_pair and a warp spanning the boundary rows
    // diverges only in forming its ghost:
    //  fm = 0:     F (face i of cell 0, flag 1) = central(cell 0, its wall ghost)
    //  fm = 1:     F (face i of cell 1, flag 2) = central; F' (face o of cell 0, flag 1) = JST
    //              whose outer neighbour (ii) is the wall ghost of cell 0
    //  fm = M - 1: F (face i of cell M-1, flag 5) = JST whose outer neighbour (o) is the
    //              far-field ghost; F' (face o of cell M-2, flag 4) = central
    //  fm = M:     F' (face o of cell M-1, flag 5) = central(cell M-1, its far-field ghost)
    // A central flux is the pair's shared central/ALE part, its dissipation switched off. Rows
    // outside the grid hold finite placeholders, which the switched-off terms multiply by zero.
    const T len = sqrt_(nix * nix + niz * niz);
    St<T> O = staged(S, sidx(fr + 1, fc)), L = Lin;
    St<T> Rs = staged(S, sidx(fr - 1, fc)), II = staged(S, sidx(fr - 2, fc));
    if (fm == 0) {
      Rs = wall_ghost_st(L, nix, niz, gx, gz);
    } else if (fm == 1) {
      const T wx = S.z[vidx(fr - 1, fc + 1)] - S.z[vidx(fr - 1, fc)];
      const T wz = S.x[vidx(fr - 1, fc)] - S.x[vidx(fr - 1, fc + 1)];
      const T wgx = (S.vx[vidx(fr - 1, fc)] + S.vx[vidx(fr - 1, fc + 1)]) / 2.0;
      const T wgz = (S.vz[vidx(fr - 1, fc)] + S.vz[vidx(fr - 1, fc + 1)]) / 2.0;
      II = wall_ghost_st(Rs, wx, wz, wgx, wgz);
    } else if (fm == M - 1) {
      O = farfield_ghost_st(L, mach, in);
    } else if (fm == M) {
      L = farfield_ghost_st(Rs, mach, in);
    }
    const T sl = S.s_rad[fc * (kTM + 2) + fr + 1], sr = S.s_rad[fc * (kTM + 2) + fr];
    const bool edge = fm == 0 || fm == M;
    Flux<T> F, Fp;
    jst_pair(O, L, Rs, II, nix, niz, len, vn, sl, sr, in, F, Fp, !edge && fm != 1,
             !edge && fm != M - 1);
    if (want_i) Fi_out = F;
    if (want_o)
#pragma unroll
      for (int k = 0; k < 4; ++k) S.fo[k][fc][fr - 1] = Fp.f[k];
  };
  T ia = lift<T>(1.0);
  // make_area (f90:287-293) from the corners bi, fi, fo, bo
  auto inv_area = [&](const T& bix, const T& biz, const T& fix, const T& fiz, const T& box,
                      const T& boz) {
    const T fox = S.x[vidx(r + 1, c + 1)], foz = S.z[vidx(r + 1, c + 1)];
    const T area = abs_c((fox - bix) * (boz - fiz) - (foz - biz) * (box - fix)) / 2.0;
    return T(1.0 / area);
  };
  if (own) {
    if constexpr (Pre) {
      const St<T> L = staged(S, sidx(r, c));
      const Vtx bi = vtx(r, c), bo = vtx(r + 1, c), fi = vtx(r, c + 1);
      angular_face(r, c, true, c > 0, Fb, L, bi, bo);
      radial_face(r, c, true, r > 0, Fi, L, bi, fi);
      ia = inv_area(bi.x, bi.z, fi.x, fi.z, bo.x, bo.z);
    } else {
      angular_face(r, c, true, c > 0, Fb, staged(S, sidx(r, c)), vtx(r, c), vtx(r + 1, c));
      radial_face(r, c, true, r > 0, Fi, staged(S, sidx(r, c)), vtx(r, c), vtx(r, c + 1));
    }
  }
  if (tid < tm) {
    Flux<T> unused;
    angular_face(tid, tn, false, true, unused, staged(S, sidx(tid, tn)), vtx(tid, tn),
                 vtx(tid + 1, tn));
  } else if (tid < tm + tn) {
    Flux<T> unused;
    radial_face(tm, tid - tm, false, true, unused, staged(S, sidx(tm, tid - tm)),
                vtx(tm, tid - tm), vtx(tm, tid - tm + 1));
  }
  __syncthreads();
  if (!own) return;
  if constexpr (!Pre)
    ia = inv_area(S.x[vidx(r, c)], S.z[vidx(r, c)], S.x[vidx(r, c + 1)], S.z[vidx(r, c + 1)],
                  S.x[vidx(r + 1, c)], S.z[vidx(r + 1, c)]);
  const int n = n0 + c;
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

// One tile: staging (phase 1), then phases 2-4.
template <class T, bool Full, bool Pre>
__device__ __forceinline__ void tile_run(TileSmem<T>& S, const Instance& in, const T& mach,
                                         int m0, int n0, int tm_in, int tn_in, const double* Ui,
                                         const double* Xi, const double* Vi, const double* dUi,
                                         const double* dXi, const double* dVi, double* R,
                                         double* dR, int h) {
  const int M = in.M, N = in.N;
  const int tid = threadIdx.x;

  // 1. stage states (cross-shaped halo) and derived quantities, vertices and grid velocities.
  // A thread first issues all of its global loads (at most two staged states and two vertex
  // pairs: kStaged = 432 and kVerts = 297 are below 2 * kThreads), then derives and stores, so
  // its loads are in flight together instead of one round after another. The second-round
  // states go to the highest threads and the second-round vertices to the lowest, so that no
  // warp derives a second state and also stages a second vertex. A partial tile stages its
  // (tm + 4) x (tn + 4) states and (tm + 1) x (tn + 1) vertices at their places in the full
  // tile's layout; the places it leaves unwritten are read by none of its faces.
  static_assert(kStaged <= 2 * kThreads && kVerts <= 2 * kThreads, "two staging rounds");
  const int tm = Full ? kTM : tm_in, tn = Full ? kTN : tn_in;
  const int sr = tm + 4, ns = sr * (tn + 4), vr = tm + 1, nv = vr * (tn + 1);
  auto state_item = [&](int k) { return k == 0 ? tid : tid + ns - kThreads; };
  auto state_valid = [&](int k, int e) { return (k == 0 || e >= kThreads) && e < ns; };
  double2 sa[2], sb[2], xv[2], vv[2];
  int64_t sj[2], vj[2];
  bool sval[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int e = state_item(k);
    const int r = e % sr - 2, c = e / sr - 2;
    const bool corner = (r < 0 || r >= tm) && (c < 0 || c >= tn);
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
    if (ev < nv) {  // vm <= M, vn <= N
      const int vm = m0 + ev % vr, vn = n0 + ev / vr;
      vj[k] = vm + (int64_t)(M + 1) * vn;
      xv[k] = __ldg(reinterpret_cast<const double2*>(Xi + 2 * vj[k]));
      if (Vi) vv[k] = __ldg(reinterpret_cast<const double2*>(Vi + 2 * vj[k]));
    }
  }
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int e = state_item(k);
    if (state_valid(k, e)) {
      const int i = sidx(e % sr - 2, e / sr - 2);
      if (sval[k]) {
        const double* dq = dUi ? dUi + 8 * sj[k] : nullptr;
        const St<T> st = derive<T>(with_part<T>(sa[k].x, dq, 0, h), with_part<T>(sa[k].y, dq, 2, h),
                                   with_part<T>(sb[k].x, dq, 4, h), with_part<T>(sb[k].y, dq, 6, h));
        S.rho[i] = st.rho; S.j1[i] = st.j1; S.j2[i] = st.j2; S.e[i] = st.e;
        S.p[i] = st.p; S.ir[i] = st.ir; S.cs[i] = st.cs;
      } else {  // outside the grid or an unused corner: finite placeholders
        S.rho[i] = lift<T>(1.0); S.j1[i] = lift<T>(0.0); S.j2[i] = lift<T>(0.0);
        S.e[i] = lift<T>(1.0); S.p[i] = lift<T>(1.0); S.ir[i] = lift<T>(1.0);
        S.cs[i] = lift<T>(1.0);
      }
    }
    const int ev = tid + k * kThreads;
    if (ev < nv) {
      const int i = vidx(ev % vr, ev / vr);
      S.x[i] = with_part<T>(xv[k].x, dXi, 4 * vj[k], h);
      S.z[i] = with_part<T>(xv[k].y, dXi, 4 * vj[k] + 2, h);
      S.vx[i] = with_part<T>(vv[k].x, dVi, 4 * vj[k], h);
      S.vz[i] = with_part<T>(vv[k].y, dVi, 4 * vj[k] + 2, h);
    }
  }
  __syncthreads();

  tile_compute<T, Full, Pre>(S, in, mach, m0, n0, tm_in, tn_in, R, dR, h);
}

// Residual: three CTAs per SM (80 registers, with a few spills); on the 256-instance 129x129
// batch this runs 11 % faster than two CTAs at 120 registers and 4 % faster than four at 64.
// Tangent (twice the shared memory): two CTAs per SM.
template <class T>
constexpr int kMinBlocks = std::is_same<T, double>::value ? 3 : 2;

// Pre: see tile_compute (for the residual two launch variants of identical results, chosen by
// the autotuner; the tangent uses Pre = false).
template <class T, bool Pre>
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
  const int tm = min(kTM, M - m0), tn = min(kTN, N - n0);
  if (tm == kTM && tn == kTN)
    tile_run<T, true, Pre>(S, in, mach, m0, n0, tm, tn, Ui, Xi, Vi, dUi, dXi, dVi, R, dR, h);
  else
    tile_run<T, false, false>(S, in, mach, m0, n0, tm, tn, Ui, Xi, Vi, dUi, dXi, dVi, R, dR, h);
}

static const char* const kVariantNames[2] = {"loads per use", "own cell preloaded"};

int launch_residual_tiled(const eb_batch* b, const double* X, const double* V, const double* U,
                          double* R, cudaStream_t stream, int max_tiles) {
  const Table t = make_table(b);
  const dim3 grid(max_tiles, b->n_inst);
  return tune::launch_tuned(
      "residual_tiled", b->n_cells, max_tiles, 2, 0, kVariantNames, stream, [&](int v) {
        auto kernel = v == 0 ? k_residual_tiled<double, false> : k_residual_tiled<double, true>;
        if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(TileSmem<double>)) != cudaSuccess)
          return check_launch("compute_odes attribute");
        kernel<<<grid, kThreads, sizeof(TileSmem<double>), stream>>>(
            t, X, V, U, nullptr, nullptr, nullptr, nullptr, R, nullptr);
        return check_launch("compute_odes");
      });
}

int launch_tangent_tiled(const eb_batch* b, const double* X, const double* V, const double* U,
                         const double* dU, const double* dX, const double* dV, const double* dMa,
                         double* dR, double* R, cudaStream_t stream, int max_tiles) {
  // One variant only: in dual arithmetic the compiler's multiply-add contraction follows the
  // code layout, so the preloading variant's tangent differs in the last bits; a fixed variant
  // keeps the tangent deterministic.
  const Table t = make_table(b);
  const dim3 grid(2 * max_tiles, b->n_inst);
  auto kernel = k_residual_tiled<D1, false>;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sizeof(TileSmem<D1>)) != cudaSuccess)
    return check_launch("apply_odes_tangent attribute");
  kernel<<<grid, kThreads, sizeof(TileSmem<D1>), stream>>>(t, X, V, U, dX, dV, dU, dMa, R, dR);
  return check_launch("apply_odes_tangent");
}

int residual_tiles(int M, int N) { return ((M + kTM - 1) / kTM) * ((N + kTN - 1) / kTN); }

}  // namespace eb
