// Matrix-free reverse (adjoint) products of the residual: for a cotangent w,
//   d_states = (dR/dU)^T w,  d_vertices = (dR/dX)^T w,  d_velocities = (dR/dV)^T w,
//   d_mach = (dR/dMa)^T w (one per instance),
// the products the reference forms from stored complex-step Jacobians (apply_odes_wrt_states_rev,
// apply_odes_wrt_vertices_rev, apply_odes_wrt_mach_rev; src/spatial_discretization.f90:604-650,
// 875-918, 1044-1072), here in one stencil pass that recomputes the face quantities and runs
// them in reverse (tile_faces_rev.cuh): no Jacobian is built or stored, and every output element
// is gathered by the one CTA that owns it (no atomics).
//
// R_c = -(F_b + F_f + F_i + F_o) / area_c (f90:370-436), so a face flux feeding cell c has the
// adjoint q_c = -w_c / area_c and the cell's area the adjoint (w_c . S_c) / area_c^2 with S_c the
// sum of its face fluxes. One CTA owns a tile of kTM x kTN cells (their states) and the vertices
// at their lower-left corners (plus the last vertex row / column of the grid). It stages the
// states with a three-cell halo, the vertices, and q and the area of the cells with a two-cell
// halo, then evaluates in reverse every face whose stencil reaches an owned state or whose
// geometry or cells touch an owned vertex: angular faces of rows [-1, kTM) x columns
// [-1, kTN + 2), radial faces of rows [-1, kTM + 2) x columns [-1, kTN]. A face's adjoints for
// its four stencil states are added to the owned ones stencil position by stencil position,
// with a barrier between positions (within one position and direction no two faces reach the
// same state); its normal / grid-velocity adjoints and w . F for its two cells go to per-face
// and per-cell slots, from which every owned vertex gathers its faces and cells in a fixed
// order. The angular index is periodic for the states; vertex column N is a variable of its own
// (cell N-1's forward corners) distinct from column 0 (cell 0's backward corners), so geometry
// adjoints are credited per cell, and the one face column between cells N-1 and 0 is reversed
// once per cell there. Halo geometry is staged through the periodic wrap, which assumes a closed
// O-grid (vertex column N equal to column 0, as the reference's grids are).
//
// A complex cotangent (the reference's complex vectors) is two real products: the CTA pair
// 2 t + h of tile t carries part h.

#include "autotune.cuh"
#include "common.cuh"
#include "tile_faces_rev.cuh"

namespace eb {
namespace adj {

constexpr int kTM = 32, kTN = 8, kThreads = 256;
constexpr int kSR = kTM + 6, kSC = kTN + 6;        // staged states: rows, columns [-3, k + 3)
constexpr int kStaged = kSR * kSC;
constexpr int kVR = kTM + 5, kVC = kTN + 5;        // staged vertices: [-2, k + 3)
constexpr int kVerts = kVR * kVC;
constexpr int kQR = kTM + 4, kQC = kTN + 4;        // cells with q and area: [-2, k + 2)
constexpr int kQCells = kQR * kQC;
constexpr int kAR = kTM + 1, kAC = kTN + 3;        // angular faces: rows [-1, kTM), cols [-1, kTN+2)
constexpr int kRR = kTM + 3, kRC = kTN + 2;        // radial faces: rows [-1, kTM+2), cols [-1, kTN]
constexpr int kNA = kAR * kAC, kNR = kRR * kRC;
constexpr int kER = kTM + 1, kEC = kTN + 1;        // cells whose area adjoint is formed: [-1, k)
constexpr int kECells = kER * kEC;

struct Smem {
  double rho[kStaged], j1[kStaged], j2[kStaged], e[kStaged], p[kStaged], ir[kStaged],
      cs[kStaged];
  double x[kVerts], z[kVerts], vx[kVerts], vz[kVerts];
  double q[4][kQCells];       // -w / area
  double area[kQCells];
  double wF[4][kECells];      // w . (flux through face b, f, i, o) of the cell
  double ga[4][kNA];          // angular faces: adjoints of (nx, nz, gx, gz)
  double gr[4][kNR];          // radial faces
  double gw[4][kRC];          // the wall-ghost use of the wall face (radial faces of row 1)
  double ac[kECells];         // area adjoint x sign(cross) / 2 of the cell
  double gu[4][kTN][kTM];     // owned states' adjoints
};

__device__ __forceinline__ int sidx(int r, int c) { return (c + 3) * kSR + (r + 3); }
__device__ __forceinline__ int vidx(int r, int c) { return (c + 2) * kVR + (r + 2); }
__device__ __forceinline__ int qidx(int r, int c) { return (c + 2) * kQR + (r + 2); }
__device__ __forceinline__ int eidx(int r, int c) { return (c + 1) * kER + (r + 1); }
__device__ __forceinline__ int aidx(int r, int c) { return (c + 1) * kAR + (r + 1); }
__device__ __forceinline__ int ridx(int r, int c) { return (c + 1) * kRR + (r + 1); }

__device__ __forceinline__ Sd staged(const Smem& S, int i) {
  return Sd{S.rho[i], S.j1[i], S.j2[i], S.e[i], S.p[i], S.ir[i], S.cs[i]};
}

__device__ __forceinline__ void load_q(const Smem& S, int r, int c, double (&q)[4]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) q[k] = S.q[k][qidx(r, c)];
}

// The result of one face in reverse: the conserved-variable adjoints of its four stencil states
// (positions 0..3: ll, l, r, rr of an angular face; (fr + 1), fr, (fr - 1), (fr - 2) of a radial
// one), the adjoints of its normal and grid velocity, of the wall face's (radial faces of grid
// row 1), and w . F of its two cells.
struct FaceAdj {
  double u[4][4];
  double n[4];   // nx, nz, gx, gz
  double nw[4];  // the wall face's nx, nz, gx, gz
  double wl, wr; // w_l . F, w_r . F'
};

__device__ __forceinline__ void add_raw(double (&u)[4], const Sd& b) {
  u[0] += b.rho;
  u[1] += b.j1;
  u[2] += b.j2;
  u[3] += b.e;
}

// Angular face between cells (fr, fc) [l] and (fr, fc - 1) [r] in reverse with the flux
// adjoints Fb (cell l) and Fpb (cell r); the stencil line (fr, fc + 1 .. fc - 2).
__device__ void angular_rev(const Smem& S, const Instance& in, int fr, int fc,
                            const double (&Fb)[4], const double (&Fpb)[4], FaceAdj& A) {
  const Sd ll = staged(S, sidx(fr, fc + 1)), l = staged(S, sidx(fr, fc));
  const Sd r = staged(S, sidx(fr, fc - 1)), rr = staged(S, sidx(fr, fc - 2));
  const double nbx = S.z[vidx(fr, fc)] - S.z[vidx(fr + 1, fc)];
  const double nbz = S.x[vidx(fr + 1, fc)] - S.x[vidx(fr, fc)];
  const double gx = (S.vx[vidx(fr + 1, fc)] + S.vx[vidx(fr, fc)]) / 2.0;
  const double gz = (S.vz[vidx(fr + 1, fc)] + S.vz[vidx(fr, fc)]) / 2.0;
  const double vn = gx * nbx + gz * nbz;
  const double len = sqrt_(nbx * nbx + nbz * nbz);
  const double sl = sensor(r.p, l.p, ll.p), sr = sensor(rr.p, r.p, l.p);
  Sd llb = zero_st(), lb = zero_st(), rb = zero_st(), rrb = zero_st();
  double nxb = 0.0, nzb = 0.0, lenb = 0.0, vnb = 0.0, slb = 0.0, srb = 0.0;
  double F[4], Fp[4];
  jst_pair_rev(ll, l, r, rr, nbx, nbz, len, vn, sl, sr, in, Fb, Fpb, llb, lb, rb, rrb, nxb, nzb,
               lenb, vnb, slb, srb, F, Fp);
  sensor_rev(r.p, l.p, ll.p, slb, rb.p, lb.p, llb.p);
  sensor_rev(rr.p, r.p, l.p, srb, rrb.p, rb.p, lb.p);
  derive_rev(ll, llb);
  derive_rev(l, lb);
  derive_rev(r, rb);
  derive_rev(rr, rrb);
  add_raw(A.u[0], llb);
  add_raw(A.u[1], lb);
  add_raw(A.u[2], rb);
  add_raw(A.u[3], rrb);
  if (len > 0.0) {
    nxb += lenb * nbx / len;
    nzb += lenb * nbz / len;
  }
  A.n[0] += nxb + vnb * gx;
  A.n[1] += nzb + vnb * gz;
  A.n[2] += vnb * nbx;
  A.n[3] += vnb * nbz;
  A.wl = 0.0;
  A.wr = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    A.wl += Fb[k] * F[k];
    A.wr += Fpb[k] * Fp[k];
  }
}

// Radial face between cells (fr, fc) [l] and (fr - 1, fc) [r] (grid row fm) in reverse, with
// make_ode's boundary cases (f90:401-436); the Mach adjoint is left to k_mach_adjoint.
__device__ void radial_rev(const Smem& S, const Instance& in, int fm, int fr, int fc,
                           const double (&Fb)[4], const double (&Fpb)[4], FaceAdj& A) {
  const int M = in.M;
  const double nix = S.z[vidx(fr, fc + 1)] - S.z[vidx(fr, fc)];
  const double niz = S.x[vidx(fr, fc)] - S.x[vidx(fr, fc + 1)];
  const double gx = (S.vx[vidx(fr, fc)] + S.vx[vidx(fr, fc + 1)]) / 2.0;
  const double gz = (S.vz[vidx(fr, fc)] + S.vz[vidx(fr, fc + 1)]) / 2.0;
  const double vn = gx * nix + gz * niz;
  double nxb = 0.0, nzb = 0.0, gxb = 0.0, gzb = 0.0, vnb = 0.0, lenb = 0.0;
  double F[4] = {0.0, 0.0, 0.0, 0.0}, Fp[4] = {0.0, 0.0, 0.0, 0.0};
  double machb = 0.0;
  const double len = sqrt_(nix * nix + niz * niz);
  if (fm == 0) {  // wall face of cell 0: central flux with the wall ghost (same face geometry)
    const Sd C = staged(S, sidx(fr, fc));
    const Sd G = wall_ghost_st(C, nix, niz, gx, gz);
    const Flux<double> f = central(C, G, nix, niz, vn);
    Sd Cb = zero_st(), Gb = zero_st();
    central_rev(C, G, nix, niz, vn, Fb, Cb, Gb, nxb, nzb, vnb);
    wall_ghost_rev(C, nix, niz, gx, gz, Gb, Cb, nxb, nzb, gxb, gzb);
    derive_rev(C, Cb);
    add_raw(A.u[1], Cb);
#pragma unroll
    for (int k = 0; k < 4; ++k) F[k] = f.f[k];
  } else if (fm == M) {  // far-field face of cell M-1: central flux with the far-field ghost
    const Sd C = staged(S, sidx(fr - 1, fc));
    const Sd G = farfield_ghost_st(C, in.mach, in);
    const Flux<double> f = central(C, G, -nix, -niz, -vn);
    Sd Cb = zero_st(), Gb = zero_st();
    double mxb = 0.0, mzb = 0.0, mvb = 0.0;
    central_rev(C, G, -nix, -niz, -vn, Fpb, Cb, Gb, mxb, mzb, mvb);
    nxb -= mxb;
    nzb -= mzb;
    vnb -= mvb;
    farfield_ghost_rev(C, in.mach, in, Gb, Cb, machb);
    derive_rev(C, Cb);
    add_raw(A.u[2], Cb);
#pragma unroll
    for (int k = 0; k < 4; ++k) Fp[k] = f.f[k];
  } else {
    const Sd O = staged(S, sidx(fr + 1, fc)), L = staged(S, sidx(fr, fc));
    const Sd Rs = staged(S, sidx(fr - 1, fc));
    Sd Ob = zero_st(), Lb = zero_st(), Rb = zero_st(), Ib = zero_st();
    const double zero4[4] = {0.0, 0.0, 0.0, 0.0};
    if (fm == 1) {
      // cell 1: central; cell 0: JST whose outer neighbour is its wall ghost, whose sensor
      // uses the ghost (the ghost is built with the wall face's geometry, row fr - 1)
      const Flux<double> f = central(L, Rs, nix, niz, vn);
      central_rev(L, Rs, nix, niz, vn, Fb, Lb, Rb, nxb, nzb, vnb);
      const double wx = S.z[vidx(fr - 1, fc + 1)] - S.z[vidx(fr - 1, fc)];
      const double wz = S.x[vidx(fr - 1, fc)] - S.x[vidx(fr - 1, fc + 1)];
      const double wgx = (S.vx[vidx(fr - 1, fc)] + S.vx[vidx(fr - 1, fc + 1)]) / 2.0;
      const double wgz = (S.vz[vidx(fr - 1, fc)] + S.vz[vidx(fr - 1, fc + 1)]) / 2.0;
      const Sd G = wall_ghost_st(Rs, wx, wz, wgx, wgz);
      const double sr = sensor(G.p, Rs.p, L.p), sl = sensor(Rs.p, L.p, O.p);
      Sd Gb = zero_st();
      double mxb = 0.0, mzb = 0.0, mvb = 0.0, srb = 0.0, slb = 0.0, Fj[4], Fu[4];
      jst_pair_rev(G, Rs, L, O, -nix, -niz, len, -vn, sr, sl, in, Fpb, zero4, Gb, Rb, Lb, Ob,
                   mxb, mzb, lenb, mvb, srb, slb, Fj, Fu);
      nxb -= mxb;
      nzb -= mzb;
      vnb -= mvb;
      sensor_rev(G.p, Rs.p, L.p, srb, Gb.p, Rb.p, Lb.p);
      sensor_rev(Rs.p, L.p, O.p, slb, Rb.p, Lb.p, Ob.p);
      double wxb = 0.0, wzb = 0.0, wgxb = 0.0, wgzb = 0.0;
      wall_ghost_rev(Rs, wx, wz, wgx, wgz, Gb, Rb, wxb, wzb, wgxb, wgzb);
      A.nw[0] += wxb;
      A.nw[1] += wzb;
      A.nw[2] += wgxb;
      A.nw[3] += wgzb;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        F[k] = f.f[k];
        Fp[k] = Fj[k];
      }
    } else {
      const Sd II = staged(S, sidx(fr - 2, fc));
      if (fm == M - 1) {
        // cell M-1: JST whose outer neighbour is its far-field ghost (also in its sensor);
        // cell M-2: central
        const Sd G = farfield_ghost_st(L, in.mach, in);
        const double sl = sensor(G.p, L.p, Rs.p), sr = sensor(II.p, Rs.p, L.p);
        Sd Gb = zero_st();
        double slb = 0.0, srb = 0.0, Fu[4];
        jst_pair_rev(G, L, Rs, II, nix, niz, len, vn, sl, sr, in, Fb, zero4, Gb, Lb, Rb, Ib,
                     nxb, nzb, lenb, vnb, slb, srb, F, Fu);
        sensor_rev(G.p, L.p, Rs.p, slb, Gb.p, Lb.p, Rb.p);
        sensor_rev(II.p, Rs.p, L.p, srb, Ib.p, Rb.p, Lb.p);
        farfield_ghost_rev(L, in.mach, in, Gb, Lb, machb);
        const Flux<double> f = central(Rs, L, -nix, -niz, -vn);
        double mxb = 0.0, mzb = 0.0, mvb = 0.0;
        central_rev(Rs, L, -nix, -niz, -vn, Fpb, Rb, Lb, mxb, mzb, mvb);
        nxb -= mxb;
        nzb -= mzb;
        vnb -= mvb;
#pragma unroll
        for (int k = 0; k < 4; ++k) Fp[k] = f.f[k];
      } else {
        const double sl = sensor(Rs.p, L.p, O.p), sr = sensor(II.p, Rs.p, L.p);
        double slb = 0.0, srb = 0.0;
        jst_pair_rev(O, L, Rs, II, nix, niz, len, vn, sl, sr, in, Fb, Fpb, Ob, Lb, Rb, Ib, nxb,
                     nzb, lenb, vnb, slb, srb, F, Fp);
        sensor_rev(Rs.p, L.p, O.p, slb, Rb.p, Lb.p, Ob.p);
        sensor_rev(II.p, Rs.p, L.p, srb, Ib.p, Rb.p, Lb.p);
      }
      derive_rev(II, Ib);
      add_raw(A.u[3], Ib);
    }
    derive_rev(O, Ob);
    derive_rev(L, Lb);
    derive_rev(Rs, Rb);
    add_raw(A.u[0], Ob);
    add_raw(A.u[1], Lb);
    add_raw(A.u[2], Rb);
  }
  if (len > 0.0) {
    nxb += lenb * nix / len;
    nzb += lenb * niz / len;
  }
  A.n[0] += nxb + vnb * gx;
  A.n[1] += nzb + vnb * gz;
  A.n[2] += gxb + vnb * nix;
  A.n[3] += gzb + vnb * niz;
  A.wl = 0.0;
  A.wr = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    A.wl += Fb[k] * F[k];
    A.wr += Fpb[k] * Fp[k];
  }
}

__device__ __forceinline__ void clear(FaceAdj& A) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
#pragma unroll
    for (int k = 0; k < 4; ++k) A.u[i][k] = 0.0;
    A.n[i] = A.nw[i] = 0.0;
  }
  A.wl = A.wr = 0.0;
}

// MinBlocks = 2: capped at 128 registers (with spills) so that two CTAs share an SM;
// MinBlocks = 1: no cap, one CTA per SM. The same code, so the two give identical results.
template <int MinBlocks>
__global__ void __launch_bounds__(kThreads, MinBlocks)
    k_residual_adjoint(Table t, const double* X, const double* V, const double* U,
                       const double* W, int cstride, double* gU, double* gX, double* gV) {
  extern __shared__ __align__(16) unsigned char adj_smem[];
  Smem& S = *reinterpret_cast<Smem*>(adj_smem);
  const Instance in = t.dev ? t.dev[blockIdx.y] : t.single;
  const int M = in.M, N = in.N;
  const int h = cstride == 2 ? (int)(blockIdx.x & 1) : 0;
  const int tile = cstride == 2 ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
  const int tiles_m = (M + kTM - 1) / kTM;
  if (tile >= tiles_m * ((N + kTN - 1) / kTN)) return;
  const int m0 = (tile % tiles_m) * kTM, n0 = (tile / tiles_m) * kTN;
  const double* Ui = U + 4 * in.cell_offset;
  const double* Wi = W + 4 * cstride * in.cell_offset;
  const double* Xi = X + 2 * in.vert_offset;
  const double* Vi = V ? V + 2 * in.vert_offset : nullptr;
  const int tid = threadIdx.x;
  auto wrap_n = [&](int n) {
    while (n < 0) n += N;
    while (n >= N) n -= N;
    return n;
  };

  // 1. states (cross-shaped halo of three; the rest finite placeholders no face reads),
  //    vertices and grid velocities (periodic through the closed grid's wrap)
  for (int e = tid; e < kStaged; e += kThreads) {
    const int r = e % kSR - 3, c = e / kSR - 3;
    const bool corner = (r < -1 || r >= kTM) && (c < -1 || c > kTN);
    const int m = m0 + r;
    Sd st{1.0, 0.0, 0.0, 1.0, 1.0, 1.0, 1.0};
    if (!corner && m >= 0 && m < M) {
      const double* q = Ui + 4 * (m + (int64_t)M * wrap_n(n0 + c));
      const double2 a = __ldg(reinterpret_cast<const double2*>(q));
      const double2 b = __ldg(reinterpret_cast<const double2*>(q + 2));
      st = derive<double>(a.x, a.y, b.x, b.y);
    }
    S.rho[e] = st.rho; S.j1[e] = st.j1; S.j2[e] = st.j2; S.e[e] = st.e;
    S.p[e] = st.p; S.ir[e] = st.ir; S.cs[e] = st.cs;
  }
  for (int e = tid; e < kVerts; e += kThreads) {
    const int i = e % kVR - 2, j = e / kVR - 2;
    const int vm = min(max(m0 + i, 0), M);
    int vn = n0 + j;
    if (vn < 0) vn += N;
    if (vn > N) vn -= N;
    vn = min(max(vn, 0), N);
    const int64_t vj = vm + (int64_t)(M + 1) * vn;
    const double2 xv = __ldg(reinterpret_cast<const double2*>(Xi + 2 * vj));
    const double2 vv = Vi ? __ldg(reinterpret_cast<const double2*>(Vi + 2 * vj))
                          : make_double2(0.0, 0.0);
    S.x[e] = xv.x;
    S.z[e] = xv.y;
    S.vx[e] = vv.x;
    S.vz[e] = vv.y;
  }
  for (int e = tid; e < 4 * kTM * kTN; e += kThreads) (&S.gu[0][0][0])[e] = 0.0;
  for (int e = tid; e < 4 * kNA; e += kThreads) (&S.ga[0][0])[e] = 0.0;
  for (int e = tid; e < 4 * kNR; e += kThreads) (&S.gr[0][0])[e] = 0.0;
  for (int e = tid; e < 4 * kRC; e += kThreads) (&S.gw[0][0])[e] = 0.0;
  for (int e = tid; e < 4 * kECells; e += kThreads) (&S.wF[0][0])[e] = 0.0;
  __syncthreads();
  // 2. per cell: area (make_area, f90:287-293) and q = -w / area (0 outside the grid)
  for (int e = tid; e < kQCells; e += kThreads) {
    const int r = e % kQR - 2, c = e / kQR - 2;
    const int m = m0 + r;
    const double bix = S.x[vidx(r, c)], biz = S.z[vidx(r, c)];
    const double fix = S.x[vidx(r, c + 1)], fiz = S.z[vidx(r, c + 1)];
    const double fox = S.x[vidx(r + 1, c + 1)], foz = S.z[vidx(r + 1, c + 1)];
    const double box = S.x[vidx(r + 1, c)], boz = S.z[vidx(r + 1, c)];
    double area = 1.0, q[4] = {0.0, 0.0, 0.0, 0.0};
    if (m >= 0 && m < M) {
      area = abs_c((fox - bix) * (boz - fiz) - (foz - biz) * (box - fix)) / 2.0;
      const double* w = Wi + 4 * cstride * (m + (int64_t)M * wrap_n(n0 + c));
#pragma unroll
      for (int k = 0; k < 4; ++k) q[k] = -__ldg(w + cstride * k + h) / area;
    }
    S.area[e] = area;
#pragma unroll
    for (int k = 0; k < 4; ++k) S.q[k][e] = q[k];
  }
  __syncthreads();

  // 3. faces in reverse, one face per thread and round. The face lists span the tile's part
  // inside the grid (tm x tn cells): angular faces of rows [-1, tm) x columns [-1, tn + 2),
  // radial faces of rows [-1, tm + 2) x columns [-1, tn], the full lists (kNA + kNR faces, three
  // rounds) for a full tile. The faces a partial tile leaves out reach no owned state, vertex or
  // cell; their slots keep the zeros of phase 1.
  const int tm = min(kTM, M - m0), tn = min(kTN, N - n0);
  const int a_rows = tm + 1, r_rows = tm + 3;
  const int na = a_rows * (tn + 3), nr = r_rows * (tn + 2);
  const int rounds = (na + nr + kThreads - 1) / kThreads;
  for (int round = 0; round < rounds; ++round) {
    const int f = tid + kThreads * round;
    const bool angular = f < na;
    const bool radial = !angular && f < na + nr;
    int fr = 0, fc = 0;
    if (angular) {
      fr = f % a_rows - 1;
      fc = f / a_rows - 1;
    } else if (radial) {
      fr = (f - na) % r_rows - 1;
      fc = (f - na) / r_rows - 1;
    }
    const int fm = m0 + fr;
    FaceAdj A;
    clear(A);
    bool have = false;
    if (angular && fm >= 0 && fm < M) {
      have = true;
      double Fb[4], Fpb[4];
      load_q(S, fr, fc, Fb);
      load_q(S, fr, fc - 1, Fpb);
      // geometry is credited to canonical cells only (grid column n0 + fc of cell l, n0 + fc -
      // 1 of cell r, both in [0, N)); where exactly one of the two is canonical the face is
      // reversed once per cell and only that cell's part enters the geometry
      const bool can_l = n0 + fc >= 0 && n0 + fc < N, can_r = n0 + fc - 1 >= 0 && n0 + fc - 1 < N;
      if (can_l == can_r) {
        angular_rev(S, in, fr, fc, Fb, Fpb, A);
        if (!can_l)
#pragma unroll
          for (int k = 0; k < 4; ++k) A.n[k] = 0.0;
      } else {
        double Fa[4], Fpa[4], Fc[4], Fpc[4];  // the canonical cell's part, the other part
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          Fa[k] = can_l ? Fb[k] : 0.0;
          Fpa[k] = can_l ? 0.0 : Fpb[k];
          Fc[k] = can_l ? 0.0 : Fb[k];
          Fpc[k] = can_l ? Fpb[k] : 0.0;
        }
        FaceAdj B;
        clear(B);
        angular_rev(S, in, fr, fc, Fa, Fpa, A);
        angular_rev(S, in, fr, fc, Fc, Fpc, B);
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int k = 0; k < 4; ++k) A.u[i][k] += B.u[i][k];
        const double wl = A.wl + B.wl, wr = A.wr + B.wr;
        A.wl = wl;
        A.wr = wr;
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) S.ga[k][aidx(fr, fc)] = A.n[k];
      if (fr >= -1 && fr < kTM && fc >= -1 && fc < kTN) S.wF[0][eidx(fr, fc)] = A.wl;
      if (fr >= -1 && fr < kTM && fc - 1 >= -1 && fc - 1 < kTN) S.wF[1][eidx(fr, fc - 1)] = A.wr;
    } else if (radial && fm >= 0 && fm <= M) {
      have = true;
      double Fb[4], Fpb[4];
      load_q(S, fr, fc, Fb);
      load_q(S, fr - 1, fc, Fpb);
      radial_rev(S, in, fm, fr, fc, Fb, Fpb, A);
      const bool can = n0 + fc >= 0 && n0 + fc < N;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        S.gr[k][ridx(fr, fc)] = can ? A.n[k] : 0.0;
        if (fm == 1) S.gw[k][fc + 1] = can ? A.nw[k] : 0.0;
      }
      if (fr >= -1 && fr < kTM && fc >= -1 && fc < kTN) S.wF[2][eidx(fr, fc)] = A.wl;
      if (fr - 1 >= -1 && fr - 1 < kTM && fc >= -1 && fc < kTN) S.wF[3][eidx(fr - 1, fc)] = A.wr;
    }
    // state adjoints, one stencil position and direction at a time
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        __syncthreads();
        if (have && (dir == 0 ? angular : radial)) {
          const int sr = dir == 0 ? fr : fr + 1 - k, sc = dir == 0 ? fc + 1 - k : fc;
          if (sr >= 0 && sr < kTM && sc >= 0 && sc < kTN)
#pragma unroll
            for (int v = 0; v < 4; ++v) S.gu[v][sc][sr] += A.u[k][v];
        }
      }
    }
  }
  __syncthreads();

  // 4. area adjoints of the cells around the owned vertices: (w . S) / area^2, times
  //    sign(cross) / 2 (area = |cross| / 2), for canonical cells of the grid
  for (int e = tid; e < kECells; e += kThreads) {
    const int r = e % kER - 1, c = e / kER - 1;
    const int m = m0 + r, n = n0 + c;
    double a = 0.0;
    if (m >= 0 && m < M && n >= 0 && n < N) {
      const double ws = ((S.wF[0][e] + S.wF[1][e]) + S.wF[2][e]) + S.wF[3][e];
      const double ar = S.area[qidx(r, c)];
      const double bix = S.x[vidx(r, c)], biz = S.z[vidx(r, c)];
      const double fix = S.x[vidx(r, c + 1)], fiz = S.z[vidx(r, c + 1)];
      const double fox = S.x[vidx(r + 1, c + 1)], foz = S.z[vidx(r + 1, c + 1)];
      const double box = S.x[vidx(r + 1, c)], boz = S.z[vidx(r + 1, c)];
      const double cross = (fox - bix) * (boz - fiz) - (foz - biz) * (box - fix);
      // the slots hold q . F = -(w . F) / area, so (w . S) / area^2 = -ws / area
      a = -ws / ar * sgn_c(cross) / 2.0;
    }
    S.ac[e] = a;
  }
  __syncthreads();

  // 5. owned states
  const int64_t cell_base = in.cell_offset;
  for (int e = tid; gU && e < kTM * kTN; e += kThreads) {
    const int r = e % kTM, c = e / kTM;
    const int m = m0 + r, n = n0 + c;
    if (m < M && n < N) {
      double* o = gU + 4 * cstride * (cell_base + m + (int64_t)M * n);
#pragma unroll
      for (int v = 0; v < 4; ++v) o[cstride * v + h] = S.gu[v][c][r];
    }
  }
  // 6. owned vertices: rows [0, kTM) of the tile (and row M), columns [0, kTN) (and column N)
  if (gX || gV) {
    for (int e = tid; e < (kTM + 1) * (kTN + 1); e += kThreads) {
      const int i = e % (kTM + 1), j = e / (kTM + 1);
      const int vm = m0 + i, vn = n0 + j;
      const bool row_ok = (i < kTM && vm < M) || vm == M;
      const bool col_ok = (j < kTN && vn < N) || vn == N;
      if (!row_ok || !col_ok) continue;
      double xb = 0.0, zb = 0.0, vxb = 0.0, vzb = 0.0;
      // angular faces: (i - 1, j) has this vertex at its upper end, (i, j) at its lower end
      if (m0 + i - 1 >= 0) {
        const int a = aidx(i - 1, j);
        zb -= S.ga[0][a];
        xb += S.ga[1][a];
        vxb += S.ga[2][a] / 2.0;
        vzb += S.ga[3][a] / 2.0;
      }
      if (i < kTM) {
        const int a = aidx(i, j);
        zb += S.ga[0][a];
        xb -= S.ga[1][a];
        vxb += S.ga[2][a] / 2.0;
        vzb += S.ga[3][a] / 2.0;
      }
      // radial faces: (i, j - 1) has this vertex at its right end, (i, j) at its left end
      {
        const int a = ridx(i, j - 1), b = ridx(i, j);
        zb += S.gr[0][a] - S.gr[0][b];
        xb += S.gr[1][b] - S.gr[1][a];
        vxb += (S.gr[2][a] + S.gr[2][b]) / 2.0;
        vzb += (S.gr[3][a] + S.gr[3][b]) / 2.0;
      }
      // the wall face in the ghost of cell 0 (radial faces of grid row 1)
      if (vm == 0) {
        zb += S.gw[0][j] - S.gw[0][j + 1];
        xb += S.gw[1][j + 1] - S.gw[1][j];
        vxb += (S.gw[2][j] + S.gw[2][j + 1]) / 2.0;
        vzb += (S.gw[3][j] + S.gw[3][j + 1]) / 2.0;
      }
      // areas: this vertex is corner bi of cell (i, j), fi of (i, j - 1), fo of (i - 1, j - 1)
      // and bo of (i - 1, j)
      auto corner = [&](int r, int c, int which) {
        if (r < -1 || r >= kTM || c < -1 || c >= kTN) return;
        const double a = S.ac[eidx(r, c)];
        if (a == 0.0) return;
        const double bix = S.x[vidx(r, c)], biz = S.z[vidx(r, c)];
        const double fix = S.x[vidx(r, c + 1)], fiz = S.z[vidx(r, c + 1)];
        const double fox = S.x[vidx(r + 1, c + 1)], foz = S.z[vidx(r + 1, c + 1)];
        const double box = S.x[vidx(r + 1, c)], boz = S.z[vidx(r + 1, c)];
        // cross = (fo - bi).x (bo - fi).z - (fo - bi).z (bo - fi).x
        switch (which) {
          case 0:  // bi
            xb -= a * (boz - fiz);
            zb += a * (box - fix);
            break;
          case 1:  // fi
            xb += a * (foz - biz);
            zb -= a * (fox - bix);
            break;
          case 2:  // fo
            xb += a * (boz - fiz);
            zb -= a * (box - fix);
            break;
          default:  // bo
            xb -= a * (foz - biz);
            zb += a * (fox - bix);
            break;
        }
      };
      corner(i, j, 0);
      corner(i, j - 1, 1);
      corner(i - 1, j - 1, 2);
      corner(i - 1, j, 3);
      const int64_t v = in.vert_offset + vm + (int64_t)(M + 1) * vn;
      if (gX) {
        gX[cstride * (2 * v) + h] = xb;
        gX[cstride * (2 * v + 1) + h] = zb;
      }
      if (gV) {
        gV[cstride * (2 * v) + h] = vxb;
        gV[cstride * (2 * v + 1) + h] = vzb;
      }
    }
  }
}

// d_mach = (dR/dMa)^T w per instance: only the far-field faces (grid rows M - 1 and M) depend on
// the Mach number, through the far-field ghost (f90:269-274) in the flux and in the sensor of
// cell M - 1. One CTA per instance; each thread reverses the far-field faces of a stride of
// columns and the CTA sums them in a fixed order.
__global__ void __launch_bounds__(256) k_mach_adjoint(Table t, const double* X,
                                                      const double* V, const double* U,
                                                      const double* W, int cstride,
                                                      double* gMa) {
  const Instance in = t.dev ? t.dev[blockIdx.x] : t.single;
  const int M = in.M, N = in.N;
  const double* Ui = U + 4 * in.cell_offset;
  const double* Wi = W + 4 * cstride * in.cell_offset;
  const double* Xi = X + 2 * in.vert_offset;
  const double* Vi = V ? V + 2 * in.vert_offset : nullptr;
  __shared__ double part[2][256];
  auto state = [&](int m, int n) {
    const double* q = Ui + 4 * (m + (int64_t)M * n);
    return derive<double>(q[0], q[1], q[2], q[3]);
  };
  auto vert = [&](const double* A, int m, int n, int d) {
    return A ? A[2 * (m + (int64_t)(M + 1) * n) + d] : 0.0;
  };
  for (int h = 0; h < cstride; ++h) {
    double acc = 0.0;
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
      auto qcell = [&](int m, double (&q)[4]) {
        const double bix = vert(Xi, m, n, 0), biz = vert(Xi, m, n, 1);
        const double fix = vert(Xi, m, n + 1, 0), fiz = vert(Xi, m, n + 1, 1);
        const double fox = vert(Xi, m + 1, n + 1, 0), foz = vert(Xi, m + 1, n + 1, 1);
        const double box = vert(Xi, m + 1, n, 0), boz = vert(Xi, m + 1, n, 1);
        const double area = abs_c((fox - bix) * (boz - fiz) - (foz - biz) * (box - fix)) / 2.0;
        const double* w = Wi + 4 * cstride * (m + (int64_t)M * n);
        for (int k = 0; k < 4; ++k) q[k] = -w[cstride * k + h] / area;
      };
      for (int fm = M - 1; fm <= M; ++fm) {
        const double nix = vert(Xi, fm, n + 1, 1) - vert(Xi, fm, n, 1);
        const double niz = vert(Xi, fm, n, 0) - vert(Xi, fm, n + 1, 0);
        const double gx = (vert(Vi, fm, n, 0) + vert(Vi, fm, n + 1, 0)) / 2.0;
        const double gz = (vert(Vi, fm, n, 1) + vert(Vi, fm, n + 1, 1)) / 2.0;
        const double vn = gx * nix + gz * niz;
        double machb = 0.0, a = 0.0, b = 0.0, c = 0.0, d = 0.0;
        if (fm == M) {  // cell M-1's outer face: central flux with the far-field ghost
          double q[4];
          qcell(M - 1, q);
          const Sd C = state(M - 1, n);
          const Sd G = farfield_ghost_st(C, in.mach, in);
          Sd Cb = zero_st(), Gb = zero_st();
          central_rev(C, G, -nix, -niz, -vn, q, Cb, Gb, a, b, c);
          farfield_ghost_rev(C, in.mach, in, Gb, Cb, machb);
        } else {  // cell M-1's inner face: JST with the ghost as its outer state and sensor
          double q[4];
          qcell(M - 1, q);
          const Sd L = state(M - 1, n), Rs = state(M - 2, n), II = state(M - 3, n);
          const Sd G = farfield_ghost_st(L, in.mach, in);
          const double sl = sensor(G.p, L.p, Rs.p), sr = sensor(II.p, Rs.p, L.p);
          const double len = sqrt_(nix * nix + niz * niz);
          Sd Gb = zero_st(), Lb = zero_st(), Rb = zero_st(), Ib = zero_st();
          double slb = 0.0, srb = 0.0, F[4], Fu[4];
          const double z4[4] = {0.0, 0.0, 0.0, 0.0};
          jst_pair_rev(G, L, Rs, II, nix, niz, len, vn, sl, sr, in, q, z4, Gb, Lb, Rb, Ib, a, b,
                       c, d, slb, srb, F, Fu);
          sensor_rev(G.p, L.p, Rs.p, slb, Gb.p, Lb.p, Rb.p);
          farfield_ghost_rev(L, in.mach, in, Gb, Lb, machb);
        }
        acc += machb;
      }
    }
    part[h][threadIdx.x] = acc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int h = 0; h < cstride; ++h) {
      double s = 0.0;
      for (int k = 0; k < (int)blockDim.x; ++k) s += part[h][k];
      gMa[cstride * blockIdx.x + h] = s;
    }
  }
}

int tiles(int M, int N) { return ((M + kTM - 1) / kTM) * ((N + kTN - 1) / kTN); }

}  // namespace adj
}  // namespace eb

using namespace eb;

extern "C" int eb_apply_odes_adjoint(const eb_batch* b, const double* X, const double* V,
                                     const double* U, const double* w, int is_complex,
                                     double* d_states, double* d_vertices,
                                     double* d_velocities, double* d_mach, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, V, U, w, d_states, d_vertices, d_velocities, d_mach);
  if (!X || !U || !w) return fail(EB_ERR_ARG, "null array");
  if (!d_states && !d_vertices && !d_velocities && !d_mach) return EB_OK;
  if (is_complex != 0 && is_complex != 1) return fail(EB_ERR_ARG, "is_complex must be 0 or 1");
  int dim = b->max_dim;
  if (b->n_inst == 1 && b->d_table == nullptr) dim = std::max(b->single.M, b->single.N);
  if (dim < 5) return fail(EB_ERR_ARG, "batch max_dim must be the largest M or N");
  if (b->n_inst > 65535) return fail(EB_ERR_ARG, "at most 65535 instances per batch");
  const Table t = make_table(b);
  const int cs = is_complex ? 2 : 1;
  cudaStream_t st = EB_STREAM(stream);
  if (d_states || d_vertices || d_velocities) {
    auto launch = [&](int v) {
      auto kernel = v == 0 ? adj::k_residual_adjoint<2> : adj::k_residual_adjoint<1>;
      if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(adj::Smem)) != cudaSuccess)
        return check_launch("apply_odes_adjoint attribute");
      kernel<<<dim3(cs * adj::tiles(dim, dim), b->n_inst), adj::kThreads, sizeof(adj::Smem),
               st>>>(t, X, V, U, w, cs, d_states, d_vertices, d_velocities);
      return check_launch("apply_odes_adjoint");
    };
    static const char* const kNames[2] = {"2 CTAs/SM (128 registers)", "1 CTA/SM"};
    if (int rc = tune::launch_tuned(is_complex ? "residual_adjoint complex" : "residual_adjoint",
                                    b->n_cells, dim, 2, 0, kNames, st, launch))
      return rc;
  }
  if (d_mach) {
    adj::k_mach_adjoint<<<b->n_inst, 256, 0, st>>>(t, X, V, U, w, cs, d_mach);
    return check_launch("apply_odes_adjoint mach");
  }
  return EB_OK;
}
