// One dual width of the tiled states Jacobian (jac_tiled.cu): included once per width inside
// its own namespace, with EB_JT_WIDTH the number of conserved variables of the seeded state
// differentiated per pass over the faces (4: one pass; 2: two passes, half the live state).

// The four conserved variables of the seeded state are differentiated kW at a time (kGroups
// passes over the faces): two-component duals halve the live derivative state, which lets two
// CTAs share an SM, for a second evaluation of the values.
constexpr int kW = EB_JT_WIDTH;
constexpr int kGroups = 4 / kW;
// the part of a 4 x 4 block one pass forms: its columns G kW .. G kW + kW - 1
constexpr int kBlk = 4 * kW;
using D4 = Dual<double, kW>;

struct Smem {
  double rho[kStaged], j1[kStaged], j2[kStaged], e[kStaged];
  double p[kStaged], ir[kStaged], cs[kStaged];
  double x[kVerts], z[kVerts], vx[kVerts], vz[kVerts];
  double nb[kBlk][kTN][kTM];  // derivative (block part) of the neighbour face's flux, per cell
};

// Staged state i, seeded (conserved variables G kW .. G kW + kW - 1 as the dual components,
// derived quantities in dual arithmetic) or plain.
template <bool Seed, int G>
__device__ __forceinline__ auto state(const Smem& S, int i) {
  if constexpr (Seed) {
    D4 u[4] = {lift<D4>(S.rho[i]), lift<D4>(S.j1[i]), lift<D4>(S.j2[i]), lift<D4>(S.e[i])};
#pragma unroll
    for (int j = 0; j < kW; ++j) u[G * kW + j].d[j] = 1.0;
    return derive<D4>(u[0], u[1], u[2], u[3]);
  } else {
    return St<double>{S.rho[i], S.j1[i], S.j2[i], S.e[i], S.p[i], S.ir[i], S.cs[i]};
  }
}

// A flux as four-component duals (a flux that does not depend on the seeded state has zero
// derivatives).
template <class T>
__device__ __forceinline__ Flux<D4> lift_flux(const Flux<T>& f) {
  Flux<D4> r;
#pragma unroll
  for (int k = 0; k < 4; ++k) r.f[k] = lift<D4>(f.f[k]);
  return r;
}

// Angular face between cells (fr, fc) [l] and (fr, fc - 1) [r]: the stencil line is
// (fr, fc + 1), (fr, fc), (fr, fc - 1), (fr, fc - 2); position K is seeded. F is the flux of
// cell l through its face b, Fp that of cell r through its face f.
template <int K, int G>
__device__ __forceinline__ void angular_pair(const Smem& S, const Instance& in, int fr, int fc,
                                             Flux<D4>& F, Flux<D4>& Fp) {
  const auto ll = state<K == 0, G>(S, sidx(fr, fc + 1));
  const auto l = state<K == 1, G>(S, sidx(fr, fc));
  const auto r = state<K == 2, G>(S, sidx(fr, fc - 1));
  const auto rr = state<K == 3, G>(S, sidx(fr, fc - 2));
  const double nbx = S.z[vidx(fr, fc)] - S.z[vidx(fr + 1, fc)];
  const double nbz = S.x[vidx(fr + 1, fc)] - S.x[vidx(fr, fc)];
  const double vn = (S.vx[vidx(fr + 1, fc)] + S.vx[vidx(fr, fc)]) / 2.0 * nbx +
                    (S.vz[vidx(fr + 1, fc)] + S.vz[vidx(fr, fc)]) / 2.0 * nbz;
  const double len = sqrt_(nbx * nbx + nbz * nbz);
  // the angular sensors centred on l and r (argument order of the residual kernel's)
  const auto sl = sensor(r.p, l.p, ll.p);
  const auto sr = sensor(rr.p, r.p, l.p);
  jst_pair(ll, l, r, rr, nbx, nbz, len, vn, sl, sr, in, F, Fp);
}

// Radial face between cells (fr, fc) [l] and (fr - 1, fc) [r] (grid row fm = m0 + fr): the
// stencil line is (fr + 1), (fr), (fr - 1), (fr - 2) in column fc; position K is seeded. F is
// the flux of cell l through its face i, Fp that of cell r through its face o; the boundary
// rows follow make_ode's five cases (f90:401-436).
template <int K, int G>
__device__ __forceinline__ void radial_pair(const Smem& S, const Instance& in, int fm, int fr,
                                            int fc, Flux<D4>& F, Flux<D4>& Fp) {
  const int M = in.M;
  const double nix = S.z[vidx(fr, fc + 1)] - S.z[vidx(fr, fc)];
  const double niz = S.x[vidx(fr, fc)] - S.x[vidx(fr, fc + 1)];
  const double gx = (S.vx[vidx(fr, fc)] + S.vx[vidx(fr, fc + 1)]) / 2.0;
  const double gz = (S.vz[vidx(fr, fc)] + S.vz[vidx(fr, fc + 1)]) / 2.0;
  const double vn = gx * nix + gz * niz;
  const double mach = in.mach;
#pragma unroll
  for (int k = 0; k < 4; ++k) F.f[k] = Fp.f[k] = lift<D4>(0.0);
  if (fm == 0) {  // wall face of cell 0 (flag 1): central flux with the wall ghost
    const auto C = state<K == 1, G>(S, sidx(fr, fc));
    F = lift_flux(central(C, wall_ghost_st(C, nix, niz, gx, gz), nix, niz, vn));
    return;
  }
  if (fm == M) {  // far-field face of cell M-1 (flag 5): central flux with the ghost
    const auto C = state<K == 2, G>(S, sidx(fr - 1, fc));
    Fp = lift_flux(central(C, farfield_ghost_st(C, mach, in), -nix, -niz, -vn));
    return;
  }
  const double len = sqrt_(nix * nix + niz * niz);
  const auto O = state<K == 0, G>(S, sidx(fr + 1, fc));
  const auto L = state<K == 1, G>(S, sidx(fr, fc));
  const auto Rs = state<K == 2, G>(S, sidx(fr - 1, fc));
  if (fm == 1) {
    // face i of cell 1 (flag 2): central; face o of cell 0 (flag 1): JST whose outer neighbour
    // is the wall ghost of cell 0. Sensors: at cell 0 from its wall ghost, at cell 1 interior.
    F = lift_flux(central(L, Rs, nix, niz, vn));
    const double wx = S.z[vidx(fr - 1, fc + 1)] - S.z[vidx(fr - 1, fc)];
    const double wz = S.x[vidx(fr - 1, fc)] - S.x[vidx(fr - 1, fc + 1)];
    const double wgx = (S.vx[vidx(fr - 1, fc)] + S.vx[vidx(fr - 1, fc + 1)]) / 2.0;
    const double wgz = (S.vz[vidx(fr - 1, fc)] + S.vz[vidx(fr - 1, fc + 1)]) / 2.0;
    const auto gh = wall_ghost_st(Rs, wx, wz, wgx, wgz);
    const auto sr = sensor(gh.p, Rs.p, L.p);
    const auto sl = sensor(Rs.p, L.p, O.p);
    Fp = lift_flux(jst(gh, Rs, L, O, -nix, -niz, len, -vn, sr, sl, in));
    return;
  }
  const auto II = state<K == 3, G>(S, sidx(fr - 2, fc));
  if (fm == M - 1) {
    // face i of cell M-1 (flag 5): JST whose outer neighbour is the far-field ghost; face o of
    // cell M-2 (flag 4): central. Sensors: at cell M-1 from its ghost, at cell M-2 interior.
    const auto gh = farfield_ghost_st(L, mach, in);
    const auto sl = sensor(gh.p, L.p, Rs.p);
    const auto sr = sensor(II.p, Rs.p, L.p);
    F = lift_flux(jst(gh, L, Rs, II, nix, niz, len, vn, sl, sr, in));
    Fp = lift_flux(central(Rs, L, -nix, -niz, -vn));
    return;
  }
  // interior face (one of the four stencil states is seeded, so the fluxes are duals)
  const auto sl = sensor(Rs.p, L.p, O.p);
  const auto sr = sensor(II.p, Rs.p, L.p);
  jst_pair(O, L, Rs, II, nix, niz, len, vn, sl, sr, in, F, Fp);
}

// Finishes a block part: J <- -acc / area for an active slot, 0 for a slot the reference does
// not write (f90:727-746); kBlk consecutive doubles of one cell's column-major block.
__device__ __forceinline__ void store_block(double* out, const double (&acc)[kBlk], double area,
                                            bool active) {
  double2* o = reinterpret_cast<double2*>(out);
#pragma unroll
  for (int e = 0; e < kBlk; e += 2)
    o[e / 2] = active ? make_double2(-acc[e] / area, -acc[e + 1] / area) : make_double2(0.0, 0.0);
}

__device__ __forceinline__ void add_to(double (&acc)[kBlk], const double (&b)[kBlk]) {
#pragma unroll
  for (int e = 0; e < kBlk; ++e) acc[e] = acc[e] + b[e];
}

// One seeded stencil position K of the angular faces (Radial = false) or the radial faces:
// evaluate this thread's face, pass the neighbour's derivative block through shared memory, and
// advance this cell's blocks.
template <bool Radial, int K, int G>
__device__ __forceinline__ void seed_step(Smem& S, const Instance& in, int m0, int n0,
                                          double (&acc_c)[kBlk], double (&acc_x)[kBlk],
                                          double area, double* Jc, int64_t slot_stride) {
  const int M = in.M, N = in.N;
  const int tid = threadIdx.x, r = tid % kTM, c = tid / kTM;
  const int m = m0 + r;
  auto exists = [&](int rr, int cc) {
    return rr >= 0 && cc >= 0 && rr < kTM && cc < kTN && m0 + rr < M && n0 + cc < N;
  };
  const bool own = exists(r, c);
  double fo[kBlk];  // this cell's own face, differentiated
#pragma unroll
  for (int e = 0; e < kBlk; ++e) fo[e] = 0.0;
  {
    int fr = r, fc = c;  // the face this thread evaluates
    int tr, tc;          // the cell that receives its neighbour flux
    bool eval;
    if (!Radial) {
      eval = m < M && (own || exists(r, c - 1));
      tr = r;
      tc = c - 1;
    } else if (c < kTN) {
      eval = m <= M && n0 + c < N;
      tr = r - 1;
      tc = c;
    } else {  // threads (r < kTN, kTN): the radial faces past the tile's outer row
      fr = kTM;
      fc = r;
      eval = r < kTN && exists(kTM - 1, r);
      tr = kTM - 1;
      tc = r;
    }
    if (eval) {
      Flux<D4> F, Fp;
      if (!Radial) angular_pair<K, G>(S, in, fr, fc, F, Fp);
      else radial_pair<K, G>(S, in, m0 + fr, fr, fc, F, Fp);
      if (exists(tr, tc)) {
#pragma unroll
        for (int r4 = 0; r4 < 4; ++r4)
#pragma unroll
          for (int i = 0; i < kW; ++i) S.nb[r4 + 4 * i][tc][tr] = Fp.f[r4].d[i];
      }
      if (fr == r && fc == c && own) {
#pragma unroll
        for (int r4 = 0; r4 < 4; ++r4)
#pragma unroll
          for (int i = 0; i < kW; ++i) fo[r4 + 4 * i] = F.f[r4].d[i];
      }
    }
  }
  __syncthreads();
  if (own) {
    double fn[kBlk];  // the neighbour's face, differentiated
#pragma unroll
    for (int e = 0; e < kBlk; ++e) fn[e] = S.nb[e][c][r];
    // angular: own face b seeded at (f, c, b, bb)[K], the f neighbour's at (ff, f, c, b)[K];
    // radial: own face i seeded at (o, c, i, ii)[K], the o neighbour's at (oo, o, c, i)[K]
    constexpr int s_own = Radial ? (K == 0 ? kO : K == 1 ? kC : K == 2 ? kI : kII)
                                 : (K == 0 ? kF : K == 1 ? kC : K == 2 ? kB : kBB);
    constexpr int s_nb = Radial ? (K == 0 ? kOO : K == 1 ? kO : K == 2 ? kC : kI)
                                : (K == 0 ? kFF : K == 1 ? kF : K == 2 ? kC : kB);
    static_assert(s_own >= 0 && s_own < 9 && s_nb >= 0 && s_nb < 9, "stencil slot out of range");
    double* out_own = Jc + slot_stride * s_own + kBlk * G;
    double* out_nb = Jc + slot_stride * s_nb + kBlk * G;
    if constexpr (K == 0) {
      store_block(out_nb, fn, area, slot_active(s_nb, m, M));
#pragma unroll
      for (int e = 0; e < kBlk; ++e) acc_x[e] = fo[e];
    } else if constexpr (K == 1) {
      if constexpr (!Radial) {
#pragma unroll
        for (int e = 0; e < kBlk; ++e) acc_c[e] = fo[e];
      } else {
        add_to(acc_c, fo);
      }
      add_to(acc_x, fn);
      store_block(out_nb, acc_x, area, slot_active(s_nb, m, M));
    } else if constexpr (K == 2) {
#pragma unroll
      for (int e = 0; e < kBlk; ++e) acc_x[e] = fo[e];
      add_to(acc_c, fn);
      if constexpr (Radial) store_block(out_nb, acc_c, area, true);
    } else {
      store_block(out_own, fo, area, slot_active(s_own, m, M));
      add_to(acc_x, fn);
      store_block(out_nb, acc_x, area, slot_active(s_nb, m, M));
    }
  }
  __syncthreads();
}

// The eight seed steps of one pass (component group G of the seeded states).
template <int G>
__device__ __forceinline__ void all_steps(Smem& S, const Instance& in, int m0, int n0,
                                          double (&acc_c)[kBlk], double (&acc_x)[kBlk], double area,
                                          double* Jc, int64_t slot_stride) {
  seed_step<false, 0, G>(S, in, m0, n0, acc_c, acc_x, area, Jc, slot_stride);
  seed_step<false, 1, G>(S, in, m0, n0, acc_c, acc_x, area, Jc, slot_stride);
  seed_step<false, 2, G>(S, in, m0, n0, acc_c, acc_x, area, Jc, slot_stride);
  seed_step<false, 3, G>(S, in, m0, n0, acc_c, acc_x, area, Jc, slot_stride);
  seed_step<true, 0, G>(S, in, m0, n0, acc_c, acc_x, area, Jc, slot_stride);
  seed_step<true, 1, G>(S, in, m0, n0, acc_c, acc_x, area, Jc, slot_stride);
  seed_step<true, 2, G>(S, in, m0, n0, acc_c, acc_x, area, Jc, slot_stride);
  seed_step<true, 3, G>(S, in, m0, n0, acc_c, acc_x, area, Jc, slot_stride);
}

__global__ void __launch_bounds__(kThreads, kW == 4 ? 1 : 2)
    k_jac_states_tiled(Table t, const double* X, const double* V, const double* U, double* J) {
  extern __shared__ __align__(16) unsigned char jt_smem[];
  Smem& S = *reinterpret_cast<Smem*>(jt_smem);
  const Instance in = t.dev ? t.dev[blockIdx.y] : t.single;
  const int M = in.M, N = in.N;
  const int tiles_m = (M + kTM - 1) / kTM;
  const int tiles = tiles_m * ((N + kTN - 1) / kTN);
  const int tile = blockIdx.x;
  if (tile >= tiles) return;
  const int m0 = (tile % tiles_m) * kTM, n0 = (tile / tiles_m) * kTN;
  const double* Ui = U + 4 * in.cell_offset;
  const double* Xi = X + 2 * in.vert_offset;
  const double* Vi = V ? V + 2 * in.vert_offset : nullptr;
  const int tid = threadIdx.x;
  // stage states (cross-shaped halo; corners and rows outside the grid get finite placeholders
  // that no face reads) with their derived quantities, vertices and grid velocities
  for (int e = tid; e < kStaged; e += kThreads) {
    const int r = e % kSR - 2, c = e / kSR - 2;
    const bool corner = (r < 0 || r >= kTM) && (c < 0 || c > kTN);
    const int m = m0 + r;
    St<double> st{1.0, 0.0, 0.0, 1.0, 1.0, 1.0, 1.0};
    if (!corner && m >= 0 && m < M) {
      int n = n0 + c;  // periodic in the angular index: n0 + c lies in [-2, N + kTN + 1]
      while (n < 0) n += N;
      while (n >= N) n -= N;
      const double* q = Ui + 4 * (m + (int64_t)M * n);
      const double2 a = __ldg(reinterpret_cast<const double2*>(q));
      const double2 b = __ldg(reinterpret_cast<const double2*>(q + 2));
      st = derive<double>(a.x, a.y, b.x, b.y);
    }
    S.rho[e] = st.rho; S.j1[e] = st.j1; S.j2[e] = st.j2; S.e[e] = st.e;
    S.p[e] = st.p; S.ir[e] = st.ir; S.cs[e] = st.cs;
  }
  for (int e = tid; e < kVerts; e += kThreads) {
    const int vm = min(m0 + e % kVR, M), vn = min(n0 + e / kVR, N);
    const int64_t vj = vm + (int64_t)(M + 1) * vn;
    const double2 xv = __ldg(reinterpret_cast<const double2*>(Xi + 2 * vj));
    const double2 vv = Vi ? __ldg(reinterpret_cast<const double2*>(Vi + 2 * vj))
                          : make_double2(0.0, 0.0);
    S.x[e] = xv.x;
    S.z[e] = xv.y;
    S.vx[e] = vv.x;
    S.vz[e] = vv.y;
  }
  __syncthreads();

  const int r = tid % kTM, c = tid / kTM;
  double area = 1.0;
  if (c < kTN) {  // make_area (f90:287-293), as the residual kernel forms it
    const double bix = S.x[vidx(r, c)], biz = S.z[vidx(r, c)];
    const double fix = S.x[vidx(r, c + 1)], fiz = S.z[vidx(r, c + 1)];
    const double fox = S.x[vidx(r + 1, c + 1)], foz = S.z[vidx(r + 1, c + 1)];
    const double box = S.x[vidx(r + 1, c)], boz = S.z[vidx(r + 1, c)];
    area = abs_c((fox - bix) * (boz - fiz) - (foz - biz) * (box - fix)) / 2.0;
  }
  const int64_t slot_stride = 16 * (int64_t)M * N;
  double* Jc = J + 144 * in.cell_offset + 16 * ((int64_t)(m0 + r) + (int64_t)M * (n0 + c));
  double acc_c[kBlk], acc_x[kBlk];
  all_steps<0>(S, in, m0, n0, acc_c, acc_x, area, Jc, slot_stride);
  if constexpr (kGroups > 1) all_steps<1>(S, in, m0, n0, acc_c, acc_x, area, Jc, slot_stride);
}

