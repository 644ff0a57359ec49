// Cell-face physics of the 2D Euler ALE discretization, generic over the scalar type.
//
// Restates the per-cell operator of PyEulerALE (`src/spatial_discretization.f90`):
// pressure, wave-speed integral, physical flux, JST face flux with ALE term, wall / far-field
// ghost states, cell geometry and the 5-case radial boundary logic of `make_ode`. Every
// function is a template over independent scalar types for states (TS), vertices (TX),
// vertex velocities (TV) and the Mach number (TM), so one source yields the FP64 residual,
// forward tangents, Jacobian blocks and exact second derivatives (see scalar.cuh).
//
// The evaluation keeps the reference's orientation rules: every cell evaluates its four
// faces in its own orientation (l = this cell), because `max_c` is asymmetric and a
// face-once evaluation would change the dissipation of near-equal spectral radii / sensors.
#pragma once

#include <cstdint>

#include "scalar.cuh"

namespace eb {

// Constants are macros so that device code can bind them to reference parameters.
#define kGamma 1.4               // heat_ratio, f90:55
#define kGm1 (kGamma - 1.0)      // (heat_ratio - 1)

// Per-instance parameters, in the layout of `eb_instance` (include/euler_b200.h).
struct Instance {
  int32_t M, N;             // cells in the radial / angular direction
  int64_t cell_offset;      // first cell of the instance in the packed cell arrays
  int64_t vert_offset;      // first vertex of the instance in the packed vertex arrays
  int64_t wall_offset;      // first wall face of the instance in the packed wall arrays
  double mach;              // free-stream Mach number
  double cos_aoa, sin_aoa;  // cos / sin of the angle of attack (host-evaluated)
  double k2, k4, c4;        // JST constants (jst_k2, jst_k4, jst_c4, f90:64-66)
  double chord, xc, zc;     // coefficient length and moment centre (core.py:65-66)
};

template <class T>
struct S4 {
  T v[4];
};
template <class T>
struct P2 {
  T x, z;
};

template <class R, class X>
EB_HD S4<R> lift4(const S4<X>& s) {
  S4<R> r;
#pragma unroll
  for (int k = 0; k < 4; ++k) r.v[k] = lift<R>(s.v[k]);
  return r;
}

// get_pressure, f90:128-133.
template <class T>
EB_HD T pressure(const S4<T>& s) {
  return kGm1 * (s.v[3] - (s.v[1] * s.v[1] + s.v[2] * s.v[2]) / s.v[0] / 2.0);
}

// get_wave_integral, f90:142-148: |j.n/rho| + sqrt(gamma p / rho) |n|.
template <class TS, class TN>
EB_HD auto wave_integral(const S4<TS>& s, const P2<TN>& n) {
  return abs_c((n.x * s.v[1] + n.z * s.v[2]) / s.v[0]) +
         sqrt_(kGamma * pressure(s) / s.v[0]) * sqrt_(n.x * n.x + n.z * n.z);
}

// make_physical_flux, f90:159-171.
template <class TS, class TN>
EB_HD auto physical_flux(const S4<TS>& s, const P2<TN>& n) {
  using R = promote_t<TS, TN>;
  const R vi = lift<R>((n.x * s.v[1] + n.z * s.v[2]) / s.v[0]);
  const TS p = pressure(s);
  S4<R> f;
  f.v[0] = s.v[0] * vi;
  f.v[1] = s.v[1] * vi + n.x * p;
  f.v[2] = s.v[2] * vi + n.z * p;
  f.v[3] = (s.v[3] + p) * vi;
  return f;
}

// make_face_flux without the optional outer states (no artificial dissipation), f90:197, 219.
template <class R, class TL, class TR, class TN, class TV>
EB_HD S4<R> face_flux_central(const S4<TL>& l, const S4<TR>& r, const P2<TN>& n,
                              const P2<TV>& gv) {
  const auto fl = physical_flux(l, n);
  const auto fr = physical_flux(r, n);
  const auto vn = gv.x * n.x + gv.z * n.z;
  S4<R> f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const R c = lift<R>((lift<R>(fl.v[k]) + lift<R>(fr.v[k])) / 2.0);
    f.v[k] = c - lift<R>((lift<R>(l.v[k]) + lift<R>(r.v[k])) / 2.0 * lift<R>(vn));
  }
  return f;
}

// make_face_flux with JST dissipation, f90:189-220.
template <class R, class TLL, class TL, class TR, class TRR, class TN, class TV>
EB_HD S4<R> face_flux_jst(const S4<TLL>& ll, const S4<TL>& l, const S4<TR>& r,
                          const S4<TRR>& rr, const P2<TN>& n, const P2<TV>& gv,
                          const Instance& in) {
  const auto fl = physical_flux(l, n);
  const auto fr = physical_flux(r, n);
  const R lam_l = lift<R>(wave_integral(l, n));
  const R lam_r = lift<R>(wave_integral(r, n));
  const R p_ll = lift<R>(pressure(ll)), p_l = lift<R>(pressure(l));
  const R p_r = lift<R>(pressure(r)), p_rr = lift<R>(pressure(rr));
  const R lam = max_c(lam_l, lam_r);
  const R sensor = max_c(abs_c(p_ll - 2.0 * p_l + p_r) / (p_ll + 2.0 * p_l + p_r),
                         abs_c(p_l - 2.0 * p_r + p_rr) / (p_l + 2.0 * p_r + p_rr));
  const R coef2 = in.k2 * sensor * lam;
  const R coef4 = max_c(0.0, in.k4 * lam - in.c4 * coef2);
  const R vn = lift<R>(gv.x * n.x + gv.z * n.z);
  S4<R> f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const R L = lift<R>(l.v[k]), Rr = lift<R>(r.v[k]);
    const R LL = lift<R>(ll.v[k]), RR = lift<R>(rr.v[k]);
    R c = (lift<R>(fl.v[k]) + lift<R>(fr.v[k])) / 2.0;
    c = c - (coef2 * (Rr - L) - coef4 * (RR - 3.0 * Rr + 3.0 * L - LL));
    f.v[k] = c - (L + Rr) / 2.0 * vn;
  }
  return f;
}

// make_wall_ghost_state, f90:231-240: reflect the momentum relative to the moving wall.
template <class TS, class TN, class TV>
EB_HD auto wall_ghost(const S4<TS>& w, const P2<TN>& n, const P2<TV>& gv) {
  using R = promote_t<TS, promote_t<TN, TV>>;
  const R proj = lift<R>(n.x * (w.v[1] - gv.x * w.v[0])) + lift<R>(n.z * (w.v[2] - gv.z * w.v[0]));
  const R nn = lift<R>(n.x * n.x + n.z * n.z);
  S4<R> g;
  g.v[0] = lift<R>(w.v[0]);
  g.v[1] = lift<R>(w.v[1]) - 2.0 * lift<R>(n.x) * proj / nn;
  g.v[2] = lift<R>(w.v[2]) - 2.0 * lift<R>(n.z) * proj / nn;
  g.v[3] = lift<R>(w.v[3]);
  return g;
}

// make_free_stream_state, f90:250-259 (cos/sin of the angle of attack evaluated on the host).
template <class TM>
EB_HD S4<TM> free_stream(const TM& mach, const Instance& in) {
  const TM speed = mach * sqrt_(kGamma);
  S4<TM> s;
  s.v[0] = lift<TM>(1.0);
  s.v[1] = speed * in.cos_aoa;
  s.v[2] = speed * in.sin_aoa;
  s.v[3] = 1.0 / kGm1 + speed * speed / 2.0;
  return s;
}

// make_farfield_ghost_state, f90:269-274.
template <class TM, class TS>
EB_HD auto farfield_ghost(const TM& mach, const S4<TS>& u, const Instance& in) {
  using R = promote_t<TM, TS>;
  const S4<TM> fs = free_stream(mach, in);
  S4<R> g;
#pragma unroll
  for (int k = 0; k < 4; ++k) g.v[k] = lift<R>(2.0 * fs.v[k]) - lift<R>(u.v[k]);
  return g;
}

// make_normal, f90:306-311: (z2 - z1, x1 - x2), |n| = edge length.
template <class T>
EB_HD P2<T> normal(const P2<T>& a, const P2<T>& b) {
  return P2<T>{b.z - a.z, a.x - b.x};
}

// make_grid_velo, f90:320-324.
template <class T>
EB_HD P2<T> grid_velo(const P2<T>& a, const P2<T>& b) {
  return P2<T>{(a.x + b.x) / 2.0, (a.z + b.z) / 2.0};
}

// make_area, f90:287-293.
template <class T>
EB_HD T area(const P2<T>& bi, const P2<T>& fi, const P2<T>& fo, const P2<T>& bo) {
  const T d1x = fo.x - bi.x, d1z = fo.z - bi.z;
  const T d2x = bo.x - fi.x, d2z = bo.z - fi.z;
  return abs_c(d1x * d2z - d1z * d2x) / 2.0;
}

// get_boundary_flag, f90:450-464, with 0-based radial index m.
EB_HD int boundary_flag(int M, int m) {
  if (m == 0) return 1;
  if (m == 1) return 2;
  if (m == M - 2) return 4;
  if (m == M - 1) return 5;
  return 3;
}

// Stencil slots in the order of the reference's Jacobian storage (f90:699-707).
enum Slot { kC = 0, kB = 1, kBB = 2, kF = 3, kFF = 4, kI = 5, kII = 6, kO = 7, kOO = 8 };
// Vertex corners (f90:511-518): backward-inward, forward-inward, forward-outward, backward-outward.
enum Corner { kBI = 0, kFI = 1, kFO = 2, kBO = 3 };
// Faces of a cell, in the summation order of make_ode (f90:395-400).
enum Face { kFaceB = 0, kFaceF = 1, kFaceI = 2, kFaceO = 3 };

// The complete local input of one cell's ODE.
template <class TS, class TX, class TV, class TM>
struct Cell {
  P2<TX> x[4];  // vertices at the corners (Corner order)
  P2<TV> w[4];  // vertex velocities at the corners
  S4<TS> u[9];  // stencil states (Slot order)
  TM mach;
  int flag;
};

template <class TS, class TX, class TV, class TM>
using cell_result_t = promote_t<TS, promote_t<TX, promote_t<TV, TM>>>;

// Geometry shared by the four faces.
template <class TX, class TV>
struct Geometry {
  TX area;
  P2<TX> n[4];  // normals per Face
  P2<TV> g[4];  // grid velocities per Face
};

template <class TX, class TV>
EB_HD Geometry<TX, TV> geometry(const P2<TX>* x, const P2<TV>* w) {
  Geometry<TX, TV> g;
  g.area = area(x[kBI], x[kFI], x[kFO], x[kBO]);
  g.n[kFaceI] = normal(x[kBI], x[kFI]);
  g.n[kFaceF] = normal(x[kFI], x[kFO]);
  g.n[kFaceO] = normal(x[kFO], x[kBO]);
  g.n[kFaceB] = normal(x[kBO], x[kBI]);
  g.g[kFaceI] = grid_velo(w[kBI], w[kFI]);
  g.g[kFaceF] = grid_velo(w[kFI], w[kFO]);
  g.g[kFaceO] = grid_velo(w[kFO], w[kBO]);
  g.g[kFaceB] = grid_velo(w[kBO], w[kBI]);
  return g;
}

// Flux through face q of a cell, in the cell's own orientation (the select case of
// make_ode, f90:392-434). `u(slot)` provides the stencil state of a slot (letting callers
// seed tangents on the fly); R is the common result type.
template <class R, class SP, class TX, class TV, class TM>
EB_HD S4<R> face(int q, int flag, const SP& u, const Geometry<TX, TV>& g, const TM& mach,
                 const Instance& in) {
  switch (q) {
    case kFaceB:
      return face_flux_jst<R>(u(kF), u(kC), u(kB), u(kBB), g.n[kFaceB], g.g[kFaceB], in);
    case kFaceF:
      return face_flux_jst<R>(u(kB), u(kC), u(kF), u(kFF), g.n[kFaceF], g.g[kFaceF], in);
    case kFaceI:
      switch (flag) {
        case 1: {
          const auto c = u(kC);
          const auto gh = wall_ghost(c, g.n[kFaceI], g.g[kFaceI]);
          return face_flux_central<R>(c, gh, g.n[kFaceI], g.g[kFaceI]);
        }
        case 2:
          return face_flux_central<R>(u(kC), u(kI), g.n[kFaceI], g.g[kFaceI]);
        case 5: {
          const auto c = u(kC);
          const auto gh = farfield_ghost(mach, c, in);
          return face_flux_jst<R>(gh, c, u(kI), u(kII), g.n[kFaceI], g.g[kFaceI], in);
        }
        default:
          return face_flux_jst<R>(u(kO), u(kC), u(kI), u(kII), g.n[kFaceI], g.g[kFaceI], in);
      }
    default:  // kFaceO
      switch (flag) {
        case 1: {
          const auto c = u(kC);
          const auto gh = wall_ghost(c, g.n[kFaceI], g.g[kFaceI]);
          return face_flux_jst<R>(gh, c, u(kO), u(kOO), g.n[kFaceO], g.g[kFaceO], in);
        }
        case 4:
          return face_flux_central<R>(u(kC), u(kO), g.n[kFaceO], g.g[kFaceO]);
        case 5: {
          const auto c = u(kC);
          const auto gh = farfield_ghost(mach, c, in);
          return face_flux_central<R>(c, gh, g.n[kFaceO], g.g[kFaceO]);
        }
        default:
          return face_flux_jst<R>(u(kI), u(kC), u(kO), u(kOO), g.n[kFaceO], g.g[kFaceO], in);
      }
  }
}

// State provider returning the cell's own stencil states.
template <class TS>
struct PlainStates {
  const S4<TS>* u;
  EB_HD const S4<TS>& operator()(int s) const { return u[s]; }
};

// make_ode, f90:370-436: -(F_b + F_f + F_i + F_o) / area.
template <class TS, class TX, class TV, class TM>
EB_HD S4<cell_result_t<TS, TX, TV, TM>> make_ode(const Cell<TS, TX, TV, TM>& c,
                                                 const Instance& in) {
  using R = cell_result_t<TS, TX, TV, TM>;
  const Geometry<TX, TV> g = geometry(c.x, c.w);
  const PlainStates<TS> u{c.u};
  const S4<R> fb = face<R>(kFaceB, c.flag, u, g, c.mach, in);
  const S4<R> ff = face<R>(kFaceF, c.flag, u, g, c.mach, in);
  const S4<R> fi = face<R>(kFaceI, c.flag, u, g, c.mach, in);
  const S4<R> fo = face<R>(kFaceO, c.flag, u, g, c.mach, in);
  const R a = lift<R>(g.area);
  S4<R> ode;
#pragma unroll
  for (int k = 0; k < 4; ++k) ode.v[k] = -(((fb.v[k] + ff.v[k]) + fi.v[k]) + fo.v[k]) / a;
  return ode;
}

// Whether face q of a cell with boundary flag `flag` depends on stencil slot s (directly or
// through a ghost state built from the centre state).
EB_HD bool face_uses_slot(int q, int flag, int s) {
  switch (q) {
    case kFaceB: return s == kF || s == kC || s == kB || s == kBB;
    case kFaceF: return s == kB || s == kC || s == kF || s == kFF;
    case kFaceI:
      switch (flag) {
        case 1: return s == kC;
        case 2: return s == kC || s == kI;
        case 5: return s == kC || s == kI || s == kII;
        default: return s == kO || s == kC || s == kI || s == kII;
      }
    default:
      switch (flag) {
        case 1: return s == kC || s == kO || s == kOO;
        case 4: return s == kC || s == kO;
        case 5: return s == kC;
        default: return s == kI || s == kC || s == kO || s == kOO;
      }
  }
}

// Slots whose Jacobian block the reference computes (the guards of f90:727-746).
EB_HD bool slot_active(int s, int m, int M) {
  switch (s) {
    case kI: return m > 0;
    case kII: return m > 1;
    case kO: return m < M - 1;
    case kOO: return m < M - 2;
    default: return true;
  }
}

// Radial / angular offsets of the stencil slots.
EB_HD int slot_dm(int s) {
  switch (s) {
    case kI: return -1;
    case kII: return -2;
    case kO: return 1;
    case kOO: return 2;
    default: return 0;
  }
}
EB_HD int slot_dn(int s) {
  switch (s) {
    case kB: return -1;
    case kBB: return -2;
    case kF: return 1;
    case kFF: return 2;
    default: return 0;
  }
}
EB_HD int wrap(int n, int N) {
  n %= N;
  return n < 0 ? n + N : n;
}

}  // namespace eb
