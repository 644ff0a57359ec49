// Face arithmetic of the tiled stencil kernels (the residual, its matrix-free tangent and the
// states Jacobian): a staged state with its derived quantities, the pressure sensor, the wall and
// far-field ghost states, and the central / JST face fluxes of make_face_flux
// (src/spatial_discretization.f90:189-274), including the evaluation of one face for both of its
// cells (jst_pair).
//
// Every function is a template over the scalar types of its arguments, each of which may be a
// plain double or a dual number (scalar.cuh): the residual uses double throughout, the tangent
// one-component duals throughout, and the Jacobian kernel seeds one stencil state at a time, so
// that only that state (and what depends on it) carries derivative components while the other
// states and the geometry stay plain doubles. The result type is the widest argument type; with
// all arguments of one type the arithmetic is exactly the single-type evaluation.
#pragma once

#include "physics.cuh"

namespace eb {

// The widest of several comparable scalar types.
template <class A, class... Rest>
struct promote_all {
  using type = A;
};
template <class A, class B, class... Rest>
struct promote_all<A, B, Rest...> {
  using type = typename promote_all<promote_t<A, B>, Rest...>::type;
};
template <class... Ts>
using promote_all_t = typename promote_all<Ts...>::type;

// a * b + c: one fused multiply-add for plain doubles, the dual product and sum otherwise.
template <class A, class B, class C>
__device__ __forceinline__ promote_t<A, promote_t<B, C>> fmad(const A& a, const B& b,
                                                             const C& c) {
  if constexpr (std::is_same<A, double>::value && std::is_same<B, double>::value &&
                std::is_same<C, double>::value)
    return fma(a, b, c);
  else
    return a * b + c;
}

template <class T>
struct St {  // a state with its derived quantities
  T rho, j1, j2, e, p, ir, cs;
};

template <class T>
__device__ __forceinline__ St<T> derive(const T& rho, const T& j1, const T& j2, const T& e) {
  St<T> s;
  s.rho = rho;
  s.j1 = j1;
  s.j2 = j2;
  s.e = e;
  s.ir = 1.0 / rho;
  s.p = kGm1 * (e - (j1 * j1 + j2 * j2) * s.ir * 0.5);
  s.cs = sqrt_(kGamma * s.p * s.ir);
  return s;
}

// The JST pressure sensor |pa - 2 pb + pc| / (pa + 2 pb + pc) (f90:208-211).
template <class A, class B, class C>
__device__ __forceinline__ auto sensor(const A& pa, const B& pb, const C& pc) {
  return abs_c(pa - 2.0 * pb + pc) / (pa + 2.0 * pb + pc);
}

// max_c(0, c) (f90:111-120 with x = 0): 0 only if 0 > Re c + 1e-8.
template <class T>
__device__ __forceinline__ T max_c0(const T& c) {
  return (0.0 > value(c) + 1e-8) ? lift<T>(0.0) : c;
}

// Wall ghost (make_wall_ghost_state, f90:231-240) of state s for face normal n, grid velocity g.
template <class TS, class TG>
__device__ __forceinline__ St<promote_t<TS, TG>> wall_ghost_st(const St<TS>& s, const TG& nx,
                                                               const TG& nz, const TG& gx,
                                                               const TG& gz) {
  using R = promote_t<TS, TG>;
  const R proj = nx * (s.j1 - gx * s.rho) + nz * (s.j2 - gz * s.rho);
  const TG nn = nx * nx + nz * nz;
  return derive<R>(lift<R>(s.rho), s.j1 - 2.0 * nx * proj / nn, s.j2 - 2.0 * nz * proj / nn,
                   lift<R>(s.e));
}

// Far-field ghost (make_farfield_ghost_state, f90:269-274): 2 U_inf - U.
template <class TS, class TM>
__device__ __forceinline__ St<promote_t<TS, TM>> farfield_ghost_st(const St<TS>& s,
                                                                   const TM& mach,
                                                                   const Instance& in) {
  using R = promote_t<TS, TM>;
  const TM speed = mach * sqrt_(kGamma);
  const TM f1 = speed * in.cos_aoa, f2 = speed * in.sin_aoa;
  const TM fe = 1.0 / kGm1 + speed * speed / 2.0;
  return derive<R>(lift<R>(2.0 - s.rho), lift<R>(2.0 * f1 - s.j1), lift<R>(2.0 * f2 - s.j2),
                   lift<R>(2.0 * fe - s.e));
}

template <class T>
struct Flux {
  T f[4];
};

// Central part + ALE term of make_face_flux (f90:197, 219) for l, r through normal (nx, nz)
// with grid-velocity flux vn = g.n.
template <class TL, class TR, class TG>
__device__ __forceinline__ Flux<promote_all_t<TL, TR, TG>> central(const St<TL>& l,
                                                                   const St<TR>& r,
                                                                   const TG& nx, const TG& nz,
                                                                   const TG& vn) {
  using R = promote_all_t<TL, TR, TG>;
  const auto vl = (nx * l.j1 + nz * l.j2) * l.ir;
  const auto vr = (nx * r.j1 + nz * r.j2) * r.ir;
  Flux<R> F;
  F.f[0] = lift<R>((l.rho * vl + r.rho * vr) / 2.0 - (l.rho + r.rho) / 2.0 * vn);
  F.f[1] = lift<R>(((l.j1 * vl + nx * l.p) + (r.j1 * vr + nx * r.p)) / 2.0 -
                   (l.j1 + r.j1) / 2.0 * vn);
  F.f[2] = lift<R>(((l.j2 * vl + nz * l.p) + (r.j2 * vr + nz * r.p)) / 2.0 -
                   (l.j2 + r.j2) / 2.0 * vn);
  F.f[3] = lift<R>(((l.e + l.p) * vl + (r.e + r.p) * vr) / 2.0 - (l.e + r.e) / 2.0 * vn);
  return F;
}

// make_face_flux with JST dissipation (f90:189-220); s1, s2 are the sensors centred on l and r.
template <class TLL, class TL, class TR, class TRR, class TG, class TS1, class TS2>
__device__ __forceinline__ Flux<promote_all_t<TLL, TL, TR, TRR, TG, TS1, TS2>> jst(
    const St<TLL>& ll, const St<TL>& l, const St<TR>& r, const St<TRR>& rr, const TG& nx,
    const TG& nz, const TG& len, const TG& vn, const TS1& s1, const TS2& s2,
    const Instance& in) {
  using R = promote_all_t<TLL, TL, TR, TRR, TG, TS1, TS2>;
  const auto vl = (nx * l.j1 + nz * l.j2) * l.ir;
  const auto vr = (nx * r.j1 + nz * r.j2) * r.ir;
  const auto lam = max_c(abs_c(vl) + l.cs * len, abs_c(vr) + r.cs * len);
  const auto coef2 = in.k2 * max_c(s1, s2) * lam;
  const auto coef4 = max_c0(in.k4 * lam - in.c4 * coef2);
  Flux<R> F;
  const R lv[4] = {lift<R>(l.rho), lift<R>(l.j1), lift<R>(l.j2), lift<R>(l.e)};
  const R rv[4] = {lift<R>(r.rho), lift<R>(r.j1), lift<R>(r.j2), lift<R>(r.e)};
  const R llv[4] = {lift<R>(ll.rho), lift<R>(ll.j1), lift<R>(ll.j2), lift<R>(ll.e)};
  const R rrv[4] = {lift<R>(rr.rho), lift<R>(rr.j1), lift<R>(rr.j2), lift<R>(rr.e)};
  const R fl[4] = {lift<R>(l.rho * vl), lift<R>(l.j1 * vl + nx * l.p),
                   lift<R>(l.j2 * vl + nz * l.p), lift<R>((l.e + l.p) * vl)};
  const R fr[4] = {lift<R>(r.rho * vr), lift<R>(r.j1 * vr + nx * r.p),
                   lift<R>(r.j2 * vr + nz * r.p), lift<R>((r.e + r.p) * vr)};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    R c = (fl[k] + fr[k]) / 2.0;
    c = c - (coef2 * (rv[k] - lv[k]) - coef4 * (rrv[k] - 3.0 * rv[k] + 3.0 * lv[k] - llv[k]));
    F.f[k] = c - (lv[k] + rv[k]) / 2.0 * vn;
  }
  return F;
}

// Both orientations of one JST face: F = make_face_flux(ll, l, r, rr, n) for the cell l and
// F' = make_face_flux(rr, r, l, ll, -n) for the cell r (f90:189-220). Mathematically F' shares
// F's central and ALE parts and its first and third differences, all negated; the orientations
// differ only in the asymmetric max_c decisions (spectral radius and sensor), which are taken per
// orientation as the reference takes them. The shared parts are formed once: the central flux
// minus the grid-velocity flux as (F(l) + F(r)) . n / 2 - (l + r) vn / 2 with the face-relative
// normal velocities vl - vn and vr - vn, and the third difference in F's orientation.
// diss / diss_p = false switch an orientation's dissipation off (its coefficients are zero), which
// leaves the central flux with the grid-velocity term (f90:197, 219) of the boundary-adjacent faces;
// the states then need only be finite.
template <class TLL, class TL, class TR, class TRR, class TG, class TSL, class TSR>
__device__ __forceinline__ void jst_pair(
    const St<TLL>& ll, const St<TL>& l, const St<TR>& r, const St<TRR>& rr, const TG& nx,
    const TG& nz, const TG& len, const TG& vn, const TSL& sl, const TSR& sr, const Instance& in,
    Flux<promote_all_t<TLL, TL, TR, TRR, TG, TSL, TSR>>& F,
    Flux<promote_all_t<TLL, TL, TR, TRR, TG, TSL, TSR>>& Fp, bool diss = true,
    bool diss_p = true) {
  using R = promote_all_t<TLL, TL, TR, TRR, TG, TSL, TSR>;
  const auto vl = (nx * l.j1 + nz * l.j2) * l.ir;
  const auto vr = (nx * r.j1 + nz * r.j2) * r.ir;
  // F' sees the normal velocities -vr, -vl: abs_c takes its derivative's sign from the value
  // with zeros as positive, so at a zero velocity the two orientations' derivatives differ
  // (the values, and plain-double results, do not)
  const auto al = abs_c(vl) + l.cs * len;
  const auto ar = abs_c(vr) + r.cs * len;
  const auto alp = abs_c(-vl) + l.cs * len;
  const auto arp = abs_c(-vr) + r.cs * len;
  const auto lam = max_c(al, ar);
  const auto lamp = max_c(arp, alp);
  const auto coef2 = in.k2 * max_c(sl, sr) * lam;
  const auto coef2p = in.k2 * max_c(sr, sl) * lamp;
  const auto coef4 = max_c0(in.k4 * lam - in.c4 * coef2);
  const auto coef4p = max_c0(in.k4 * lamp - in.c4 * coef2p);
  const auto wl = vl - vn;
  const auto wr = vr - vn;
  const auto ps = l.p + r.p;
  const R ca[4] = {lift<R>(0.5 * fmad(l.rho, wl, r.rho * wr)),
                   lift<R>(0.5 * fmad(l.j1, wl, fmad(r.j1, wr, nx * ps))),
                   lift<R>(0.5 * fmad(l.j2, wl, fmad(r.j2, wr, nz * ps))),
                   lift<R>(0.5 * fmad(l.e, wl, fmad(r.e, wr, fmad(l.p, vl, r.p * vr))))};
  const R lv[4] = {lift<R>(l.rho), lift<R>(l.j1), lift<R>(l.j2), lift<R>(l.e)};
  const R rv[4] = {lift<R>(r.rho), lift<R>(r.j1), lift<R>(r.j2), lift<R>(r.e)};
  const R llv[4] = {lift<R>(ll.rho), lift<R>(ll.j1), lift<R>(ll.j2), lift<R>(ll.e)};
  const R rrv[4] = {lift<R>(rr.rho), lift<R>(rr.j1), lift<R>(rr.j2), lift<R>(rr.e)};
  const R zero = lift<R>(0.0);
  const R c2 = diss ? lift<R>(coef2) : zero, c4 = diss ? lift<R>(coef4) : zero;
  const R c2p = diss_p ? lift<R>(coef2p) : zero, c4p = diss_p ? lift<R>(coef4p) : zero;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const R d1 = rv[k] - lv[k];
    const R d3 = fmad(3.0, lv[k], fmad(-3.0, rv[k], rrv[k])) - llv[k];
    F.f[k] = fmad(c4, d3, fmad(-c2, d1, ca[k]));
    Fp.f[k] = fmad(-c4p, d3, fmad(c2p, d1, -ca[k]));
  }
}

}  // namespace eb
