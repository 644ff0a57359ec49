// Reverse (adjoint) mode of the face arithmetic in tile_faces.cuh, in plain doubles: given the
// forward inputs and the adjoints of a function's outputs, each routine recomputes what it needs
// of the forward values and adds the adjoints of its inputs. Together they differentiate
// make_face_flux with its ghost states and sensors (src/spatial_discretization.f90:189-274) in
// reverse, so a matrix-free vector-Jacobian product w^T dR/d(U, X, V, Ma) costs a few face
// evaluations per cell instead of the Jacobian blocks.
//
// A state adjoint has the seven components of St: the conserved variables and the derived
// pressure, 1/rho and speed of sound. derive_rev folds the derived components into the conserved
// ones. The branch primitives keep the forward decisions: abs_c's derivative is sign(x) with
// zeros counted as positive, max_c passes the adjoint to the argument it selected.
#pragma once

#include "tile_faces.cuh"

namespace eb {

using Sd = St<double>;

__device__ __forceinline__ Sd zero_st() { return Sd{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}; }

__device__ __forceinline__ double sgn_c(double x) { return x < 0.0 ? -1.0 : 1.0; }

// derive (ir = 1/rho, p = (g - 1)(e - |j|^2 ir / 2), cs = sqrt(g p ir)) in reverse: moves the
// adjoints of p, ir and cs of state s into b's conserved components (and clears them).
__device__ __forceinline__ void derive_rev(const Sd& s, Sd& b) {
  if (b.cs != 0.0) {
    const double t = b.cs * kGamma / (2.0 * s.cs);
    b.p += t * s.ir;
    b.ir += t * s.p;
  }
  b.e += kGm1 * b.p;
  b.j1 -= kGm1 * s.j1 * s.ir * b.p;
  b.j2 -= kGm1 * s.j2 * s.ir * b.p;
  b.ir -= kGm1 * 0.5 * (s.j1 * s.j1 + s.j2 * s.j2) * b.p;
  b.rho -= s.ir * s.ir * b.ir;
  b.p = b.ir = b.cs = 0.0;
}

// sensor(pa, pb, pc) = |pa - 2 pb + pc| / (pa + 2 pb + pc) in reverse.
__device__ __forceinline__ void sensor_rev(double pa, double pb, double pc, double sb,
                                           double& pab, double& pbb, double& pcb) {
  const double n = pa - 2.0 * pb + pc, d = pa + 2.0 * pb + pc;
  const double nb = sb * sgn_c(n) / d, db = -sb * fabs(n) / (d * d);
  pab += nb + db;
  pbb += 2.0 * (db - nb);
  pcb += nb + db;
}

// v = (nx j1 + nz j2) ir (the normal velocity) in reverse.
__device__ __forceinline__ void normal_velocity_rev(const Sd& s, double nx, double nz, double vb,
                                                    Sd& b, double& nxb, double& nzb) {
  b.ir += vb * (nx * s.j1 + nz * s.j2);
  const double tb = vb * s.ir;
  nxb += tb * s.j1;
  nzb += tb * s.j2;
  b.j1 += tb * nx;
  b.j2 += tb * nz;
}

// central (the central flux with the ALE term) in reverse, for the flux adjoint Fb.
__device__ __forceinline__ void central_rev(const Sd& l, const Sd& r, double nx, double nz,
                                            double vn, const double (&Fb)[4], Sd& lb, Sd& rb,
                                            double& nxb, double& nzb, double& vnb) {
  const double vl = (nx * l.j1 + nz * l.j2) * l.ir;
  const double vr = (nx * r.j1 + nz * r.j2) * r.ir;
  const double h0 = 0.5 * Fb[0], h1 = 0.5 * Fb[1], h2 = 0.5 * Fb[2], h3 = 0.5 * Fb[3];
  const double vlb = h0 * l.rho + h1 * l.j1 + h2 * l.j2 + h3 * (l.e + l.p);
  const double vrb = h0 * r.rho + h1 * r.j1 + h2 * r.j2 + h3 * (r.e + r.p);
  lb.rho += h0 * (vl - vn);
  lb.j1 += h1 * (vl - vn);
  lb.j2 += h2 * (vl - vn);
  lb.e += h3 * (vl - vn);
  lb.p += h1 * nx + h2 * nz + h3 * vl;
  rb.rho += h0 * (vr - vn);
  rb.j1 += h1 * (vr - vn);
  rb.j2 += h2 * (vr - vn);
  rb.e += h3 * (vr - vn);
  rb.p += h1 * nx + h2 * nz + h3 * vr;
  nxb += h1 * (l.p + r.p);
  nzb += h2 * (l.p + r.p);
  vnb -= h0 * (l.rho + r.rho) + h1 * (l.j1 + r.j1) + h2 * (l.j2 + r.j2) + h3 * (l.e + r.e);
  normal_velocity_rev(l, nx, nz, vlb, lb, nxb, nzb);
  normal_velocity_rev(r, nx, nz, vrb, rb, nxb, nzb);
}

// Both orientations of a JST face (jst_pair) in reverse, for the flux adjoints Fb (of F, cell l)
// and Fpb (of F', cell r). With Fpb = 0 it is the reverse of the single-orientation jst of cell l
// (the same flux). Returns the forward fluxes in F, Fp.
__device__ __forceinline__ void jst_pair_rev(const Sd& ll, const Sd& l, const Sd& r,
                                             const Sd& rr, double nx, double nz, double len,
                                             double vn, double sl, double sr,
                                             const Instance& in, const double (&Fb)[4],
                                             const double (&Fpb)[4], Sd& llb, Sd& lb, Sd& rb,
                                             Sd& rrb, double& nxb, double& nzb, double& lenb,
                                             double& vnb, double& slb, double& srb,
                                             double (&F)[4], double (&Fp)[4]) {
  const double vl = (nx * l.j1 + nz * l.j2) * l.ir;
  const double vr = (nx * r.j1 + nz * r.j2) * r.ir;
  const double al = fabs(vl) + l.cs * len, ar = fabs(vr) + r.cs * len;
  const double alp = fabs(-vl) + l.cs * len, arp = fabs(-vr) + r.cs * len;
  const bool sel_l = al > ar + 1e-8, sel_lp = arp > alp + 1e-8;    // lam = al? / lamp = arp?
  const bool sel_s = sl > sr + 1e-8, sel_sp = sr > sl + 1e-8;      // sm = sl? / smp = sr?
  const double lam = sel_l ? al : ar, lamp = sel_lp ? arp : alp;
  const double sm = sel_s ? sl : sr, smp = sel_sp ? sr : sl;
  const double coef2 = in.k2 * sm * lam, coef2p = in.k2 * smp * lamp;
  const double t4 = in.k4 * lam - in.c4 * coef2, t4p = in.k4 * lamp - in.c4 * coef2p;
  const bool z4 = 0.0 > t4 + 1e-8, z4p = 0.0 > t4p + 1e-8;
  const double coef4 = z4 ? 0.0 : t4, coef4p = z4p ? 0.0 : t4p;
  const double wl = vl - vn, wr = vr - vn, ps = l.p + r.p;
  const double ca[4] = {0.5 * fma(l.rho, wl, r.rho * wr),
                        0.5 * fma(l.j1, wl, fma(r.j1, wr, nx * ps)),
                        0.5 * fma(l.j2, wl, fma(r.j2, wr, nz * ps)),
                        0.5 * fma(l.e, wl, fma(r.e, wr, fma(l.p, vl, r.p * vr)))};
  const double lv[4] = {l.rho, l.j1, l.j2, l.e}, rv[4] = {r.rho, r.j1, r.j2, r.e};
  const double llv[4] = {ll.rho, ll.j1, ll.j2, ll.e}, rrv[4] = {rr.rho, rr.j1, rr.j2, rr.e};
  double lvb[4], rvb[4], llvb[4], rrvb[4], cab[4];
  double coef4b = 0.0, coef4pb = 0.0, coef2b = 0.0, coef2pb = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double d1 = rv[k] - lv[k];
    const double d3 = fma(3.0, lv[k], fma(-3.0, rv[k], rrv[k])) - llv[k];
    F[k] = fma(coef4, d3, fma(-coef2, d1, ca[k]));
    Fp[k] = fma(-coef4p, d3, fma(coef2p, d1, -ca[k]));
    cab[k] = Fb[k] - Fpb[k];
    const double d1b = coef2p * Fpb[k] - coef2 * Fb[k];
    const double d3b = coef4 * Fb[k] - coef4p * Fpb[k];
    coef4b += d3 * Fb[k];
    coef4pb -= d3 * Fpb[k];
    coef2b -= d1 * Fb[k];
    coef2pb += d1 * Fpb[k];
    lvb[k] = 3.0 * d3b - d1b;
    rvb[k] = d1b - 3.0 * d3b;
    rrvb[k] = d3b;
    llvb[k] = -d3b;
  }
  // the shared central / ALE part
  const double h0 = 0.5 * cab[0], h1 = 0.5 * cab[1], h2 = 0.5 * cab[2], h3 = 0.5 * cab[3];
  const double wlb = h0 * l.rho + h1 * l.j1 + h2 * l.j2 + h3 * l.e;
  const double wrb = h0 * r.rho + h1 * r.j1 + h2 * r.j2 + h3 * r.e;
  lb.rho += lvb[0] + h0 * wl;
  lb.j1 += lvb[1] + h1 * wl;
  lb.j2 += lvb[2] + h2 * wl;
  lb.e += lvb[3] + h3 * wl;
  rb.rho += rvb[0] + h0 * wr;
  rb.j1 += rvb[1] + h1 * wr;
  rb.j2 += rvb[2] + h2 * wr;
  rb.e += rvb[3] + h3 * wr;
  llb.rho += llvb[0];
  llb.j1 += llvb[1];
  llb.j2 += llvb[2];
  llb.e += llvb[3];
  rrb.rho += rrvb[0];
  rrb.j1 += rrvb[1];
  rrb.j2 += rrvb[2];
  rrb.e += rrvb[3];
  const double psb = h1 * nx + h2 * nz;
  nxb += h1 * ps;
  nzb += h2 * ps;
  lb.p += h3 * vl + psb;
  rb.p += h3 * vr + psb;
  double vlb = h3 * l.p + wlb, vrb = h3 * r.p + wrb;
  vnb -= wlb + wrb;
  // coef4 = max_c0(k4 lam - c4 coef2), coef2 = k2 max_c(s, s') lam (both orientations)
  const double t4b = z4 ? 0.0 : coef4b, t4pb = z4p ? 0.0 : coef4pb;
  double lamb = in.k4 * t4b, lampb = in.k4 * t4pb;
  coef2b -= in.c4 * t4b;
  coef2pb -= in.c4 * t4pb;
  const double smb = in.k2 * lam * coef2b, smpb = in.k2 * lamp * coef2pb;
  lamb += in.k2 * sm * coef2b;
  lampb += in.k2 * smp * coef2pb;
  if (sel_s) slb += smb; else srb += smb;
  if (sel_sp) srb += smpb; else slb += smpb;
  const double alb = sel_l ? lamb : 0.0, arb = sel_l ? 0.0 : lamb;
  const double arpb = sel_lp ? lampb : 0.0, alpb = sel_lp ? 0.0 : lampb;
  // al = |vl| + cs_l len, alp = |-vl| + cs_l len, and the same for r
  vlb += sgn_c(vl) * alb - sgn_c(-vl) * alpb;
  vrb += sgn_c(vr) * arb - sgn_c(-vr) * arpb;
  lb.cs += len * (alb + alpb);
  rb.cs += len * (arb + arpb);
  lenb += l.cs * (alb + alpb) + r.cs * (arb + arpb);
  normal_velocity_rev(l, nx, nz, vlb, lb, nxb, nzb);
  normal_velocity_rev(r, nx, nz, vrb, rb, nxb, nzb);
}

// Wall ghost of state s (wall_ghost_st) in reverse: gb is the ghost's seven-component adjoint
// (consumed); adds to s's conserved components and to the wall normal / grid velocity adjoints.
__device__ __forceinline__ void wall_ghost_rev(const Sd& s, double nx, double nz, double gx,
                                               double gz, Sd gb, Sd& sb, double& nxb,
                                               double& nzb, double& gxb, double& gzb) {
  const Sd g = wall_ghost_st(s, nx, nz, gx, gz);
  derive_rev(g, gb);
  const double proj = nx * (s.j1 - gx * s.rho) + nz * (s.j2 - gz * s.rho);
  const double nn = nx * nx + nz * nz;
  const double a = 2.0 * proj / nn;  // g.j1 = s.j1 - nx a, g.j2 = s.j2 - nz a
  sb.rho += gb.rho;
  sb.j1 += gb.j1;
  sb.j2 += gb.j2;
  sb.e += gb.e;
  const double ab = -(gb.j1 * nx + gb.j2 * nz);
  nxb -= gb.j1 * a;
  nzb -= gb.j2 * a;
  const double projb = 2.0 * ab / nn, nnb = -a * ab / nn;
  nxb += 2.0 * nx * nnb + projb * (s.j1 - gx * s.rho);
  nzb += 2.0 * nz * nnb + projb * (s.j2 - gz * s.rho);
  sb.j1 += projb * nx;
  sb.j2 += projb * nz;
  sb.rho -= projb * (nx * gx + nz * gz);
  gxb -= projb * nx * s.rho;
  gzb -= projb * nz * s.rho;
}

// Far-field ghost 2 U_inf(Ma) - s (farfield_ghost_st) in reverse: gb is the ghost's
// seven-component adjoint (consumed); adds to s's conserved components and to the Mach adjoint.
__device__ __forceinline__ void farfield_ghost_rev(const Sd& s, double mach, const Instance& in,
                                                   Sd gb, Sd& sb, double& machb) {
  const Sd g = farfield_ghost_st(s, mach, in);
  derive_rev(g, gb);
  sb.rho -= gb.rho;
  sb.j1 -= gb.j1;
  sb.j2 -= gb.j2;
  sb.e -= gb.e;
  const double rg = sqrt_(kGamma), speed = mach * rg;
  machb += 2.0 * rg * (gb.j1 * in.cos_aoa + gb.j2 * in.sin_aoa + gb.e * speed);
}

}  // namespace eb
