// Jacobian kernels of the residual and the forces, templated on the base scalar B:
// B = double gives the Jacobian blocks (replacing the complex-step procedures of
// src/spatial_discretization.f90:552-1256); B = Dual<double, 2> with a direction on the states,
// vertices or velocities gives their directional derivatives (second-order routines).
#pragma once

#include "common.cuh"

namespace eb {

// Face flux kept out of line: the Jacobian kernels evaluate it up to 16 times per cell with
// wide dual types, and inlining every call makes the nested-dual kernels very large.
template <class R, class SP, class TX, class TV, class TM>
__device__ __noinline__ S4<R> face_call(int q, int flag, const SP& u, const Geometry<TX, TV>& g,
                                        const TM& mach, const Instance& in) {
  return face<R>(q, flag, u, g, mach, in);
}

// State provider for the states Jacobian: the states of slot `seed_slot` carry the identity
// tangent, every other state a zero tangent; B-level values may carry a direction.
template <class B>
struct SeededStates {
  const Plain* p;
  const Direction* d;  // null when the direction does not target the states
  int seed_slot;
  EB_HD S4<Dual<B, 4>> operator()(int s) const {
    S4<Dual<B, 4>> r;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const B b = bval<B>(p->u[s].v[k], d ? d->ur[s].v[k] : 0.0, d ? d->ui[s].v[k] : 0.0);
      r.v[k] = seed<B, 4>(b, s == seed_slot ? k : -1);
    }
    return r;
  }
};

// d(odes)/d(states) blocks (compute_odes_wrt_states, f90:666-750). B = double gives the
// Jacobian; B = Dual<double,2> with a direction gives its directional derivatives. Each slot's
// block sums only the faces that read that slot (others contribute exactly zero).
template <class B, int Dir>
__global__ void __launch_bounds__(128) k_jac_states(Table t, int64_t n_cells, const double* X,
                                                    const double* V, const double* U,
                                                    const double* D, double* J, double* Jre,
                                                    double* Jim) {
  using TX = std::conditional_t<Dir == kDirVertices, B, double>;
  using TV = std::conditional_t<Dir == kDirVelocities, B, double>;
  using R = Dual<B, 4>;
  const Instance in = t.dev ? t.dev[blockIdx.y] : t.single;  // grid y = instance
  const int64_t cells = (int64_t)in.M * in.N;
  for (int64_t local = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; local < cells;
       local += (int64_t)gridDim.x * blockDim.x) {
    Plain p;
    load_plain(in, local, X, V, U, p);
    Direction dir;
    if (Dir != kDirNone) load_direction(in, p, Dir, D, dir);
    P2<TX> x[4];
    P2<TV> w[4];
    typed_corners<TX, B>(p.x, dir.xr, dir.xi, Dir == kDirVertices, x);
    typed_corners<TV, B>(p.w, dir.xr, dir.xi, Dir == kDirVelocities, w);
    const Geometry<TX, TV> geo = geometry(x, w);
    const B area_b = lift<B>(geo.area);
    const int64_t slot_stride = 16 * (int64_t)in.M * in.N;
    const int64_t base = 144 * in.cell_offset + 16 * local;
    for (int s = 0; s < 9; ++s) {
      const int64_t o = base + slot_stride * s;
      if (!slot_active(s, p.m, in.M)) {
        for (int e = 0; e < 16; ++e) store_b<B>(lift<B>(0.0), o + e, J, Jre, Jim);
        continue;
      }
      const SeededStates<B> prov{&p, Dir == kDirStates ? &dir : nullptr, s};
      B acc[4][4];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[r][i] = lift<B>(0.0);
      for (int q = 0; q < 4; ++q) {
        if (!face_uses_slot(q, p.flag, s)) continue;
        const S4<R> f = face_call<R>(q, p.flag, prov, geo, in.mach, in);
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int i = 0; i < 4; ++i) acc[r][i] = acc[r][i] + f.v[r].d[i];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int r = 0; r < 4; ++r) store_b<B>(-acc[r][i] / area_b, o + r + 4 * i, J, Jre, Jim);
    }
  }
}

// d(odes)/d(vertices) or d(odes)/d(velocities) blocks (f90:933-993, 1087-1143).
template <class B, int Dir, bool Velo>
__global__ void __launch_bounds__(128) k_jac_vertexlike(Table t, int64_t n_cells,
                                                        const double* X, const double* V,
                                                        const double* U, const double* D,
                                                        double* J, double* Jre, double* Jim) {
  using TS = std::conditional_t<Dir == kDirStates, B, double>;
  using TXb = std::conditional_t<Dir == kDirVertices, B, double>;
  using TVb = std::conditional_t<Dir == kDirVelocities, B, double>;
  // the seeded variable is Dual<B, 2>; the other geometry variable keeps its base type
  using TX = std::conditional_t<Velo, TXb, Dual<B, 2>>;
  using TV = std::conditional_t<Velo, Dual<B, 2>, TVb>;
  const Instance in = t.dev ? t.dev[blockIdx.y] : t.single;  // grid y = instance
  const int64_t cells = (int64_t)in.M * in.N;
  for (int64_t local = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; local < cells;
       local += (int64_t)gridDim.x * blockDim.x) {
    Plain p;
    load_plain(in, local, X, V, U, p);
    Direction dir;
    if (Dir != kDirNone) load_direction(in, p, Dir, D, dir);
    Cell<TS, TX, TV, double> c;
    c.mach = in.mach;
    c.flag = p.flag;
#pragma unroll
    for (int s = 0; s < 9; ++s)
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if constexpr (std::is_same<TS, double>::value) {
          c.u[s].v[k] = p.u[s].v[k];
        } else {
          c.u[s].v[k] = bval<B>(p.u[s].v[k], Dir == kDirStates ? dir.ur[s].v[k] : 0.0,
                                Dir == kDirStates ? dir.ui[s].v[k] : 0.0);
        }
      }
    P2<B> xb[4], wb[4];
    typed_corners<B, B>(p.x, dir.xr, dir.xi, Dir == kDirVertices, xb);
    typed_corners<B, B>(p.w, dir.xr, dir.xi, Dir == kDirVelocities, wb);
    P2<TXb> xo[4];
    P2<TVb> wo[4];
    typed_corners<TXb, B>(p.x, dir.xr, dir.xi, Dir == kDirVertices, xo);
    typed_corners<TVb, B>(p.w, dir.xr, dir.xi, Dir == kDirVelocities, wo);
    const int64_t slot_stride = 8 * (int64_t)in.M * in.N;
    const int64_t base = 32 * in.cell_offset + 8 * local;
    for (int k = 0; k < 4; ++k) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if constexpr (Velo) {
          c.x[j] = xo[j];
          c.w[j].x = seed<B, 2>(wb[j].x, j == k ? 0 : -1);
          c.w[j].z = seed<B, 2>(wb[j].z, j == k ? 1 : -1);
        } else {
          c.w[j] = wo[j];
          c.x[j].x = seed<B, 2>(xb[j].x, j == k ? 0 : -1);
          c.x[j].z = seed<B, 2>(xb[j].z, j == k ? 1 : -1);
        }
      }
      const auto o = make_ode(c, in);
      const int64_t off = base + slot_stride * k;
#pragma unroll
      for (int d = 0; d < 2; ++d)
#pragma unroll
        for (int r = 0; r < 4; ++r) store_b<B>(o.v[r].d[d], off + r + 4 * d, J, Jre, Jim);
    }
  }
}

// d(odes)/d(mach) (compute_odes_wrt_mach, f90:552-593): only the far-field row is non-zero.
template <class B, int Dir>
__global__ void __launch_bounds__(128) k_jac_mach(Table t, int64_t n_cells, const double* X,
                                                  const double* V, const double* U,
                                                  const double* D, double* J, double* Jre,
                                                  double* Jim) {
  using TS = std::conditional_t<Dir == kDirStates, B, double>;
  using TX = std::conditional_t<Dir == kDirVertices, B, double>;
  using TV = std::conditional_t<Dir == kDirVelocities, B, double>;
  const Instance in = t.dev ? t.dev[blockIdx.y] : t.single;  // grid y = instance
  const int64_t cells = (int64_t)in.M * in.N;
  for (int64_t local = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; local < cells;
       local += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = in.cell_offset + local;
    const int m = (int)(local % in.M);
    if (m != in.M - 1) {
      for (int r = 0; r < 4; ++r) store_b<B>(lift<B>(0.0), 4 * g + r, J, Jre, Jim);
      continue;
    }
    Plain p;
    load_plain(in, local, X, V, U, p);
    Direction dir;
    if (Dir != kDirNone) load_direction(in, p, Dir, D, dir);
    Cell<TS, TX, TV, Dual<B, 1>> c;
    c.flag = p.flag;
    c.mach = seed<B, 1>(lift<B>(in.mach), 0);
    typed_corners<TX, B>(p.x, dir.xr, dir.xi, Dir == kDirVertices, c.x);
    typed_corners<TV, B>(p.w, dir.xr, dir.xi, Dir == kDirVelocities, c.w);
#pragma unroll
    for (int s = 0; s < 9; ++s)
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if constexpr (std::is_same<TS, double>::value) {
          c.u[s].v[k] = p.u[s].v[k];
        } else {
          c.u[s].v[k] = bval<B>(p.u[s].v[k], Dir == kDirStates ? dir.ur[s].v[k] : 0.0,
                                Dir == kDirStates ? dir.ui[s].v[k] : 0.0);
        }
      }
    const auto o = make_ode(c, in);
#pragma unroll
    for (int r = 0; r < 4; ++r) store_b<B>(o.v[r].d[0], 4 * g + r, J, Jre, Jim);
  }
}

// d(forces)/d(states) (f90:1188-1213) and its directional derivatives.
template <class B, int Dir>
__global__ void k_jac_forces_states(Table t, int64_t n_wall, const double* X, const double* U,
                                    const double* D, double* J, double* Jre, double* Jim) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_wall;
       g += (int64_t)gridDim.x * blockDim.x) {
    const Instance in = t.wall(g);
    const int n = (int)(g - in.wall_offset), M = in.M;
    const double* Xi = X + 2 * in.vert_offset;
    const int64_t va = (int64_t)(M + 1) * n, vb = (int64_t)(M + 1) * (n + 1);
    const S4<double> u = ld4(U + 4 * (in.cell_offset + (int64_t)M * n));
    P2<B> a, b;
    {
      const P2<double> a0 = ld2(Xi + 2 * va), b0 = ld2(Xi + 2 * vb);
      const double* Dx = D + 4 * in.vert_offset;
      const bool dx = Dir == kDirVertices;
      a.x = bval<B>(a0.x, dx ? Dx[4 * va] : 0.0, dx ? Dx[4 * va + 1] : 0.0);
      a.z = bval<B>(a0.z, dx ? Dx[4 * va + 2] : 0.0, dx ? Dx[4 * va + 3] : 0.0);
      b.x = bval<B>(b0.x, dx ? Dx[4 * vb] : 0.0, dx ? Dx[4 * vb + 1] : 0.0);
      b.z = bval<B>(b0.z, dx ? Dx[4 * vb + 2] : 0.0, dx ? Dx[4 * vb + 3] : 0.0);
    }
    const P2<B> nv = normal(a, b);
    S4<Dual<B, 4>> us;
    const double* Du = D + 8 * (in.cell_offset + (int64_t)M * n);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const bool du = Dir == kDirStates;
      us.v[k] = seed<B, 4>(bval<B>(u.v[k], du ? Du[2 * k] : 0.0, du ? Du[2 * k + 1] : 0.0), k);
    }
    const Dual<B, 4> p = pressure(us);
    const int64_t o = 8 * (in.wall_offset + n);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      store_b<B>(p.d[i] * nv.x, o + 2 * i, J, Jre, Jim);
      store_b<B>(p.d[i] * nv.z, o + 2 * i + 1, J, Jre, Jim);
    }
  }
}

// d(forces)/d(vertices) (f90:1227-1256) and its directional derivatives.
template <class B, int Dir>
__global__ void k_jac_forces_vertices(Table t, int64_t n_wall, const double* X,
                                      const double* U, const double* D, double* J, double* Jre,
                                      double* Jim) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_wall;
       g += (int64_t)gridDim.x * blockDim.x) {
    const Instance in = t.wall(g);
    const int n = (int)(g - in.wall_offset), M = in.M, N = in.N;
    const double* Xi = X + 2 * in.vert_offset;
    const int64_t va = (int64_t)(M + 1) * n, vb = (int64_t)(M + 1) * (n + 1);
    const S4<double> u = ld4(U + 4 * (in.cell_offset + (int64_t)M * n));
    S4<B> ub;
    const double* Du = D + 8 * (in.cell_offset + (int64_t)M * n);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const bool du = Dir == kDirStates;
      ub.v[k] = bval<B>(u.v[k], du ? Du[2 * k] : 0.0, du ? Du[2 * k + 1] : 0.0);
    }
    const B p = pressure(ub);
    const P2<double> a0 = ld2(Xi + 2 * va), b0 = ld2(Xi + 2 * vb);
    const double* Dx = D + 4 * in.vert_offset;
    const bool dx = Dir == kDirVertices;
    P2<B> a, b;
    a.x = bval<B>(a0.x, dx ? Dx[4 * va] : 0.0, dx ? Dx[4 * va + 1] : 0.0);
    a.z = bval<B>(a0.z, dx ? Dx[4 * va + 2] : 0.0, dx ? Dx[4 * va + 3] : 0.0);
    b.x = bval<B>(b0.x, dx ? Dx[4 * vb] : 0.0, dx ? Dx[4 * vb + 1] : 0.0);
    b.z = bval<B>(b0.z, dx ? Dx[4 * vb + 2] : 0.0, dx ? Dx[4 * vb + 3] : 0.0);
    for (int k = 0; k < 2; ++k) {
      P2<Dual<B, 2>> as, bs;
      as.x = seed<B, 2>(a.x, k == 0 ? 0 : -1);
      as.z = seed<B, 2>(a.z, k == 0 ? 1 : -1);
      bs.x = seed<B, 2>(b.x, k == 1 ? 0 : -1);
      bs.z = seed<B, 2>(b.z, k == 1 ? 1 : -1);
      const P2<Dual<B, 2>> nv = normal(as, bs);
      // layout (2, 2, N, 2) per instance: d + 2*(e + 2*(n + N*k)), instance base 8*wall_offset
      const int64_t base = 8 * in.wall_offset + 4 * (n + (int64_t)N * k);
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        store_b<B>(p * nv.x.d[e], base + 2 * e, J, Jre, Jim);
        store_b<B>(p * nv.z.d[e], base + 2 * e + 1, J, Jre, Jim);
      }
    }
  }
}


}  // namespace eb
