// Shared device-side helpers of the kernel translation units: the instance table, stencil
// loading, typed (dual-number) construction of cell inputs and complex load/store helpers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <initializer_list>
#include <cstring>
#include <string>
#include <type_traits>

#include "../../include/euler_b200.h"
#include "physics.cuh"

namespace eb {

// Error reporting (defined in euler_kernels.cu).
int fail(int code, const char* msg);
int check_launch(const char* what);
int validate(const eb_batch* b);
// Grid of a per-instance kernel (y = instance; defined in euler_kernels.cu).
int per_instance_grid(const eb_batch* b, bool vertices, int per_item, int threads, dim3& grid);


static_assert(sizeof(Instance) == sizeof(eb_instance), "instance layout mismatch");

// Instance table as seen by the kernels.
struct Table {
  const Instance* dev;  // device table (null: use `single`)
  int n;
  Instance single;

  // Instance whose member `off` range contains g (binary search over a sorted table).
  template <int64_t Instance::*Off>
  __device__ __forceinline__ Instance find(int64_t g) const {
    if (dev == nullptr) return single;
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (dev[mid].*Off <= g) lo = mid; else hi = mid - 1;
    }
    return dev[lo];
  }
  __device__ __forceinline__ Instance cell(int64_t g) const { return find<&Instance::cell_offset>(g); }
  __device__ __forceinline__ Instance wall(int64_t g) const { return find<&Instance::wall_offset>(g); }
  __device__ __forceinline__ Instance vert(int64_t g) const { return find<&Instance::vert_offset>(g); }
};

inline Table make_table(const eb_batch* b) {
  Table t;
  t.dev = reinterpret_cast<const Instance*>(b->d_table);
  t.n = b->n_inst;
  std::memcpy(&t.single, &b->single, sizeof(Instance));
  return t;
}

inline int grid_for(int64_t n, int threads) {
  int64_t blocks = (n + threads - 1) / threads;
  const int64_t cap = 148 * 64;  // persistent-style cap: 148 SMs x 64 resident waves
  if (blocks > cap) blocks = cap;
  return (int)(blocks < 1 ? 1 : blocks);
}

// ---- loading ---------------------------------------------------------------------------

struct Plain {
  P2<double> x[4], w[4];
  S4<double> u[9];
  int m, n, flag;
};

__device__ __forceinline__ P2<double> ld2(const double* p) {
  const double2 v = *reinterpret_cast<const double2*>(p);
  return P2<double>{v.x, v.y};
}
__device__ __forceinline__ S4<double> ld4(const double* p) {
  const double2 a = *reinterpret_cast<const double2*>(p);
  const double2 b = *reinterpret_cast<const double2*>(p + 2);
  return S4<double>{{a.x, a.y, b.x, b.y}};
}

// Gathers the cell's stencil (the associate blocks of f90:510-530). Radial neighbours past
// the boundary are not read (the reference associates them but never uses them).
__device__ __forceinline__ void load_plain(const Instance& in, int64_t local, const double* X,
                                           const double* V, const double* U, Plain& p) {
  const int M = in.M, N = in.N;
  const int m = (int)(local % M), n = (int)(local / M);
  p.m = m;
  p.n = n;
  p.flag = boundary_flag(M, m);
  const double* Xi = X + 2 * in.vert_offset;
  const int64_t v_bi = m + (int64_t)(M + 1) * n, v_fi = m + (int64_t)(M + 1) * (n + 1);
  p.x[kBI] = ld2(Xi + 2 * v_bi);
  p.x[kFI] = ld2(Xi + 2 * v_fi);
  p.x[kFO] = ld2(Xi + 2 * (v_fi + 1));
  p.x[kBO] = ld2(Xi + 2 * (v_bi + 1));
  if (V) {
    const double* Vi = V + 2 * in.vert_offset;
    p.w[kBI] = ld2(Vi + 2 * v_bi);
    p.w[kFI] = ld2(Vi + 2 * v_fi);
    p.w[kFO] = ld2(Vi + 2 * (v_fi + 1));
    p.w[kBO] = ld2(Vi + 2 * (v_bi + 1));
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) p.w[k] = P2<double>{0.0, 0.0};
  }
  const double* Ui = U + 4 * in.cell_offset;
#pragma unroll
  for (int s = 0; s < 9; ++s) {
    const int mm = m + slot_dm(s);
    if (mm < 0 || mm >= M) {
      p.u[s] = S4<double>{{0.0, 0.0, 0.0, 0.0}};
      continue;
    }
    const int nn = wrap(n + slot_dn(s), N);
    p.u[s] = ld4(Ui + 4 * (mm + (int64_t)M * nn));
  }
}

// Complex direction (re / im parts) at the cell's stencil, for one variable kind.
struct Direction {
  P2<double> xr[4], xi[4];  // vertices or velocities
  S4<double> ur[9], ui[9];  // states
};

enum DirKind { kDirNone = -1, kDirStates = 0, kDirVertices = 1, kDirVelocities = 2 };

__device__ __forceinline__ void load_direction(const Instance& in, const Plain& p, int kind,
                                               const double* D, Direction& d) {
  const int M = in.M, N = in.N, m = p.m, n = p.n;
  if (kind == kDirStates) {
    const double* Di = D + 8 * in.cell_offset;
#pragma unroll
    for (int s = 0; s < 9; ++s) {
      const int mm = m + slot_dm(s);
      if (mm < 0 || mm >= M) {
        d.ur[s] = S4<double>{{0.0, 0.0, 0.0, 0.0}};
        d.ui[s] = d.ur[s];
        continue;
      }
      const double* q = Di + 8 * (mm + (int64_t)M * wrap(n + slot_dn(s), N));
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        d.ur[s].v[k] = q[2 * k];
        d.ui[s].v[k] = q[2 * k + 1];
      }
    }
  } else {
    const double* Di = D + 4 * in.vert_offset;
    const int64_t v[4] = {m + (int64_t)(M + 1) * n, m + (int64_t)(M + 1) * (n + 1),
                          m + 1 + (int64_t)(M + 1) * (n + 1), m + 1 + (int64_t)(M + 1) * n};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double* q = Di + 4 * v[k];
      d.xr[k] = P2<double>{q[0], q[2]};
      d.xi[k] = P2<double>{q[1], q[3]};
    }
  }
}

// ---- typed construction ------------------------------------------------------------------

using D2 = Dual<double, 2>;

// B-typed value from a plain value and (optionally) its two directional tangents.
template <class B>
EB_HD B bval(double v, double re, double im);
template <>
EB_HD double bval<double>(double v, double, double) {
  return v;
}
template <>
EB_HD D2 bval<D2>(double v, double re, double im) {
  D2 r;
  r.v = v;
  r.d[0] = re;
  r.d[1] = im;
  return r;
}

// Tangent-seeded scalar: value `b`, tangent components e_i (Dual<B, K>).
template <class B, int K>
EB_HD Dual<B, K> seed(const B& b, int i) {
  Dual<B, K> r;
  r.v = b;
#pragma unroll
  for (int j = 0; j < K; ++j) r.d[j] = lift<B>(j == i ? 1.0 : 0.0);
  return r;
}

// Typed vertex / velocity arrays: T is B when the direction targets this variable, else double.
template <class T, class B>
EB_HD void typed_corners(const P2<double>* x, const P2<double>* dr, const P2<double>* di,
                         bool with_dir, P2<T>* out) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if constexpr (std::is_same<T, double>::value) {
      out[k] = x[k];
    } else {
      out[k].x = bval<B>(x[k].x, with_dir ? dr[k].x : 0.0, with_dir ? di[k].x : 0.0);
      out[k].z = bval<B>(x[k].z, with_dir ? dr[k].z : 0.0, with_dir ? di[k].z : 0.0);
    }
  }
}

template <class T>
EB_HD void store_b(const T& v, int64_t idx, double* J, double* Jre, double* Jim) {
  if constexpr (std::is_same<T, double>::value) {
    J[idx] = v;
  } else {
    if (J) J[idx] = v.v;
    Jre[idx] = v.d[0];
    Jim[idx] = v.d[1];
  }
}


struct C2 {
  double re, im;
};
__device__ __forceinline__ C2 ldc(const double* p) {
  const double2 v = *reinterpret_cast<const double2*>(p);
  return C2{v.x, v.y};
}
__device__ __forceinline__ void stc(double* p, C2 c) {
  *reinterpret_cast<double2*>(p) = make_double2(c.re, c.im);
}

// Arrays are read and written as 16-byte vectors (4-component states, complex values, pairs of
// coordinates): every array argument must be 16-byte aligned, and a misaligned one is rejected
// with EB_ERR_ARG before any launch (null pointers pass).
inline int aligned16(std::initializer_list<const void*> ptrs) {
  for (const void* q : ptrs)
    if (reinterpret_cast<uintptr_t>(q) & 15) return fail(EB_ERR_ARG, "arrays must be 16-byte aligned");
  return EB_OK;
}

}  // namespace eb

#define EB_STREAM(s) reinterpret_cast<cudaStream_t>(s)
#define EB_ALIGNED(...)                              \
  do {                                               \
    int _rc = eb::aligned16({__VA_ARGS__});          \
    if (_rc != EB_OK) return _rc;                    \
  } while (0)

#define EB_VALIDATE(b)            \
  do {                            \
    int _rc = eb::validate(b);    \
    if (_rc != EB_OK) return _rc; \
  } while (0)
