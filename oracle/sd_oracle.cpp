// CPU oracle for the PyEulerALE spatial discretization -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, in C++17 complex(8) arithmetic, the Fortran module
// `src/spatial_discretization.f90` of PyEulerALE v1.1.5 (the reference). It is the
// checker for the CUDA library in `pyeulerale_b200/`: only `tests/`, the smoke check
// and the CPU baseline leg of `bench.py` load it. The product path never calls it.
//
// Parity pins: the oracle, driven through the reference's unmodified Python class
// (`src/py_euler_ale/core.py`) via the f2py-compatible shim in `oracle/shim.py`,
// reproduces the reference's committed golden outputs
// (`examples/response/Ma0p05.out`, `Ma0p5.out`, `examples/gain/Ma0p10.out`, `Ma0p50.out`)
// and passes the reference's 20 unit tests (`tests/test_linearization.py`).
//
// Arrays follow the Fortran layouts exactly (column-major, 0-based here):
//   vertices/velocities (2, M+1, N+1) complex, states/odes (4, M, N) complex,
//   d(odes)/d(states) (4, 4, M, N, 9) real, d(odes)/d(vertices) (4, 2, M, N, 4) real,
//   d(odes)/d(mach) (4, 1, M, N) real, forces (2, N) complex,
//   d(forces)/d(states) (2, 4, N) real, d(forces)/d(vertices) (2, 2, N, 2) real.
// Complex arrays are interleaved (re, im) doubles.
//
// Build: `make -C oracle` (g++ -O3 -mavx2 -mfma -fcx-fortran-rules -fopenmp).

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cplx = std::complex<double>;

// Parameters of the Fortran module (f90:52-66).
constexpr double kStep = 1e-12;                                   // complex-step size, f90:52
constexpr double kDegToRad = 0.0174532925199432957692369;        // f90:54
constexpr double kGamma = 1.4;                                    // f90:55

struct Params {
  double aoa;  // angle of attack in degrees (module variable `aoa`, f90:63)
  double k2;   // jst_k2, f90:64
  double k4;   // jst_k4, f90:65
  double c4;   // jst_c4, f90:66
};

struct S4 { cplx v[4]; };
struct P2 { cplx x, z; };

// abs_c, f90:97-102: |re| + i*im*sign(1, re) (sign honours -0.0).
inline cplx abs_c(cplx x) {
  return cplx(std::fabs(x.real()), x.imag() * std::copysign(1.0, x.real()));
}

// max_c, f90:111-120: x only if Re x > Re y + 1e-8, else y.
inline cplx max_c(cplx x, cplx y) { return (x.real() > y.real() + 1e-8) ? x : y; }

// get_pressure, f90:128-133.
inline cplx pressure(const S4& s) {
  return (kGamma - 1.0) * (s.v[3] - (s.v[1] * s.v[1] + s.v[2] * s.v[2]) / s.v[0] / 2.0);
}

// get_wave_integral, f90:142-148.
inline cplx wave_integral(const S4& s, const P2& n) {
  return abs_c((n.x * s.v[1] + n.z * s.v[2]) / s.v[0]) +
         std::sqrt(kGamma * pressure(s) / s.v[0]) * std::sqrt(n.x * n.x + n.z * n.z);
}

// make_physical_flux, f90:159-171.
inline S4 physical_flux(const S4& s, const P2& n) {
  cplx vi = (n.x * s.v[1] + n.z * s.v[2]) / s.v[0];
  cplx p = pressure(s);
  S4 f;
  f.v[0] = s.v[0] * vi;
  f.v[1] = s.v[1] * vi + n.x * p;
  f.v[2] = s.v[2] * vi + n.z * p;
  f.v[3] = (s.v[3] + p) * vi;
  return f;
}

// make_face_flux, f90:189-220. `ll`/`rr` null means the optional arguments are absent
// (no artificial dissipation on that face).
inline S4 face_flux(const S4* ll, const S4& l, const S4& r, const S4* rr, const P2& n,
                    const P2& gv, const Params& prm) {
  S4 fl = physical_flux(l, n), fr = physical_flux(r, n);
  S4 flux;
  for (int k = 0; k < 4; ++k) flux.v[k] = (fl.v[k] + fr.v[k]) / 2.0;
  if (ll && rr) {
    cplx lam_l = wave_integral(l, n), lam_r = wave_integral(r, n);
    cplx p_ll = pressure(*ll), p_l = pressure(l), p_r = pressure(r), p_rr = pressure(*rr);
    cplx lam = max_c(lam_l, lam_r);
    cplx sensor = max_c(abs_c(p_ll - 2.0 * p_l + p_r) / (p_ll + 2.0 * p_l + p_r),
                        abs_c(p_l - 2.0 * p_r + p_rr) / (p_l + 2.0 * p_r + p_rr));
    cplx coef2 = prm.k2 * sensor * lam;
    cplx coef4 = max_c(cplx(0.0, 0.0), prm.k4 * lam - prm.c4 * coef2);
    for (int k = 0; k < 4; ++k) {
      flux.v[k] = flux.v[k] - (coef2 * (r.v[k] - l.v[k]) -
                               coef4 * (rr->v[k] - 3.0 * r.v[k] + 3.0 * l.v[k] - ll->v[k]));
    }
  }
  cplx vn = gv.x * n.x + gv.z * n.z;
  for (int k = 0; k < 4; ++k) flux.v[k] = flux.v[k] - (l.v[k] + r.v[k]) / 2.0 * vn;
  return flux;
}

// make_wall_ghost_state, f90:231-240.
inline S4 wall_ghost(const S4& w, const P2& n, const P2& gv) {
  cplx proj = n.x * (w.v[1] - gv.x * w.v[0]) + n.z * (w.v[2] - gv.z * w.v[0]);
  cplx nn = n.x * n.x + n.z * n.z;
  S4 g;
  g.v[0] = w.v[0];
  g.v[1] = w.v[1] - 2.0 * n.x * proj / nn;
  g.v[2] = w.v[2] - 2.0 * n.z * proj / nn;
  g.v[3] = w.v[3];
  return g;
}

// make_free_stream_state, f90:250-259.
inline S4 free_stream(cplx mach, const Params& prm) {
  cplx speed = mach * std::sqrt(kGamma);
  double a = kDegToRad * prm.aoa;
  S4 s;
  s.v[0] = 1.0;
  s.v[1] = speed * std::cos(a);
  s.v[2] = speed * std::sin(a);
  s.v[3] = 1.0 / (kGamma - 1.0) + speed * speed / 2.0;
  return s;
}

// make_farfield_ghost_state, f90:269-274.
inline S4 farfield_ghost(cplx mach, const S4& u, const Params& prm) {
  S4 fs = free_stream(mach, prm), g;
  for (int k = 0; k < 4; ++k) g.v[k] = 2.0 * fs.v[k] - u.v[k];
  return g;
}

// make_area, f90:287-293.
inline cplx area(const P2& bi, const P2& fi, const P2& fo, const P2& bo) {
  P2 d1{fo.x - bi.x, fo.z - bi.z}, d2{bo.x - fi.x, bo.z - fi.z};
  return abs_c(d1.x * d2.z - d1.z * d2.x) / 2.0;
}

// make_normal, f90:306-311.
inline P2 normal(const P2& a, const P2& b) { return P2{b.z - a.z, a.x - b.x}; }

// make_grid_velo, f90:320-324.
inline P2 grid_velo(const P2& a, const P2& b) { return P2{(a.x + b.x) / 2.0, (a.z + b.z) / 2.0}; }

// get_boundary_flag, f90:450-464 (m is 0-based here).
inline int boundary_flag(int M, int m) {
  if (m == 0) return 1;
  if (m == 1) return 2;
  if (m == M - 2) return 4;
  if (m == M - 1) return 5;
  return 3;
}

// The cell's complete local input: 4 vertices, 4 vertex velocities, 9 stencil states.
struct Stencil {
  P2 x[4];   // bi, fi, fo, bo
  P2 v[4];   // bi, fi, fo, bo
  S4 u[9];   // c, b, bb, f, ff, i, ii, o, oo (the Jacobian slot order of f90:699-707)
  int flag;
};
enum { C = 0, B = 1, BB = 2, F = 3, FF = 4, I = 5, II = 6, O = 7, OO = 8 };

// make_ode, f90:370-436.
S4 make_ode(cplx mach, const Stencil& s, const Params& prm) {
  const P2 &bi = s.x[0], &fi = s.x[1], &fo = s.x[2], &bo = s.x[3];
  cplx a = area(bi, fi, fo, bo);
  P2 n_i = normal(bi, fi), n_f = normal(fi, fo), n_o = normal(fo, bo), n_b = normal(bo, bi);
  P2 g_i = grid_velo(s.v[0], s.v[1]), g_f = grid_velo(s.v[1], s.v[2]);
  P2 g_o = grid_velo(s.v[2], s.v[3]), g_b = grid_velo(s.v[3], s.v[0]);
  const S4* u = s.u;
  S4 fb = face_flux(&u[F], u[C], u[B], &u[BB], n_b, g_b, prm);
  S4 ff = face_flux(&u[B], u[C], u[F], &u[FF], n_f, g_f, prm);
  S4 fi_, fo_;
  switch (s.flag) {
    case 1: {
      S4 g = wall_ghost(u[C], n_i, g_i);
      fi_ = face_flux(nullptr, u[C], g, nullptr, n_i, g_i, prm);
      fo_ = face_flux(&g, u[C], u[O], &u[OO], n_o, g_o, prm);
      break;
    }
    case 2:
      fi_ = face_flux(nullptr, u[C], u[I], nullptr, n_i, g_i, prm);
      fo_ = face_flux(&u[I], u[C], u[O], &u[OO], n_o, g_o, prm);
      break;
    case 3:
      fi_ = face_flux(&u[O], u[C], u[I], &u[II], n_i, g_i, prm);
      fo_ = face_flux(&u[I], u[C], u[O], &u[OO], n_o, g_o, prm);
      break;
    case 4:
      fi_ = face_flux(&u[O], u[C], u[I], &u[II], n_i, g_i, prm);
      fo_ = face_flux(nullptr, u[C], u[O], nullptr, n_o, g_o, prm);
      break;
    default: {
      S4 g = farfield_ghost(mach, u[C], prm);
      fi_ = face_flux(&g, u[C], u[I], &u[II], n_i, g_i, prm);
      fo_ = face_flux(nullptr, u[C], g, nullptr, n_o, g_o, prm);
      break;
    }
  }
  S4 ode;
  for (int k = 0; k < 4; ++k) ode.v[k] = -(fb.v[k] + ff.v[k] + fi_.v[k] + fo_.v[k]) / a;
  return ode;
}

// ---------------------------------------------------------------------------------------
// Array access in the Fortran layouts (0-based indices).
struct Grid {
  int M, N;
  const cplx* X;  // (2, M+1, N+1)
  const cplx* V;  // (2, M+1, N+1)
  const cplx* U;  // (4, M, N)
  P2 vert(const cplx* A, int m, int n) const {
    const cplx* p = A + 2 * (m + (M + 1) * n);
    return P2{p[0], p[1]};
  }
  S4 state(int m, int n) const {
    S4 s;
    if (m < 0 || m >= M) {  // out-of-range associate of the reference; never used
      for (int k = 0; k < 4; ++k) s.v[k] = 0.0;
      return s;
    }
    const cplx* p = U + 4 * (m + M * n);
    for (int k = 0; k < 4; ++k) s.v[k] = p[k];
    return s;
  }
  // Gathers the cell's stencil (the associate blocks of f90:510-530).
  Stencil gather(int m, int n) const {
    Stencil s;
    s.x[0] = vert(X, m, n);
    s.x[1] = vert(X, m, n + 1);
    s.x[2] = vert(X, m + 1, n + 1);
    s.x[3] = vert(X, m + 1, n);
    s.v[0] = vert(V, m, n);
    s.v[1] = vert(V, m, n + 1);
    s.v[2] = vert(V, m + 1, n + 1);
    s.v[3] = vert(V, m + 1, n);
    auto wrap = [&](int k) { return ((k % N) + N) % N; };
    s.u[C] = state(m, n);
    s.u[B] = state(m, wrap(n - 1));
    s.u[BB] = state(m, wrap(n - 2));
    s.u[F] = state(m, wrap(n + 1));
    s.u[FF] = state(m, wrap(n + 2));
    s.u[I] = state(m - 1, n);
    s.u[II] = state(m - 2, n);
    s.u[O] = state(m + 1, n);
    s.u[OO] = state(m + 2, n);
    s.flag = boundary_flag(M, m);
    return s;
  }
};

inline int wrapn(int k, int N) { return ((k % N) + N) % N; }

// Cells whose Jacobian slot k exists (the `if (m > 1)` ... guards of f90:727-746).
inline bool slot_active(int k, int m, int M) {
  switch (k) {
    case I: return m > 0;
    case II: return m > 1;
    case O: return m < M - 1;
    case OO: return m < M - 2;
    default: return true;
  }
}

int g_threads = 1;  // OpenMP threads used by the oracle (1 = serial like the reference)

}  // namespace

extern "C" {

struct sdo_params { double aoa, k2, k4, c4; };

static Params to_params(const sdo_params* p) { return Params{p->aoa, p->k2, p->k4, p->c4}; }

void sdo_set_threads(int n) { g_threads = n > 0 ? n : 1; }

int sdo_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// set_free_stream_state, f90:471-482.
void sdo_set_free_stream_state(const sdo_params* p, double mre, double mim, int M, int N,
                               double* states) {
  Params prm = to_params(p);
  S4 fs = free_stream(cplx(mre, mim), prm);
  cplx* U = reinterpret_cast<cplx*>(states);
  for (long c = 0; c < (long)M * N; ++c)
    for (int k = 0; k < 4; ++k) U[4 * c + k] = fs.v[k];
}

// compute_odes, f90:496-537.
void sdo_compute_odes(const sdo_params* p, double mre, double mim, int M, int N,
                      const double* X, const double* V, const double* U, double* R) {
  Params prm = to_params(p);
  Grid g{M, N, reinterpret_cast<const cplx*>(X), reinterpret_cast<const cplx*>(V),
         reinterpret_cast<const cplx*>(U)};
  cplx mach(mre, mim);
  cplx* out = reinterpret_cast<cplx*>(R);
#pragma omp parallel for collapse(2) schedule(static) num_threads(g_threads)
  for (int n = 0; n < N; ++n)
    for (int m = 0; m < M; ++m) {
      S4 o = make_ode(mach, g.gather(m, n), prm);
      for (int k = 0; k < 4; ++k) out[4 * (m + (long)M * n) + k] = o.v[k];
    }
}

// compute_odes_wrt_mach, f90:552-593: only the far-field row depends on the Mach number.
void sdo_compute_odes_wrt_mach(const sdo_params* p, double mre, double mim, int M, int N,
                               const double* X, const double* V, const double* U,
                               double* jac) {
  Params prm = to_params(p);
  Grid g{M, N, reinterpret_cast<const cplx*>(X), reinterpret_cast<const cplx*>(V),
         reinterpret_cast<const cplx*>(U)};
  std::memset(jac, 0, sizeof(double) * 4 * (size_t)M * N);
  cplx mach(mre, mim + kStep);
  for (int n = 0; n < N; ++n) {
    Stencil s = g.gather(M - 1, n);
    s.flag = boundary_flag(M, M - 1);
    S4 o = make_ode(mach, s, prm);
    for (int k = 0; k < 4; ++k) jac[4 * ((M - 1) + (long)M * n) + k] = o.v[k].imag() / kStep;
  }
}

// apply_odes_wrt_mach_fwd, f90:604-621.
void sdo_apply_odes_wrt_mach_fwd(int M, int N, const double* jac, const double* d_mach,
                                 double* d_odes) {
  cplx dm(d_mach[0], d_mach[1]);
  cplx* out = reinterpret_cast<cplx*>(d_odes);
  for (long c = 0; c < (long)M * N; ++c)
    for (int k = 0; k < 4; ++k) out[4 * c + k] = jac[4 * c + k] * dm;
}

// apply_odes_wrt_mach_rev, f90:632-650.
void sdo_apply_odes_wrt_mach_rev(int M, int N, const double* jac, const double* d_odes,
                                 double* d_mach) {
  const cplx* w = reinterpret_cast<const cplx*>(d_odes);
  cplx acc = 0.0;
  for (long c = 0; c < (long)M * N; ++c) {
    cplx t = 0.0;
    for (int k = 0; k < 4; ++k) t += w[4 * c + k] * jac[4 * c + k];
    acc += t;
  }
  d_mach[0] = acc.real();
  d_mach[1] = acc.imag();
}

// compute_odes_wrt_states, f90:666-750: complex-step 4x4 blocks for the 9 stencil slots.
void sdo_compute_odes_wrt_states(const sdo_params* p, double mre, double mim, int M, int N,
                                 const double* X, const double* V, const double* U,
                                 double* jac) {
  Params prm = to_params(p);
  Grid g{M, N, reinterpret_cast<const cplx*>(X), reinterpret_cast<const cplx*>(V),
         reinterpret_cast<const cplx*>(U)};
  cplx mach(mre, mim);
  const size_t slot_stride = (size_t)16 * M * N;
#pragma omp parallel for collapse(2) schedule(static) num_threads(g_threads)
  for (int n = 0; n < N; ++n)
    for (int m = 0; m < M; ++m) {
      Stencil base = g.gather(m, n);
      for (int k = 0; k < 9; ++k) {
        if (!slot_active(k, m, M)) continue;  // block left untouched, as in the reference
        for (int i = 0; i < 4; ++i) {
          Stencil s = base;
          s.u[k].v[i] += cplx(0.0, kStep);
          S4 o = make_ode(mach, s, prm);
          double* blk = jac + slot_stride * k + 16 * (m + (size_t)M * n);
          for (int r = 0; r < 4; ++r) blk[r + 4 * i] = o.v[r].imag() / kStep;
        }
      }
    }
}

// convert_odes_wrt_states, f90:765-814, restated in O(nnz): for every block row the
// candidate columns of the 9-point stencil are listed with the reference's if-chain
// priority, coincident columns keep the first match, and columns are emitted in
// ascending order with 1-based indices. Returns the number of blocks written or -1 if
// `capacity` is too small.
long sdo_convert_odes_wrt_states(int M, int N, const double* jac, double* data,
                                 int32_t* indices, int32_t* indptr, long capacity) {
  const size_t slot_stride = (size_t)16 * M * N;
  long ptr = 0;
  indptr[0] = 1;
  struct Cand { long col; int prio; int slot; };
  for (int n = 0; n < N; ++n)
    for (int m = 0; m < M; ++m) {
      Cand c[9];
      int nc = 0;
      auto add = [&](int mm, int nn, int prio, int slot) {
        if (mm < 0 || mm >= M) return;
        c[nc++] = Cand{(long)mm + (long)M * nn, prio, slot};
      };
      // Order and slots of the if-chain of f90:786-803.
      add(m, wrapn(n - 1, N), 0, B);
      add(m, wrapn(n - 2, N), 1, BB);
      add(m - 1, n, 2, I);
      add(m - 2, n, 3, II);
      add(m, n, 4, C);
      add(m + 1, n, 5, O);
      add(m + 2, n, 6, OO);
      add(m, wrapn(n + 1, N), 7, F);
      add(m, wrapn(n + 2, N), 8, FF);
      std::sort(c, c + nc, [](const Cand& a, const Cand& b) {
        return a.col != b.col ? a.col < b.col : a.prio < b.prio;
      });
      for (int j = 0; j < nc; ++j) {
        if (j > 0 && c[j].col == c[j - 1].col) continue;
        if (ptr >= capacity) return -1;
        const double* blk = jac + slot_stride * c[j].slot + 16 * (m + (size_t)M * n);
        std::memcpy(data + 16 * ptr, blk, 16 * sizeof(double));
        indices[ptr] = (int32_t)(c[j].col + 1);
        ++ptr;
      }
      indptr[m + (long)M * n + 1] = (int32_t)(ptr + 1);
    }
  return ptr;
}

// apply_odes_wrt_states_fwd, f90:825-864.
void sdo_apply_odes_wrt_states_fwd(int M, int N, const double* jac, const double* d_states,
                                   double* d_odes) {
  const cplx* x = reinterpret_cast<const cplx*>(d_states);
  cplx* y = reinterpret_cast<cplx*>(d_odes);
  const size_t slot_stride = (size_t)16 * M * N;
  for (int n = 0; n < N; ++n)
    for (int m = 0; m < M; ++m) {
      const int nb[9][2] = {{m, n}, {m, wrapn(n - 1, N)}, {m, wrapn(n - 2, N)},
                            {m, wrapn(n + 1, N)}, {m, wrapn(n + 2, N)}, {m - 1, n},
                            {m - 2, n}, {m + 1, n}, {m + 2, n}};
      cplx acc[4] = {0.0, 0.0, 0.0, 0.0};
      // Summation order of f90:856-861: c, b, bb, f, ff, then ii, i, oo, o.
      const int order[9] = {C, B, BB, F, FF, II, I, OO, O};
      for (int q = 0; q < 9; ++q) {
        int k = order[q];
        if (!slot_active(k, m, M)) continue;
        const double* blk = jac + slot_stride * k + 16 * (m + (size_t)M * n);
        const cplx* xv = x + 4 * (nb[k][0] + (size_t)M * nb[k][1]);
        for (int r = 0; r < 4; ++r) {
          cplx t = 0.0;
          for (int i = 0; i < 4; ++i) t += blk[r + 4 * i] * xv[i];
          acc[r] += t;
        }
      }
      for (int r = 0; r < 4; ++r) y[4 * (m + (size_t)M * n) + r] = acc[r];
    }
}

// apply_odes_wrt_states_rev, f90:875-918 (scatter-add in the reference's order).
void sdo_apply_odes_wrt_states_rev(int M, int N, const double* jac, const double* d_odes,
                                   double* d_states) {
  const cplx* w = reinterpret_cast<const cplx*>(d_odes);
  cplx* y = reinterpret_cast<cplx*>(d_states);
  const size_t slot_stride = (size_t)16 * M * N;
  for (long c = 0; c < 4L * M * N; ++c) y[c] = 0.0;
  for (int n = 0; n < N; ++n)
    for (int m = 0; m < M; ++m) {
      const int nb[9][2] = {{m, n}, {m, wrapn(n - 1, N)}, {m, wrapn(n - 2, N)},
                            {m, wrapn(n + 1, N)}, {m, wrapn(n + 2, N)}, {m - 1, n},
                            {m - 2, n}, {m + 1, n}, {m + 2, n}};
      const cplx* wv = w + 4 * (m + (size_t)M * n);
      for (int k = 0; k < 9; ++k) {
        if (!slot_active(k, m, M)) continue;
        const double* blk = jac + slot_stride * k + 16 * (m + (size_t)M * n);
        cplx* yv = y + 4 * (nb[k][0] + (size_t)M * nb[k][1]);
        for (int i = 0; i < 4; ++i) {
          cplx t = 0.0;
          for (int r = 0; r < 4; ++r) t += wv[r] * blk[r + 4 * i];
          yv[i] += t;
        }
      }
    }
}

// compute_odes_wrt_vertices, f90:933-993, and compute_odes_wrt_velocities, f90:1087-1143:
// complex-step 4x2 blocks for the cell's 4 vertices (bi, fi, fo, bo).
static void odes_wrt_vertexlike(const sdo_params* p, double mre, double mim, int M, int N,
                                const double* X, const double* V, const double* U,
                                double* jac, bool velocities) {
  Params prm = to_params(p);
  Grid g{M, N, reinterpret_cast<const cplx*>(X), reinterpret_cast<const cplx*>(V),
         reinterpret_cast<const cplx*>(U)};
  cplx mach(mre, mim);
  const size_t slot_stride = (size_t)8 * M * N;
#pragma omp parallel for collapse(2) schedule(static) num_threads(g_threads)
  for (int n = 0; n < N; ++n)
    for (int m = 0; m < M; ++m) {
      Stencil base = g.gather(m, n);
      for (int k = 0; k < 4; ++k)
        for (int d = 0; d < 2; ++d) {
          Stencil s = base;
          P2& tgt = velocities ? s.v[k] : s.x[k];
          (d == 0 ? tgt.x : tgt.z) += cplx(0.0, kStep);
          S4 o = make_ode(mach, s, prm);
          double* blk = jac + slot_stride * k + 8 * (m + (size_t)M * n);
          for (int r = 0; r < 4; ++r) blk[r + 4 * d] = o.v[r].imag() / kStep;
        }
    }
}

void sdo_compute_odes_wrt_vertices(const sdo_params* p, double mre, double mim, int M, int N,
                                   const double* X, const double* V, const double* U,
                                   double* jac) {
  odes_wrt_vertexlike(p, mre, mim, M, N, X, V, U, jac, false);
}

void sdo_compute_odes_wrt_velocities(const sdo_params* p, double mre, double mim, int M,
                                     int N, const double* X, const double* V, const double* U,
                                     double* jac) {
  odes_wrt_vertexlike(p, mre, mim, M, N, X, V, U, jac, true);
}

// apply_odes_wrt_vertices_fwd, f90:1005-1032 (also used for the velocities).
void sdo_apply_odes_wrt_vertices_fwd(int M, int N, const double* jac,
                                     const double* d_vertices, double* d_odes) {
  const cplx* x = reinterpret_cast<const cplx*>(d_vertices);
  cplx* y = reinterpret_cast<cplx*>(d_odes);
  const size_t slot_stride = (size_t)8 * M * N;
  for (int n = 0; n < N; ++n)
    for (int m = 0; m < M; ++m) {
      const int vx[4][2] = {{m, n}, {m, n + 1}, {m + 1, n + 1}, {m + 1, n}};
      cplx acc[4] = {0.0, 0.0, 0.0, 0.0};
      for (int k = 0; k < 4; ++k) {
        const double* blk = jac + slot_stride * k + 8 * (m + (size_t)M * n);
        const cplx* xv = x + 2 * (vx[k][0] + (size_t)(M + 1) * vx[k][1]);
        for (int r = 0; r < 4; ++r) acc[r] += blk[r] * xv[0] + blk[r + 4] * xv[1];
      }
      for (int r = 0; r < 4; ++r) y[4 * (m + (size_t)M * n) + r] = acc[r];
    }
}

// apply_odes_wrt_vertices_rev, f90:1044-1072.
void sdo_apply_odes_wrt_vertices_rev(int M, int N, const double* jac, const double* d_odes,
                                     double* d_vertices) {
  const cplx* w = reinterpret_cast<const cplx*>(d_odes);
  cplx* y = reinterpret_cast<cplx*>(d_vertices);
  const size_t slot_stride = (size_t)8 * M * N;
  for (long c = 0; c < 2L * (M + 1) * (N + 1); ++c) y[c] = 0.0;
  for (int n = 0; n < N; ++n)
    for (int m = 0; m < M; ++m) {
      const int vx[4][2] = {{m, n}, {m, n + 1}, {m + 1, n + 1}, {m + 1, n}};
      const cplx* wv = w + 4 * (m + (size_t)M * n);
      for (int k = 0; k < 4; ++k) {
        const double* blk = jac + slot_stride * k + 8 * (m + (size_t)M * n);
        cplx* yv = y + 2 * (vx[k][0] + (size_t)(M + 1) * vx[k][1]);
        for (int d = 0; d < 2; ++d) {
          cplx t = 0.0;
          for (int r = 0; r < 4; ++r) t += wv[r] * blk[r + 4 * d];
          yv[d] += t;
        }
      }
    }
}

// compute_forces, f90:1156-1174.
void sdo_compute_forces(int M, int N, const double* X, const double* U, double* F) {
  Grid g{M, N, reinterpret_cast<const cplx*>(X), nullptr, reinterpret_cast<const cplx*>(U)};
  cplx* out = reinterpret_cast<cplx*>(F);
  for (int n = 0; n < N; ++n) {
    cplx p = pressure(g.state(0, n));
    P2 nv = normal(g.vert(g.X, 0, n), g.vert(g.X, 0, n + 1));
    out[2 * n] = p * nv.x;
    out[2 * n + 1] = p * nv.z;
  }
}

// compute_forces_wrt_states, f90:1188-1213.
void sdo_compute_forces_wrt_states(int M, int N, const double* X, const double* U,
                                   double* jac) {
  Grid g{M, N, reinterpret_cast<const cplx*>(X), nullptr, reinterpret_cast<const cplx*>(U)};
  for (int n = 0; n < N; ++n) {
    P2 nv = normal(g.vert(g.X, 0, n), g.vert(g.X, 0, n + 1));
    for (int i = 0; i < 4; ++i) {
      S4 s = g.state(0, n);
      s.v[i] += cplx(0.0, kStep);
      cplx p = pressure(s);
      jac[0 + 2 * (i + 4 * n)] = (p * nv.x).imag() / kStep;
      jac[1 + 2 * (i + 4 * n)] = (p * nv.z).imag() / kStep;
    }
  }
}

// apply_forces_wrt_states_fwd, f90:1333-1348.
void sdo_apply_forces_wrt_states_fwd(int M, int N, const double* jac, const double* d_states,
                                     double* d_forces) {
  const cplx* x = reinterpret_cast<const cplx*>(d_states);
  cplx* y = reinterpret_cast<cplx*>(d_forces);
  for (int n = 0; n < N; ++n) {
    const cplx* xv = x + 4 * ((size_t)M * n);
    for (int d = 0; d < 2; ++d) {
      cplx t = 0.0;
      for (int i = 0; i < 4; ++i) t += jac[d + 2 * (i + 4 * n)] * xv[i];
      y[2 * n + d] = t;
    }
  }
}

// apply_forces_wrt_states_rev, f90:1359-1375.
void sdo_apply_forces_wrt_states_rev(int M, int N, const double* jac, const double* d_forces,
                                     double* d_states) {
  const cplx* w = reinterpret_cast<const cplx*>(d_forces);
  cplx* y = reinterpret_cast<cplx*>(d_states);
  for (long c = 0; c < 4L * M * N; ++c) y[c] = 0.0;
  for (int n = 0; n < N; ++n) {
    cplx* yv = y + 4 * ((size_t)M * n);
    for (int i = 0; i < 4; ++i) {
      cplx t = 0.0;
      for (int d = 0; d < 2; ++d) t += w[2 * n + d] * jac[d + 2 * (i + 4 * n)];
      yv[i] = t;
    }
  }
}

// compute_forces_wrt_vertices, f90:1227-1256.
void sdo_compute_forces_wrt_vertices(int M, int N, const double* X, const double* U,
                                     double* jac) {
  Grid g{M, N, reinterpret_cast<const cplx*>(X), nullptr, reinterpret_cast<const cplx*>(U)};
  for (int n = 0; n < N; ++n) {
    cplx p = pressure(g.state(0, n));
    for (int k = 0; k < 2; ++k)
      for (int e = 0; e < 2; ++e) {
        P2 a = g.vert(g.X, 0, n), b = g.vert(g.X, 0, n + 1);
        P2& t = (k == 0) ? a : b;
        (e == 0 ? t.x : t.z) += cplx(0.0, kStep);
        P2 nv = normal(a, b);
        jac[0 + 2 * (e + 2 * (n + (size_t)N * k))] = (p * nv.x).imag() / kStep;
        jac[1 + 2 * (e + 2 * (n + (size_t)N * k))] = (p * nv.z).imag() / kStep;
      }
  }
}

// apply_forces_wrt_vertices_fwd, f90:1267-1288.
void sdo_apply_forces_wrt_vertices_fwd(int M, int N, const double* jac,
                                       const double* d_vertices, double* d_forces) {
  const cplx* x = reinterpret_cast<const cplx*>(d_vertices);
  cplx* y = reinterpret_cast<cplx*>(d_forces);
  for (int n = 0; n < N; ++n) {
    const cplx* a = x + 2 * ((size_t)(M + 1) * n);
    const cplx* b = x + 2 * ((size_t)(M + 1) * (n + 1));
    for (int d = 0; d < 2; ++d) {
      cplx t0 = jac[d + 2 * (0 + 2 * (n + (size_t)N * 0))] * a[0] +
                jac[d + 2 * (1 + 2 * (n + (size_t)N * 0))] * a[1];
      cplx t1 = jac[d + 2 * (0 + 2 * (n + (size_t)N * 1))] * b[0] +
                jac[d + 2 * (1 + 2 * (n + (size_t)N * 1))] * b[1];
      y[2 * n + d] = t0 + t1;
    }
  }
}

// apply_forces_wrt_vertices_rev, f90:1299-1322.
void sdo_apply_forces_wrt_vertices_rev(int M, int N, const double* jac, const double* d_forces,
                                       double* d_vertices) {
  const cplx* w = reinterpret_cast<const cplx*>(d_forces);
  cplx* y = reinterpret_cast<cplx*>(d_vertices);
  for (long c = 0; c < 2L * (M + 1) * (N + 1); ++c) y[c] = 0.0;
  for (int n = 0; n < N; ++n) {
    for (int k = 0; k < 2; ++k) {
      cplx* yv = y + 2 * ((size_t)(M + 1) * (n + k));
      for (int e = 0; e < 2; ++e) {
        cplx t = w[2 * n] * jac[0 + 2 * (e + 2 * (n + (size_t)N * k))] +
                 w[2 * n + 1] * jac[1 + 2 * (e + 2 * (n + (size_t)N * k))];
        yv[e] += t;
      }
    }
  }
}

}  // extern "C"
