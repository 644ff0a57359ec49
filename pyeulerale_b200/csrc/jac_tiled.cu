// Tiled d(odes)/d(states) Jacobian (eb_compute_odes_wrt_states, replacing the complex-step
// compute_odes_wrt_states of src/spatial_discretization.f90:666-750): the nine 4 x 4 blocks of
// every cell, in the reference layout (4, 4, M, N, 9).
//
// It follows the tiled residual kernel: one CTA stages a tile of states (with a two-cell cross
// halo, periodic in the angular index) and its vertices in shared memory, derives 1/rho, p and
// c once per staged state, and evaluates every face once for both of its cells (jst_pair,
// tile_faces.cuh). A face's flux depends on the four states of its stencil line (ll, l, r, rr);
// the face is evaluated four times, each time with one of the four seeded as a four-component
// dual number (the other three and the geometry stay plain doubles), which gives the 4 x 4
// derivative blocks of both cells' fluxes with respect to that state. A cell's block for slot s
// sums the derivatives of its faces with respect to the state in slot s; the reference sums the
// same face terms in the same order, -(((F_b + F_f) + F_i) + F_o) / area (f90:395-400). The
// sensors (f90:208-211) are recomputed from the staged pressures with the seeded one dual.
//
// The seeded state's four conserved variables are differentiated kW at a time: with kW = 4 one
// pass over the faces (255 registers, one CTA per SM), with kW = 2 two passes that repeat the
// value arithmetic but hold half the derivative state (two CTAs per SM). Each derivative
// component is formed by the same operations either way, so both give identical blocks.
//
// Layout of a CTA: a tile of kTM = 32 radial x kTN = 7 angular cells on 256 threads; thread
// (r, c), c < 8, evaluates the angular face between cells (r, c - 1) and (r, c), so the tile's
// 32 x 8 angular faces take one evaluation per thread, and thread (r, c < 7) the radial face
// between cells (r - 1, c) and (r, c), the seven radial faces past the tile's outer row going to
// threads (r < 7, 7). A face's flux for its own cell (r, c) stays in the thread; the flux for the
// neighbour goes through shared memory. Per seeded stencil position each cell's blocks are
// finished in a fixed order (angular: ff, f, bb, b; radial: oo, o, c, ii, i), so a thread keeps
// at most two unfinished blocks.
//
// Compiled without FMA contraction (as the other Jacobian kernels): the values of the seeded
// dual evaluation then equal the plain ones bit for bit, so branch decisions (abs_c, max_c) at
// exact ties, e.g. an exact free stream, are those of the reference.

#include "common.cuh"
#include "autotune.cuh"
#include "tile_faces.cuh"

namespace eb {
namespace jt {

constexpr int kTM = 32;                 // radial cells per tile
constexpr int kTN = 7;                  // angular cells per tile
constexpr int kThreads = kTM * (kTN + 1);
constexpr int kSR = kTM + 4;            // staged rows (radial halo 2)
constexpr int kSC = kTN + 4;            // staged columns (angular halo 2)
constexpr int kStaged = kSR * kSC;
constexpr int kVR = kTM + 1, kVC = kTN + 1;
constexpr int kVerts = kVR * kVC;

__device__ __forceinline__ int sidx(int r, int c) { return (c + 2) * kSR + (r + 2); }
__device__ __forceinline__ int vidx(int r, int c) { return c * kVR + r; }

namespace w4 {
#define EB_JT_WIDTH 4
#include "jac_tiled_pass.cuh"
#undef EB_JT_WIDTH
}  // namespace w4

namespace w2 {
#define EB_JT_WIDTH 2
#include "jac_tiled_pass.cuh"
#undef EB_JT_WIDTH
}  // namespace w2

int tiles(int M, int N) { return ((M + kTM - 1) / kTM) * ((N + kTN - 1) / kTN); }

}  // namespace jt

// One launch of the W-wide pass (namespace w4 or w2).
template <int W>
int launch_width(const eb_batch* b, const Table& t, int dim, const double* X, const double* V,
                 const double* U, double* J, cudaStream_t stream) {
  using namespace jt;
  auto kernel = W == 4 ? w4::k_jac_states_tiled : w2::k_jac_states_tiled;
  const int smem = W == 4 ? (int)sizeof(w4::Smem) : (int)sizeof(w2::Smem);
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
      cudaSuccess)
    return check_launch("compute_odes_wrt_states attribute");
  kernel<<<dim3(tiles(dim, dim), b->n_inst), kThreads, smem, stream>>>(t, X, V, U, J);
  return check_launch("compute_odes_wrt_states");
}

int launch_jac_states_tiled(const eb_batch* b, const double* X, const double* V,
                            const double* U, double* J, cudaStream_t stream) {
  int dim = b->max_dim;
  if (b->n_inst == 1 && b->d_table == nullptr) dim = std::max(b->single.M, b->single.N);
  if (dim < 5) return fail(EB_ERR_ARG, "batch max_dim must be the largest M or N");
  if (b->n_inst > 65535) return fail(EB_ERR_ARG, "at most 65535 instances per batch");
  const Table t = make_table(b);
  static const char* const kNames[2] = {"width 4, 1 CTA/SM", "width 2, 2 CTAs/SM"};
  return tune::launch_tuned("jac_states_tiled", b->n_cells, dim, 2, 0, kNames, stream,
                            [&](int v) {
                              return v == 0 ? launch_width<4>(b, t, dim, X, V, U, J, stream)
                                            : launch_width<2>(b, t, dim, X, V, U, J, stream);
                            });
}

}  // namespace eb
