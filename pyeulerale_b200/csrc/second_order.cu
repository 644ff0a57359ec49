// C ABI of the second-order building blocks: directional derivatives of the Jacobians with
// nested duals (B = Dual<double, 2>: the real and imaginary parts of a complex direction).
// They replace the four complex-step Jacobian rebuilds per call of the reference's
// finite-difference second-order routines (src/py_euler_ale/core.py:718-1275).

#include "jacobian_kernels.cuh"

using namespace eb;

extern "C" {

#define EB_DIR_DISPATCH(KERNEL, ...)                                                        \
  switch (dir_kind) {                                                                       \
    case kDirStates:                                                                        \
      KERNEL<D2, kDirStates><<<jgrid, 128, 0, EB_STREAM(stream)>>>(__VA_ARGS__); \
      break;                                                                                \
    case kDirVertices:                                                                      \
      KERNEL<D2, kDirVertices><<<jgrid, 128, 0, EB_STREAM(stream)>>>(__VA_ARGS__); \
      break;                                                                                \
    case kDirVelocities:                                                                    \
      KERNEL<D2, kDirVelocities><<<jgrid, 128, 0, EB_STREAM(stream)>>>(__VA_ARGS__); \
      break;                                                                                \
    default:                                                                                \
      return fail(EB_ERR_ARG, "dir_kind must be 0 (states), 1 (vertices) or 2 (velocities)"); \
  }


int eb_odes_wrt_mach_dir(const eb_batch* b, const double* X, const double* V, const double* U,
                         int dir_kind, const double* d, double* J_re, double* J_im,
                         void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, V, U, d, J_re, J_im);
  if (!X || !U || !d || !J_re || !J_im) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  dim3 jgrid;
  if (int rc = per_instance_grid(b, false, 1, 128, jgrid)) return rc;
  EB_DIR_DISPATCH(k_jac_mach, t, b->n_cells, X, V, U, d, nullptr, J_re, J_im);
  return check_launch("odes_wrt_mach_dir");
}

int eb_odes_wrt_states_dir(const eb_batch* b, const double* X, const double* V,
                           const double* U, int dir_kind, const double* d, double* J_re,
                           double* J_im, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, V, U, d, J_re, J_im);
  if (!X || !U || !d || !J_re || !J_im) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  dim3 jgrid;
  if (int rc = per_instance_grid(b, false, 1, 128, jgrid)) return rc;
  EB_DIR_DISPATCH(k_jac_states, t, b->n_cells, X, V, U, d, nullptr, J_re, J_im);
  return check_launch("odes_wrt_states_dir");
}

int eb_odes_wrt_vertices_dir(const eb_batch* b, const double* X, const double* V,
                             const double* U, int dir_kind, const double* d, double* J_re,
                             double* J_im, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, V, U, d, J_re, J_im);
  if (!X || !U || !d || !J_re || !J_im) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  dim3 g;
  if (int rc = per_instance_grid(b, false, 1, 128, g)) return rc;
  cudaStream_t s = EB_STREAM(stream);
  switch (dir_kind) {
    case kDirStates:
      k_jac_vertexlike<D2, kDirStates, false><<<g, 128, 0, s>>>(t, b->n_cells, X, V, U, d,
                                                                nullptr, J_re, J_im);
      break;
    case kDirVertices:
      k_jac_vertexlike<D2, kDirVertices, false><<<g, 128, 0, s>>>(t, b->n_cells, X, V, U, d,
                                                                  nullptr, J_re, J_im);
      break;
    case kDirVelocities:
      k_jac_vertexlike<D2, kDirVelocities, false><<<g, 128, 0, s>>>(t, b->n_cells, X, V, U, d,
                                                                    nullptr, J_re, J_im);
      break;
    default:
      return fail(EB_ERR_ARG, "dir_kind must be 0 (states), 1 (vertices) or 2 (velocities)");
  }
  return check_launch("odes_wrt_vertices_dir");
}

int eb_forces_wrt_states_dir(const eb_batch* b, const double* X, const double* U,
                             int dir_kind, const double* d, double* J_re, double* J_im,
                             void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, U, d, J_re, J_im);
  if (!X || !U || !d || !J_re || !J_im) return fail(EB_ERR_ARG, "null array");
  if (dir_kind != kDirStates && dir_kind != kDirVertices)
    return fail(EB_ERR_ARG, "forces depend on states and vertices only");
  const Table t = make_table(b);
  const int g = grid_for(b->n_wall, 128);
  cudaStream_t s = EB_STREAM(stream);
  if (dir_kind == kDirStates)
    k_jac_forces_states<D2, kDirStates><<<g, 128, 0, s>>>(t, b->n_wall, X, U, d, nullptr, J_re, J_im);
  else
    k_jac_forces_states<D2, kDirVertices><<<g, 128, 0, s>>>(t, b->n_wall, X, U, d, nullptr, J_re, J_im);
  return check_launch("forces_wrt_states_dir");
}

int eb_forces_wrt_vertices_dir(const eb_batch* b, const double* X, const double* U,
                               int dir_kind, const double* d, double* J_re, double* J_im,
                               void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, U, d, J_re, J_im);
  if (!X || !U || !d || !J_re || !J_im) return fail(EB_ERR_ARG, "null array");
  if (dir_kind != kDirStates && dir_kind != kDirVertices)
    return fail(EB_ERR_ARG, "forces depend on states and vertices only");
  const Table t = make_table(b);
  const int g = grid_for(b->n_wall, 128);
  cudaStream_t s = EB_STREAM(stream);
  if (dir_kind == kDirStates)
    k_jac_forces_vertices<D2, kDirStates><<<g, 128, 0, s>>>(t, b->n_wall, X, U, d, nullptr, J_re, J_im);
  else
    k_jac_forces_vertices<D2, kDirVertices><<<g, 128, 0, s>>>(t, b->n_wall, X, U, d, nullptr, J_re, J_im);
  return check_launch("forces_wrt_vertices_dir");
}

}  // extern "C"
