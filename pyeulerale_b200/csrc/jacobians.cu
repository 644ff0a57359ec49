// C ABI of the first-order Jacobians (dual-number kernels of jacobian_kernels.cuh with
// B = double), replacing the complex-step procedures of src/spatial_discretization.f90.

#include "jacobian_kernels.cuh"

using namespace eb;

namespace eb {
// The tiled states Jacobian (jac_tiled.cu).
int launch_jac_states_tiled(const eb_batch* b, const double* X, const double* V,
                            const double* U, double* J, cudaStream_t stream);
}  // namespace eb

extern "C" {

int eb_compute_odes_wrt_mach(const eb_batch* b, const double* X, const double* V,
                             const double* U, double* J, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, V, U, J);
  if (!X || !U || !J) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  dim3 jgrid;
  if (int rc = per_instance_grid(b, false, 1, 128, jgrid)) return rc;
  k_jac_mach<double, kDirNone><<<jgrid, 128, 0, EB_STREAM(stream)>>>(
      t, b->n_cells, X, V, U, nullptr, J, nullptr, nullptr);
  return check_launch("compute_odes_wrt_mach");
}

int eb_compute_odes_wrt_states(const eb_batch* b, const double* X, const double* V,
                               const double* U, double* J, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, V, U, J);
  if (!X || !U || !J) return fail(EB_ERR_ARG, "null array");
  return launch_jac_states_tiled(b, X, V, U, J, EB_STREAM(stream));
}

// The per-cell states Jacobian (one thread per cell, each block from its own face evaluations).
// Kept as the plain variant for comparison; the tiled kernel serves eb_compute_odes_wrt_states.
int eb_compute_odes_wrt_states_untiled(const eb_batch* b, const double* X, const double* V,
                                       const double* U, double* J, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, V, U, J);
  if (!X || !U || !J) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  dim3 jgrid;
  if (int rc = per_instance_grid(b, false, 1, 128, jgrid)) return rc;
  k_jac_states<double, kDirNone><<<jgrid, 128, 0, EB_STREAM(stream)>>>(
      t, b->n_cells, X, V, U, nullptr, J, nullptr, nullptr);
  return check_launch("compute_odes_wrt_states_untiled");
}

int eb_compute_odes_wrt_vertices(const eb_batch* b, const double* X, const double* V,
                                 const double* U, double* J, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, V, U, J);
  if (!X || !U || !J) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  dim3 jgrid;
  if (int rc = per_instance_grid(b, false, 1, 128, jgrid)) return rc;
  k_jac_vertexlike<double, kDirNone, false>
      <<<jgrid, 128, 0, EB_STREAM(stream)>>>(t, b->n_cells, X, V, U,
                                                                  nullptr, J, nullptr, nullptr);
  return check_launch("compute_odes_wrt_vertices");
}

int eb_compute_odes_wrt_velocities(const eb_batch* b, const double* X, const double* V,
                                   const double* U, double* J, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, V, U, J);
  if (!X || !U || !J) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  dim3 jgrid;
  if (int rc = per_instance_grid(b, false, 1, 128, jgrid)) return rc;
  k_jac_vertexlike<double, kDirNone, true>
      <<<jgrid, 128, 0, EB_STREAM(stream)>>>(t, b->n_cells, X, V, U,
                                                                  nullptr, J, nullptr, nullptr);
  return check_launch("compute_odes_wrt_velocities");
}

int eb_compute_forces_wrt_states(const eb_batch* b, const double* X, const double* U,
                                 double* J, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, U, J);
  if (!X || !U || !J) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  k_jac_forces_states<double, kDirNone><<<grid_for(b->n_wall, 128), 128, 0, EB_STREAM(stream)>>>(
      t, b->n_wall, X, U, nullptr, J, nullptr, nullptr);
  return check_launch("compute_forces_wrt_states");
}

int eb_compute_forces_wrt_vertices(const eb_batch* b, const double* X, const double* U,
                                   double* J, void* stream) {
  EB_VALIDATE(b);
  EB_ALIGNED(X, U, J);
  if (!X || !U || !J) return fail(EB_ERR_ARG, "null array");
  const Table t = make_table(b);
  k_jac_forces_vertices<double, kDirNone>
      <<<grid_for(b->n_wall, 128), 128, 0, EB_STREAM(stream)>>>(t, b->n_wall, X, U, nullptr, J,
                                                                 nullptr, nullptr);
  return check_launch("compute_forces_wrt_vertices");
}

}  // extern "C"
