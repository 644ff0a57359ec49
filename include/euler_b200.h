/*
 * euler_b200 -- C ABI of the B200 (sm_100a) spatial discretization of the 2D Euler ALE
 * equations on O-grids, a drop-in for the native layer of PyEulerALE v1.1.5.
 *
 * The reference reaches its native code through the f2py module
 * `py_euler_ale.euler_ale.spatial_discretization` (src/spatial_discretization.f90, bound by
 * meson.build:21-35): 20 procedures plus 4 module variables (aoa, jst_k2, jst_k4, jst_c4,
 * f90:63-66) that are set before each call (src/py_euler_ale/core.py:258-263). Each entry
 * point below replaces one of those procedures; the module variables become fields of
 * `eb_instance`, so calls are reentrant and instances with different parameters can be
 * batched.
 *
 * Conventions
 *  - All array pointers are DEVICE pointers (FP64). Layouts are the reference's Fortran
 *    layouts (column-major): vertices / velocities (2, M+1, N+1), states / odes (4, M, N),
 *    d(odes)/d(states) (4, 4, M, N, 9), d(odes)/d(vertices|velocities) (4, 2, M, N, 4),
 *    d(odes)/d(mach) (4, 1, M, N), forces (2, N), d(forces)/d(states) (2, 4, N),
 *    d(forces)/d(vertices) (2, 2, N, 2). Complex arrays are interleaved (re, im) doubles.
 *  - Every array pointer must be 16-byte aligned (the kernels move states, complex values and
 *    coordinate pairs as 16-byte vectors); a misaligned array is rejected with EB_ERR_ARG
 *    before anything is launched.
 *  - The states, vertices and velocities are real here: the reference stores them as
 *    complex128 only to run its complex-step differentiation, and its public API exposes
 *    their real parts (core.py:159-211).
 *  - Several grids ("instances") may be packed back to back: instance i owns cells
 *    [cell_offset, cell_offset + M*N) and vertices [vert_offset, vert_offset + (M+1)(N+1)).
 *    Per-cell arrays are indexed with the cell offset times the per-cell size (4 for states,
 *    144 for d(odes)/d(states), ...), per-vertex arrays with the vertex offset times 2, and
 *    per-wall-face arrays (forces) with the instance's angular offset `wall_offset`.
 *  - `stream` is a cudaStream_t (NULL = legacy default stream). Calls are asynchronous
 *    unless stated; nothing allocates device memory except where stated.
 *  - Return value: EB_OK or a negative EB_ERR_* code; eb_last_error() describes it.
 *  - Grids need M >= 4 radial and N >= 5 angular cells (the 9-point stencil reaches two
 *    cells in each direction; the reference indexes out of bounds below that).
 */
#ifndef EULER_B200_H
#define EULER_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EB_OK 0
#define EB_ERR_ARG (-1)      /* invalid argument (sizes, null pointer, table) */
#define EB_ERR_CUDA (-2)     /* a CUDA runtime call failed */
#define EB_ERR_NOCONV (-3)   /* an iterative solve hit its iteration limit */
#define EB_ERR_NAN (-4)      /* a NaN / Inf appeared in a solve */

/* One grid with its flow parameters (104 bytes). */
typedef struct eb_instance {
  int32_t M;            /* cells in the radial direction (num_radial) */
  int32_t N;            /* cells in the angular direction (num_angular) */
  int64_t cell_offset;  /* first cell of this instance in the packed per-cell arrays */
  int64_t vert_offset;  /* first vertex of this instance in the packed per-vertex arrays */
  int64_t wall_offset;  /* first wall face of this instance in the packed per-wall arrays */
  double mach;          /* free-stream Mach number */
  double cos_aoa;       /* cos(angle of attack) -- the reference's `aoa` in degrees, f90:253 */
  double sin_aoa;       /* sin(angle of attack) */
  double k2, k4, c4;    /* JST constants jst_k2, jst_k4, jst_c4 (f90:64-66) */
  double chord;         /* coefficient_length (core.py:65) */
  double xc, zc;        /* coefficient_center (core.py:66) */
} eb_instance;

/* A set of instances. For a single grid set n_inst = 1, d_table = NULL and fill `single`;
 * otherwise d_table is a DEVICE array of n_inst (at most 65535) instances sorted by
 * cell_offset, and max_dim must hold the largest M or N: the per-instance kernels run one grid
 * row per instance sized by it (EB_ERR_ARG otherwise). */
typedef struct eb_batch {
  const eb_instance* d_table;
  int32_t n_inst;
  int32_t max_dim;      /* largest M or N over the instances (0: only `single` is used) */
  int64_t n_cells;      /* total cells over all instances */
  int64_t n_verts;      /* total vertices over all instances */
  int64_t n_wall;       /* total wall faces (sum of N) over all instances */
  eb_instance single;
} eb_batch;

/* Text of the last error on the calling thread. */
const char* eb_last_error(void);
/* Library version string. */
const char* eb_version(void);

/* ---- residual and forces -------------------------------------------------------------- */

/* set_free_stream_state, f90:471-482: U(:, m, n) = free-stream state of each instance. */
int eb_set_free_stream_state(const eb_batch* b, double* U, void* stream);

/* compute_odes, f90:496-537: R = R(Ma, U, X, V). V may be NULL (static grid). */
int eb_compute_odes(const eb_batch* b, const double* X, const double* V, const double* U,
                    double* R, void* stream);

/* The same residual by the plain one-thread-per-cell kernel (every stencil state read from
 * global memory, the reference's per-face recomputation); a baseline for the tiled kernel. */
int eb_compute_odes_untiled(const eb_batch* b, const double* X, const double* V,
                            const double* U, double* R, void* stream);

/* compute_forces, f90:1156-1174: F(:, n) = p(U(:, 1, n)) * normal(X(:, 1, n), X(:, 1, n+1)).
 * F is real (2, N) per instance at 2*wall_offset. coef (optional, may be NULL) receives per
 * instance (c_d, c_l, c_m) as core.py:1277-1364 defines them, with the instance's chord and
 * moment centre; the wall sums are warp-shuffle reductions, one CTA per instance. */
int eb_compute_forces(const eb_batch* b, const double* X, const double* U, double* F,
                      double* coef, void* stream);

/* ---- Jacobians (replacing the complex-step procedures) ------------------------------- */

/* compute_odes_wrt_mach, f90:552-593. J: (4, 1, M, N) per instance, 4*cell_offset. */
int eb_compute_odes_wrt_mach(const eb_batch* b, const double* X, const double* V,
                             const double* U, double* J, void* stream);
/* compute_odes_wrt_states, f90:666-750. J: (4, 4, M, N, 9) per instance, 144*cell_offset.
 * Blocks the reference does not compute (slots reaching past the radial boundary) are 0.
 * Tiled kernel: each face evaluated once for both cells, per seeded stencil state. */
int eb_compute_odes_wrt_states(const eb_batch* b, const double* X, const double* V,
                               const double* U, double* J, void* stream);
/* The same Jacobian by the plain one-thread-per-cell kernel (each slot's block from that cell's
 * own face evaluations, as the reference's per-cell complex step); a baseline for the tiled
 * kernel. */
int eb_compute_odes_wrt_states_untiled(const eb_batch* b, const double* X, const double* V,
                                       const double* U, double* J, void* stream);
/* compute_odes_wrt_vertices, f90:933-993. J: (4, 2, M, N, 4) per instance, 32*cell_offset. */
int eb_compute_odes_wrt_vertices(const eb_batch* b, const double* X, const double* V,
                                 const double* U, double* J, void* stream);
/* compute_odes_wrt_velocities, f90:1087-1143. Same layout as the vertices. */
int eb_compute_odes_wrt_velocities(const eb_batch* b, const double* X, const double* V,
                                   const double* U, double* J, void* stream);
/* compute_forces_wrt_states, f90:1188-1213. J: (2, 4, N) per instance, 8*wall_offset. */
int eb_compute_forces_wrt_states(const eb_batch* b, const double* X, const double* U,
                                 double* J, void* stream);
/* compute_forces_wrt_vertices, f90:1227-1256. J: (2, 2, N, 2) per instance, 8*wall_offset. */
int eb_compute_forces_wrt_vertices(const eb_batch* b, const double* X, const double* U,
                                   double* J, void* stream);

/* ---- Jacobian products (complex vectors, real Jacobians) ------------------------------ */

/* apply_odes_wrt_mach_fwd / _rev, f90:604-650. d_mach: one complex per instance. */
int eb_apply_odes_wrt_mach_fwd(const eb_batch* b, const double* J, const double* d_mach,
                               double* d_odes, void* stream);
int eb_apply_odes_wrt_mach_rev(const eb_batch* b, const double* J, const double* d_odes,
                               double* d_mach, void* stream);
/* apply_odes_wrt_states_fwd / _rev, f90:825-918. The reverse product gathers the
 * transposed stencil (no atomics, deterministic). */
int eb_apply_odes_wrt_states_fwd(const eb_batch* b, const double* J, const double* d_states,
                                 double* d_odes, void* stream);
int eb_apply_odes_wrt_states_rev(const eb_batch* b, const double* J, const double* d_odes,
                                 double* d_states, void* stream);
/* apply_odes_wrt_vertices_fwd / _rev, f90:1005-1072 (also used with the velocity
 * Jacobians, core.py:480-481, 508-509). */
int eb_apply_odes_wrt_vertices_fwd(const eb_batch* b, const double* J,
                                   const double* d_vertices, double* d_odes, void* stream);
int eb_apply_odes_wrt_vertices_rev(const eb_batch* b, const double* J, const double* d_odes,
                                   double* d_vertices, void* stream);
/* apply_forces_wrt_states_fwd / _rev, f90:1333-1375. */
int eb_apply_forces_wrt_states_fwd(const eb_batch* b, const double* J, const double* d_states,
                                   double* d_forces, void* stream);
int eb_apply_forces_wrt_states_rev(const eb_batch* b, const double* J, const double* d_forces,
                                   double* d_states, void* stream);
/* apply_forces_wrt_vertices_fwd / _rev, f90:1267-1322. */
int eb_apply_forces_wrt_vertices_fwd(const eb_batch* b, const double* J,
                                     const double* d_vertices, double* d_forces, void* stream);
int eb_apply_forces_wrt_vertices_rev(const eb_batch* b, const double* J,
                                     const double* d_forces, double* d_vertices, void* stream);

/* Matrix-free forward tangent: dR = dR/dU.dU + dR/dX.dX + dR/dV.dV + dR/dMa.dMa in one
 * stencil pass (forward-mode duals, no stored Jacobian). Complex dU (4,M,N), dX/dV (2,M+1,N+1),
 * dMa (one complex per instance); any of them may be NULL (zero). R (optional) receives the
 * residual itself. */
int eb_apply_odes_tangent(const eb_batch* b, const double* X, const double* V, const double* U,
                          const double* dU, const double* dX, const double* dV,
                          const double* dMa, double* dR, double* R, void* stream);

/* Matrix-free reverse products for the cotangent w (4, M, N): d_states = (dR/dU)^T w
 * (4, M, N), d_vertices = (dR/dX)^T w and d_velocities = (dR/dV)^T w (2, M+1, N+1), d_mach =
 * (dR/dMa)^T w (one per instance): what apply_odes_wrt_states_rev, apply_odes_wrt_vertices_rev
 * and apply_odes_wrt_mach_rev (f90:604-650, 875-918, 1044-1072) give with the stored Jacobians,
 * in one reverse pass over the faces (no Jacobian built). is_complex = 1: w and the outputs are
 * interleaved complex (the transposes are of the real Jacobians, no conjugation); 0: real.
 * Outputs are overwritten; any of them may be NULL (not formed). Grids must be closed
 * O-grids (vertex column N equal to column 0). */
int eb_apply_odes_adjoint(const eb_batch* b, const double* X, const double* V, const double* U,
                          const double* w, int is_complex, double* d_states, double* d_vertices,
                          double* d_velocities, double* d_mach, void* stream);

/* ---- BSR form of d(odes)/d(states) --------------------------------------------------- */

/* convert_odes_wrt_states, f90:765-814, for a single instance: data (4, 4, nnzb), 1-based
 * int32 indices (nnzb) and index_pointers (M*N + 1) exactly as the reference emits them,
 * nnzb = (9M - 6) N. */
int eb_convert_odes_wrt_states(const eb_batch* b, const double* J, double* data,
                               int32_t* indices, int32_t* index_pointers, void* stream);
/* y = (A - shift*I) x for the BSR matrix A of one instance (complex x, y). */
int eb_bsr_shifted_spmv(int64_t n_rows, const double* data, const int32_t* indices,
                        const int32_t* index_pointers, double shift_re, double shift_im,
                        const double* x, double* y, void* stream);

/* ---- resolvent: restarted complex GMRES ------------------------------------------------ */

typedef struct eb_gmres_options {
  double tol;              /* relative residual ||b - A x|| / ||b|| to reach (e.g. 1e-10) */
  int32_t restart;         /* Krylov vectors per cycle */
  int32_t max_iterations;  /* limit on Arnoldi steps over all cycles (bounded run time) */
  int32_t check_every;     /* Arnoldi steps between convergence reads on the host */
  int32_t use_initial_guess; /* 1: start from the given x, 0: from zero */
} eb_gmres_options;

typedef struct eb_gmres_info {
  int32_t iterations;      /* Arnoldi steps taken by this system */
  int32_t cycles;          /* restart cycles of the call */
  int32_t converged;       /* 1 if the true relative residual reached tol */
  int32_t reserved;
  double rel_residual;     /* final true relative residual */
} eb_gmres_info;

/* Device workspace (bytes) for eb_gmres_solve with these systems. host_table: HOST copy of
 * the batch's instance table (NULL for a single instance); sys_inst: instance of each system
 * (NULL: all systems on instance 0). */
int64_t eb_gmres_workspace_bytes(const eb_batch* b, const eb_instance* host_table, int n_sys,
                                 const int32_t* sys_inst, int restart);

/* Solves n_sys systems (A_i - shift_s I) x_s = b_s (adjoint = 1: (A_i - shift_s I)^H x_s = b_s,
 * the transposed solve of solve_odes_wrt_states_adj, core.py:567-599) where A_i is the
 * d(odes)/d(states) Jacobian J of the system's instance. shifts: HOST array of n_sys complex
 * (interleaved). rhs / x: DEVICE complex vectors, system-major (system s occupies 4*M*N complex
 * entries after the previous systems'). Right-preconditioned by the inverse diagonal blocks.
 * info: HOST array of n_sys. Returns EB_ERR_NOCONV at the iteration limit (x holds the last
 * iterate) and EB_ERR_NAN if a residual became non-finite. Synchronises `stream`. */
int eb_gmres_solve(const eb_batch* b, const eb_instance* host_table, const double* J, int n_sys,
                   const int32_t* sys_inst, const double* shifts, int adjoint,
                   const double* rhs, double* x, const eb_gmres_options* opt, void* workspace,
                   int64_t workspace_bytes, eb_gmres_info* info, void* stream);

/* Scratch-free GMRES: the same solve as eb_gmres_solve (same arguments minus the
 * workspace), for callers that cannot allocate device memory -- a host program whose device
 * memory belongs to another runtime's pool, or a loop that may not allocate once running. Its
 * workspace is a 48 MiB array in the library's device memory, held by every GPU that loads the
 * library until the process exits; systems needing more (eb_gmres_workspace_bytes) are
 * rejected with EB_ERR_ARG. The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress); under CUDA's lazy module loading (the default) that lookup is also
 * when the device commits the 48 MiB, so the first call is itself a device allocation: make it
 * once at start-up, on each device, before the loop that may not allocate and before any
 * stream capture. Later calls allocate nothing. All calls share
 * the array: calls that overlap on the GPU (other streams, other host threads) race and must be
 * serialised by the caller. No counterpart in the reference (its solver allocates on every
 * call, core.py:512-599). */
int eb_gmres_solve_noalloc(const eb_batch* b, const eb_instance* host_table, const double* J,
                           int n_sys, const int32_t* sys_inst, const double* shifts,
                           int adjoint, const double* rhs, double* x,
                           const eb_gmres_options* opt, eb_gmres_info* info, void* stream);

/* Many shifts of one instance by GMRES preconditioned with the ring-LU factors of a few nearby
 * "anchor" shifts: system s (shift s, right-hand side s) is right-preconditioned by
 * (J - a_k I)^-1 with k = sys_anchor[s], the anchors' factors being those eb_ringlu_factor_many
 * left in ringlu_workspace (anchor k at ringlu_workspace + k * ringlu_stride). Each Arnoldi step
 * applies every anchor's factors once to all of its systems (at most 8 per anchor) as a forward
 * ring sweep over several right-hand sides; anchors whose systems have all converged drop out.
 * Forward solves only (the frequency response's (dR/dU - s I) dU = rhs, core.py:533-565 per
 * shift in the reference); single instance. workspace: eb_gmres_workspace_bytes(b, NULL, n_sys,
 * NULL, restart) bytes; aux: eb_gmres_anchored_aux_bytes bytes, 256-byte aligned. Other
 * arguments, statuses and info as eb_gmres_solve (EB_ERR_NOCONV leaves the unconverged systems'
 * last iterates in x; a caller solves those directly). Synchronises `stream`. */
int64_t eb_gmres_anchored_aux_bytes(int M, int N, int n_sys, int n_anchors,
                                    const int32_t* sys_anchor);
int eb_gmres_solve_anchored(const eb_batch* b, const double* J, int n_sys, const double* shifts,
                            const double* rhs, double* x, const eb_gmres_options* opt,
                            int n_anchors, const int32_t* sys_anchor, const void* ringlu_workspace,
                            int64_t ringlu_stride, void* workspace, int64_t workspace_bytes,
                            void* aux, int64_t aux_bytes, eb_gmres_info* info, void* stream);

/* ---- resolvent: direct ring-block LU ----------------------------------------------------- */

/* Device workspace (bytes) holding the block-LU factors of one M x N instance: 3 M dense
 * (4N)^2 complex super-blocks (Dinv, L1, C1' per ring: 768 M N^2 bytes; 1.6 GB at 129x129,
 * 12.9 GB at 257x257, 25.8 GB at 513x257), the rings' real 4 x 4 block diagonals (B2, C2), two
 * scratch super-blocks, pivots and solve vectors. */
int64_t eb_ringlu_workspace_bytes(int M, int N);

/* Factors A = J - shift I (J: d(odes)/d(states) of the single instance in `b`) by block
 * Gaussian elimination over the radial rings, pivoting inside each ring block. The factors
 * serve eb_ringlu_solve for both A and A^H. Synchronises `stream`; EB_ERR_NAN if a ring block
 * is singular. */
int eb_ringlu_factor(const eb_batch* b, const double* J, double shift_re, double shift_im,
                     void* workspace, int64_t workspace_bytes, void* stream);

/* eb_ringlu_factor for n_shifts systems J[s] - shift_s I at once, all of the grid size of the
 * single instance in `b`: J[s] (host array of device pointers) is system s's d(odes)/d(states)
 * (the same pointer for every s for a frequency sweep, different ones for several instances of
 * equal size), shifts[2 s], shifts[2 s + 1] its shift (real, imaginary; host array), and its
 * workspace starts at workspace + s * workspace_stride (stride >= eb_ringlu_workspace_bytes, a
 * multiple of 256; workspace 256-byte aligned). Each step of the elimination runs as one launch
 * over all systems, so a frequency sweep factors its shifts together instead of one after
 * another (the reference factors J - s I with SuperLU once per reduced frequency,
 * examples/response/run.py:138-144, and once per PTC step, :117-120). Each workspace then serves
 * eb_ringlu_solve / eb_ringlu_solve_many. Synchronises `stream`; EB_ERR_NAN if a ring block of
 * any system is singular. */
int eb_ringlu_factor_many(const eb_batch* b, const double* const* J, int n_shifts,
                          const double* shifts, void* workspace, int64_t workspace_stride,
                          void* stream);

/* x = A^-1 rhs (adjoint = 1: x = A^-H rhs) with the factors of eb_ringlu_factor for the same
 * J and shift, then iterative refinement x += A^-1 (rhs - A x) until ||rhs - A x|| / ||rhs||
 * <= tol or max_refine refinements (EB_ERR_NOCONV). rhs, x: complex (4, M, N) reference
 * layout; rel_residual (host, optional) receives the final relative residual. This replaces
 * solve_odes_wrt_states_fwd / _adj (core.py:533-599). Synchronises `stream`. */
int eb_ringlu_solve(const eb_batch* b, const double* J, double shift_re, double shift_im,
                    int adjoint, const void* workspace, int64_t workspace_bytes,
                    const double* rhs, double* x, double tol, int max_refine,
                    double* rel_residual, void* stream);

/* eb_ringlu_solve for the n_shifts factorisations of one eb_ringlu_factor_many call: system s
 * uses J[s], shift s, the workspace at workspace + s * workspace_stride, rhs[s] and x[s] (host
 * arrays of device pointers). The triangular sweeps of all systems run as batched launches;
 * refinement passes continue until every system reaches tol. rel_residuals (host, optional,
 * n_shifts entries) receives the final relative residuals. Synchronises `stream`. */
int eb_ringlu_solve_many(const eb_batch* b, const double* const* J, int n_shifts,
                         const double* shifts, int adjoint, const void* workspace,
                         int64_t workspace_stride, const double* const* rhs, double* const* x,
                         double tol, int max_refine, double* rel_residuals, void* stream);

/* ---- measurement ------------------------------------------------------------------------- */

/* FP64 throughput probe (the FP64 roofline denominator of the stencil kernels): 8 * sms CTAs of
 * 256 threads, each thread 8 independent chains of `iterations` fused multiply-adds (2 flops
 * each); `sink` (one device double) is written only in a case that does not occur. No
 * counterpart in the reference. */
int eb_fp64_fma_probe(int64_t iterations, int sms, double* sink, void* stream);

/* FP64 tensor-core throughput probe (the denominator of the dense ring-LU products): 4 * sms
 * CTAs of 256 threads, each warp 8 independent accumulators updated `iterations` times by
 * mma.sync.m8n8k4.f64 (512 flops each). No counterpart in the reference. */
int eb_fp64_mma_probe(int64_t iterations, int sms, double* sink, void* stream);

/* The ring LU's dense product as a library call: C_z = alpha A_z B_z + beta C_z for z < batch,
 * complex double (interleaved), column-major, no transposes, A_z = A + z stride_a complex
 * elements (likewise B, C); alpha and beta real, beta == 0 does not read C. variant: -1 the
 * default (2), 0 the register-staged double buffer, 1 the cp.async three-stage ring on 64 x 64
 * tiles, 2 a two-stage ring on 64 x 32 tiles (identical results). In the reference the dense products of its solves are SuperLU's and BLAS's
 * (core.py:533-599). */
int eb_zgemm_strided_batched(int M, int N, int K, double alpha, const double* A, int lda,
                             int64_t stride_a, const double* B, int ldb, int64_t stride_b,
                             double beta, double* C, int ldc, int64_t stride_c, int batch,
                             int variant, void* stream);

/* ---- launch-variant autotuner -------------------------------------------------------------- */

/* Kernels with several launch variants of identical results (the states Jacobian: dual width 4
 * at one CTA per SM or width 2 at two) time each variant on the first call for a problem size
 * and keep the fastest (EB_AUTOTUNE=0, or a stream being captured: the default variant, untimed).
 * Writes the choices and their times as text into buf (len bytes, NUL-terminated) and returns
 * the report's full length. No counterpart in the reference (which has no GPU kernels). */
int eb_autotune_report(char* buf, int len);

/* ---- PTC/SER steady state ---------------------------------------------------------------- */

/* Device workspace (bytes) of eb_ptc_run for an M x N instance and at most max_steps steps: the
 * ring-LU factors of one shift, two complex vectors, the control block and the history. */
int64_t eb_ptc_workspace_bytes(int M, int N, int max_steps);

/* The pseudo-transient continuation with switched evolution relaxation of the reference's
 * example driver (examples/response/run.py:84-123) for one instance, on the device: each step
 * evaluates R(U) into R, rel = max|R| / max|R_0| (R_0: the residual of U on entry), records rel,
 * stops if rel <= rtol or rel is not finite, else builds the states Jacobian into J and updates
 * U += Re((J - shift I)^-1 (-R)) with shift = (ser / rel)^-1 (ring-block LU, one refinement
 * step). At most max_steps steps. The first step runs eagerly, the others replay one captured
 * CUDA graph; the control values stay on the device and the host reads one stop flag per step.
 * On return U is the final state, R and J its residual and Jacobian (of the state before the
 * last update when max_steps ends the loop), history (HOST, 2 max_steps) the pairs (max|R|,
 * rel) of the steps and *n_steps their count. EB_ERR_NAN if rel became non-finite or a ring block was singular;
 * reaching max_steps is not an error (as in the example driver). Synchronises `stream`. */
int eb_ptc_run(const eb_batch* b, const double* X, const double* V, double* U, double* R,
               double* J, double ser, double rtol, int max_steps, void* workspace,
               int64_t workspace_bytes, double* history, int* n_steps, void* stream);

/* ---- pressure coefficients --------------------------------------------------------------- */
/* cp (real, one per cell, packed like the cells) of the states U: ((gamma-1)(E - |j|^2/2/rho) -
 * 1) / q with q = gamma Ma^2 / 2 per instance (compute_pressure_coefficients,
 * core.py:1423-1449). */
int eb_compute_pressure_coefficients(const eb_batch* b, const double* U, double* cp,
                                     void* stream);

/* d_cp (complex, one per cell) = dcp/dU . d_states (complex (4, M, N) per instance)
 * (apply_pressure_coefficients_wrt_states_fwd, core.py:1451-1488). */
int eb_apply_pressure_coefficients_wrt_states_fwd(const eb_batch* b, const double* U,
                                                  const double* d_states, double* d_cp,
                                                  void* stream);

/* ---- second-order building blocks ------------------------------------------------------ */
/* Directional derivatives of the Jacobians: with a complex direction d on the variable
 * `dir_kind` (0 = states, 1 = vertices, 2 = velocities), these write dJ/de along Re(d) to
 * J_re and along Im(d) to J_im, in the layout of the corresponding Jacobian. They replace the
 * four complex-step Jacobian rebuilds of each second-order routine (core.py:718-1275). */
int eb_odes_wrt_mach_dir(const eb_batch* b, const double* X, const double* V, const double* U,
                         int dir_kind, const double* d, double* J_re, double* J_im,
                         void* stream);
int eb_odes_wrt_states_dir(const eb_batch* b, const double* X, const double* V,
                           const double* U, int dir_kind, const double* d, double* J_re,
                           double* J_im, void* stream);
int eb_odes_wrt_vertices_dir(const eb_batch* b, const double* X, const double* V,
                             const double* U, int dir_kind, const double* d, double* J_re,
                             double* J_im, void* stream);
int eb_forces_wrt_states_dir(const eb_batch* b, const double* X, const double* U,
                             int dir_kind, const double* d, double* J_re, double* J_im,
                             void* stream);
int eb_forces_wrt_vertices_dir(const eb_batch* b, const double* X, const double* U,
                               int dir_kind, const double* d, double* J_re, double* J_im,
                               void* stream);

#ifdef __cplusplus
}
#endif

#endif /* EULER_B200_H */
