/*
 * magasm.h -- C ABI of the B200 (sm_100a) Nedelec element-assembly library.
 *
 * This is the drop-in boundary for MagPackage's assembly path. MATLAB reaches
 * it through the MEX gateways in magpackage_b200/mex/ (same names and
 * argument lists as the reference's gateways) and a plain C host reaches it
 * directly (magpackage_b200/harness/replay.c). No torch or CUDA C++ types
 * appear in the signatures: pointers are plain, streams are passed as void*
 * (a cudaStream_t, NULL = the legacy default stream).
 *
 * Every entry point returns MAG_OK (0) or a negative MAG_E* status and sets a
 * thread-local message readable with mag_last_error(). Nothing here calls
 * exit(), traps or asserts on the device; bad inputs are reported, not
 * dereferenced.
 *
 * Index conventions. The MEX-compatible entry points (mag_mex_*) take the
 * reference's exact layout: MATLAB column-major doubles, 1-based node/dof ids
 * stored as doubles, Signs as +-1 doubles. The handle-based entry points take
 * int32 0-based arrays in device memory: T [Ne][4], dofs [Ne][6] (-1 = no dof,
 * the reference's dof 0), tags [Ne] (1-based material tags as in RegionTags).
 * Row-major [Ne][k] equals MATLAB's [k x Ne] column-major, so the same buffer
 * serves both.
 */
#ifndef MAGASM_H
#define MAGASM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MAG_OK 0
#define MAG_E_ARG (-1)       /* bad argument (null pointer, size, count) */
#define MAG_E_RANGE (-2)     /* index out of range (node, dof, tag) */
#define MAG_E_GEOMETRY (-3)  /* degenerate element (det == 0 or not finite) */
#define MAG_E_CUDA (-4)      /* CUDA runtime error */
#define MAG_E_TIMEOUT (-5)   /* a bounded device-side wait gave up */
#define MAG_E_NOMEM (-6)     /* device allocation failed */
#define MAG_E_UNSUPPORTED (-7)

typedef struct mag_mesh mag_mesh; /* opaque, device-resident mesh + CSR plan */

typedef struct {
    int64_t num_nodes;
    int64_t num_elements;
    int64_t num_dofs;       /* CSR rows/cols */
    int64_t nnz;            /* structural nonzeros (union of element couplings) */
    int64_t num_incidences; /* (element, local edge) pairs with a dof */
    int32_t max_row_nnz;
    int32_t wide_positions; /* 1 if some row exceeds 31 entries */
    int32_t signs_derived;  /* 1 if signs equal the Mesh.m:134 rule and are not stored */
    int32_t schedule;       /* MAG_SCHEDULE_* used by the Jacobian assembly */
    int32_t tile_blocks;    /* CTA blocks of MAG_SCHEDULE_TILE_BLOCKS (0 = not available) */
    int32_t tile_colors;    /* largest number of element colour classes in one of its blocks */
    int64_t device_bytes;   /* memory held by the handle */
    int32_t shared_blocks;  /* row blocks of MAG_SCHEDULE_SHARED_ROW_BLOCKS (0 = not available) */
    int32_t reserved0;      /* 0 */
    int32_t nz_pass;        /* 1 if MAG_SCHEDULE_NZ_ROW_BLOCKS is available for this mesh */
    double tile_evals_per_elem; /* element evaluations per element and assembly of the tile schedule */
    double tile_plan_ms;    /* host time to build its plan */
} mag_mesh_info;

/* Jacobian assembly schedules; all give identical bits. */
#define MAG_OPTION_SCHEDULE 1
#define MAG_OPTION_TILE_VARIANT 2 /* launch shape of the tile schedule's Jacobian kernel: 0 = 320 threads x
                                     2 CTAs/SM (default), 1 = 288 x 2, 2 = 256 x 2, 3 = 512 x 1; same bits */
#define MAG_OPTION_TILE_PREFETCH 3 /* staging depth of the tile schedule: how many waves of resident CTAs
                                      ahead a CTA prefetches its successor block's records into L2
                                      (0 = none, 1 = default, 2); same bits */
#define MAG_SCHEDULE_TWO_PASS 0   /* element kernel + row reduction through an HBM scratch slab */
#define MAG_SCHEDULE_RETIRED_1 1  /* retired (a persistent launch over an L2 scratch ring); rejected */
#define MAG_SCHEDULE_ROW_BLOCKS 2 /* one launch, no scratch: per-row element recompute */
#define MAG_SCHEDULE_SHARED_ROW_BLOCKS 3 /* as 2, each block's distinct elements evaluated once in shared
                                            memory (standard curl table, else runs as 2) */
#define MAG_SCHEDULE_RETIRED_4 4  /* retired (as 3 with the block's nodes and edge values staged first:
                                     slower than 3); rejected */
#define MAG_SCHEDULE_NZ_ROW_BLOCKS 5     /* as 3, each off-diagonal entry placed by its (at most two)
                                            contributing incidences and the block's nonzeros stored in one
                                            pass; only diagonals and residuals are summed per row (meshes
                                            whose off-diagonal entries have more than two contributions,
                                            e.g. repeated dofs, run as 3) */
#define MAG_SCHEDULE_TILE_BLOCKS 6 /* one launch, no scratch: blocks of whole rows whose edges start in a
                                      4x4x4-layer spatial tile of nodes; one thread per incident element
                                      (about 1.5 evaluations per element) writes its rows' off-diagonal
                                      entries into the block's values in colour phases (no two elements of
                                      a colour share an entry), diagonals and residuals are summed per row
                                      in element order. Needs rows of at most 31 entries and off-diagonal
                                      entries of at most two contributions (standard curl table; else the
                                      row-block schedules run). The default when available */

/* ---- library ------------------------------------------------------------ */

int mag_version(void);
const char *mag_last_error(void);
/* Threading. Every handle-based entry point only enqueues work on its stream and
 * returns; mag_sync waits for the stream (MAG_E_CUDA with the CUDA error text if
 * work on it failed). Different handles may be used from different host threads at
 * once; one handle is used by one thread at a time. The MEX entry points run one at
 * a time (they share the mesh cache and the staging buffers) and return with their
 * outputs on the host, as the reference's gateways do (they are single-threaded
 * callees of MATLAB: assemble_jacobian_kernel_mex.cpp:8-153). */
int mag_sync(void *stream);

/* ---- topology ------------------------------------------------------------ */

/* Mesh.generateEdges (src/Mesh.m:114-138) on the GPU. d_T: int32 [Ne][4],
 * 0-based nodes. Outputs (device): d_edges [E][2] 0-based (lexicographic by
 * (min,max) node; capacity 6*Ne rows), d_t2e [Ne][6] 0-based edge ids,
 * d_sign [Ne][6] (+1 iff the local start node has the smaller id). *E_out is
 * written on the host after the call completes (the call synchronises). */
int mag_generate_edges(const int32_t *d_T, int64_t Ne, int64_t Nn, int32_t *d_edges,
                       int32_t *d_t2e, int8_t *d_sign, int64_t *E_out, void *stream);

/* ---- mesh handle: one-time CSR plan -------------------------------------- */

/* Copies the mesh into the handle's layout and builds, on the GPU, the CSR
 * pattern of the dof-dof coupling (rows/cols = dofs, columns sorted) and the
 * per-row incidence list (element, local edge, position of each of its six
 * couplings inside the row) that the assembly's fixed-order reduction uses.
 * This is the reference's unique()/sparse() structure work (Mesh.m:126-135,
 * Assembler.m:37-38) done once per mesh. d_signs may be NULL (derive from T,
 * the Mesh.m:134-135 rule); when given and equal to that rule it is not stored.
 * All inputs are device pointers; the handle keeps its own copies. */
int mag_mesh_create(const double *d_P, int64_t Nn, const int32_t *d_T, int64_t Ne,
                    const int32_t *d_dofs, const int8_t *d_signs, const int32_t *d_tags,
                    int64_t num_dofs, mag_mesh **out, void *stream);
int mag_mesh_destroy(mag_mesh *mesh);
int mag_mesh_get_info(const mag_mesh *mesh, mag_mesh_info *info);
/* Handle options (MAG_OPTION_*). */
int mag_mesh_set_option(mag_mesh *mesh, int option, int64_t value);
/* Autotune the tile schedule's Newton Jacobian on the caller's state: every launch shape
 * (MAG_OPTION_TILE_VARIANT) x staging depth (MAG_OPTION_TILE_PREFETCH) is timed `reps` times
 * (CUDA events on `stream`) and the fastest is kept in the handle. times_ms, when not NULL,
 * receives the mean ms of each pair, index variant * 3 + depth (12 entries). The outputs of
 * every candidate are the same bits, so d_vals and d_res hold the Jacobian and residual at
 * d_sol afterwards. MAG_E_UNSUPPORTED when the mesh runs another schedule. */
int mag_mesh_tune(mag_mesh *mesh, const double *d_sol, double *d_vals, double *d_res, int reps,
                  double *times_ms, int *variant, int *depth, void *stream);
/* Synchronise `stream` and report whether the last assemblies completed: MAG_E_RANGE if a
 * kernel of the tile schedule found a plan index out of range and skipped it (an internal
 * error: the results are incomplete). The status is cleared once reported. No assembly
 * kernel waits on another CTA or kernel. */
int mag_mesh_check(mag_mesh *mesh, void *stream);
/* Copy the structural pattern out (device buffers: row_ptr [num_dofs+1], col_idx [nnz]). */
int mag_mesh_pattern(const mag_mesh *mesh, int64_t *d_row_ptr, int32_t *d_col_idx, void *stream);

/* Quadrature and reference basis, exactly what Assembler.m passes to the MEX
 * (Assembler.m:30-32,191-193): Qw [nq], CurlRef and ValRef [6 x 3 x nq]
 * column-major (entry (i,c,q) at i + 6c + 18q). Host pointers; nq <= 16. */
int mag_mesh_set_quadrature(mag_mesh *mesh, const double *qw, int nq, const double *curl_ref,
                            const double *val_ref);

/* Material tables in the layout of Assembler.packMaterialData
 * (src/Assembler.m:270-304): eight host arrays indexed by tag-1, nmat entries
 * each, breaks/coefs concatenated. Consumed by MexMaterialUtils.hpp:24-87's
 * rule (binary search, Horner, linear extrapolation past maxB, clamps). */
int mag_mesh_set_materials(mag_mesh *mesh, const double *lin_nu, const double *is_nonlinear,
                           const double *max_bsq, int nmat, const double *breaks, int nbreaks,
                           const double *coefs, int ncoefs, const double *spline_start,
                           const double *spline_count, const double *coef_start);

/* ---- assembly into the structural CSR (device buffers) -------------------- */

/* Newton Jacobian values and residual: the work of
 * assemble_jacobian_kernel_mex.cpp:61-152 followed by the sparse() sums of
 * Assembler.m:205-206,214-215, fused. d_sol [num_dofs] is SolA; d_vals [nnz]
 * receives J (ignored when calc_j == 0, like CalcJ = false); d_res [num_dofs]
 * receives the residual. Values are summed per nonzero in ascending element
 * order by a fixed-order reduction: deterministic, no floating-point atomics. */
int mag_assemble_jacobian(mag_mesh *mesh, const double *d_sol, double *d_vals, double *d_res,
                          int calc_j, void *stream);

/* Curl-curl stiffness K(nu) with a per-element reluctivity d_nu [Ne]
 * (assemble_curl_curl_kernel_mex.cpp:18-121 + Assembler.m:37-38). Under
 * MAG_SCHEDULE_NZ_ROW_BLOCKS (the default when available) one launch without the element
 * scratch; under the other schedules the element kernel and the row reduction. Same bits. */
int mag_assemble_stiffness(mag_mesh *mesh, const double *d_nu, double *d_vals, void *stream);

/* Harmonic-balance assembly (assemble_hbfem_kernel_mex.cpp:26-258, called through
 * Assembler.assembleHBFEM by HBFEMSolver.m:78,96; that wrapper is absent from the
 * reference). Harmonic field d_sol_re/d_sol_im [K][num_dofs] (= MATLAB's [Ndof x K]
 * column-major; imaginary part may be NULL), AFT matrices D [K][N] (D(t,h) at
 * h*N + t) and P [N][K] (P(h,t) at t*K + h), imaginary parts may be NULL. Writes
 * the harmonic residual d_res_re/d_res_im [K][num_dofs] (the gateway's R triplets
 * summed as sparse() does) and, when d_vals is not NULL, the DC-reluctivity block
 * on the CSR pattern; harmonic k's Jacobian block is Scalings[k] * d_vals. The
 * spline coefficient offsets come from mag_mesh_set_materials (the gateway never
 * sets them, so it is defined only for linear materials). K <= 16. */
int mag_assemble_hbfem(mag_mesh *mesh, const double *d_sol_re, const double *d_sol_im, int K,
                       const double *d_d_re, const double *d_d_im, const double *d_p_re, const double *d_p_im,
                       int N, double *d_vals, double *d_res_re, double *d_res_im, void *stream);

/* Newton residual at d_sol with the tangent evaluated at a seeded state: per
 * element the flux density B of d_sol scaled by d_bscale[e] (the learned warm
 * start's first Jacobian; no counterpart in the reference). Same outputs as
 * mag_assemble_jacobian with calc_j = 1; d_bscale = 1 everywhere reproduces it
 * to rounding. Standard curl table only. */
int mag_assemble_jacobian_seeded(mag_mesh *mesh, const double *d_sol, const double *d_bscale,
                                 double *d_vals, double *d_res, void *stream);

/* Per-element scale of the seeded tangent: beta_e = (|B_e| + |B_hat_e|)/(2|B_e|),
 * B_e the flux density of d_sol and |B_hat_e|^2 where the element's nonlinear
 * nu(|B|^2) equals d_nu_hat[e] (a predicted reluctivity), i.e. the tangent at the
 * midpoint between the current and the predicted state, clamped to the trust region
 * [1/max_scale, max_scale] (max_scale >= 1). beta = 1 for linear materials,
 * d_nu_hat[e] <= 0 or B_e = 0. No counterpart in the reference. */
int mag_seed_midpoint(mag_mesh *mesh, const double *d_sol, const double *d_nu_hat, double max_scale,
                      double *d_bscale, void *stream);

/* Sigma-weighted Nedelec mass M(sigma) (assemble_mass_kernel_mex.cpp:17-127 +
 * Assembler.m:52-53,71-72). d_sigma [Ne], or NULL for sigma = 1 (the
 * reference's empty Coeffs, assemble_mass_kernel_mex.cpp:155,187). */
int mag_assemble_mass(mag_mesh *mesh, const double *d_sigma, double *d_vals, void *stream);

/* Source vector F (assemble_source_kernel_mex.cpp:16-114 + Assembler.m:87-89).
 * d_js [Ne][3] current density per element; d_out [num_dofs]. */
int mag_assemble_source(mag_mesh *mesh, const double *d_js, double *d_out, void *stream);

/* Winding (coil current) vector C = sparse(I(valid), 1, V(valid), num_dofs, 1) as a dense
 * d_out [num_dofs] (assemble_winding_kernel_mex.cpp:13-127 + Assembler.m:134-161): the
 * elements tagged coil_id, direction d_dir_field [Ne][3] (device; NULL = the uniform host
 * direction dir[3]) times scale (Turns / CrossSectionArea), integrated against the basis
 * of mag_mesh_set_quadrature's ValRef. Summed in ascending element order. */
int mag_assemble_winding(mag_mesh *mesh, int coil_id, const double *d_dir_field, const double *dir,
                         double scale, double *d_out, void *stream);

/* Element magnetic flux density B [Ne][3] and |B|^2 [Ne] at the solution
 * d_sol (the per-element curl of PostProcessor.computeElementB,
 * src/post/PostProcessor.m:64-126, evaluated as the Jacobian kernel does). */
int mag_element_b(mag_mesh *mesh, const double *d_sol, double *d_b, double *d_bsq, void *stream);

/* MATLAB sparse() storage: drop entries whose value is exactly zero (MATLAB
 * keeps no explicit zeros). Inputs: a CSR over nrows rows. Outputs must hold
 * nrows+1 / nnz entries; *nnz_out is written on the host (the call synchronises).
 * d_vals_out may alias nothing of the inputs. */
int mag_csr_drop_zeros(const int64_t *d_row_ptr, const int32_t *d_col_idx, const double *d_vals,
                       int64_t nrows, int64_t *d_row_ptr_out, int32_t *d_col_out,
                       double *d_vals_out, int64_t *nnz_out, void *stream);

/* ---- batched complex frequency-domain assembly ------------------------------ */

typedef struct mag_batch mag_batch;

/* A_i = K_i(nu_i) + j*omega_i*M_i(sigma_i) for n independent meshes, the system
 * FrequencySolver.solve forms (src/solver/FrequencySolver.m:87,125,131) without
 * its regularisation term, assembled in ONE launch over a work queue of
 * (mesh, block) items: variants 0-3 take the meshes' row blocks (persistent CTAs;
 * incidences per CTA x CTAs per SM), variants 4-5 their tile blocks (one CTA per
 * item; threads per CTA), available when every mesh has a tile plan. d_nu[i] and
 * d_sigma[i] are per-element device arrays (d_sigma[i] may be NULL: sigma = 1);
 * d_vals[i] receives complex128 values (re, im interleaved) on mesh i's
 * structural pattern; omega in rad/s. Creation times every available variant on
 * these inputs, keeps the fastest, and captures its launch in a CUDA graph.
 * Every variant gives the same bits. */
int mag_batch_create(mag_mesh *const *meshes, int n, const double *const *d_nu,
                     const double *const *d_sigma, const double *omega, double *const *d_vals,
                     mag_batch **out, void *stream);
/* Replays the captured graph on `stream`. */
int mag_batch_assemble(mag_batch *batch, void *stream);
/* The chosen variant, its description, and the time (ms) each variant took
 * during creation (times[] must hold mag_batch_variants() entries). */
int mag_batch_variants(void);
int mag_batch_tuning(const mag_batch *batch, int *chosen, double *times_ms, char *name, int name_len);
/* Use variant `variant` (0 .. mag_batch_variants()-1) instead of the tuned one and
 * capture it again; MAG_E_UNSUPPORTED if it is not available for these meshes. */
int mag_batch_select(mag_batch *batch, int variant);
int mag_batch_destroy(mag_batch *batch);

/* ---- per-element reluctivity predictor (no counterpart in the reference) ---- */

/* A 4 -> 64 -> 64 -> 64 -> 1 SiLU MLP whose hidden GEMMs run on the 5th-generation
 * tensor cores (BF16 operands, FP32 accumulation in tensor memory) with FP32
 * master weights and Adam. It predicts log-reluctivity per element from the
 * previous steps' |B|, the source and the material, to seed the first Jacobian
 * of a Newton solve (mag_seed_midpoint + mag_assemble_jacobian_seeded).
 * Parameters: W1[64][4] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] w4[64] b4.
 * Feature arrays are [rows][4] float32 and 16-byte aligned. SiLU is evaluated
 * with the hardware tanh approximation (relative error ~2^-11, below the BF16
 * rounding of every layer input). */
typedef struct mag_mlp mag_mlp;
int mag_mlp_num_params(void);
int mag_mlp_create(const float *init_params, mag_mlp **out);
int mag_mlp_destroy(mag_mlp *mlp);
int mag_mlp_get_params(const mag_mlp *mlp, float *host_params);
int mag_mlp_set_params(mag_mlp *mlp, const float *host_params);
/* y[rows] = f(feats[rows][4]); z[rows][3][64] (pre-activations) may be NULL. */
int mag_mlp_forward(mag_mlp *mlp, const float *d_feats, int64_t rows, float *d_y, float *d_z, void *stream);
/* nu = clamp(exp(y * y_scale + y_shift), nu_min, nu_max) written to d_nu[d_rows[i]]
 * (d_rows NULL: d_nu[i]). */
int mag_mlp_predict_nu(mag_mlp *mlp, const float *d_feats, int64_t rows, const int32_t *d_rows,
                       double y_scale, double y_shift, double nu_min, double nu_max, double *d_nu,
                       void *stream);
/* Forward + backward of L = sum_i loss_scale/2 * (y_i - target_i)^2: d_grad[num_params]
 * (NULL: internal buffer), summed over rows in a fixed order. d_y [rows], d_z [rows][3][64]. */
int mag_mlp_gradient(mag_mlp *mlp, const float *d_feats, const float *d_target, int64_t rows,
                     float loss_scale, float *d_y, float *d_z, float *d_grad, void *stream);
/* One Adam step (lr, betas 0.9/0.999) on the mean-squared error of a minibatch. */
int mag_mlp_train_step(mag_mlp *mlp, const float *d_feats, const float *d_target, int64_t rows,
                       float lr, float *d_y, float *d_z, void *stream);
/* One epoch of mag_mlp_train_step over minibatches of `batch` rows in the order of the
 * device permutation d_perm [rows] (a last partial minibatch is skipped): each minibatch is
 * gathered on the device into d_xb [batch][4] and d_tb [batch] (16-byte aligned), so the
 * host only enqueues launches. d_loss (or NULL) accumulates the sum of squared errors of
 * every minibatch before its step. d_y [batch], d_z [batch][3][64] are workspace. */
int mag_mlp_train_epoch(mag_mlp *mlp, const float *d_feats, const float *d_target, int64_t rows,
                        const int64_t *d_perm, int64_t batch, float lr, float *d_xb, float *d_tb, float *d_y,
                        float *d_z, float *d_loss, void *stream);
/* Synchronise; MAG_E_TIMEOUT if a tensor-core completion wait gave up since the last
 * check (the status is cleared once reported). The outputs of that call are incomplete. */
int mag_mlp_check(mag_mlp *mlp, void *stream);
/* Polls a kernel makes on a tensor-core completion before it gives up (then it waits
 * for the MMAs it issued, frees its tensor memory, records MAG_E_TIMEOUT and returns);
 * 0 restores the default bound (about a second). Small values exist to test that path. */
int mag_mlp_set_spin_limit(mag_mlp *mlp, int64_t polls);

/* ---- sparse algebra for the Newton driver ------------------------------------
 * CSR arguments: d_row_ptr [n+1] int64, d_col_idx [nnz] int32, d_vals [nnz]. */

/* y = A x (the products of TransientSolver.m:289-300). */
int mag_csr_spmv(int64_t n, const int64_t *d_row_ptr, const int32_t *d_col_idx, const double *d_vals,
                 const double *d_x, double *d_y, void *stream);

/* Dirichlet elimination in place: A <- M_free A M_free + M_fixed and
 * rhs[fixed] = 0 (BoundaryCondition.applyDirichlet, src/BoundaryCondition.m:81-112).
 * d_fixed [n] is nonzero for a fixed dof; d_rhs may be NULL. Entries that
 * become zero stay in the pattern (MATLAB's result would not store them). */
int mag_csr_apply_dirichlet(int64_t n, const int64_t *d_row_ptr, const int32_t *d_col_idx, double *d_vals,
                            const uint8_t *d_fixed, double *d_rhs, void *stream);

/* Preconditioned conjugate gradients, the stand-in for the reference's MUMPS
 * solve (LinearSolver.solve, src/solver/LinearSolver.m:22-46), for symmetric
 * positive definite A. d_x holds the initial guess and receives the solution;
 * stops when ||b - A x|| <= rtol ||b|| (recursive residual) or after max_iter
 * iterations. Jacobi preconditioner, plus the auxiliary gradient space when set.
 * Deterministic (fixed-order reductions). Outputs: iterations, ||r||/||b||,
 * status 1 converged / 2 iteration limit / 3 breakdown (returns MAG_E_GEOMETRY).
 * Synchronises the host once per 32 iterations. */
typedef struct mag_pcg mag_pcg;
int mag_pcg_create(int64_t n, mag_pcg **out);
int mag_pcg_destroy(mag_pcg *pcg);
/* Optional auxiliary gradient space for the preconditioner:
 * z = D^-1 r + G (dn_inv .* (G^T r)), with G [n x ni] the discrete gradient
 * (edge-node incidence, +-1) restricted to free edges and interior nodes, given
 * both as G and as G^T in CSR, and dn_inv = 1 / diag(G^T A G). The arrays stay
 * owned by the caller and must outlive the solves. ni = 0 removes it. */
int mag_pcg_set_aux(mag_pcg *pcg, int64_t ni, const int64_t *d_g_row_ptr, const int32_t *d_g_col_idx,
                    const double *d_g_vals, const int64_t *d_gt_row_ptr, const int32_t *d_gt_col_idx,
                    const double *d_gt_vals, const double *d_dn_inv);
int mag_pcg_solve(mag_pcg *pcg, const int64_t *d_row_ptr, const int32_t *d_col_idx, const double *d_vals,
                  const double *d_b, double *d_x, double rtol, int max_iter, int *iters, double *relres,
                  int *status, void *stream);

/* Per-element reluctivity nu(|B|^2) and d nu / d|B|^2 at the solution d_sol
 * (the values the Jacobian kernel evaluates, MexMaterialUtils.hpp:24-87);
 * needs mag_mesh_set_materials. Either output may be NULL. */
int mag_element_nu(mag_mesh *mesh, const double *d_sol, double *d_nu, double *d_dnu, void *stream);

/* ---- MEX-compatible entry points (host buffers, reference layout) ---------
 * Every mag_mex_* entry point below (except mag_mex_jacobian_noalloc) keeps the
 * device form of the last two meshes it was given, per device: P, T, Dofs and Signs
 * converted to the library's layout and, for the sparse-returning calls, the CSR
 * pattern. A call finds its mesh by the sizes and a 128-bit content hash of those
 * four arrays (Tags hashed apart and reconverted when they change), so a Newton loop
 * calling with the same mesh uploads only SolA, while an array changed in place, or
 * a new array at a reused address, is converted afresh. The calls hold one library
 * lock for their duration. */

/* Release the device memory of the cached MEX meshes. */
int mag_mex_cache_clear(void);

/* [I,J,V,R_idx,R_val] = assemble_jacobian_kernel_mex(P,T,Dofs,Signs,Tags,SolA,
 *   Qw,CurlRef,lin,isNon,maxB,brk,coe,start,cnt,coeStart,calcJ)
 * (src/mex/assemble_jacobian_kernel_mex.cpp:8-153, 17 inputs). All arrays are
 * host doubles in MATLAB layout; outputs are host buffers sized 36*Ne (I,J,V;
 * untouched when calc_j == 0) and 6*Ne (R_idx, R_val), triplets in the
 * reference's order (element-major, local column j outer, row i inner). */
int mag_mex_jacobian(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                     const double *Signs, const double *Tags, const double *SolA, int64_t Ndof,
                     const double *Qw, int nq, const double *CurlRef, const double *lin,
                     const double *isNon, const double *maxB, int nmat, const double *brk,
                     int nbrk, const double *coe, int ncoe, const double *start,
                     const double *cnt, const double *coeStart, int calc_j, double *I,
                     double *J, double *V, double *R_idx, double *R_val);

/* [I,J,V] = assemble_curl_curl_kernel_mex(P,T,Dofs,Signs,Nu,Qw,CurlRef)
 * (src/mex/assemble_curl_curl_kernel_mex.cpp:18-121). */
int mag_mex_curl_curl(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                      const double *Signs, const double *Nu, const double *Qw, int nq,
                      const double *CurlRef, double *I, double *J, double *V);

/* [I,J,V] = assemble_mass_kernel_mex(P,T,Dofs,Signs,Coeffs,Qw,ValRef)
 * (src/mex/assemble_mass_kernel_mex.cpp:17-127). ncoeffs != Ne means sigma = 1. */
int mag_mex_mass(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                 const double *Signs, const double *Coeffs, int64_t ncoeffs, const double *Qw,
                 int nq, const double *ValRef, double *I, double *J, double *V);

/* [I,V] = assemble_source_kernel_mex(P,T,Dofs,Signs,Js,Qw,ValRef)
 * (src/mex/assemble_source_kernel_mex.cpp:16-114): Js [3 x Ne]; outputs 6*Ne. */
int mag_mex_source(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                   const double *Signs, const double *Js, const double *Qw, int nq, const double *ValRef,
                   double *I, double *V);

/* [I,V] = assemble_winding_kernel_mex(P,T,Dofs,Signs,Tags,CoilID,DirField,UniDir,Scale,Qw,ValRef)
 * (src/mex/assemble_winding_kernel_mex.cpp:13-127): DirField [3 x Ne] or NULL (the
 * empty []: UniDir [3] for every element); I = V = 0 for elements outside the coil.
 * Outputs 6*Ne. */
int mag_mex_winding(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                    const double *Signs, const double *Tags, double CoilID, const double *DirField,
                    const double *UniDir, double Scale, const double *Qw, int nq, const double *ValRef,
                    double *I, double *V);

/* ---- MATLAB sparse results of the MEX-compatible entry points --------------
 * The sparse() that Assembler.m applies to the gateways' triplets
 * (Assembler.m:37-38 stiffness, :52-53 and :71-72 mass, :205-215 Jacobian and
 * residual) done on the GPU: the host receives MATLAB's compressed-column
 * storage (jc [n+1], ir [nnz] as 64-bit mwIndex, pr [nnz]) instead of 36*Ne
 * triplets. Duplicates are summed in ascending element order, exact zeros are
 * dropped and entries of missing dofs (Dofs == 0) are skipped, as the
 * (I > 0) & (J > 0) filter and sparse() do. The MEX gateways return it when
 * given their optional trailing argument. */
typedef struct mag_sparse mag_sparse;

/* J = sparse(I, J, V, Ndof, Ndof) and R = full(sparse(R_idx, 1, R_val, Ndof, 1))
 * of mag_mex_jacobian's outputs (same inputs). R is a host buffer [Ndof].
 * *J_out is left NULL when calc_j == 0. */
int mag_mex_jacobian_sparse(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                            const double *Signs, const double *Tags, const double *SolA, int64_t Ndof,
                            const double *Qw, int nq, const double *CurlRef, const double *lin,
                            const double *isNon, const double *maxB, int nmat, const double *brk, int nbrk,
                            const double *coe, int ncoe, const double *start, const double *cnt,
                            const double *coeStart, int calc_j, mag_sparse **J_out, double *R);
/* K = sparse(I, J, V, Ndof, Ndof) of mag_mex_curl_curl's outputs. */
int mag_mex_curl_curl_sparse(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                             const double *Signs, const double *Nu, const double *Qw, int nq,
                             const double *CurlRef, int64_t Ndof, mag_sparse **out);
/* M = sparse(I, J, V, Ndof, Ndof) of mag_mex_mass's outputs. */
int mag_mex_mass_sparse(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                        const double *Signs, const double *Coeffs, int64_t ncoeffs, const double *Qw, int nq,
                        const double *ValRef, int64_t Ndof, mag_sparse **out);
/* Size (n x n) and number of stored entries. */
int mag_sparse_info(const mag_sparse *sp, int64_t *n, int64_t *nnz);
/* Copy into host arrays jc [n+1], ir [nnz], pr [nnz] (mxGetJc / mxGetIr / mxGetPr
 * of mxCreateSparse(n, n, nnz, mxREAL)). */
int mag_sparse_copy(const mag_sparse *sp, uint64_t *jc, uint64_t *ir, double *pr);
int mag_sparse_destroy(mag_sparse *sp);

/* Allocation-free form of mag_mex_jacobian, for callers that cannot allocate
 * device memory: a MEX function working on mxGPUArray buffers owned by
 * MATLAB's allocator, a host inside another runtime's memory pool or under a
 * fixed budget, or a path where cudaMalloc must not run. (No counterpart in
 * the reference, whose MEX kernels run on the host.)
 * The caller owns everything: d_* are device arrays in the reference's MEX
 * layout (P [3*Nn], T [4*Ne] and Dofs/Signs [6*Ne] as doubles, 1-based;
 * Tags [Ne]; SolA [Ndof]); outputs d_I/d_J/d_V [36*Ne] (untouched when
 * calc_j == 0) and d_Ridx/d_Rval [6*Ne] on the device. Qw, CurlRef and the
 * material tables are host arrays, as in mag_mex_jacobian. The element blocks
 * go to a static device array inside the library (Ne <= 32768, nmat <= 64,
 * nbrk <= 4096, ncoe <= 16384; larger sizes return MAG_E_UNSUPPORTED), which
 * every GPU that loads the library holds until exit. The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress, once per
 * device): make it before any stream capture begins. Each call copies the host
 * tables and synchronises `stream`.
 * With lazy module loading (CUDA's default) the first call on a device is when the
 * array is committed on the device, and it can fail with MAG_E_CUDA when the
 * device has no memory left, so make it early. Calls share the array: calls
 * that overlap on the GPU race and must be serialised. Synchronises `stream` to
 * report index errors (MAG_E_RANGE; the offending elements' values are NaN). */
int mag_mex_jacobian_noalloc(const double *d_P, int64_t Nn, const double *d_T, int64_t Ne,
                             const double *d_Dofs, const double *d_Signs, const double *d_Tags,
                             const double *d_SolA, int64_t Ndof, const double *Qw, int nq,
                             const double *CurlRef, const double *lin, const double *isNon,
                             const double *maxB, int nmat, const double *brk, int nbrk,
                             const double *coe, int ncoe, const double *start, const double *cnt,
                             const double *coeStart, int calc_j, double *d_I, double *d_J,
                             double *d_V, double *d_Ridx, double *d_Rval, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MAGASM_H */
