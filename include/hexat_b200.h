/*
 * hexat_b200.h -- C ABI of the B200-native inner-solve library for HEXA(T)
 * v069 (voxel Hex8 linear elasticity + topology optimisation).
 *
 * The library replaces, on one GPU, the reference's Julia/CUDA.jl routines
 * for the linear solve, the Helmholtz density filter and the element stress.
 * Reference paths below are relative to the reference project root
 * (v069_2025_12_09_HEXAS_TOPO_anti_checkerboard/).
 *
 * Conventions (identical to the reference's data layout):
 *  - nodes: nN x 3 Float32, Julia column-major (x of node n at n, y at nN+n,
 *    z at 2nN+n);  elements: nE x 8 Int64, column-major, 1-based, corner
 *    order of src/Core/Element.jl:8-17;  bc_indicator: nN x 3 Float32
 *    column-major, > 0 means the DOF is fixed;  f, u: 3nN interleaved
 *    (dof = 3*node + component);  per-element arrays have length nE.
 *  - Every call is blocking: results are in the caller's buffers on return.
 *    The caller owns all buffers; no pointer is retained after a call.
 *  - Device-array calls read their inputs on the context's own stream.  Each
 *    call first orders that stream after the work already queued on the
 *    legacy default CUDA stream (stream 0, where e.g. PyTorch queues by
 *    default); inputs written on any other stream must be complete (the
 *    caller synchronises that stream first).
 *  - Every call returns an hx_status and never throws across the ABI.
 *    hx_last_error() describes the last failure of a context.
 *  - Nothing falls back to the CPU: without a usable device, calls return
 *    HX_NO_DEVICE / HX_CUDA_ERROR.
 */
#ifndef HEXAT_B200_H
#define HEXAT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HX_API __attribute__((visibility("default")))

typedef enum hx_status {
  HX_OK = 0,
  HX_NOT_CONVERGED = 1, /* iteration or wall-clock limit reached */
  HX_STALLED = 2,       /* accepted stagnation / refinement made no progress */
  HX_BREAKDOWN = 3,     /* p.Ap <= 0 or NaN */
  HX_NONFINITE = 4,     /* NaN/Inf in the residual */
  HX_OOM = 5,
  HX_BAD_ARG = 6,
  HX_CUDA_ERROR = 7,
  HX_NO_DEVICE = 8,
  HX_DIVERGED = 9 /* residual exploded or grew 100x over its best */
} hx_status;

typedef enum hx_dtype { HX_F32 = 0, HX_F64 = 1 } hx_dtype;

typedef enum hx_precision {
  HX_PREC_FP64 = 0,     /* plain FP64 Jacobi-PCG */
  HX_PREC_MIXED32 = 1   /* FP32 PCG with FP64 reliable updates (true-residual
                           replacement, FP64 dots, FP64 convergence test);
                           any other value returns HX_BAD_ARG */
} hx_precision;

typedef enum hx_preconditioner {
  HX_PC_JACOBI = 0,
  HX_PC_LEARNED = 1, /* CNN preconditioner inside flexible CG (needs weights) */
  HX_PC_NONE = 2,
  HX_PC_MULTIGRID = 3 /* geometric multigrid V-cycle (FP32) inside flexible CG
                         (FP64 vectors, or FP32 with FP64 reliable updates under
                         HX_PREC_MIXED32): the GPU replacement of the reference's
                         CPU algebraic multigrid (GPUSolver.jl:168-268) */
} hx_preconditioner;

typedef struct hx_solve_opts {
  int32_t precision;       /* hx_precision */
  int32_t preconditioner;  /* hx_preconditioner */
  double tol;              /* stop when ||r||/||b|| < tol */
  int32_t max_iter;
  int32_t warm_start;      /* 1: u_inout holds the initial guess */
  double shift_factor;     /* shift s = shift_factor * max(diag over free DOFs) */
  double wall_limit_ms;    /* 0: no limit */
  int32_t check_every;     /* host poll period in iterations (0: automatic) */
  int32_t keep_best;       /* 1: keep the best iterate (reference semantics) */
  double inner_tol;        /* mixed precision: the FP32 recursive residual is
                              replaced by the FP64 true residual each time it
                              has dropped by this factor (default 0.1); with
                              HX_PC_MULTIGRID by its cube */
  int32_t max_refine;      /* reserved */
  int32_t ref_retry;       /* 1: reference retry/shift-escalation semantics */
  int32_t divergence_checks; /* 1: explosion and 100x-over-best checks */
  int32_t verify_true_residual; /* 1: recompute ||b-Au|| in FP64 at the end */
  int32_t learned_no_fallback; /* 1: learned FCG without the Jacobi fallback */
  int32_t multigrid_fallback;  /* 1 (with ref_retry): after a failed or stagnated
                                  Jacobi attempt switch to HX_PC_MULTIGRID, as the
                                  reference's "jacobi_amg" switches to AMG
                                  (GPUSolver.jl:540-579) */
  int32_t mg_smooth_degree;    /* multigrid: Chebyshev degree of each pre- and
                                  post-smoothing, 1..8 (0: the default, 2) */
  int32_t reserved[3];
} hx_solve_opts;

typedef struct hx_solve_report {
  int32_t status;       /* hx_status of the solve */
  int32_t iterations;   /* CG iterations (all inner iterations when mixed) */
  int32_t refinements;  /* mixed: FP64 residual replacements; FP64 forms:
                           restarts from the iterate because the true
                           residual was still above tol when the recursive
                           one converged (ref_retry = 0 only) */
  int32_t attempts;     /* retry attempts used (ref_retry) */
  int32_t fallback_used;/* a fallback preconditioner finished the solve:
                           learned -> Jacobi, or Jacobi -> multigrid */
  int32_t zero_rhs;     /* 1: ||f_free|| == 0, u = 0 returned */
  double rel_res;       /* recursive residual at stop (reference final_rel_res) */
  double true_rel_res;  /* ||b - (K+sI)u|| / ||b|| recomputed in FP64 */
  double shift;         /* diagonal shift actually used */
  double time_setup_ms;
  double time_solve_ms;
  double time_total_ms;
  double time_device_ms;   /* CUDA-event time of the call on the context stream */
  double kernel_launches;  /* kernels launched by the call (graph nodes included) */
  double time_precond_setup_ms; /* multigrid hierarchy set-up (part of time_solve_ms;
                                   0 for the other preconditioners) */
  double reserved[1];
} hx_solve_report;

typedef struct hx_ctx hx_ctx;

/* ---- context -------------------------------------------------------------
 * One context per host thread; it owns one CUDA stream and the cached device
 * buffers (the counterpart of the reference's GLOBAL_HELMHOLTZ_CACHE,
 * src/Optimization/GPUHelmholtz.jl:12-33).  Uses the primary context of
 * `device`, as CUDA.jl does (src/Main.jl:179). */
HX_API hx_status hx_create(hx_ctx **out, int32_t device);
HX_API void hx_destroy(hx_ctx *ctx);
HX_API const char *hx_last_error(const hx_ctx *ctx);
HX_API void hx_default_opts(hx_solve_opts *opts);
HX_API const char *hx_status_string(int32_t status);
/* The context's CUDA stream (a cudaStream_t), for callers that bracket
 * library calls with their own CUDA events. */
HX_API hx_status hx_get_stream(const hx_ctx *ctx, void **stream);
/* Total kernels this context has launched (graph nodes included). */
HX_API int64_t hx_kernel_launches(const hx_ctx *ctx);

/* ---- mesh, material, boundary conditions ---------------------------------
 * hx_set_grid: the structured mesh of src/Mesh/Mesh.jl:23-60 (generate_mesh)
 * with nx*ny*nz elements of size dx*dy*dz.
 * hx_set_mesh: any node/element arrays in the reference layout.  A mesh whose
 * nodes sit on a lattice (generate_mesh output, or its pruned subset from
 * src/Mesh/MeshPruner.jl:18-112) is embedded in its bounding grid so the
 * structured kernels run; absent elements get zero stiffness and nodes
 * without stiffness are held fixed (what reconstruct_full_solution,
 * MeshPruner.jl:120-138, returns for them).  Element size is taken from the
 * first element, as src/Solvers/GPUSolver.jl:136-145 does.
 * hx_set_bc: src/Core/Boundary.jl:135-160 bc_indicator. */
HX_API hx_status hx_set_grid(hx_ctx *ctx, int64_t nx, int64_t ny, int64_t nz,
                             double dx, double dy, double dz);
HX_API hx_status hx_set_mesh(hx_ctx *ctx, const float *nodes, int64_t n_nodes,
                             const int64_t *elements, int64_t n_elem);
HX_API hx_status hx_set_material(hx_ctx *ctx, double E, double nu);
HX_API hx_status hx_set_bc(hx_ctx *ctx, const float *bc_indicator,
                           int64_t n_nodes);
/* Grid shape of the current mesh (elements per axis) and the mapping of the
 * caller's node/element numbering to grid positions (-1: none). */
HX_API hx_status hx_get_grid(const hx_ctx *ctx, int64_t dims[3], double h[3]);

/* ---- stiffness operator ---------------------------------------------------
 * y = sum_e factor_e * Ke * x_e over all elements, no boundary conditions,
 * no shift: src/Solvers/CPUSolver.jl:50-94 apply_stiffness, with
 * factor_e = E*density_e (0 for skipped elements).  Host arrays in the
 * caller's numbering. */
HX_API hx_status hx_apply_stiffness(hx_ctx *ctx, int32_t dtype, const void *x,
                                    const void *factor, void *y);
/* Allocation-free K(f)x -- no counterpart in the reference.
 * Some callers cannot let a library allocate device memory: cudaMalloc and
 * cudaFree synchronize the device (stalling every other stream of a caller
 * that keeps work in flight), and a host runtime that pools device memory
 * itself (CUDA.jl in the reference's Julia host) may hold most of the
 * device, so a foreign allocation fails.  This entry point computes
 * y = K(f)x on the structured nx*ny*nz grid (no boundary conditions, no
 * shift, as hx_apply_stiffness) and *xKx = x.y (FP64, deterministic), all
 * arrays FP64 DEVICE pointers in grid numbering (x 16-byte aligned; factor,
 * y and xKx 8-byte aligned; a misaligned pointer returns HX_BAD_ARG before
 * any GPU work), on `stream` (a cudaStream_t; NULL = default stream).  It allocates nothing: its scratch
 * (one partial sum per CTA plus a completion counter) lives in a static
 * device array of 256 + 8*HX_NOALLOC_MAX_BLOCKS bytes that every GPU
 * loading the library holds until exit.  Grids needing more than
 * HX_NOALLOC_MAX_BLOCKS CTAs (beyond about 1880 x 1880 nodes per plane)
 * are rejected with HX_BAD_ARG.  The first call on a device resolves the
 * array's device address (cudaGetSymbolAddress) with that device current;
 * make that first call before any stream capture.  All calls on a device
 * share the array: calls that overlap on the GPU race, so order them
 * (e.g. on one stream).  Returns without waiting for the GPU. */
#define HX_NOALLOC_MAX_BLOCKS 16384
HX_API hx_status hx_apply_stiffness_noalloc(int64_t nx, int64_t ny, int64_t nz,
                                            double dx, double dy, double dz,
                                            double nu, const double *x,
                                            const double *factor, double *y,
                                            double *xKx, void *stream);
/* Jacobi diagonal, src/Solvers/CPUSolver.jl:109-148. */
HX_API hx_status hx_diagonal(hx_ctx *ctx, int32_t dtype, const void *factor,
                             void *diag);

/* ---- linear solve ---------------------------------------------------------
 * Solves (K_ff + s I) u_f = f_f on the free DOFs by Jacobi-PCG with
 * M^-1 = 1/(diag + s) (src/Solvers/GPUSolver.jl:274-609, M_inv at :402).
 * factor: per-element stiffness factor (E*density, or the caller's SIMP
 * modulus).  u_inout: initial guess when opts->warm_start, full-length
 * solution (zeros at fixed DOFs) on return.  Host arrays of `dtype`. */
HX_API hx_status hx_solve(hx_ctx *ctx, int32_t dtype, const void *f,
                          const void *factor, void *u_inout,
                          const hx_solve_opts *opts, hx_solve_report *report);
/* The same with FP64 device pointers in grid numbering (no host traffic). */
HX_API hx_status hx_solve_device(hx_ctx *ctx, const double *f_dev,
                                 const double *factor_dev, double *u_dev,
                                 const hx_solve_opts *opts,
                                 hx_solve_report *report);

/* The solver of this context's drop-in solves (hx_solve_system_gpu,
 * hx_solve_system_grid).  The reference reads
 * config["solver_parameters"]["preconditioner"] on every solve
 * (src/Solvers/GPUSolver.jl:320-324): "jacobi" = (HX_PC_JACOBI,
 * HX_PREC_FP64, multigrid_fallback 0); "jacobi_amg", the default of
 * configs/default.yaml:191 and of this library = (HX_PC_JACOBI,
 * HX_PREC_FP64, 1); "amg" = (HX_PC_MULTIGRID, HX_PREC_FP64, 0), the
 * multigrid preconditioner from the first attempt (prec_name "GMG").
 * HX_PREC_MIXED32 and HX_PC_LEARNED (needs loaded networks; prec_name
 * "Learned", or "Jacobi" when it fell back) are further choices.  The
 * retry and shift-escalation semantics apply to every choice. */
HX_API hx_status hx_set_dropin_solver(hx_ctx *ctx, int32_t preconditioner, int32_t precision,
                                      int32_t multigrid_fallback);

/* Drop-in for GPUSolver.solve_system_gpu(nodes, elements, E, nu,
 * bc_indicator, f, density; max_iter, tol, shift_factor,
 * min_stiffness_threshold, u_guess) -> (x_full, final_rel_res, prec_name),
 * src/Solvers/GPUSolver.jl:611-627 (called from
 * src/Solvers/IterativeSolver.jl:27-39).  Elements with density <
 * min_stiffness_threshold are inactive (GPUSolver.jl:128); factor =
 * E*density (:147).  u_guess may be NULL (cold start).  Writes x_full
 * (3*n_nodes), *final_rel_res and the preconditioner name.  Failure
 * handling as the reference's with its default preconditioner "jacobi_amg"
 * (configs/default.yaml:191): three attempts with shift escalation, and
 * after a failed or stagnated Jacobi attempt the geometric multigrid
 * preconditioner in place of the CPU AMG (prec_name "GMG"). */
HX_API hx_status hx_solve_system_gpu(
    hx_ctx *ctx, const float *nodes, int64_t n_nodes, const int64_t *elements,
    int64_t n_elem, float E, float nu, const float *bc_indicator,
    const float *f, const float *density, int32_t max_iter, double tol,
    float shift_factor, float min_stiffness_threshold, const float *u_guess,
    float *x_full, double *final_rel_res, char *prec_name,
    int32_t prec_name_cap);

/* The same solve on the unpruned structured mesh of generate_mesh
 * (nx*ny*nz elements of dx*dy*dz; src/Mesh/Mesh.jl:23-60), given by its
 * dimensions instead of node and element arrays, with the reference's
 * pruning done on the device: elements with density < min_stiffness_threshold
 * get zero stiffness and nodes left without stiffness are held at 0 -- the
 * x_full the reference's prune_system / solve / reconstruct_full_solution
 * returns (src/Solvers/Solver.jl:60-91,158-160, src/Mesh/MeshPruner.jl).
 * The host only copies: no per-element or per-node host work.  Arrays in the
 * grid's numbering (generate_mesh's own). */
HX_API hx_status hx_solve_system_grid(
    hx_ctx *ctx, int64_t nx, int64_t ny, int64_t nz, double dx, double dy,
    double dz, float E, float nu, const float *bc_indicator, const float *f,
    const float *density, int32_t max_iter, double tol, float shift_factor,
    float min_stiffness_threshold, const float *u_guess, float *x_full,
    double *final_rel_res, char *prec_name, int32_t prec_name_cap);

/* ---- Helmholtz PDE density filter ------------------------------------------
 * (r^2 K + M) x = T rho with T the lumped vol/8 scatter, Jacobi-CG (at most
 * max_iter iterations, residual tested every 10), element value = mean of
 * its 8 nodes: src/Optimization/GPUHelmholtz.jl:39-229.  ref_compat=1 uses
 * the reference element whose top face sits at z=+dz (Element.jl:106-107,
 * an element 1.5*dz tall); ref_compat=0 the geometric element.  Structured
 * grids only (the reference always filters the full grid). */
HX_API hx_status hx_filter(hx_ctx *ctx, int32_t dtype, const void *rho,
                           void *rho_out, double radius, int32_t ref_compat,
                           double tol, int32_t max_iter,
                           hx_solve_report *report);
HX_API hx_status hx_filter_device(hx_ctx *ctx, const double *rho_dev,
                                  double *out_dev, double radius,
                                  int32_t ref_compat, double tol,
                                  int32_t max_iter, hx_solve_report *report);
/* Drop-in for GPUHelmholtz.apply_gpu_filter!(density, nElem_x, nElem_y,
 * nElem_z, dx, dy, dz, radius, elements, tol) -> (filtered, time, iters, res),
 * src/Optimization/GPUHelmholtz.jl:344-376.  On failure returns a non-OK
 * status (the reference returned Float32[] to request its CPU fallback). */
HX_API hx_status hx_apply_gpu_filter(hx_ctx *ctx, const float *density,
                                     int64_t nelem_x, int64_t nelem_y,
                                     int64_t nelem_z, double dx, double dy,
                                     double dz, double radius, double tol,
                                     int32_t ref_compat, float *filtered,
                                     double *time_s, int32_t *iters,
                                     double *res);

/* ---- stress ----------------------------------------------------------------
 * Centre-point stress with modulus E*density[e] for density > 1e-6:
 * principal values (descending, 3 per element), von Mises, Voigt
 * (xx,yy,zz,xy,yz,xz), L1 = sum |principal|, unit direction of the largest
 * principal stress (sign: largest-magnitude component positive; the
 * reference's LAPACK sign is arbitrary).  src/Core/Stress.jl:10-100.
 * Outputs are element-major (principal[3e+i], voigt[6e+i], dir[3e+i]),
 * i.e. the memory layout of the reference's 3 x nE / 6 x nE matrices. */
HX_API hx_status hx_stress(hx_ctx *ctx, int32_t dtype, const void *u,
                           const void *density, double E, double nu,
                           void *principal, void *vonmises, void *voigt,
                           void *l1, void *dir);
/* p-norm aggregate of the element von Mises stresses (no reference
 * counterpart; the stress-constrained loop's aggregate):
 * *pnorm = (sum_e vm_e^P)^(1/P), vm as in hx_stress (0 for void elements),
 * formed as max(vm) * (sum (vm/max)^P)^(1/P) in FP64 on the device;
 * *vmax = max vm (may be NULL).  P >= 1 (8 in the stress-aggregated loop). */
HX_API hx_status hx_stress_pnorm(hx_ctx *ctx, int32_t dtype, const void *u,
                                 const void *density, double E, double nu,
                                 double P, double *pnorm, double *vmax);
/* Drop-in for Stress.compute_stress_field(nodes, elements, U, E, nu,
 * density), src/Core/Stress.jl:57-100. */
HX_API hx_status hx_compute_stress_field(
    hx_ctx *ctx, const float *nodes, int64_t n_nodes, const int64_t *elements,
    int64_t n_elem, const float *U, float E, float nu, const float *density,
    float *principal, float *vonmises, float *voigt, float *l1, float *dir);

/* ---- result file ------------------------------------------------------------
 * Drop-in for export_binary_for_web(filename, nodes, elements, density,
 * l1_stress, principal_field, geom, threshold, iter, current_radius, config),
 * src/IO/Postprocessing.jl:159-262: the "webdata" file the reference's
 * viewers and its checkpoint restart (src/IO/Configuration.jl:31-77) read.
 * Magic 0x48455841 ("HEXA"), version 2, iter, radius, threshold, count, dx,
 * dy, dz, then for the elements with density >= threshold, in element order:
 * centroids (3 Float32 each), densities, L1 stress signed by the principal
 * stress of largest magnitude; then the JSON text's byte length and the text
 * (the caller serialises its config, as the reference's JSON.json does).
 * The selection and the per-element values are computed on the device; no
 * file is written when no element passes (*count = 0).  Needs the mesh in
 * grid numbering (hx_set_grid, or generate_mesh order through hx_set_mesh).
 * hx_export_webdata: host arrays of dtype (principal: 3 values per element,
 * element-major); _device: FP64 device arrays. */
HX_API hx_status hx_export_webdata(hx_ctx *ctx, const char *path, int32_t dtype,
                                   const void *density, const void *l1_stress,
                                   const void *principal, float threshold,
                                   int32_t iter, float current_radius,
                                   const char *json, int64_t json_len,
                                   int64_t *count);
HX_API hx_status hx_export_webdata_device(hx_ctx *ctx, const char *path,
                                          const double *density_dev,
                                          const double *l1_dev,
                                          const double *principal_dev,
                                          float threshold, int32_t iter,
                                          float current_radius, const char *json,
                                          int64_t json_len, int64_t *count);

/* ---- compliance, sensitivities, OC update ------------------------------------
 * hx_compliance: c = f.u in FP64 (src/Main.jl:428 computes it on the host).
 * hx_element_energy: ce_e = u_e^T Ke u_e with unit modulus (no reference
 * counterpart; the compliance sensitivity of the OC method is
 * dc_e = -p*rho^(p-1)*(E0-Emin)*ce_e).
 * hx_oc_update: optimality-criteria update with bisection on the volume
 * multiplier (no reference counterpart: the reference updates by stress
 * ratio, src/Optimization/TopOpt.jl:260-402; this is the published OC method
 * of the top88/top3d family).  See the library documentation for the exact
 * rule. */
HX_API hx_status hx_compliance(hx_ctx *ctx, int32_t dtype, const void *f,
                               const void *u, double *c);
HX_API hx_status hx_element_energy(hx_ctx *ctx, int32_t dtype, const void *u,
                                   void *ce);
HX_API hx_status hx_oc_update(hx_ctx *ctx, int32_t dtype, const void *x,
                              const void *dc, const void *dv, double volfrac,
                              double move, void *xnew, double *lambda,
                              int32_t *steps);

/* ---- density update -----------------------------------------------------------------
 * Drop-in for TopologyOptimization.update_density!(density, l1_stress_norm_field,
 * protected_elements_mask, E, l1_stress_allowable, iter, number_of_iterations,
 * original_density, min_density, max_density, config, elements, is_annealing)
 * -> (max_change, R_length, current_threshold, filter_time, filter_iters,
 * filter_res), src/Optimization/TopOpt.jl:139-405, on the structured grid of
 * params->nelem (elements in grid order, as the reference's density vector).
 * Float32 host arrays of n = nx*ny*nz entries, updated in place like the
 * Julia vectors: density (and l1_stress when stress regularisation is on);
 * protected_mask is one byte per element (non-zero = protected).
 * mode HX_UPDATE_STRESS_RATIO (the reference): optional stress
 * regularisation filter, radius schedule with the 1.2 h guard and R/2.5,
 * proposal clamp((l1/allowable)/E, min, max) (original density where
 * protected), Helmholtz filter with the reference element, clamp, culling of
 * at most floor(active * max_culling_ratio) of the weakest elements below
 * threshold * iter / number_of_iterations (ties in element order), protected
 * re-enforce; every per-element step in the reference's Float32 arithmetic,
 * the filters in FP64 (radius, sizes and tolerance rounded to Float32 as the
 * reference's filter workspace does, at most 200 iterations).
 * mode HX_UPDATE_OC (no reference counterpart): dc (the compliance
 * sensitivities, required) is Helmholtz-filtered with the same radius and
 * the density takes one optimality-criteria step (bisection on the volume
 * multiplier, unit volumes, oc_volfrac, oc_move), then the clamp and the
 * protected re-enforce; no culling (current_threshold 0).
 * filtered_out (optional, n floats) receives the filtered proposal (or the
 * filtered dc), rounded to Float32. */
typedef enum hx_update_mode { HX_UPDATE_STRESS_RATIO = 0, HX_UPDATE_OC = 1 } hx_update_mode;
typedef struct hx_update_params {
  int64_t nelem[3];     /* config geometry nElem_x/y/z_computed */
  double h[3];          /* dx/dy/dz_computed (used as Float32) */
  double max_domain_dim;
  double filter_tolerance;            /* solver_parameters (default 1e-5) */
  double stress_regularization_ratio; /* optimization_parameters (default 0) */
  double filter_R_init_perc;          /* (default 0) */
  double filter_R_interm_perc;        /* (default 0) */
  double filter_R_final_perc;         /* (default 0) */
  double filter_R_interm_iter_perc;   /* (default 50) */
  double final_density_threshold;     /* (default 0.95) */
  double max_culling_ratio;           /* (default 0.1) */
  int32_t mode;                       /* hx_update_mode */
  int32_t reserved0;
  double oc_volfrac, oc_move;         /* HX_UPDATE_OC only */
  double reserved[4];
} hx_update_params;
typedef struct hx_update_result {
  double max_change, R_length, current_threshold, filter_time, filter_res;
  int32_t filter_iters;
  int32_t culled;       /* elements set to min_density by the culling */
  double reserved[2];
} hx_update_result;
HX_API void hx_default_update_params(hx_update_params *params);
HX_API hx_status hx_update_density(hx_ctx *ctx, float *density, float *l1_stress,
                                   const uint8_t *protected_mask, float E,
                                   float l1_stress_allowable, int32_t iter,
                                   int32_t number_of_iterations,
                                   const float *original_density, float min_density,
                                   float max_density, const hx_update_params *params,
                                   const float *dc, float *filtered_out,
                                   hx_update_result *result);

/* ---- device-resident optimisation loop pieces ---------------------------------------
 * No reference counterpart (the OC loop is the published method).  FP64
 * device arrays in grid numbering; need a grid mesh (hx_set_grid).  With
 * hx_filter_device and hx_solve_device they keep an OC iteration on the
 * device.  fac = emin + max(rho,0)^p (e0 - emin);  dc = -p max(rho,0)^(p-1)
 * (e0 - emin) u_e^T Ke u_e;  *c = f.u (FP64);  OC bisection as hx_oc_update
 * (dv NULL: unit volumes). */
HX_API hx_status hx_simp_device(hx_ctx *ctx, const double *rho_dev, double p,
                                double e0, double emin, double *fac_dev);
HX_API hx_status hx_sensitivity_device(hx_ctx *ctx, const double *rho_dev,
                                       const double *u_dev, double p, double e0,
                                       double emin, double *dc_dev);
HX_API hx_status hx_compliance_device(hx_ctx *ctx, const double *f_dev,
                                      const double *u_dev, double *c);
HX_API hx_status hx_oc_update_device(hx_ctx *ctx, const double *x_dev,
                                     const double *dc_dev, const double *dv_dev,
                                     double volfrac, double move,
                                     double *xnew_dev, double *lambda,
                                     int32_t *steps);

/* ---- learned preconditioner -----------------------------------------------------
 * No reference counterpart.  z = D^-1/2 (I + sum_l R_l^T E_l^T G_l^T G_l E_l R_l) D^-1/2 r
 * for l = HX_NET_FIRST_LEVEL .. HX_NET_FIRST_LEVEL + 2: R_l restricts a nodal
 * field to node-grid level l (each level halves the grid, full weighting)
 * and R_l^T is its exact transpose; E_l lifts a field to 6 channels
 * (x, density * x); G_l is a 3D CNN of 4 conv3d layers (3x3x3, no bias,
 * 6 -> 16 -> 16 -> 16 -> 16 channels, BF16 weights and activations, FP32
 * accumulation on the tensor cores) and G_l^T its transposed convolutions.
 * Symmetric positive definite for every choice of weights; zero weights give
 * Jacobi.  hx_solve with preconditioner HX_PC_LEARNED applies it in flexible
 * CG (Notay, one stored direction) and falls back to Jacobi-PCG from the
 * current iterate on breakdown or stagnation (report->fallback_used).
 * Parameters: HX_NET_PARAMS floats, the 3 networks one after the other
 * (finest level first), each 4 layers of [27 taps][16 out][16 in] weights;
 * input channels >= 6 of each first layer are forced to zero. */
#define HX_NET_FIRST_LEVEL 2
#define HX_NET_PARAMS (3 * 4 * 27 * 256)
HX_API hx_status hx_net_init(hx_ctx *ctx, uint64_t seed);
HX_API hx_status hx_net_set_params(hx_ctx *ctx, const float *params);
HX_API hx_status hx_net_get_params(hx_ctx *ctx, float *params);
/* y = G^T G x0 with the FIRST network on an nx*ny*nz NODE grid from host
 * arrays [node][16] (FP32, rounded to BF16; channels >= 6 of x0 and dy are
 * ignored, those of y are zero) and grads = d<dy, y>/dparams (HX_NET_PARAMS
 * values, zero for the other networks; gradient check). */
HX_API hx_status hx_net_forward_backward(hx_ctx *ctx, int32_t nx, int32_t ny,
                                         int32_t nz, const float *x0,
                                         const float *dy, float *y,
                                         float *grads);
/* Operator inputs of the network (Jacobi scaling, density feature) for the
 * FP64 device factors `fac` on the current mesh and BCs. */
HX_API hx_status hx_net_prepare(hx_ctx *ctx, const double *fac_dev);
/* Failure detection of the tensor-core convolution (no reference
 * counterpart): launches one convolution CTA whose load barrier is never
 * armed, so its bounded wait (about a second at most) runs out; the kernel
 * records the timeout and returns without a fault.  *detected = 1 when the
 * host saw it; the call then runs an ordinary convolution on the same
 * context and returns HX_OK only if that succeeds.  Clears the packed
 * weights' staging and re-packs them from the loaded parameters. */
HX_API hx_status hx_selftest_wait_timeout(hx_ctx *ctx, int32_t *detected);
/* z = P r, the learned preconditioner of the prepared operator (FP64 device
 * vectors, grid numbering); z = 0 when r vanishes on the free DOFs. */
HX_API hx_status hx_net_apply(hx_ctx *ctx, const double *r_dev, double *z_dev);
/* z = V r, one V-cycle of the geometric multigrid preconditioner of the last
 * multigrid-preconditioned solve (HX_PC_MULTIGRID) on this context: FP64
 * device vectors, grid numbering, r zero on the fixed DOFs.  No reference
 * counterpart (the reference's AMG is applied inside its solve only,
 * src/Solvers/GPUSolver.jl:513-516).  HX_BAD_ARG before such a solve. */
HX_API hx_status hx_gmg_apply(hx_ctx *ctx, const double *r_dev, double *z_dev);
/* One Adam step on a residual (and error) of the prepared operator (FP64
 * device vectors, grid numbering; r = f - K x, e = u* - x).  With z the
 * preconditioned vector of r:  loss_kind 0: *loss = (z-e)^T K (z-e) / e^T K e
 * (needs e);  loss_kind 1: *loss = |D^-1/2 (K z - r)|^2 / |D^-1/2 r|^2
 * (e unused, may be NULL). */
HX_API hx_status hx_net_train_step(hx_ctx *ctx, const double *r_dev,
                                   const double *e_dev, double lr,
                                   int32_t loss_kind, double *loss);
/* The same over a batch: the gradients of `count` pairs (arrays of device
 * pointers; e_devs may be NULL for loss_kind 1) are summed before one Adam
 * step; *loss = their mean loss. */
HX_API hx_status hx_net_train_batch(hx_ctx *ctx, const double *const *r_devs,
                                    const double *const *e_devs, int32_t count,
                                    double lr, int32_t loss_kind, double *loss);
/* FP64 Jacobi-PCG from zero on (f, fac) storing the iterate every `every`
 * (even) iterations into snaps_dev[count][3*nodes] until rtol `tol`;
 * *taken = snapshots stored.  Training data for the network. */
HX_API hx_status hx_pcg_snapshots(hx_ctx *ctx, const double *f_dev,
                                  const double *fac_dev, int32_t every,
                                  int32_t count, double tol, double *snaps_dev,
                                  int32_t *taken);
/* r = f - K(fac) x on the free DOFs (0 on fixed ones), FP64 device arrays. */
HX_API hx_status hx_residual_device(hx_ctx *ctx, const double *f_dev,
                                    const double *fac_dev, const double *x_dev,
                                    double *r_dev);

/* ---- instrumentation ---------------------------------------------------------
 * Average device time (CUDA events on the context stream) of `reps`
 * back-to-back launches of one kernel on the buffers of the last hx_solve /
 * hx_solve_device (kernel ids below); inputs are left unchanged except the
 * kernels' scratch outputs.  Used by the benchmark for the live roofline. */
enum {
  HX_KERNEL_PCG_STEP_FP64 = 0,   /* fused p/x update + K.p + p.q reduction */
  HX_KERNEL_PCG_UPDATE_FP64 = 1, /* r update + r.z, r.r reductions */
  HX_KERNEL_APPLY_FP64 = 2,      /* plain K.x */
  HX_KERNEL_PCG_STEP_FP32 = 3,
  HX_KERNEL_FILTER_MATVEC = 4,
  HX_KERNEL_CONV3 = 5,           /* one 16 -> 16 BF16 conv3d layer on the node grid */
  HX_KERNEL_NET_APPLY = 6,       /* one learned-preconditioner application */
  HX_KERNEL_FCG_STEP_FP32 = 7    /* flexible-CG step of the mixed learned solve:
                                    p = z + beta p_old, x update, K.p, p.q */
};
HX_API hx_status hx_time_kernel(hx_ctx *ctx, int32_t kernel, int32_t reps,
                                double *avg_ms);

#ifdef __cplusplus
}
#endif
#endif /* HEXAT_B200_H */
