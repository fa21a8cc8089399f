// hx_solver.h -- device-level solver entry points (grid numbering, FP64
// device arrays) used by the C ABI layer.
#pragma once
#include "hx_internal.h"

namespace hx {
void ensure_workspace(hx_ctx* c);
void upload_bc(hx_ctx* c);
hx_status solve_grid(hx_ctx* c, const double* f, const double* fac, double* u,
                     const hx_solve_opts& o, hx_solve_report* rep);
// Filter on the grid g with element size h (FP64 device arrays, grid numbering).
hx_status filter_grid(hx_ctx* c, const Grid& g, const double h[3], const double* rho, double* out,
                      double radius, int ref_compat, double tol, int max_iter,
                      hx_solve_report* rep);
// Average time of `reps` launches of one kernel on the last solve's buffers.
hx_status time_kernel(hx_ctx* c, int kernel, int reps, double* avg_ms);
}  // namespace hx
