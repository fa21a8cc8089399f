// hx_solver.h -- device-level solver entry points (grid numbering, FP64
// device arrays) used by the C ABI layer.
#pragma once
#include <functional>

#include "hx_internal.h"

namespace hx {
// device-state plumbing shared by the solvers
CgState fresh_state(double tol, int max_iter, int check_every, bool divchecks, bool keep_best);
void put_state(hx_ctx* c, int slot, const CgState& s);
CgState get_state(hx_ctx* c, int slot);
int auto_batch(const Grid& g, int check_every);
// Capture `reps` x body into one CUDA graph and launch it until the state of
// `slot` leaves HX_RUNNING, `max_launches` (> 0) launches were made, the wall
// limit passed, or keep_going (if given) returns false for the state read
// after a launch.
CgState run_batched(hx_ctx* c, int slot, int reps, const std::function<void()>& body,
                    double wall_limit_ms, double t0, bool* timed_out, int max_launches,
                    const std::function<bool(const CgState&)>& keep_going = {});
// node masks, diagonal, shift and M^-1 (FP64) for `fac`; returns max diag
double jacobi_setup_public(hx_ctx* c, const double* fac, double shift_factor, double* shift_out);
template <typename T>
CgState pcg_fused(hx_ctx* c, int slot, const T* fac, const T* b, T* x, bool warm, T shift,
                  const ElemCoef<T>& K, T* r, T* P0, T* P1, T* q, const T* minv, T* xbest,
                  const CgState& init, int check_every, double wall_ms, double t0,
                  bool* timed_out);
// learned preconditioner (hx_net.cu)
void net_init(hx_ctx* c, uint64_t seed);
void net_set_params(hx_ctx* c, const float* params);
void net_get_params(hx_ctx* c, float* params);
void net_forward_backward(hx_ctx* c, int nx, int ny, int nz, const float* x0, const float* dy,
                          float* y, float* grads);
double net_train_step(hx_ctx* c, const double* const* r, const double* const* e, int count,
                      double lr, int loss_kind);
void net_prepare(hx_ctx* c, const double* fac);
bool conv_wait_selftest(hx_ctx* c);
void net_apply_vec(hx_ctx* c, const double* r, double* z);
// Timing bodies on the prepared network: 0 = one 16 -> 16 conv layer on the
// node grid, 1 = one preconditioner application (lift, 8 layers, output).
std::function<void()> net_time_body(hx_ctx* c, int which);
CgState solve_learned(hx_ctx* c, const double* fac, const double* b, double* x, bool warm,
                      double shift, const hx_solve_opts& o, double t0, bool* timed_out,
                      int* fallback, int* iters_out);
CgState solve_learned_mixed(hx_ctx* c, const double* fac, const double* b, double* x, bool warm,
                            double shift, const hx_solve_opts& o, double t0, bool* timed_out,
                            int* fallback, int* iters_out);
// Mixed-precision flexible CG with the multigrid V-cycle (hx_net.cu's FP32
// loop with FP64 reliable updates; Jacobi-PCG finishes a stalled solve).
CgState solve_gmg_mixed(hx_ctx* c, const double* fac, const double* b, double* x, bool warm,
                            double shift, const hx_solve_opts& o, double t0, bool* timed_out,
                            int* fallback, int* iters_out);
CgState solve_mixed(hx_ctx* c, const double* fac, const double* b, double* x, bool warm,
                    double shift, const hx_solve_opts& o, double t0, bool* timed_out,
                    int* inner_total);
int pcg_snapshots(hx_ctx* c, const double* f, const double* fac, int every, int count,
                  double tol, double* snaps);
void ensure_workspace(hx_ctx* c);
void upload_bc(hx_ctx* c);
hx_status solve_grid(hx_ctx* c, const double* f, const double* fac, double* u,
                     const hx_solve_opts& o, hx_solve_report* rep);
// Filter on the grid g with element size h (FP64 device arrays, grid numbering).
hx_status filter_grid(hx_ctx* c, const Grid& g, const double h[3], const double* rho, double* out,
                      double radius, int ref_compat, double tol, int max_iter,
                      hx_solve_report* rep);
// update_density! of the reference (or the OC step) on Float32 host arrays
// (hx_update.cu); see hx_update_density.
hx_status update_density(hx_ctx* c, float* density, float* l1, const uint8_t* prot, float E,
                         float allow, int it, int n_iter, const float* orig, float min_d,
                         float max_d, const hx_update_params& p, const float* dc,
                         float* filtered_out, hx_update_result* res);
void update_radius_schedule(const hx_update_params& p, int it, int n_iter, double* R_length,
                            double* R_effective);
// export_binary_for_web from element arrays in grid numbering on the device
// (T = double or float; principal: 3 values per element) (hx_export.cu).
template <typename T>
hx_status export_webdata(hx_ctx* c, const char* path, const T* dens, const T* l1, const T* pr,
                         float threshold, int iter, float radius, const char* json,
                         int64_t json_len, int64_t* count_out);
// geometric multigrid (hx_gmg.cu): hierarchy for `fac` (after the Jacobi
// set-up of the solve), one V-cycle z = V(r), the flexible-CG coefficients
// of a preconditioned residual, and the FP64 FCG solve it preconditions
// default Chebyshev degree of the multigrid smoothing
constexpr int GMG_DEFAULT_DEGREE = 2;
void gmg_setup(hx_ctx* c, const double* fac, double shift);
template <typename T>
void gmg_vcycle(hx_ctx* c, const T* r, T* z);
template <typename T>
void launch_fcg_coeffs(cudaStream_t s, const T* z, const T* q_old, const T* r, int64_t n,
                       double* partials, CgState* st);
CgState solve_gmg(hx_ctx* c, const double* fac, const double* b, double* x, bool warm,
                  double shift, const hx_solve_opts& o, double t0, bool* timed_out,
                  int* iters_out);
// Average time of `reps` launches of one kernel on the last solve's buffers.
hx_status time_kernel(hx_ctx* c, int kernel, int reps, double* avg_ms);
}  // namespace hx
