// hx_solver.cu -- host orchestration of the device solvers: Jacobi set-up,
// the FP64 PCG loop (CUDA-graph batches, device-side scalars, host poll),
// mixed-precision iterative refinement, the Helmholtz filter CG, and the
// reference retry semantics.
#include <chrono>
#include <cmath>
#include <functional>
#include <limits>

#include "hx_solver.h"

namespace hx {

int64_t& launch_counter() {
  static thread_local int64_t n = 0;
  return n;
}

int current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return dev;
}

int sm_count() {
  static std::atomic<int> cache[64];  // 0: not yet queried
  const int dev = current_device();
  const bool tracked = dev >= 0 && dev < 64;
  if (tracked) {
    const int n = cache[dev].load(std::memory_order_relaxed);
    if (n > 0) return n;
  }
  int n = 0;
  if (dev < 0 || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return 148;  // not cached: the next call asks again
  }
  if (n <= 0) return 148;
  if (tracked) cache[dev].store(n, std::memory_order_relaxed);
  return n;
}

ElemCoef<double> make_elem_coef(double dx, double dy, double dz, double nu) {
  ElemCoef<double> K{};
  const double lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  const double mu = 1.0 / (2.0 * (1.0 + nu));
  const double h[3] = {dx, dy, dz};
  auto m = [&](int a, int sg) { return sg ? h[a] / 6.0 : h[a] / 2.0; };
  auto s = [&](int a, int sg) { return sg ? 2.0 / h[a] : 0.0; };
  for (int c = 0; c < 3; ++c) {
    const int j = (c + 1) % 3, k = (c + 2) % 3;
    for (int sg = 0; sg < 8; ++sg) {
      const int b[3] = {sg & 1, (sg >> 1) & 1, (sg >> 2) & 1};
      const double S[3] = {s(0, b[0]), s(1, b[1]), s(2, b[2])};
      const double M[3] = {m(0, b[0]), m(1, b[1]), m(2, b[2])};
      const double all = S[0] * M[1] * M[2] + M[0] * S[1] * M[2] + M[0] * M[1] * S[2];
      K.dg[c][sg] = ((lam + mu) * S[c] * M[j] * M[k] + mu * all) / 8.0;
    }
    double kd = 0;
    for (int sg = 0; sg < 8; ++sg) kd += K.dg[c][sg];
    K.kd[c] = kd;
  }
  for (int k = 0; k < 3; ++k)
    for (int sk = 0; sk < 2; ++sk) {
      K.lam[k][sk] = lam * m(k, sk) / 8.0;
      K.mu[k][sk] = mu * m(k, sk) / 8.0;
    }
  return K;
}

ElemCoef<float> to_float(const ElemCoef<double>& k) {
  ElemCoef<float> f{};
  for (int c = 0; c < 3; ++c) {
    for (int s = 0; s < 8; ++s) f.dg[c][s] = (float)k.dg[c][s];
    for (int s = 0; s < 2; ++s) {
      f.lam[c][s] = (float)k.lam[c][s];
      f.mu[c][s] = (float)k.mu[c][s];
    }
    f.kd[c] = (float)k.kd[c];
  }
  return f;
}

static double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------------------
// Workspace
// ---------------------------------------------------------------------------
void ensure_workspace(hx_ctx* c) {
  if (!c->h_state) HX_CUDA(cudaMallocHost(&c->h_state, 4 * sizeof(CgState)));
  c->d_state.ensure(4);
  const size_t nb = std::max<size_t>(mv_max_blocks(c->g), 64ull * sm_count());
  c->d_partials.ensure(4 * nb);
  c->d_scalars.ensure(16);
}

void upload_bc(hx_ctx* c) {
  const int64_t nn = c->g.nodes();
  c->d_bcfree.ensure(nn);
  if (c->bcfree.size() != (size_t)nn) c->bcfree.assign(nn, 7);  // no BC given: all free
  HX_CUDA(cudaMemcpyAsync(c->d_bcfree.p, c->bcfree.data(), nn, cudaMemcpyHostToDevice, c->stream));
  c->bc_dirty = false;
}

CgState fresh_state(double tol, int max_iter, int check_every, bool divchecks,
                    bool keep_best) {
  CgState s{};
  s.tol = tol;
  s.max_iter = max_iter;
  s.check_every = std::max(1, check_every);
  s.explode = divchecks ? 1000.0 : 0.0;
  s.div_ratio = divchecks ? 100.0 : 0.0;
  s.keep_best = keep_best ? 1 : 0;
  s.best_rel = INFINITY;
  s.status = HX_RUNNING;
  return s;
}

void put_state(hx_ctx* c, int slot, const CgState& s) {
  c->h_state[slot] = s;
  HX_CUDA(cudaMemcpyAsync(c->d_state.p + slot, c->h_state + slot, sizeof(CgState),
                          cudaMemcpyHostToDevice, c->stream));
}

CgState get_state(hx_ctx* c, int slot) {
  HX_CUDA(cudaMemcpyAsync(c->h_state + slot, c->d_state.p + slot, sizeof(CgState),
                          cudaMemcpyDeviceToHost, c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  return c->h_state[slot];
}

// Run `body` (a sequence of launches on c->stream) `reps` times as one CUDA
// graph launch per poll; stop when the state in `slot` leaves RUNNING, the
// wall-clock limit is hit, or after `max_launches` graph launches (0: no
// limit).  Returns the final state.
CgState run_batched(hx_ctx* c, int slot, int reps, const std::function<void()>& body,
                    double wall_limit_ms, double t0, bool* timed_out, int max_launches,
                    const std::function<bool(const CgState&)>& keep_going) {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const int64_t before = launch_counter();
  HX_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  try {
    for (int i = 0; i < reps; ++i) body();
  } catch (...) {
    cudaStreamEndCapture(c->stream, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  const int64_t per_graph = launch_counter() - before;
  launch_counter() = before;  // captured, not yet launched
  HX_CUDA(cudaStreamEndCapture(c->stream, &graph));
  cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  HX_CUDA(ie);
  CgState st{};
  *timed_out = false;
  try {
    for (int nl = 1;; ++nl) {
      HX_CUDA(cudaGraphLaunch(exec, c->stream));
      launch_counter() += per_graph;
      st = get_state(c, slot);
      if (st.status != HX_RUNNING) break;
      if (max_launches > 0 && nl >= max_launches) break;
      if (keep_going && !keep_going(st)) break;
      if (wall_limit_ms > 0 && now_ms() - t0 > wall_limit_ms) {
        *timed_out = true;
        break;
      }
    }
  } catch (...) {
    cudaGraphExecDestroy(exec);
    throw;
  }
  HX_CUDA(cudaGraphExecDestroy(exec));
  return st;
}

int auto_batch(const Grid& g, int check_every) {
  if (check_every > 0) return check_every;
  const int64_t n = g.dofs();
  if (n > 4000000) return 16;
  if (n > 400000) return 32;
  return 64;
}

// Jacobi set-up: node masks, diagonal, shift, M^-1 (FP64) into c->d_minv.
// Returns max diagonal over free DOFs.
double jacobi_setup_public(hx_ctx* c, const double* fac, double shift_factor, double* shift_out) {
  const Grid& g = c->g;
  const int64_t nn = g.nodes(), n = g.dofs();
  c->d_nmask.ensure(nn);
  c->d_minv.ensure(n);
  put_state(c, 3, CgState{});
  launch_node_diag<double>(c->stream, fac, c->d_bcfree.p, c->d_nmask.p, c->d_minv.p, g, c->K,
                           c->d_partials.p, c->d_state.p + 3, c->d_scalars.p);
  double maxd = 0;
  HX_CUDA(cudaMemcpyAsync(&c->h_state[3].aux[0], c->d_scalars.p, sizeof(double),
                          cudaMemcpyDeviceToHost, c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  maxd = c->h_state[3].aux[0];
  const double shift = shift_factor * maxd;
  launch_minv<double>(c->stream, c->d_nmask.p, c->d_minv.p, c->d_minv.p, nn, shift);
  *shift_out = shift;
  return maxd;
}

// ---------------------------------------------------------------------------
// Jacobi-PCG on the fused kernels (T = double: the plain FP64 solve; T =
// float: the inner solve of mixed precision).  b must already be masked; x
// holds the initial guess (masked) when warm.  Iteration k reads p_{k-1}
// from P[(k+1)%2] and writes p_k into P[k%2]; the graph body runs two
// iterations so the buffer roles stay fixed.  On exit the pending
// x += alpha p of the last iteration is applied.  Returns the final state.
// ---------------------------------------------------------------------------
template <typename T>
CgState pcg_fused(hx_ctx* c, int slot, const T* fac, const T* b, T* x, bool warm, T shift,
                  const ElemCoef<T>& K, T* r, T* P0, T* P1, T* q, const T* minv, T* xbest,
                  const CgState& init, int check_every, double wall_ms, double t0,
                  bool* timed_out) {
  const Grid& g = c->g;
  const int64_t n = g.dofs();
  CgState* st = c->d_state.p + slot;
  put_state(c, slot, init);
  if (warm) {
    launch_matvec<T>(c->stream, 0, x, q, fac, c->d_nmask.p, g, K, shift, c->d_state.p + 3,
                     c->d_partials.p, nullptr);
    launch_cg_init<T>(c->stream, b, q, minv, r, P1, n, st, c->d_partials.p);
  } else {
    launch_fill_zero(c->stream, x, n * sizeof(T));
    launch_cg_init<T>(c->stream, b, nullptr, minv, r, P1, n, st, c->d_partials.p);
  }
  if (xbest) HX_CUDA(cudaMemcpyAsync(xbest, x, n * sizeof(T), cudaMemcpyDeviceToDevice, c->stream));
  CgState s0 = get_state(c, slot);
  if (s0.status != HX_RUNNING || init.max_iter <= 0) return s0;
  auto body = [&]() {
    launch_pcg_step<T>(c->stream, P1, P0, r, minv, x, q, fac, c->d_nmask.p, g, K, shift, st,
                       c->d_partials.p);
    launch_cg_update2<T>(c->stream, r, q, minv, n, st, c->d_partials.p);
    if (xbest) launch_axpy_state<T>(c->stream, xbest, x, P0, n, st, 1);
    launch_pcg_step<T>(c->stream, P0, P1, r, minv, x, q, fac, c->d_nmask.p, g, K, shift, st,
                       c->d_partials.p);
    launch_cg_update2<T>(c->stream, r, q, minv, n, st, c->d_partials.p);
    if (xbest) launch_axpy_state<T>(c->stream, xbest, x, P1, n, st, 2);
  };
  const int reps = std::max(1, check_every / 2);
  CgState sf = run_batched(c, slot, reps, body, wall_ms, t0, timed_out, 0);
  // apply the pending step x_{k+1} = x_k + alpha_k p_k (not after a breakdown,
  // whose alpha is invalid); p_k sits in P[(iter-1) % 2]
  if (sf.status != HX_ST_BREAKDOWN && sf.iter > 0) {
    T* pk = ((sf.iter - 1) % 2 == 0) ? P0 : P1;
    launch_axpy_state<T>(c->stream, x, x, pk, n, st, 0);
  }
  return sf;
}

template CgState pcg_fused<double>(hx_ctx*, int, const double*, const double*, double*, bool,
                                   double, const ElemCoef<double>&, double*, double*, double*,
                                   double*, const double*, double*, const CgState&, int, double,
                                   double, bool*);
template CgState pcg_fused<float>(hx_ctx*, int, const float*, const float*, float*, bool, float,
                                  const ElemCoef<float>&, float*, float*, float*, float*,
                                  const float*, float*, const CgState&, int, double, double,
                                  bool*);

static CgState pcg_fp64(hx_ctx* c, const double* fac, const double* b, double* x, bool warm,
                        double shift, const hx_solve_opts& o, double t0, bool* timed_out) {
  const int64_t n = c->g.dofs();
  double* r = c->d_r.ensure(n);
  double* P0 = c->d_p.ensure(n);
  double* P1 = c->d_p2.ensure(n);
  double* q = c->d_q.ensure(n);
  double* xbest = o.keep_best ? c->d_xbest.ensure(n) : nullptr;
  const CgState init =
      fresh_state(o.tol, o.max_iter, 1, o.divergence_checks != 0, o.keep_best != 0);
  return pcg_fused<double>(c, 0, fac, b, x, warm, shift, c->K, r, P0, P1, q, c->d_minv.p, xbest,
                           init, auto_batch(c->g, o.check_every), o.wall_limit_ms, t0, timed_out);
}

// FP64 true residual ||b - (K+sI)x|| / ||b||.
static double true_residual(hx_ctx* c, const double* fac, const double* b, const double* x,
                            double shift) {
  const Grid& g = c->g;
  const int64_t n = g.dofs();
  double* q = c->d_q.ensure(n);
  put_state(c, 3, CgState{});
  launch_matvec<double>(c->stream, 0, x, q, fac, c->d_nmask.p, g, c->K, shift, c->d_state.p + 3,
                        c->d_partials.p, nullptr);
  launch_resid_norm(c->stream, b, q, n, c->d_state.p + 3, c->d_partials.p, c->d_scalars.p);
  double v[2];
  HX_CUDA(cudaMemcpyAsync(v, c->d_scalars.p, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                          c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  return v[1] > 0 ? std::sqrt(v[0] / v[1]) : 0.0;
}

// ---------------------------------------------------------------------------
// Mixed precision: FP32 Jacobi-PCG with reliable updates.  The Krylov
// iteration (fused step + residual update) runs in FP32 with FP64 dot
// products; it accumulates its correction in d32.  Whenever the recursive
// FP32 residual has dropped by `delta` (opts.inner_tol) since the last
// replacement, or claims convergence, the host folds d32 into the FP64
// solution, recomputes the true residual b - (K+sI)x in FP64, replaces the
// FP32 residual with it and resumes with the same search direction (no
// restart).  Convergence is judged only on the FP64 true residual.
// ---------------------------------------------------------------------------
CgState solve_mixed(hx_ctx* c, const double* fac, const double* b, double* x, bool warm,
                    double shift, const hx_solve_opts& o, double t0, bool* timed_out,
                    int* inner_total) {
  const Grid& g = c->g;
  const int64_t n = g.dofs(), ne = g.elems();
  float* fac32 = c->d_fac32.ensure(ne);
  float* minv32 = c->d_minv32.ensure(n);
  float* r32 = c->d_r32.ensure(n);
  float* P0 = c->d_p32.ensure(n);
  float* P1 = c->d_p32b.ensure(n);
  float* q32 = c->d_q32.ensure(n);
  float* d32 = c->d_x32.ensure(n);
  double* q = c->d_q.ensure(n);
  launch_convert<float, double>(c->stream, fac32, fac, ne);
  launch_convert<float, double>(c->stream, minv32, c->d_minv.p, n);
  const ElemCoef<float> K32 = to_float(c->K);
  const float sh32 = (float)shift;
  CgState* so = c->d_state.p;      // FP64 outer: ||b||, true residual
  CgState* si = c->d_state.p + 1;  // FP32 Krylov iteration
  *inner_total = 0;
  // ||b||
  CgState s = fresh_state(o.tol, std::numeric_limits<int>::max(), 1, false, false);
  put_state(c, 3, CgState{});
  launch_dot(c->stream, b, b, n, c->d_state.p + 3, c->d_partials.p, c->d_scalars.p);
  double bb = 0;
  HX_CUDA(cudaMemcpyAsync(&bb, c->d_scalars.p, sizeof(double), cudaMemcpyDeviceToHost,
                          c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  s.bnorm = std::sqrt(bb);
  if (s.bnorm == 0.0) {
    launch_fill_zero(c->stream, x, n * sizeof(double));
    s.status = HX_ST_ZERO_RHS;
    s.rel_res = 0;
    return s;
  }
  put_state(c, 0, s);
  if (!warm) launch_fill_zero(c->stream, x, n * sizeof(double));
  // true residual of the initial guess -> r32 = r / ||b||
  if (warm)
    launch_matvec<double>(c->stream, 0, x, q, fac, c->d_nmask.p, g, c->K, shift,
                          c->d_state.p + 3, c->d_partials.p, nullptr);
  else
    launch_fill_zero(c->stream, q, n * sizeof(double));
  launch_ir_residual(c->stream, b, q, r32, n, so, c->d_partials.p);
  CgState so_h = get_state(c, 0);
  if (so_h.status != HX_RUNNING) return so_h;
  // FP32 iteration state: rz from the replaced residual, p_{-1} = z, alpha =
  // beta = 0; bnorm = 1 because r32 is already scaled by 1/||b||
  const double delta = (o.inner_tol > 0 && o.inner_tol < 1) ? o.inner_tol : 0.1;
  CgState init = fresh_state(o.tol, o.max_iter, 1, false, false);
  put_state(c, 1, init);
  launch_fill_zero(c->stream, d32, n * sizeof(float));
  launch_cg_init<float>(c->stream, r32, nullptr, minv32, r32, P1, n, si, c->d_partials.p);
  CgState st = get_state(c, 1);
  st.bnorm = 1.0;
  st.aux[1] = delta;
  st.aux[2] = st.rr;
  st.max_iter = o.max_iter;
  put_state(c, 1, st);
  const int reps = std::max(1, auto_batch(g, o.check_every) / 2);
  int parity = 0;  // which P buffer holds p_{k-1}: P1 when parity == 0
  for (;;) {
    float* Pin = parity ? P0 : P1;
    float* Pout = parity ? P1 : P0;
    auto body = [&]() {
      launch_pcg_step<float>(c->stream, Pin, Pout, r32, minv32, d32, q32, fac32, c->d_nmask.p, g,
                             K32, sh32, si, c->d_partials.p);
      launch_cg_update2<float>(c->stream, r32, q32, minv32, n, si, c->d_partials.p);
      launch_pcg_step<float>(c->stream, Pout, Pin, r32, minv32, d32, q32, fac32, c->d_nmask.p, g,
                             K32, sh32, si, c->d_partials.p);
      launch_cg_update2<float>(c->stream, r32, q32, minv32, n, si, c->d_partials.p);
    };
    const int it_before = st.iter;
    CgState sf = run_batched(c, 1, reps, body, o.wall_limit_ms, t0, timed_out, 0);
    const int done = sf.iter - it_before;
    *inner_total += done;
    // p_k of the last completed iteration: iterations alternate Pin -> Pout
    float* pk = (done % 2 == 1) ? Pout : Pin;
    if (done % 2 == 1) parity ^= 1;
    if (sf.status != HX_ST_BREAKDOWN && done > 0) {
      launch_axpy_state<float>(c->stream, d32, d32, pk, n, si, 0);  // pending step
    }
    // fold the FP32 correction into x and replace the residual in FP64
    launch_ir_correct(c->stream, x, d32, n, so);
    launch_fill_zero(c->stream, d32, n * sizeof(float));
    launch_matvec<double>(c->stream, 0, x, q, fac, c->d_nmask.p, g, c->K, shift,
                          c->d_state.p + 3, c->d_partials.p, nullptr);
    launch_ir_residual(c->stream, b, q, r32, n, so, c->d_partials.p);
    so_h = get_state(c, 0);
    if (so_h.status != HX_RUNNING) {
      so_h.iter = *inner_total;
      return so_h;  // converged on the true residual (or non-finite)
    }
    if (*timed_out || sf.status == HX_ST_BREAKDOWN || sf.status == HX_ST_NONFINITE ||
        sf.status == HX_ST_DIVERGED || *inner_total >= o.max_iter) {
      so_h.status = (sf.status == HX_ST_PAUSED || sf.status == HX_ST_CONVERGED ||
                     sf.status == HX_RUNNING)
                        ? HX_ST_MAXITER
                        : sf.status;
      so_h.iter = *inner_total;
      return so_h;
    }
    // resume: rz from the replaced residual (p, beta kept), alpha = 0 so the
    // next step does not re-apply the step already folded into x
    st = get_state(c, 1);
    launch_cg_init<float>(c->stream, r32, nullptr, minv32, r32, q32, n, si, c->d_partials.p);
    CgState s2 = get_state(c, 1);
    s2.bnorm = 1.0;
    s2.alpha = 0.0;
    s2.beta = st.beta;
    s2.iter = sf.iter;
    s2.aux[1] = delta;
    s2.aux[2] = s2.rr;
    s2.max_iter = o.max_iter;
    s2.status = HX_RUNNING;
    put_state(c, 1, s2);
    st = s2;
  }
}

static hx_status map_status(int st) {
  switch (st) {
    case HX_ST_CONVERGED:
    case HX_ST_ZERO_RHS:
      return HX_OK;
    case HX_ST_BREAKDOWN:
      return HX_BREAKDOWN;
    case HX_ST_NONFINITE:
      return HX_NONFINITE;
    case HX_ST_DIVERGED:
      return HX_DIVERGED;
    default:
      return HX_NOT_CONVERGED;
  }
}

// ---------------------------------------------------------------------------
// Device-level solve in grid numbering.  f, fac, u are FP64 device arrays.
// ---------------------------------------------------------------------------
hx_status solve_grid(hx_ctx* c, const double* f, const double* fac, double* u,
                     const hx_solve_opts& o, hx_solve_report* rep) {
  const double t0 = now_ms();
  HX_REQUIRE(c->has_mesh, "no mesh: call hx_set_grid or hx_set_mesh first");
  HX_REQUIRE(o.tol > 0, "tol must be > 0");
  HX_REQUIRE(o.preconditioner == HX_PC_JACOBI || o.preconditioner == HX_PC_LEARNED ||
                 o.preconditioner == HX_PC_MULTIGRID,
             "unknown preconditioner");
  HX_REQUIRE(o.preconditioner != HX_PC_LEARNED || o.precision == HX_PREC_FP64 ||
                 o.precision == HX_PREC_MIXED32,
             "the learned preconditioner runs with FP64 or FP32 (mixed) vectors");
  ensure_workspace(c);
  if (c->bc_dirty) upload_bc(c);
  const Grid& g = c->g;
  const int64_t n = g.dofs();
  double* b = c->d_b.ensure(n);
  hx_solve_report R{};
  c->gmg.setup_ms = 0;
  const int attempts = o.ref_retry ? 3 : 1;
  double factor = o.shift_factor;
  double maxd = 0, shift = 0;
  bool success = false;
  bool have_global_best = false;
  double global_lowest = INFINITY;
  double* gbest = nullptr;
  CgState last{};
  bool timed_out = false;
  int total_iters = 0;
  double t_setup = 0;
  // the reference's Jacobi -> AMG switch (GPUSolver.jl:540-579), with the
  // multigrid preconditioner in place of the CPU AMG
  bool use_mg = o.preconditioner == HX_PC_MULTIGRID;
  bool can_switch = o.ref_retry && o.multigrid_fallback && o.preconditioner == HX_PC_JACOBI;
  for (int attempt = 1; attempt <= attempts; ++attempt) {
    const double ts = now_ms();
    if (attempt == 1) {
      maxd = jacobi_setup_public(c, fac, factor, &shift);
      launch_mask_rhs<double>(c->stream, f, c->d_minv.p, b, n);
    } else {
      shift = factor * maxd;
      launch_node_diag<double>(c->stream, fac, c->d_bcfree.p, c->d_nmask.p, c->d_minv.p, g, c->K,
                               c->d_partials.p, c->d_state.p + 3, c->d_scalars.p);
      launch_minv<double>(c->stream, c->d_nmask.p, c->d_minv.p, c->d_minv.p, g.nodes(), shift);
    }
    const bool warm = o.warm_start && attempt == 1;
    if (warm) launch_mask_rhs<double>(c->stream, u, c->d_minv.p, u, n);  // zero fixed DOFs
    HX_CUDA(cudaStreamSynchronize(c->stream));
    t_setup += now_ms() - ts;
    CgState st{};
    if (o.preconditioner == HX_PC_LEARNED) {
      int fb = 0, its = 0;
      if (o.precision == HX_PREC_FP64) {
        st = solve_learned(c, fac, b, u, warm, shift, o, t0, &timed_out, &fb, &its);
      } else {
        st = solve_learned_mixed(c, fac, b, u, warm, shift, o, t0, &timed_out, &fb, &its);
        R.refinements = c->h_state[0].iter;
      }
      total_iters += its;
      R.fallback_used = fb;
    } else if (use_mg) {
      int its = 0;
      if (o.precision == HX_PREC_FP64) {
        st = solve_gmg(c, fac, b, u, warm, shift, o, t0, &timed_out, &its);
        if (o.preconditioner != HX_PC_MULTIGRID) R.fallback_used = 1;
      } else {
        int fb = 0;
        st = solve_gmg_mixed(c, fac, b, u, warm, shift, o, t0, &timed_out, &fb, &its);
        R.refinements = c->h_state[0].iter;
        R.fallback_used = fb || o.preconditioner != HX_PC_MULTIGRID;
      }
      total_iters += its;
    } else if (o.precision == HX_PREC_FP64) {
      st = pcg_fp64(c, fac, b, u, warm, shift, o, t0, &timed_out);
      total_iters += st.iter;
    } else {
      int inner = 0;
      st = solve_mixed(c, fac, b, u, warm, shift, o, t0, &timed_out, &inner);
      total_iters += inner;
      R.refinements = c->h_state[0].iter;
    }
    // The FP64 forms stop on the recursive residual, which over thousands of
    // iterations can drift below the true one.  Outside the reference's
    // retry semantics (which stop on the recursive residual, as
    // GPUSolver.jl:508 does), convergence is confirmed on the FP64 true
    // residual: while it is still above tol, the same method restarts from
    // the current iterate (at most twice, within max_iter).  The mixed forms
    // already judge convergence on the true residual.
    for (int restart = 0; restart < 2 && !o.ref_retry && o.precision == HX_PREC_FP64 &&
                          st.status == HX_ST_CONVERGED && !timed_out;
         ++restart) {
      if (true_residual(c, fac, b, u, shift) < o.tol) break;
      hx_solve_opts oc = o;
      oc.max_iter = o.max_iter - total_iters;
      if (oc.max_iter <= 0) {
        st.status = HX_ST_MAXITER;
        break;
      }
      if (o.preconditioner == HX_PC_LEARNED) {
        int fb = 0, its = 0;
        st = solve_learned(c, fac, b, u, true, shift, oc, t0, &timed_out, &fb, &its);
        total_iters += its;
        R.fallback_used |= fb;
      } else if (use_mg) {
        int its = 0;
        st = solve_gmg(c, fac, b, u, true, shift, oc, t0, &timed_out, &its);
        total_iters += its;
      } else {
        st = pcg_fp64(c, fac, b, u, true, shift, oc, t0, &timed_out);
        total_iters += st.iter;
      }
      R.refinements += 1;
    }
    last = st;
    R.attempts = attempt;
    if (st.status == HX_ST_CONVERGED || st.status == HX_ST_ZERO_RHS) {
      success = true;
      break;
    }
    if (!o.ref_retry || timed_out) break;
    // Failure handling of src/Solvers/GPUSolver.jl:536-593; its switch to
    // the host AMG goes to the multigrid preconditioner here.
    const bool diverged = st.status == HX_ST_BREAKDOWN || st.status == HX_ST_NONFINITE ||
                          st.status == HX_ST_DIVERGED;
    const bool failed_badly = diverged || st.best_rel > 0.1;
    // with a stronger preconditioner to switch to, stagnation is not accepted
    if (!failed_badly && !can_switch && st.best_rel < 5e-2) {
      if (o.keep_best)
        HX_CUDA(cudaMemcpyAsync(u, c->d_xbest.p, n * sizeof(double), cudaMemcpyDeviceToDevice,
                                c->stream));
      success = true;
      last.status = HX_ST_CONVERGED;
      R.status = HX_STALLED;
      break;
    }
    if (failed_badly || (can_switch && st.best_rel > o.tol)) {
      if (can_switch) {
        use_mg = true;  // the next attempt runs multigrid-preconditioned
        can_switch = false;
      } else if (use_mg && o.preconditioner != HX_PC_MULTIGRID) {
        use_mg = false;  // multigrid failed too: back to Jacobi, no more switching
      }
      factor *= 10.0;
    } else {
      if (st.best_rel < global_lowest && o.keep_best) {
        global_lowest = st.best_rel;
        gbest = c->d_aux5.ensure(n);
        HX_CUDA(cudaMemcpyAsync(gbest, c->d_xbest.p, n * sizeof(double),
                                cudaMemcpyDeviceToDevice, c->stream));
        have_global_best = true;
      }
      factor *= 5.0;
    }
  }
  if (!success && o.ref_retry) {
    if (have_global_best)
      HX_CUDA(cudaMemcpyAsync(u, gbest, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    else
      launch_fill_zero(c->stream, u, n * sizeof(double));
  }
  R.iterations = total_iters;
  R.zero_rhs = last.status == HX_ST_ZERO_RHS;
  R.rel_res = last.rel_res;
  R.shift = shift;
  if (o.verify_true_residual) {
    R.true_rel_res = (last.status == HX_ST_ZERO_RHS) ? 0.0 : true_residual(c, fac, b, u, shift);
  } else {
    R.true_rel_res = NAN;
  }
  HX_CUDA(cudaStreamSynchronize(c->stream));
  if (R.status == 0) R.status = timed_out ? HX_NOT_CONVERGED : map_status(last.status);
  R.time_setup_ms = t_setup;
  R.time_total_ms = now_ms() - t0;
  R.time_solve_ms = R.time_total_ms - t_setup;
  R.time_precond_setup_ms = c->gmg.setup_ms;
  if (rep) *rep = R;
  return (hx_status)R.status;
}

// ---------------------------------------------------------------------------
// Helmholtz filter in grid numbering (FP64 device arrays).
// ---------------------------------------------------------------------------
hx_status filter_grid(hx_ctx* c, const Grid& g, const double h[3], const double* rho, double* out,
                      double radius, int ref_compat, double tol, int max_iter,
                      hx_solve_report* rep) {
  const double t0 = now_ms();
  HX_REQUIRE(g.nxe > 0 && g.nye > 0 && g.nze > 0, "filter grid is empty");
  HX_REQUIRE(radius >= 0, "radius must be >= 0");
  HX_REQUIRE(max_iter >= 1, "max_iter must be >= 1");
  ensure_workspace(c);
  const size_t nbf = 4ull * cdiv(g.nxn, 32) * cdiv(g.nyn, 8) * cdiv(g.nzn, 4);
  c->d_partials.ensure(std::max<size_t>(c->d_partials.n, nbf));
  const int64_t nn = g.nodes();
  const FilterCoef F = make_filter_coef(h[0], h[1], h[2], radius, ref_compat);
  double* invd = c->f_invd.ensure(nn);
  double* x = c->f_x.ensure(nn);
  double* r = c->f_r.ensure(nn);
  double* p = c->f_p.ensure(nn);
  double* q = c->f_q.ensure(nn);
  double* b = c->f_b.ensure(nn);
  const bool same_grid = c->fg.nxe == g.nxe && c->fg.nye == g.nye && c->fg.nze == g.nze &&
                         c->fh[0] == h[0] && c->fh[1] == h[1] && c->fh[2] == h[2];
  if (!c->filt_ready || !same_grid || std::fabs(c->filt_radius - radius) > 1e-12 ||
      c->filt_compat != ref_compat) {
    c->fg = g;
    for (int a = 0; a < 3; ++a) c->fh[a] = h[a];
    launch_filter_invdiag(c->stream, invd, g, F);
    c->filt_ready = true;
    c->filt_radius = radius;
    c->filt_compat = ref_compat;
  }
  c->f_used = true;
  c->f_radius_last = radius;
  c->f_compat_last = ref_compat;
  launch_filter_rhs(c->stream, rho, b, g, F.vol8);
  launch_fill_zero(c->stream, x, nn * sizeof(double));
  CgState* st = c->d_state.p + 2;
  put_state(c, 2, fresh_state(tol, max_iter, 10, false, false));
  launch_cg_init<double>(c->stream, b, nullptr, invd, r, p, nn, st, c->d_partials.p);
  CgState s0 = get_state(c, 2);
  hx_solve_report R{};
  if (s0.status == HX_ST_ZERO_RHS) {
    // zero RHS: the reference returns the input unchanged (GPUHelmholtz.jl:179-182)
    HX_CUDA(cudaMemcpyAsync(out, rho, g.elems() * sizeof(double), cudaMemcpyDeviceToDevice,
                            c->stream));
    HX_CUDA(cudaStreamSynchronize(c->stream));
    R.status = HX_OK;
    R.time_total_ms = now_ms() - t0;
    if (rep) *rep = R;
    return HX_OK;
  }
  auto body = [&]() {
    launch_filter_matvec(c->stream, p, q, g, F, st, c->d_partials.p);
    launch_cg_update<double>(c->stream, x, p, r, q, invd, nn, st, c->d_partials.p);
    launch_cg_pupdate<double>(c->stream, p, r, invd, nn, st);
  };
  bool to = false;
  CgState sf = run_batched(c, 2, 10, body, 0.0, t0, &to, 0);
  launch_filter_extract(c->stream, x, out, g);
  HX_CUDA(cudaStreamSynchronize(c->stream));
  R.iterations = sf.iter;
  R.rel_res = sf.rel_res;
  // Reaching max_iter is the reference's normal exit too (it returns its
  // result regardless); report it but do not fail.
  R.status = (sf.status == HX_ST_CONVERGED || sf.status == HX_ST_MAXITER)
                 ? HX_OK
                 : map_status(sf.status);
  R.true_rel_res = NAN;
  R.time_total_ms = now_ms() - t0;
  R.time_solve_ms = R.time_total_ms;
  if (rep) *rep = R;
  return (hx_status)R.status;
}

hx_status time_kernel(hx_ctx* c, int kernel, int reps, double* avg_ms) {
  HX_REQUIRE(c->has_mesh, "no mesh");
  HX_REQUIRE(reps >= 1, "reps must be >= 1");
  HX_REQUIRE(avg_ms != nullptr, "avg_ms is null");
  ensure_workspace(c);
  const Grid& g = c->g;
  const int64_t n = g.dofs(), ne = g.elems();
  auto ready = [&](size_t have, size_t need) { return have >= need && need > 0; };
  CgState ts = fresh_state(0.0, 0x7fffffff, 1, false, false);
  ts.rz = 1.0;
  ts.bnorm = 1.0;
  ts.alpha = 0.0;  // the update kernels then leave x, r unchanged
  ts.beta = 0.0;
  put_state(c, 3, ts);
  CgState* st = c->d_state.p + 3;
  cudaEvent_t e0, e1;
  HX_CUDA(cudaEventCreate(&e0));
  HX_CUDA(cudaEventCreate(&e1));
  std::function<void()> body;
  if (kernel == HX_KERNEL_PCG_STEP_FP64 || kernel == HX_KERNEL_PCG_UPDATE_FP64 ||
      kernel == HX_KERNEL_APPLY_FP64) {
    HX_REQUIRE(ready(c->d_p.n, n) && ready(c->d_p2.n, n) && ready(c->d_q.n, n) &&
                   ready(c->d_r.n, n) && ready(c->d_minv.n, n) && ready(c->d_fac.n, ne) &&
                   ready(c->d_nmask.n, g.nodes()),
               "run a solve before timing its kernels");
    double* xs = c->d_aux0.ensure(n);
    HX_CUDA(cudaMemsetAsync(xs, 0, n * sizeof(double), c->stream));
    if (kernel == HX_KERNEL_PCG_STEP_FP64)
      body = [&] {
        launch_pcg_step<double>(c->stream, c->d_p.p, c->d_p2.p, c->d_r.p, c->d_minv.p, xs,
                                c->d_q.p, c->d_fac.p, c->d_nmask.p, g, c->K, 0.0, st,
                                c->d_partials.p);
      };
    else if (kernel == HX_KERNEL_PCG_UPDATE_FP64)
      body = [&] {
        launch_cg_update2<double>(c->stream, c->d_r.p, c->d_q.p, c->d_minv.p, n, st,
                                  c->d_partials.p);
      };
    else
      body = [&] {
        launch_matvec<double>(c->stream, 0, c->d_p.p, c->d_q.p, c->d_fac.p, c->d_nmask.p, g, c->K,
                              0.0, st, c->d_partials.p, nullptr);
      };
  } else if (kernel == HX_KERNEL_PCG_STEP_FP32 || kernel == HX_KERNEL_FCG_STEP_FP32) {
    HX_REQUIRE(ready(c->d_fac.n, ne) && ready(c->d_nmask.n, g.nodes()) && ready(c->d_minv.n, n) &&
                   (ready(c->d_r.n, n) || ready(c->d_b.n, n)),
               "run a solve first");
    float* f32 = c->d_fac32.ensure(ne);
    float* p32 = c->d_p32.ensure(n);
    float* p32b = c->d_p32b.ensure(n);
    float* q32 = c->d_q32.ensure(n);
    float* r32 = c->d_r32.ensure(n);
    float* m32 = c->d_minv32.ensure(n);
    float* x32 = c->d_x32.ensure(n);
    launch_convert<float, double>(c->stream, f32, c->d_fac.p, ne);
    launch_convert<float, double>(c->stream, m32, c->d_minv.p, n);
    HX_CUDA(cudaMemsetAsync(p32, 0, n * sizeof(float), c->stream));
    // the last residual, or the right-hand side after a solve that kept none
    launch_convert<float, double>(c->stream, r32, ready(c->d_r.n, n) ? c->d_r.p : c->d_b.p, n);
    HX_CUDA(cudaMemsetAsync(x32, 0, n * sizeof(float), c->stream));
    const ElemCoef<float> K32 = to_float(c->K);
    if (kernel == HX_KERNEL_PCG_STEP_FP32) {
      body = [&, f32, p32, p32b, q32, r32, m32, x32, K32] {
        launch_pcg_step<float>(c->stream, p32, p32b, r32, m32, x32, q32, f32, c->d_nmask.p, g,
                               K32, 0.0f, st, c->d_partials.p);
      };
    } else {
      // the flexible-CG step with z = the converted residual: beta = 0 gives
      // p = z != 0, so p.q > 0 and the state stays running; alpha_old = 0
      // leaves x unchanged; z.r (aux[3]) only scales the new alpha
      ts.aux[3] = 1.0;
      put_state(c, 3, ts);
      body = [&, f32, p32, p32b, q32, r32, x32, K32] {
        launch_fcg_step<float>(c->stream, p32, p32b, r32, x32, q32, f32, c->d_nmask.p, g, K32,
                               0.0f, st, c->d_partials.p);
      };
    }
  } else if (kernel == HX_KERNEL_FILTER_MATVEC) {
    HX_REQUIRE(c->f_used, "run a filter before timing its kernel");
    const FilterCoef F = make_filter_coef(c->fh[0], c->fh[1], c->fh[2], c->f_radius_last,
                                          c->f_compat_last);
    const Grid fg = c->fg;
    body = [&, F, fg] { launch_filter_matvec(c->stream, c->f_p.p, c->f_q.p, fg, F, st, c->d_partials.p); };
  } else if (kernel == HX_KERNEL_CONV3 || kernel == HX_KERNEL_NET_APPLY) {
    body = net_time_body(c, kernel == HX_KERNEL_CONV3 ? 0 : 1);
  } else {
    throw Error{HX_BAD_ARG, "unknown kernel id"};
  }
  body();  // warm-up
  HX_CUDA(cudaEventRecord(e0, c->stream));
  for (int i = 0; i < reps; ++i) body();
  HX_CUDA(cudaEventRecord(e1, c->stream));
  HX_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  HX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *avg_ms = ms / reps;
  return HX_OK;
}

}  // namespace hx
