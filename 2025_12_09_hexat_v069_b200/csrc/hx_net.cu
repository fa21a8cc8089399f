// hx_net.cu -- the convolutional preconditioner network on the host side:
// parameters, training (forward, backward, Adam, all on the GPU), PCG
// snapshots for training data, and the flexible-CG solve that applies it.
//
// Network: 4 conv3d layers (3x3x3) on the node grid, 4 -> 16 -> 16 -> 16 -> 3
// channels, ReLU after the first three; input = the Jacobi-scaled residual
// D^-1/2 r (normalised by its RMS s) and a density feature; output NN(r~).
// The preconditioner is z = D^-1 r + s D^-1/2 NN(r~): Jacobi plus a learned
// correction, so an untrained (zero) last layer reproduces Jacobi.  It is
// trained on residual/error pairs (r = b - A x_k, e = u* - x_k) taken from
// Jacobi-PCG iterates, to make z approximate e.  Applied inside flexible CG
// (Notay's FCG with one stored direction); convergence is always judged on
// the residual, and the solve falls back to Jacobi-PCG from the current
// iterate when FCG breaks down or stalls.
#include <cmath>
#include <cstring>
#include <vector>

#include "hx_cnn.h"
#include "hx_solver.h"

namespace hx {

namespace {

constexpr int LP = NET_LAYER_PARAMS;

GridN node_grid(const Grid& g) { return GridN{g.nxn, g.nyn, g.nzn}; }

bool live_param(int layer, int k) {
  const int in_real = (layer == 0) ? 4 : 16;
  const int out_real = (layer == NET_LAYERS - 1) ? 3 : 16;
  if (k >= 27 * 256) return (k - 27 * 256) < out_real;  // bias
  const int co = (k / 16) % 16, ci = k % 16;
  return co < out_real && ci < in_real;
}

void net_alloc_params(hx_ctx* c) {
  auto& N = c->net;
  N.w.ensure(NET_PARAMS);
  N.m.ensure(NET_PARAMS);
  N.v.ensure(NET_PARAMS);
  N.grad.ensure(NET_PARAMS);
  N.live.ensure(NET_PARAMS);
  N.wf.ensure(NET_LAYERS * 27 * 256);
  N.wb.ensure(NET_LAYERS * 27 * 256);
  N.scal.ensure(8);
}

void net_pack(hx_ctx* c) {
  auto& N = c->net;
  for (int l = 0; l < NET_LAYERS; ++l)
    launch_pack_weights(c->stream, N.w.p + l * LP, N.wf.p + l * 27 * 256, N.wb.p + l * 27 * 256);
}

void net_upload(hx_ctx* c, const std::vector<float>& w) {
  auto& N = c->net;
  net_alloc_params(c);
  std::vector<unsigned char> live(NET_PARAMS);
  for (int l = 0; l < NET_LAYERS; ++l)
    for (int k = 0; k < LP; ++k) live[l * LP + k] = live_param(l, k) ? 1 : 0;
  HX_CUDA(cudaMemcpyAsync(N.w.p, w.data(), NET_PARAMS * sizeof(float), cudaMemcpyHostToDevice,
                          c->stream));
  HX_CUDA(cudaMemcpyAsync(N.live.p, live.data(), NET_PARAMS, cudaMemcpyHostToDevice, c->stream));
  HX_CUDA(cudaMemsetAsync(N.m.p, 0, NET_PARAMS * sizeof(float), c->stream));
  HX_CUDA(cudaMemsetAsync(N.v.p, 0, NET_PARAMS * sizeof(float), c->stream));
  net_pack(c);
  HX_CUDA(cudaStreamSynchronize(c->stream));
  N.step = 0;
  N.ready = true;
}

void net_buffers(hx_ctx* c, int64_t nn, size_t tiles, bool train) {
  auto& N = c->net;
  const size_t a = (size_t)nn * 16;
  N.x0.ensure(a);
  N.a1.ensure(a);
  N.a2.ensure(a);
  N.a3.ensure(a);
  N.y.ensure(a);
  if (train) {
    N.da.ensure(a);
    N.db.ensure(a);
    N.part.ensure(tiles * LP);
  }
}

// forward through the 4 layers; the last layer writes `cout_last` channels
void net_forward(hx_ctx* c, const GridN& g, int cout_last) {
  auto& N = c->net;
  const __nv_bfloat16* W = N.wf.p;
  const float* w = N.w.p;
  launch_conv3(c->stream, 16, 0, N.x0.p, N.a1.p, W + 0 * 6912, w + 0 * LP + 6912, nullptr, g);
  launch_conv3(c->stream, 16, 0, N.a1.p, N.a2.p, W + 1 * 6912, w + 1 * LP + 6912, nullptr, g);
  launch_conv3(c->stream, 16, 0, N.a2.p, N.a3.p, W + 2 * 6912, w + 2 * LP + 6912, nullptr, g);
  launch_conv3(c->stream, cout_last, 1, N.a3.p, N.y.p, W + 3 * 6912, w + 3 * LP + 6912, nullptr,
               g);
}

// backward from da = dLoss/dY (16 channels): parameter gradients into N.grad
void net_backward(hx_ctx* c, const GridN& g) {
  auto& N = c->net;
  const __nv_bfloat16* Wb = N.wb.p;
  launch_conv3_wgrad(c->stream, N.a3.p, N.da.p, N.part.p, N.grad.p + 3 * LP, g);
  launch_conv3(c->stream, 16, 2, N.da.p, N.db.p, Wb + 3 * 6912, nullptr, N.a3.p, g);
  launch_conv3_wgrad(c->stream, N.a2.p, N.db.p, N.part.p, N.grad.p + 2 * LP, g);
  launch_conv3(c->stream, 16, 2, N.db.p, N.da.p, Wb + 2 * 6912, nullptr, N.a2.p, g);
  launch_conv3_wgrad(c->stream, N.a1.p, N.da.p, N.part.p, N.grad.p + 1 * LP, g);
  launch_conv3(c->stream, 16, 2, N.da.p, N.db.p, Wb + 1 * 6912, nullptr, N.a1.p, g);
  launch_conv3_wgrad(c->stream, N.x0.p, N.db.p, N.part.p, N.grad.p + 0 * LP, g);
}

// Jacobi scaling and density feature of the current operator (after a solve
// set up M^-1 for `fac`).
void net_operator_inputs(hx_ctx* c, const double* fac) {
  auto& N = c->net;
  const int64_t n = c->g.dofs();
  HX_REQUIRE(c->d_minv.n >= (size_t)n, "no Jacobi data: run a solve on this grid first");
  N.dinvs.ensure(n);
  N.feat.ensure(c->g.nodes());
  launch_sqrt(c->stream, c->d_minv.p, N.dinvs.p, n);
  launch_rho_feature(c->stream, fac, N.feat.p, c->g);
}

}  // namespace

// ---------------------------------------------------------------------------
// parameters
// ---------------------------------------------------------------------------
void net_init(hx_ctx* c, uint64_t seed) {
  std::vector<float> w(NET_PARAMS, 0.f);
  uint64_t s = seed ? seed : 0x2545F4914F6CDD1DULL;
  auto uni = [&]() {  // splitmix64 -> (0, 1)
    s += 0x9E3779B97F4A7C15ULL;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return ((z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  };
  for (int l = 0; l < NET_LAYERS; ++l) {
    const int in_real = (l == 0) ? 4 : 16;
    double std = std::sqrt(2.0 / (27.0 * in_real));
    if (l == NET_LAYERS - 1) std *= 0.1;  // start close to plain Jacobi
    for (int k = 0; k < 27 * 256; ++k) {
      const double g = std::sqrt(-2.0 * std::log(uni())) * std::cos(6.283185307179586 * uni());
      if (live_param(l, k)) w[l * LP + k] = (float)(g * std);
    }
  }
  net_upload(c, w);
}

void net_set_params(hx_ctx* c, const float* params) {
  std::vector<float> w(params, params + NET_PARAMS);
  for (int l = 0; l < NET_LAYERS; ++l)
    for (int k = 0; k < LP; ++k)
      if (!live_param(l, k)) w[l * LP + k] = 0.f;
  net_upload(c, w);
}

void net_get_params(hx_ctx* c, float* params) {
  HX_REQUIRE(c->net.ready, "network not initialised");
  HX_CUDA(cudaMemcpyAsync(params, c->net.w.p, NET_PARAMS * sizeof(float), cudaMemcpyDeviceToHost,
                          c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
}

// Forward + backward on a given node grid from host data (FP32 arrays
// [node][16]); for gradient checks.  Inputs are rounded to BF16.
void net_forward_backward(hx_ctx* c, int nx, int ny, int nz, const float* x0, const float* dy,
                          float* y, float* grads) {
  HX_REQUIRE(c->net.ready, "network not initialised");
  HX_REQUIRE(nx >= 1 && ny >= 1 && nz >= 1, "bad grid");
  const GridN g{nx, ny, nz};
  const int64_t nn = (int64_t)nx * ny * nz;
  net_buffers(c, nn, conv_num_tiles(g), true);
  auto& N = c->net;
  std::vector<__nv_bfloat16> h((size_t)nn * 16);
  for (size_t i = 0; i < h.size(); ++i) h[i] = __float2bfloat16_rn(x0[i]);
  HX_CUDA(cudaMemcpyAsync(N.x0.p, h.data(), h.size() * 2, cudaMemcpyHostToDevice, c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  net_forward(c, g, 16);
  std::vector<__nv_bfloat16> hy((size_t)nn * 16);
  HX_CUDA(cudaMemcpyAsync(hy.data(), N.y.p, hy.size() * 2, cudaMemcpyDeviceToHost, c->stream));
  for (size_t i = 0; i < h.size(); ++i) h[i] = __float2bfloat16_rn(dy[i]);
  HX_CUDA(cudaMemcpyAsync(N.da.p, h.data(), h.size() * 2, cudaMemcpyHostToDevice, c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  net_backward(c, g);
  HX_CUDA(cudaMemcpyAsync(grads, N.grad.p, NET_PARAMS * sizeof(float), cudaMemcpyDeviceToHost,
                          c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  for (size_t i = 0; i < hy.size(); ++i) y[i] = __bfloat162float(hy[i]);
}

// One Adam step on a residual/error pair of the current operator (grid,
// factors of the last solve).  r, e: FP64 device vectors (grid numbering).
double net_train_step(hx_ctx* c, const double* r, const double* e, double lr) {
  HX_REQUIRE(c->net.ready, "network not initialised");
  auto& N = c->net;
  const Grid& g = c->g;
  const int64_t n = g.dofs(), nn = g.nodes();
  const GridN gn = node_grid(g);
  HX_REQUIRE(N.dinvs.n >= (size_t)n && N.feat.n >= (size_t)nn,
             "no operator inputs: call hx_net_prepare after a solve");
  net_buffers(c, nn, conv_num_tiles(gn), true);
  ensure_workspace(c);
  // rz = r.M^-1 r for the input scaling (state slot 3)
  double* zscr = c->d_aux1.ensure(n);
  double* pscr = c->d_aux2.ensure(n);
  HX_CUDA(cudaMemsetAsync(c->d_state.p + 3, 0, sizeof(CgState), c->stream));
  launch_cg_init<double>(c->stream, r, nullptr, c->d_minv.p, zscr, pscr, n, c->d_state.p + 3,
                         c->d_partials.p);
  const double scale_mul = 1.0 / (double)n;
  launch_net_input(c->stream, r, N.dinvs.p, N.feat.p, c->d_state.p + 3, scale_mul, N.x0.p, nn);
  net_forward(c, gn, 16);
  launch_net_loss(c->stream, r, e, N.dinvs.p, N.y.p, c->d_state.p + 3, scale_mul, 1.0 / (double)n,
                  N.da.p, c->d_partials.p, c->d_state.p + 2, N.scal.p, nn);
  net_backward(c, gn);
  N.step += 1;
  launch_adam(c->stream, N.w.p, N.m.p, N.v.p, N.grad.p, N.live.p, NET_PARAMS, (float)lr, N.step);
  net_pack(c);
  double loss = 0;
  HX_CUDA(cudaMemcpyAsync(&loss, N.scal.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  return loss;
}

void net_prepare(hx_ctx* c, const double* fac) { net_operator_inputs(c, fac); }

// ---------------------------------------------------------------------------
// Flexible CG with the network preconditioner (FP64 vectors and operator,
// BF16 network).  Falls back to Jacobi-PCG from the current iterate when
// FCG breaks down, diverges, or stalls (best residual not halved over
// `stall_window` iterations).
// ---------------------------------------------------------------------------
CgState solve_learned(hx_ctx* c, const double* fac, const double* b, double* x, bool warm,
                      double shift, const hx_solve_opts& o, double t0, bool* timed_out,
                      int* fallback, int* iters_out) {
  HX_REQUIRE(c->net.ready, "learned preconditioner requested but no network is loaded");
  auto& N = c->net;
  const Grid& g = c->g;
  const int64_t n = g.dofs(), nn = g.nodes();
  const GridN gn = node_grid(g);
  net_operator_inputs(c, fac);
  net_buffers(c, nn, 0, false);
  double* r = c->d_r.ensure(n);
  double* P0 = c->d_p.ensure(n);
  double* P1 = c->d_p2.ensure(n);
  double* q = c->d_q.ensure(n);
  double* z = N.z.ensure(n);
  const double* minv = c->d_minv.p;
  CgState* st = c->d_state.p;
  const double scale_mul = 1.0 / (double)n;
  CgState init = fresh_state(o.tol, o.max_iter, 1, o.divergence_checks != 0, false);
  put_state(c, 0, init);
  if (warm) {
    launch_matvec<double>(c->stream, 0, x, q, fac, c->d_nmask.p, g, c->K, shift, c->d_state.p + 3,
                          c->d_partials.p, nullptr);
    launch_cg_init<double>(c->stream, b, q, minv, r, P1, n, st, c->d_partials.p);
  } else {
    launch_fill_zero(c->stream, x, n * sizeof(double));
    launch_cg_init<double>(c->stream, b, nullptr, minv, r, P1, n, st, c->d_partials.p);
  }
  launch_fill_zero(c->stream, q, n * sizeof(double));
  CgState s0 = get_state(c, 0);
  *fallback = 0;
  *iters_out = 0;
  if (s0.status != HX_RUNNING || o.max_iter <= 0) return s0;
  auto one = [&](double* pin, double* pout) {
    launch_net_input(c->stream, r, N.dinvs.p, N.feat.p, st, scale_mul, N.x0.p, nn);
    net_forward(c, gn, 8);
    launch_net_output(c->stream, r, minv, N.dinvs.p, N.y.p, 8, st, scale_mul, z, q,
                      c->d_partials.p, nn);
    launch_fcg_step<double>(c->stream, pin, pout, z, r, x, q, fac, c->d_nmask.p, g, c->K, shift,
                            st, c->d_partials.p);
    launch_cg_update2<double>(c->stream, r, q, minv, n, st, c->d_partials.p);
  };
  auto body = [&]() {
    one(P1, P0);
    one(P0, P1);
  };
  const int reps = std::max(1, auto_batch(g, o.check_every) / 2);
  const int stall_window = 200;
  double best = s0.rel_res;
  int best_it = 0;
  CgState sf{};
  bool stalled = false;
  // run in batches, checking the stall criterion between them
  for (;;) {
    sf = run_batched(c, 0, reps, body, o.wall_limit_ms, t0, timed_out, 1);
    if (sf.rel_res < 0.5 * best) {
      best = sf.rel_res;
      best_it = sf.iter;
    }
    if (sf.status != HX_RUNNING || *timed_out) break;
    if (sf.iter - best_it > stall_window) {
      stalled = true;
      break;
    }
  }
  // pending x += alpha p of the last completed iteration
  if (sf.status != HX_ST_BREAKDOWN && sf.iter > 0) {
    double* pk = ((sf.iter - 1) % 2 == 0) ? P0 : P1;
    launch_axpy_state<double>(c->stream, x, x, pk, n, st, 0);
  }
  *iters_out = sf.iter;
  const bool failed = stalled || sf.status == HX_ST_BREAKDOWN || sf.status == HX_ST_DIVERGED ||
                      sf.status == HX_ST_NONFINITE;
  if (!failed || *timed_out) return sf;
  // fallback: Jacobi-PCG warm-started from the current iterate
  *fallback = 1;
  hx_solve_opts oj = o;
  oj.max_iter = std::max(1, o.max_iter - sf.iter);
  oj.keep_best = 0;
  CgState sj = pcg_fused<double>(c, 0, fac, b, x, true, shift, c->K, r, P0, P1, q, minv, nullptr,
                                 fresh_state(o.tol, oj.max_iter, 1, o.divergence_checks != 0,
                                             false),
                                 auto_batch(g, o.check_every), o.wall_limit_ms, t0, timed_out);
  *iters_out += sj.iter;
  return sj;
}

// FP64 Jacobi-PCG from zero, storing x every `every` iterations (at most
// `count` snapshots, n doubles each) until convergence.  Returns the number
// of snapshots taken.
int pcg_snapshots(hx_ctx* c, const double* f, const double* fac, int every, int count,
                  double tol, double* snaps) {
  HX_REQUIRE(every >= 2 && every % 2 == 0, "snapshot period must be even and >= 2");
  const Grid& g = c->g;
  const int64_t n = g.dofs();
  ensure_workspace(c);
  if (c->bc_dirty) upload_bc(c);
  double shift = 0;
  jacobi_setup_public(c, fac, 0.0, &shift);
  double* b = c->d_b.ensure(n);
  launch_mask_rhs<double>(c->stream, f, c->d_minv.p, b, n);
  double* x = c->d_x.ensure(n);
  double* r = c->d_r.ensure(n);
  double* P0 = c->d_p.ensure(n);
  double* P1 = c->d_p2.ensure(n);
  double* q = c->d_q.ensure(n);
  CgState* st = c->d_state.p;
  put_state(c, 0, fresh_state(tol, 0x7fffffff, 1, false, false));
  launch_fill_zero(c->stream, x, n * sizeof(double));
  launch_cg_init<double>(c->stream, b, nullptr, c->d_minv.p, r, P1, n, st, c->d_partials.p);
  int taken = 0;
  auto body = [&]() {
    launch_pcg_step<double>(c->stream, P1, P0, r, c->d_minv.p, x, q, fac, c->d_nmask.p, g, c->K,
                            0.0, st, c->d_partials.p);
    launch_cg_update2<double>(c->stream, r, q, c->d_minv.p, n, st, c->d_partials.p);
    launch_pcg_step<double>(c->stream, P0, P1, r, c->d_minv.p, x, q, fac, c->d_nmask.p, g, c->K,
                            0.0, st, c->d_partials.p);
    launch_cg_update2<double>(c->stream, r, q, c->d_minv.p, n, st, c->d_partials.p);
  };
  bool to = false;
  while (taken < count) {
    CgState s = run_batched(c, 0, every / 2, body, 0.0, 0.0, &to, 1);
    HX_CUDA(cudaMemcpyAsync(snaps + (size_t)taken * n, x, n * sizeof(double),
                            cudaMemcpyDeviceToDevice, c->stream));
    ++taken;
    if (s.status != HX_RUNNING) break;
  }
  HX_CUDA(cudaStreamSynchronize(c->stream));
  return taken;
}

}  // namespace hx
