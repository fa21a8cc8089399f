// hx_net.cu -- the convolutional preconditioner network on the host side:
// parameters, training (forward, backward, Adam, all on the GPU), PCG
// snapshots for training data, and the flexible-CG solve that applies it.
//
// Network G: 4 conv3d layers (3x3x3, no bias, no activation) on the node
// grid, 6 -> 16 -> 16 -> 16 -> 16 channels.  Its input is the lifting
// E r~ = (r~, feat * r~) of the Jacobi-scaled residual r~ = D^-1/2 r / s
// (s = RMS of D^-1/2 r, which only keeps BF16 in range), feat the nodal
// density feature.  The preconditioner is
//     z = D^-1 r + s D^-1/2 E^T G^T G E r~ = D^-1/2 (I + E^T G^T G E) D^-1/2 r,
// G^T being the transposed convolutions with the same weights.  For every
// choice of weights this is symmetric positive definite (E^T G^T G E is
// positive semi-definite), so CG with it converges like PCG with any SPD
// preconditioner; zero weights give Jacobi.  Only the BF16 roundings make
// it slightly nonlinear, which flexible CG (Notay's FCG, one stored
// direction) absorbs.  A nonlinear network (ReLU, biases) was not used: it
// breaks symmetry and linearity, and FCG(1) with such a network stagnated.
//
// Training minimises, over residual/error pairs (r = b - A x_k, e = u* - x_k)
// taken from Jacobi-PCG iterates, the energy-norm error of one
// preconditioned step, loss = (z-e)^T A (z-e) / e^T A e (A e = r), or the
// scaled residual |D^-1/2 (A z - r)|^2 / |D^-1/2 r|^2.  Convergence is
// always judged on the residual, and the solve falls back to Jacobi-PCG
// from the current iterate when FCG breaks down or stalls.
#include <cmath>
#include <cstring>
#include <vector>

#include "hx_cnn.h"
#include "hx_solver.h"

namespace hx {

namespace {

constexpr int LP = NET_LAYER_PARAMS;

GridN node_grid(const Grid& g) { return GridN{g.nxn, g.nyn, g.nzn}; }

// weights [tap][co][ci]: layer 0 reads NET_IN live input channels
bool live_param(int layer, int k) {
  const int ci = k % 16;
  return layer > 0 || ci < NET_IN;
}

void net_alloc_params(hx_ctx* c) {
  auto& N = c->net;
  N.w.ensure(NET_PARAMS);
  N.m.ensure(NET_PARAMS);
  N.v.ensure(NET_PARAMS);
  N.grad.ensure(NET_PARAMS);
  N.live.ensure(NET_PARAMS);
  N.wf.ensure(NET_PARAMS);
  N.wb.ensure(NET_PARAMS);
  N.scal.ensure(8);
}

void net_pack(hx_ctx* c) {
  auto& N = c->net;
  for (int l = 0; l < NET_LAYERS; ++l)
    launch_pack_weights(c->stream, N.w.p + l * LP, N.wf.p + l * LP, N.wb.p + l * LP);
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

// Activation buffers: x0 (input), y (6-channel output, stride 8), and the
// intermediate layers (2 for application, 7 + 2 gradient buffers for training).
void net_buffers(hx_ctx* c, int64_t nn, size_t tiles, bool train) {
  auto& N = c->net;
  const size_t a = (size_t)nn * 16;
  N.x0.ensure(a);
  N.y.ensure((size_t)nn * 8);
  for (int i = 0; i < (train ? 7 : 2); ++i) N.act[i].ensure(a);
  if (train) {
    N.da.ensure(a);
    N.db.ensure(a);
    N.part.ensure(tiles * LP);
  }
}

const __nv_bfloat16* fwd_w(const hx_ctx* c, int l) { return c->net.wf.p + l * LP; }
const __nv_bfloat16* adj_w(const hx_ctx* c, int l) { return c->net.wb.p + l * LP; }

// y = G^T G x0 through two ping-pong buffers (application).
void net_apply(hx_ctx* c, const GridN& g) {
  auto& N = c->net;
  __nv_bfloat16* u = N.act[0].p;
  __nv_bfloat16* v = N.act[1].p;
  launch_conv3(c->stream, 16, N.x0.p, u, fwd_w(c, 0), g);  // A1
  launch_conv3(c->stream, 16, u, v, fwd_w(c, 1), g);       // A2
  launch_conv3(c->stream, 16, v, u, fwd_w(c, 2), g);       // A3
  launch_conv3(c->stream, 16, u, v, fwd_w(c, 3), g);       // H = G x0
  launch_conv3(c->stream, 16, v, u, adj_w(c, 3), g);       // B3
  launch_conv3(c->stream, 16, u, v, adj_w(c, 2), g);       // B2
  launch_conv3(c->stream, 16, v, u, adj_w(c, 1), g);       // B1
  launch_conv3(c->stream, 8, u, N.y.p, adj_w(c, 0), g);    // B0 = G^T H
}

// y = G^T G x0 keeping every activation for the backward pass:
// act = A1 A2 A3 H B3 B2 B1.
void net_forward_train(hx_ctx* c, const GridN& g) {
  auto& N = c->net;
  launch_conv3(c->stream, 16, N.x0.p, N.act[0].p, fwd_w(c, 0), g);
  for (int l = 1; l < 4; ++l) launch_conv3(c->stream, 16, N.act[l - 1].p, N.act[l].p, fwd_w(c, l), g);
  for (int l = 3; l >= 1; --l)
    launch_conv3(c->stream, 16, N.act[6 - l].p, N.act[7 - l].p, adj_w(c, l), g);
  launch_conv3(c->stream, 8, N.act[6].p, N.y.p, adj_w(c, 0), g);
}

// Parameter gradients into N.grad from da = dLoss/dB0 (16-channel storage).
// B0 = G^T H with H = G x0: the G^T half is differentiated first
// (E_l = dLoss/dB_l = W_{l-1} * E_{l-1}, weight gradient of a transposed use
// = wgrad(X = E, D = its input)), then the G half from dLoss/dH = W_3 * E_3
// (weight gradient of a forward use = wgrad(X = its input, D = dLoss/dout),
// dLoss/din = W^T * dLoss/dout).
void net_backward_train(hx_ctx* c, const GridN& g) {
  auto& N = c->net;
  __nv_bfloat16* e0 = N.da.p;
  __nv_bfloat16* e1 = N.db.p;
  // transposed uses: layer l maps B_{l+1} (act[6-l], H for l = 3) to B_l
  const __nv_bfloat16* bin[4] = {N.act[6].p, N.act[5].p, N.act[4].p, N.act[3].p};
  for (int l = 0; l < 4; ++l) {
    launch_conv3_wgrad(c->stream, e0, bin[l], N.part.p, N.grad.p + l * LP, false, g);
    launch_conv3(c->stream, 16, e0, e1, fwd_w(c, l), g);  // E_{l+1}; l = 3: dLoss/dH
    std::swap(e0, e1);
  }
  // forward uses: layer l maps A_l (x0 for l = 0) to A_{l+1} (H for l = 3)
  const __nv_bfloat16* ain[4] = {N.x0.p, N.act[0].p, N.act[1].p, N.act[2].p};
  for (int l = 3; l >= 0; --l) {
    launch_conv3_wgrad(c->stream, ain[l], e0, N.part.p, N.grad.p + l * LP, true, g);
    if (l > 0) {
      launch_conv3(c->stream, 16, e0, e1, adj_w(c, l), g);
      std::swap(e0, e1);
    }
  }
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
  // private copy: training steps apply the operator long after the caller's call
  double* fb = N.facbuf.ensure(c->g.elems());
  if (fb != fac)
    HX_CUDA(cudaMemcpyAsync(fb, fac, c->g.elems() * sizeof(double), cudaMemcpyDeviceToDevice,
                            c->stream));
  N.fac_last = fb;
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
    // variance-preserving for a linear layer; the last one small, so that
    // the untrained preconditioner is close to Jacobi.  (All-zero weights
    // would be a stationary point: the loss is quadratic in G.)
    double std = std::sqrt(1.0 / (27.0 * (l == 0 ? NET_IN : 16)));
    if (l == NET_LAYERS - 1) std *= 0.3;
    for (int k = 0; k < LP; ++k) {
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

// y = G^T G x0 and the parameter gradient of <dy, y> on a given node grid
// from host data (FP32 arrays [node][16], channels >= NET_IN ignored); for
// gradient checks.  Inputs are rounded to BF16.
void net_forward_backward(hx_ctx* c, int nx, int ny, int nz, const float* x0, const float* dy,
                          float* y, float* grads) {
  HX_REQUIRE(c->net.ready, "network not initialised");
  HX_REQUIRE(nx >= 1 && ny >= 1 && nz >= 1, "bad grid");
  const GridN g{nx, ny, nz};
  const int64_t nn = (int64_t)nx * ny * nz;
  net_buffers(c, nn, conv_num_tiles(g), true);
  auto& N = c->net;
  std::vector<__nv_bfloat16> h((size_t)nn * 16);
  for (size_t i = 0; i < h.size(); ++i) h[i] = __float2bfloat16_rn((i % 16) < NET_IN ? x0[i] : 0.f);
  HX_CUDA(cudaMemcpyAsync(N.x0.p, h.data(), h.size() * 2, cudaMemcpyHostToDevice, c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  net_forward_train(c, g);
  std::vector<__nv_bfloat16> hy((size_t)nn * 8);
  HX_CUDA(cudaMemcpyAsync(hy.data(), N.y.p, hy.size() * 2, cudaMemcpyDeviceToHost, c->stream));
  for (size_t i = 0; i < h.size(); ++i) h[i] = __float2bfloat16_rn((i % 16) < NET_IN ? dy[i] : 0.f);
  HX_CUDA(cudaMemcpyAsync(N.da.p, h.data(), h.size() * 2, cudaMemcpyHostToDevice, c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  net_backward_train(c, g);
  HX_CUDA(cudaMemcpyAsync(grads, N.grad.p, NET_PARAMS * sizeof(float), cudaMemcpyDeviceToHost,
                          c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  for (int64_t n = 0; n < nn; ++n)
    for (int ch = 0; ch < 16; ++ch)
      y[n * 16 + ch] = ch < 8 ? __bfloat162float(hy[n * 8 + ch]) : 0.f;
}

// One Adam step on a residual (and error) of the current operator (grid,
// factors of the last hx_net_prepare).  r, e: FP64 device vectors (grid
// numbering).
double net_train_step(hx_ctx* c, const double* r, const double* e, double lr, int loss_kind) {
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
  CgState* s3 = c->d_state.p + 3;
  CgState* s2 = c->d_state.p + 2;
  HX_CUDA(cudaMemsetAsync(s3, 0, sizeof(CgState), c->stream));
  launch_cg_init<double>(c->stream, r, nullptr, c->d_minv.p, zscr, pscr, n, s3, c->d_partials.p);
  const double scale_mul = 1.0 / (double)n;
  launch_net_lift(c->stream, r, N.dinvs.p, N.feat.p, s3, nullptr, 0, scale_mul, N.x0.p, nn);
  net_forward_train(c, gn);
  double* z = N.z.ensure(n);
  double* q = c->d_q.ensure(n);
  launch_net_output(c->stream, r, c->d_minv.p, N.dinvs.p, N.feat.p, N.y.p, s3, scale_mul, z,
                    nullptr, nullptr, nn);
  HX_CUDA(cudaMemsetAsync(s2, 0, sizeof(CgState), c->stream));
  bool host_ratio = false;
  if (loss_kind == 0) {
    // energy-norm loss of the preconditioned vector z against the error e
    HX_REQUIRE(e != nullptr, "the energy loss needs the error vector");
    launch_axpby(c->stream, zscr, z, e, n);  // d = z - e
    launch_matvec<double>(c->stream, 0, zscr, q, N.fac_last, c->d_nmask.p, g, c->K, 0.0, s3,
                          c->d_partials.p, nullptr);
    launch_net_aloss(c->stream, zscr, q, e, r, n, c->d_partials.p, s2, N.scal.p);
    launch_net_lift(c->stream, q, N.dinvs.p, N.feat.p, s3, s2, 1, scale_mul, N.da.p, nn);
  } else {
    // scaled residual loss |D^-1/2 (A z - r)|^2 / |D^-1/2 r|^2
    launch_matvec<double>(c->stream, 0, z, q, N.fac_last, c->d_nmask.p, g, c->K, 0.0, s3,
                          c->d_partials.p, nullptr);
    launch_axpby(c->stream, q, q, r, n);  // w = A z - r
    // rz(slot 2) = w.M^-1 w, pscr = M^-1 w, then zscr = A M^-1 w
    launch_cg_init<double>(c->stream, q, nullptr, c->d_minv.p, zscr, pscr, n, s2,
                           c->d_partials.p);
    launch_matvec<double>(c->stream, 0, pscr, zscr, N.fac_last, c->d_nmask.p, g, c->K, 0.0, s3,
                          c->d_partials.p, nullptr);
    launch_net_lift(c->stream, zscr, N.dinvs.p, N.feat.p, s3, nullptr, 2, scale_mul, N.da.p, nn);
    host_ratio = true;
  }
  net_backward_train(c, gn);
  N.step += 1;
  launch_adam(c->stream, N.w.p, N.m.p, N.v.p, N.grad.p, N.live.p, NET_PARAMS, (float)lr, N.step);
  net_pack(c);
  double loss = 0;
  if (host_ratio) {
    const CgState a = get_state(c, 2), b = get_state(c, 3);
    loss = b.rz > 0 ? a.rz / b.rz : 0.0;
  } else {
    HX_CUDA(cudaMemcpyAsync(&loss, N.scal.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    HX_CUDA(cudaStreamSynchronize(c->stream));
  }
  return loss;
}

void net_prepare(hx_ctx* c, const double* fac) { net_operator_inputs(c, fac); }

// z = P r with the prepared operator (FP64 device vectors, grid numbering).
void net_apply_vec(hx_ctx* c, const double* r, double* z) {
  HX_REQUIRE(c->net.ready, "network not initialised");
  auto& N = c->net;
  const Grid& g = c->g;
  const int64_t n = g.dofs(), nn = g.nodes();
  HX_REQUIRE(N.dinvs.n >= (size_t)n && N.feat.n >= (size_t)nn,
             "no operator inputs: call hx_net_prepare after a solve");
  net_buffers(c, nn, 0, false);
  ensure_workspace(c);
  CgState* s3 = c->d_state.p + 3;
  HX_CUDA(cudaMemsetAsync(s3, 0, sizeof(CgState), c->stream));
  launch_cg_init<double>(c->stream, r, nullptr, c->d_minv.p, c->d_aux1.ensure(n),
                         c->d_aux2.ensure(n), n, s3, c->d_partials.p);
  const CgState st = get_state(c, 3);
  if (st.status == HX_ST_ZERO_RHS) {  // r = 0 on the free DOFs
    launch_fill_zero(c->stream, z, n * sizeof(double));
    HX_CUDA(cudaStreamSynchronize(c->stream));
    return;
  }
  HX_REQUIRE(st.status == HX_RUNNING && st.rz > 0.0, "r is not finite");
  const double scale_mul = 1.0 / (double)n;
  launch_net_lift(c->stream, r, N.dinvs.p, N.feat.p, s3, nullptr, 0, scale_mul, N.x0.p, nn);
  net_apply(c, node_grid(g));
  launch_net_output(c->stream, r, c->d_minv.p, N.dinvs.p, N.feat.p, N.y.p, s3, scale_mul, z,
                    nullptr, nullptr, nn);
  HX_CUDA(cudaStreamSynchronize(c->stream));
}

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
    launch_net_lift(c->stream, r, N.dinvs.p, N.feat.p, st, nullptr, 0, scale_mul, N.x0.p, nn);
    net_apply(c, gn);
    launch_net_output(c->stream, r, minv, N.dinvs.p, N.feat.p, N.y.p, st, scale_mul, z, q,
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
    if (!o.learned_no_fallback && sf.iter - best_it > stall_window) {
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
  if (!failed || *timed_out || o.learned_no_fallback) return sf;
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
