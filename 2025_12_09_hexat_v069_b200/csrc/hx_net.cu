// hx_net.cu -- the learned preconditioner on the host side: parameters,
// training (forward, backward, Adam, all on the GPU), PCG snapshots for
// training data, and the flexible-CG solve that applies it.
//
// Preconditioner (symmetric positive definite for every choice of weights):
//     z = D^-1/2 (I + sum_{l=1..3} R_l^T E_l^T G_l^T G_l E_l R_l) D^-1/2 r.
// D^-1/2 r is taken as a nodal field (3 components per node of the mesh's
// node grid, level 0).  R_l restricts it to node-grid level l (each level
// halves the grid: coarse node i <-> fine node 2i, full weighting 1/2, 1,
// 1/2 per axis) and R_l^T is the exact transpose (prolongation).  E_l lifts
// a field to 6 channels (x, feat_l * x), feat_l being the density feature
// restricted to level l, and G_l is a network of 4 conv3d layers (3x3x3, no
// bias, no activation, 6 -> 16 -> 16 -> 16 -> 16 channels) with G_l^T its
// transposed convolutions.  Each term is positive semi-definite, zero
// weights give Jacobi, and the networks act only on coarse levels: a
// level-1 network costs 1/8 of one on the mesh's grid and sees twice as far,
// which is where Jacobi-PCG is slow (smooth error).  Only the BF16 roundings
// make the operator slightly nonlinear, which flexible CG (Notay's FCG, one
// stored direction) absorbs.  The input is scaled by the RMS s of D^-1/2 r
// to keep BF16 in range (z does not depend on s otherwise).  A nonlinear
// network (ReLU, biases) on the mesh's grid was tried first: it breaks
// symmetry and linearity, and FCG(1) with it stagnated.
//
// Training minimises, over residual/error pairs (r = b - A x_k, e = u* - x_k)
// taken from Jacobi-PCG iterates, the energy-norm error of one
// preconditioned step, loss = (z-e)^T A (z-e) / e^T A e (A e = r), or the
// scaled residual |D^-1/2 (A z - r)|^2 / |D^-1/2 r|^2.  Convergence is
// always judged on the residual, and the solve falls back to Jacobi-PCG
// from the current iterate when FCG breaks down or stalls.
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

#include "hx_cnn.h"
#include "hx_solver.h"

namespace hx {

namespace {

constexpr int LP = NET_LAYER_PARAMS;
constexpr int NP = NET_NET_PARAMS;

GridN level_grid(const Grid& g, int l) {
  GridN a{g.nxn, g.nyn, g.nzn};
  for (int k = 0; k < l; ++k) a = GridN{(a.nx - 1) / 2 + 1, (a.ny - 1) / 2 + 1, (a.nz - 1) / 2 + 1};
  return a;
}
int64_t nodes_of(const GridN& a) { return (int64_t)a.nx * a.ny * a.nz; }

// parameter p: network p / NP, layer (p % NP) / LP, weights [tap][co][ci];
// the first layer of each network reads NET_IN live input channels
bool live_param(int p) {
  const int layer = (p % NP) / LP, ci = p % 16;
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
  for (int l = 0; l < NET_PARAMS / LP; ++l)
    launch_pack_weights(c->stream, N.w.p + l * LP, N.wf.p + l * LP, N.wb.p + l * LP);
}

void net_upload(hx_ctx* c, const std::vector<float>& w) {
  auto& N = c->net;
  net_alloc_params(c);
  std::vector<unsigned char> live(NET_PARAMS);
  for (int p = 0; p < NET_PARAMS; ++p) live[p] = live_param(p) ? 1 : 0;
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

// Buffers of every level for the current mesh.  Application needs the
// fields, the network input/output per level and two ping-pong activation
// buffers (sized for level 1, the largest network grid); training keeps
// every activation of every level.
void net_buffers(hx_ctx* c, bool train) {
  auto& N = c->net;
  const GridN g1 = level_grid(c->g, 1);
  const size_t a1 = (size_t)nodes_of(g1) * 16;
  N.tmp[0].ensure(a1);
  N.tmp[1].ensure(a1);
  for (int l = 0; l <= NET_NETS; ++l) {
    const size_t nl = (size_t)nodes_of(level_grid(c->g, l));
    auto& L = N.lv[l];
    L.x.ensure(nl * 3);
    L.acc.ensure(nl * 3);
    L.feat.ensure(nl);
    if (l >= 1) {
      L.x0.ensure(nl * 16);
      L.y.ensure(nl * 8);
    }
    if (train) {
      L.gx.ensure(nl * 3);
      if (l >= 1)
        for (auto& a : L.act) a.ensure(nl * 16);
    }
  }
  if (train) {
    N.da.ensure(a1);
    N.db.ensure(a1);
    N.part.ensure(conv_num_tiles(g1) * LP);
  }
}

const __nv_bfloat16* fwd_w(const hx_ctx* c, int k, int l) { return c->net.wf.p + k * NP + l * LP; }
const __nv_bfloat16* adj_w(const hx_ctx* c, int k, int l) { return c->net.wb.p + k * NP + l * LP; }

// y = G_k^T G_k x0 on grid g through the two ping-pong buffers (application).
void stack_apply(hx_ctx* c, int k, const GridN& g, const __nv_bfloat16* x0, __nv_bfloat16* y) {
  __nv_bfloat16* u = c->net.tmp[0].p;
  __nv_bfloat16* v = c->net.tmp[1].p;
  launch_conv3(c->stream, 16, x0, u, fwd_w(c, k, 0), g);  // A1
  launch_conv3(c->stream, 16, u, v, fwd_w(c, k, 1), g);   // A2
  launch_conv3(c->stream, 16, v, u, fwd_w(c, k, 2), g);   // A3
  launch_conv3(c->stream, 16, u, v, fwd_w(c, k, 3), g);   // H = G x0
  launch_conv3(c->stream, 16, v, u, adj_w(c, k, 3), g);   // B3
  launch_conv3(c->stream, 16, u, v, adj_w(c, k, 2), g);   // B2
  launch_conv3(c->stream, 16, v, u, adj_w(c, k, 1), g);   // B1
  launch_conv3(c->stream, 8, u, y, adj_w(c, k, 0), g);    // B0 = G^T H (6 live channels)
}

// y = G_k^T G_k x0 keeping every activation: act = A1 A2 A3 H B3 B2 B1.
void stack_forward_train(hx_ctx* c, int k, const GridN& g, const __nv_bfloat16* x0,
                         DevBuf<__nv_bfloat16>* act, __nv_bfloat16* y) {
  launch_conv3(c->stream, 16, x0, act[0].p, fwd_w(c, k, 0), g);
  for (int l = 1; l < 4; ++l) launch_conv3(c->stream, 16, act[l - 1].p, act[l].p, fwd_w(c, k, l), g);
  for (int l = 3; l >= 1; --l) launch_conv3(c->stream, 16, act[6 - l].p, act[7 - l].p, adj_w(c, k, l), g);
  launch_conv3(c->stream, 8, act[6].p, y, adj_w(c, k, 0), g);
}

// Gradients of network k into N.grad from da = dLoss/dB0 (16-channel
// storage; overwritten).  B0 = G^T H with H = G x0: the G^T half is
// differentiated first (E_{l+1} = dLoss/dB_{l+1} = W_l * E_l; the weight
// gradient of a transposed use is wgrad(X = E_l, D = its input)), then the G
// half from dLoss/dH = W_3 * E_3 (forward use: wgrad(X = its input,
// D = dLoss/dout), dLoss/din = W^T * dLoss/dout).
void stack_backward_train(hx_ctx* c, int k, const GridN& g, const __nv_bfloat16* x0,
                          const DevBuf<__nv_bfloat16>* act, bool accumulate) {
  auto& N = c->net;
  float* grad = N.grad.p + k * NP;
  __nv_bfloat16* e0 = N.da.p;
  __nv_bfloat16* e1 = N.db.p;
  // transposed uses: layer l maps B_{l+1} (H for l = 3) to B_l
  const __nv_bfloat16* bin[4] = {act[6].p, act[5].p, act[4].p, act[3].p};
  for (int l = 0; l < 4; ++l) {
    launch_conv3_wgrad(c->stream, e0, bin[l], N.part.p, grad + l * LP, accumulate, g);
    launch_conv3(c->stream, 16, e0, e1, fwd_w(c, k, l), g);  // E_{l+1}; l = 3: dLoss/dH
    std::swap(e0, e1);
  }
  // forward uses: layer l maps A_l (x0 for l = 0) to A_{l+1} (H for l = 3)
  const __nv_bfloat16* ain[4] = {x0, act[0].p, act[1].p, act[2].p};
  for (int l = 3; l >= 0; --l) {
    launch_conv3_wgrad(c->stream, ain[l], e0, N.part.p, grad + l * LP, true, g);
    if (l > 0) {
      launch_conv3(c->stream, 16, e0, e1, adj_w(c, k, l), g);
      std::swap(e0, e1);
    }
  }
}

// lv[0].acc = sum_l R_l^T E_l^T G_l^T G_l E_l R_l lv[0].x  (coarsest level
// first: acc_l = E_l^T y_l + R^T acc_{l+1}).  `train` keeps the activations.
void precond_correction(hx_ctx* c, bool train) {
  auto& N = c->net;
  GridN gl[NET_NETS + 1];
  for (int l = 0; l <= NET_NETS; ++l) gl[l] = level_grid(c->g, l);
  for (int l = 1; l <= NET_NETS; ++l)
    launch_restrict(c->stream, 3, N.lv[l - 1].x.p, N.lv[l].x.p, gl[l - 1], gl[l], false);
  for (int l = NET_NETS; l >= 1; --l) {
    auto& L = N.lv[l];
    const int64_t nl = nodes_of(gl[l]);
    launch_lift(c->stream, L.x.p, L.feat.p, L.x0.p, nl);
    if (train)
      stack_forward_train(c, l - 1, gl[l], L.x0.p, L.act, L.y.p);
    else
      stack_apply(c, l - 1, gl[l], L.x0.p, L.y.p);
    launch_unlift(c->stream, L.y.p, L.feat.p, L.acc.p, false, nl);
    if (l < NET_NETS) launch_prolong(c->stream, N.lv[l + 1].acc.p, L.acc.p, gl[l], gl[l + 1], true);
  }
  launch_prolong(c->stream, N.lv[1].acc.p, N.lv[0].acc.p, gl[0], gl[1], false);
}

// Jacobi scaling and density features of the current operator (after a
// solve set up M^-1 for `fac`).
void net_operator_inputs(hx_ctx* c, const double* fac) {
  auto& N = c->net;
  const int64_t n = c->g.dofs();
  HX_REQUIRE(c->d_minv.n >= (size_t)n, "no Jacobi data: run a solve on this grid first");
  net_buffers(c, false);
  N.dinvs.ensure(n);
  launch_sqrt(c->stream, c->d_minv.p, N.dinvs.p, n);
  launch_rho_feature(c->stream, fac, N.lv[0].feat.p, c->g);
  for (int l = 1; l <= NET_NETS; ++l)
    launch_restrict(c->stream, 1, N.lv[l - 1].feat.p, N.lv[l].feat.p, level_grid(c->g, l - 1),
                    level_grid(c->g, l), true);
  // private copy: training steps apply the operator long after the caller's call
  double* fb = N.facbuf.ensure(c->g.elems());
  if (fb != fac)
    HX_CUDA(cudaMemcpyAsync(fb, fac, c->g.elems() * sizeof(double), cudaMemcpyDeviceToDevice,
                            c->stream));
  N.fac_last = fb;
}

void require_prepared(hx_ctx* c) {
  HX_REQUIRE(c->net.ready, "network not initialised");
  HX_REQUIRE(c->net.dinvs.n >= (size_t)c->g.dofs() && c->net.fac_last != nullptr,
             "no operator inputs: call hx_net_prepare after a solve");
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
  for (int p = 0; p < NET_PARAMS; ++p) {
    const int layer = (p % NP) / LP;
    // variance-preserving for a linear layer; the last one small, so that
    // the untrained preconditioner is close to Jacobi.  (All-zero weights
    // would be a stationary point: the loss is quadratic in G.)
    double std = std::sqrt(1.0 / (27.0 * (layer == 0 ? NET_IN : 16)));
    if (layer == NET_LAYERS - 1) std *= 0.3;
    const double g = std::sqrt(-2.0 * std::log(uni())) * std::cos(6.283185307179586 * uni());
    if (live_param(p)) w[p] = (float)(g * std);
  }
  net_upload(c, w);
}

void net_set_params(hx_ctx* c, const float* params) {
  std::vector<float> w(params, params + NET_PARAMS);
  for (int p = 0; p < NET_PARAMS; ++p)
    if (!live_param(p)) w[p] = 0.f;
  net_upload(c, w);
}

void net_get_params(hx_ctx* c, float* params) {
  HX_REQUIRE(c->net.ready, "network not initialised");
  HX_CUDA(cudaMemcpyAsync(params, c->net.w.p, NET_PARAMS * sizeof(float), cudaMemcpyDeviceToHost,
                          c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
}

// y = G^T G x0 of the first network and the gradient of <dy, y> w.r.t. its
// parameters (the other networks' gradients are zero), on a given node grid
// from host data (FP32 arrays [node][16], channels >= NET_IN ignored); for
// gradient checks.  Inputs are rounded to BF16.
void net_forward_backward(hx_ctx* c, int nx, int ny, int nz, const float* x0, const float* dy,
                          float* y, float* grads) {
  HX_REQUIRE(c->net.ready, "network not initialised");
  HX_REQUIRE(nx >= 1 && ny >= 1 && nz >= 1, "bad grid");
  const GridN g{nx, ny, nz};
  const int64_t nn = (int64_t)nx * ny * nz;
  auto& N = c->net;
  DevBuf<__nv_bfloat16> bx0, by, act[7];
  bx0.ensure(nn * 16);
  by.ensure(nn * 8);
  for (auto& a : act) a.ensure(nn * 16);
  N.da.ensure(nn * 16);
  N.db.ensure(nn * 16);
  N.part.ensure(conv_num_tiles(g) * LP);
  std::vector<__nv_bfloat16> h((size_t)nn * 16);
  for (size_t i = 0; i < h.size(); ++i) h[i] = __float2bfloat16_rn((i % 16) < NET_IN ? x0[i] : 0.f);
  HX_CUDA(cudaMemcpyAsync(bx0.p, h.data(), h.size() * 2, cudaMemcpyHostToDevice, c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  stack_forward_train(c, 0, g, bx0.p, act, by.p);
  std::vector<__nv_bfloat16> hy((size_t)nn * 8);
  HX_CUDA(cudaMemcpyAsync(hy.data(), by.p, hy.size() * 2, cudaMemcpyDeviceToHost, c->stream));
  for (size_t i = 0; i < h.size(); ++i) h[i] = __float2bfloat16_rn((i % 16) < NET_IN ? dy[i] : 0.f);
  HX_CUDA(cudaMemcpyAsync(N.da.p, h.data(), h.size() * 2, cudaMemcpyHostToDevice, c->stream));
  HX_CUDA(cudaMemsetAsync(N.grad.p, 0, NET_PARAMS * sizeof(float), c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  stack_backward_train(c, 0, g, bx0.p, act, false);
  HX_CUDA(cudaMemcpyAsync(grads, N.grad.p, NET_PARAMS * sizeof(float), cudaMemcpyDeviceToHost,
                          c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  for (int64_t n = 0; n < nn; ++n)
    for (int ch = 0; ch < 16; ++ch)
      y[n * 16 + ch] = ch < 8 ? __bfloat162float(hy[n * 8 + ch]) : 0.f;
}

// Loss of one residual (and error) of the current operator; with `grad`,
// adds its parameter gradient to N.grad (`first`: overwrite instead).
double net_loss_grad(hx_ctx* c, const double* r, const double* e, int loss_kind, bool first) {
  auto& N = c->net;
  const Grid& g = c->g;
  const int64_t n = g.dofs();
  double* zscr = c->d_aux1.ensure(n);
  double* pscr = c->d_aux2.ensure(n);
  CgState* s3 = c->d_state.p + 3;
  CgState* s2 = c->d_state.p + 2;
  // rz = r.M^-1 r for the input scaling (state slot 3)
  HX_CUDA(cudaMemsetAsync(s3, 0, sizeof(CgState), c->stream));
  launch_cg_init<double>(c->stream, r, nullptr, c->d_minv.p, zscr, pscr, n, s3, c->d_partials.p);
  const double scale_mul = 1.0 / (double)n;
  launch_field_in(c->stream, r, N.dinvs.p, s3, nullptr, 0, scale_mul, N.lv[0].x.p, n);
  precond_correction(c, true);
  double* z = N.z.ensure(n);
  double* q = c->d_q.ensure(n);
  launch_net_output(c->stream, r, c->d_minv.p, N.dinvs.p, N.lv[0].acc.p, s3, scale_mul, z,
                    nullptr, nullptr, n);
  HX_CUDA(cudaMemsetAsync(s2, 0, sizeof(CgState), c->stream));
  bool host_ratio = false;
  const double* gvec = nullptr;  // dLoss/dz up to the coefficient of the mode
  int mode = 1;
  if (loss_kind == 0) {
    // energy-norm loss of the preconditioned vector z against the error e
    HX_REQUIRE(e != nullptr, "the energy loss needs the error vector");
    launch_axpby(c->stream, zscr, z, e, n);  // d = z - e
    launch_matvec<double>(c->stream, 0, zscr, q, N.fac_last, c->d_nmask.p, g, c->K, 0.0, s3,
                          c->d_partials.p, nullptr);
    launch_net_aloss(c->stream, zscr, q, e, r, n, c->d_partials.p, s2, N.scal.p);
    gvec = q;  // 2 A d / e.r
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
    gvec = zscr;  // 2 A M^-1 w / r.M^-1 r
    mode = 2;
    host_ratio = true;
  }
  // dLoss/d(correction at level l) = R_l (s D^-1/2 dLoss/dz); each network's
  // output gradient is its lifting E_l
  launch_field_in(c->stream, gvec, N.dinvs.p, s3, s2, mode, scale_mul, N.lv[0].gx.p, n);
  for (int l = 1; l <= NET_NETS; ++l)
    launch_restrict(c->stream, 3, N.lv[l - 1].gx.p, N.lv[l].gx.p, level_grid(g, l - 1),
                    level_grid(g, l), false);
  for (int l = 1; l <= NET_NETS; ++l) {
    const GridN gl = level_grid(g, l);
    launch_lift(c->stream, N.lv[l].gx.p, N.lv[l].feat.p, N.da.p, nodes_of(gl));
    stack_backward_train(c, l - 1, gl, N.lv[l].x0.p, N.lv[l].act, !first);
  }
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

// One Adam step on the summed gradient of `count` residual (and error)
// pairs of the current operator (grid, factors of the last hx_net_prepare).
// r[i], e[i]: FP64 device vectors (grid numbering).  Returns the mean loss.
double net_train_step(hx_ctx* c, const double* const* r, const double* const* e, int count,
                      double lr, int loss_kind) {
  require_prepared(c);
  HX_REQUIRE(count >= 1, "empty batch");
  auto& N = c->net;
  net_buffers(c, true);
  ensure_workspace(c);
  double sum = 0.0;
  for (int i = 0; i < count; ++i)
    sum += net_loss_grad(c, r[i], e ? e[i] : nullptr, loss_kind, i == 0);
  N.step += 1;
  launch_adam(c->stream, N.w.p, N.m.p, N.v.p, N.grad.p, N.live.p, NET_PARAMS, (float)lr, N.step);
  net_pack(c);
  HX_CUDA(cudaStreamSynchronize(c->stream));
  return sum / count;
}

void net_prepare(hx_ctx* c, const double* fac) { net_operator_inputs(c, fac); }

// z = P r with the prepared operator (FP64 device vectors, grid numbering).
void net_apply_vec(hx_ctx* c, const double* r, double* z) {
  require_prepared(c);
  auto& N = c->net;
  const int64_t n = c->g.dofs();
  net_buffers(c, false);
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
  launch_field_in(c->stream, r, N.dinvs.p, s3, nullptr, 0, scale_mul, N.lv[0].x.p, n);
  precond_correction(c, false);
  launch_net_output(c->stream, r, c->d_minv.p, N.dinvs.p, N.lv[0].acc.p, s3, scale_mul, z,
                    nullptr, nullptr, n);
  HX_CUDA(cudaStreamSynchronize(c->stream));
}

std::function<void()> net_time_body(hx_ctx* c, int which) {
  require_prepared(c);
  auto& N = c->net;
  const Grid g = c->g;
  const int64_t n = g.dofs();
  HX_REQUIRE(c->d_r.n >= (size_t)n, "run a solve before timing the network");
  net_buffers(c, false);
  if (which == 0) {  // one 16 -> 16 layer on the level-1 grid
    const GridN g1 = level_grid(g, 1);
    HX_CUDA(cudaMemsetAsync(N.tmp[0].p, 0, (size_t)nodes_of(g1) * 16 * sizeof(__nv_bfloat16),
                            c->stream));
    return [c, g1] {
      launch_conv3(c->stream, 16, c->net.tmp[0].p, c->net.tmp[1].p, fwd_w(c, 0, 1), g1);
    };
  }
  // the state of slot 3 holds r.M^-1 r of the last solve's residual
  CgState* s3 = c->d_state.p + 3;
  HX_CUDA(cudaMemsetAsync(s3, 0, sizeof(CgState), c->stream));
  launch_cg_init<double>(c->stream, c->d_r.p, nullptr, c->d_minv.p, c->d_aux1.ensure(n),
                         c->d_aux2.ensure(n), n, s3, c->d_partials.p);
  double* z = N.z.ensure(n);
  return [c, s3, z, n] {
    auto& M = c->net;
    const double scale_mul = 1.0 / (double)n;
    launch_field_in(c->stream, c->d_r.p, M.dinvs.p, s3, nullptr, 0, scale_mul, M.lv[0].x.p, n);
    precond_correction(c, false);
    launch_net_output(c->stream, c->d_r.p, c->d_minv.p, M.dinvs.p, M.lv[0].acc.p, s3, scale_mul,
                      z, nullptr, nullptr, n);
  };
}

// ---------------------------------------------------------------------------
// Flexible CG with the network preconditioner (FP64 vectors and operator,
// BF16 network).  Falls back to Jacobi-PCG from the current iterate when
// FCG breaks down, diverges, or stalls.
// ---------------------------------------------------------------------------
CgState solve_learned(hx_ctx* c, const double* fac, const double* b, double* x, bool warm,
                      double shift, const hx_solve_opts& o, double t0, bool* timed_out,
                      int* fallback, int* iters_out) {
  HX_REQUIRE(c->net.ready, "learned preconditioner requested but no network is loaded");
  auto& N = c->net;
  const Grid& g = c->g;
  const int64_t n = g.dofs();
  net_operator_inputs(c, fac);
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
    launch_field_in(c->stream, r, N.dinvs.p, st, nullptr, 0, scale_mul, N.lv[0].x.p, n);
    precond_correction(c, false);
    launch_net_output(c->stream, r, minv, N.dinvs.p, N.lv[0].acc.p, st, scale_mul, z, q,
                      c->d_partials.p, n);
    launch_fcg_step<double>(c->stream, pin, pout, z, r, x, q, fac, c->d_nmask.p, g, c->K, shift,
                            st, c->d_partials.p);
    launch_cg_update2<double>(c->stream, r, q, minv, n, st, c->d_partials.p);
  };
  auto body = [&]() {
    one(P1, P0);
    one(P0, P1);
  };
  const int reps = std::max(1, auto_batch(g, o.check_every) / 2);
  double best = s0.rel_res;
  int best_it = 0;
  CgState sf{};
  bool stalled = false;
  // Run in batches, checking between them for stagnation: no 10% gain on
  // the best residual within max(500, iterations / 4) iterations.  (CG
  // residuals are not monotone and on hard problems halve only every few
  // hundred iterations, so a tighter test would misfire.)
  for (;;) {
    sf = run_batched(c, 0, reps, body, o.wall_limit_ms, t0, timed_out, 1);
    if (sf.rel_res < 0.9 * best) {
      best = sf.rel_res;
      best_it = sf.iter;
    }
    if (sf.status != HX_RUNNING || *timed_out) break;
    const int window = std::max(500, sf.iter / 4);
    if (!o.learned_no_fallback && sf.iter - best_it > window) {
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
