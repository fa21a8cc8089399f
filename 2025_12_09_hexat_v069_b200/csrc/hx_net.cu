// hx_net.cu -- the learned preconditioner on the host side: parameters,
// training (forward, backward, Adam, all on the GPU), PCG snapshots for
// training data, and the flexible-CG solves that apply it.
//
// Preconditioner (symmetric positive definite for every choice of weights):
//     z = D^-1/2 (I + sum_{l=NET_L0..NET_TOP} R_l^T E_l^T G_l^T G_l E_l R_l) D^-1/2 r.
// D^-1/2 r is taken as a nodal field (3 components per node of the mesh's
// node grid, level 0).  R_l restricts it to node-grid level l (each level
// halves the grid: coarse node i <-> fine node 2i, full weighting 1/2, 1,
// 1/2 per axis) and R_l^T is the exact transpose (prolongation).  E_l lifts
// a field to 6 channels (x, feat_l * x), feat_l being the density feature
// restricted to level l, and G_l is a network of 4 conv3d layers (3x3x3, no
// bias, no activation, 6 -> 16 -> 16 -> 16 -> 16 channels) with G_l^T its
// transposed convolutions.  Each term is positive semi-definite, and zero
// weights give Jacobi.  The networks act only on coarse levels (2, 3, 4): a
// level-l network costs 8^-l of one on the mesh's grid and sees 2^l times as
// far, which is where Jacobi-PCG is slow (smooth error); level 1 carries
// only the restricted field.  Only the BF16 roundings make the operator
// slightly nonlinear, which flexible CG (Notay's FCG, one stored direction)
// absorbs.  The input is scaled by the RMS s of D^-1/2 r to keep BF16 in
// range (z does not depend on s otherwise).  A nonlinear network (ReLU,
// biases) on the mesh's grid was tried first: it breaks symmetry and
// linearity, and FCG(1) with it stagnated.
//
// Training minimises, over residual/error pairs (r = b - A x_k, e = u* - x_k)
// taken from Jacobi-PCG iterates, the energy-norm error of one
// preconditioned step, loss = (z-e)^T A (z-e) / e^T A e (A e = r), or the
// scaled residual |D^-1/2 (A z - r)|^2 / |D^-1/2 r|^2.  Convergence is
// always judged on the residual, and the solve falls back to Jacobi-PCG
// from the current iterate when FCG breaks down or stalls.
#include <cmath>
#include <limits>
#include <cstring>
#include <utility>
#include <vector>

#include "hx_cnn.h"
#include "hx_solver.h"

namespace hx {

namespace {

constexpr int LP = NET_LAYER_PARAMS;
constexpr int NP = NET_NET_PARAMS;
static_assert(NET_NETS >= 1 && NET_NETS <= 3, "one side stream per level beyond the first");
static_assert(NET_L0 >= 1 && NET_TOP < 8, "level range of the networks");

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
  if (N.err.n == 0) {
    N.err.ensure(1);
    HX_CUDA(cudaMemsetAsync(N.err.p, 0, sizeof(int), c->stream));
  }
}

// Throws if a conv kernel reported a wait that ran out (and clears the flag).
void check_conv_error(hx_ctx* c) {
  if (c->net.err.n == 0) return;
  int e = 0;
  HX_CUDA(cudaMemcpyAsync(&e, c->net.err.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  if (e != 0) {
    HX_CUDA(cudaMemsetAsync(c->net.err.p, 0, sizeof(int), c->stream));
    throw Error{HX_CUDA_ERROR, "tensor-core convolution: a bounded wait ran out"};
  }
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

// Buffers of every level for the current mesh: fields on levels 1 ..
// NET_TOP, network input/output on the network levels, two ping-pong
// activation buffers for the finest network (level NET_L0, the largest) and
// two per coarser network (their side streams); training keeps every
// activation of every network.
void net_buffers(hx_ctx* c, bool train) {
  auto& N = c->net;
  const GridN g1 = level_grid(c->g, NET_L0);
  const size_t a1 = (size_t)nodes_of(g1) * 16;
  N.tmp[0].ensure(a1);
  N.tmp[1].ensure(a1);
  N.lv[0].feat.ensure((size_t)nodes_of(level_grid(c->g, 0)));  // only the feature on level 0
  ensure_workspace(c);
  const size_t need = 2 * net_output_blocks(level_grid(c->g, 0));
  if (c->d_partials.n < need) c->d_partials.ensure(need);
  for (int l = 1; l <= NET_TOP; ++l) {
    const size_t nl = (size_t)nodes_of(level_grid(c->g, l));
    auto& L = N.lv[l];
    L.x.ensure(nl * 3);
    L.acc.ensure(nl * 3);
    L.feat.ensure(nl);
    if (train) L.gx.ensure(nl * 3);
    if (l < NET_L0) continue;
    L.x0.ensure(nl * 16);
    L.y.ensure(nl * 8);
    if (train)
      for (auto& a : L.act) a.ensure(nl * 16);
    if (l > NET_L0)
      for (auto& b : L.pp) b.ensure(nl * 16);
  }
  if (!N.ev_fork) {
    HX_CUDA(cudaEventCreateWithFlags(&N.ev_fork, cudaEventDisableTiming));
    for (int i = 0; i < 2; ++i) {
      HX_CUDA(cudaStreamCreateWithFlags(&N.side[i], cudaStreamNonBlocking));
      HX_CUDA(cudaEventCreateWithFlags(&N.ev_join[i], cudaEventDisableTiming));
      HX_CUDA(cudaEventCreateWithFlags(&N.ev_x[i], cudaEventDisableTiming));
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

// y = G_k^T G_k x0 on grid g through the ping-pong buffers u, v, on stream s.
void stack_apply(hx_ctx* c, cudaStream_t s, int k, const GridN& g, const __nv_bfloat16* x0,
                 __nv_bfloat16* y, __nv_bfloat16* u, __nv_bfloat16* v) {
  int* err = c->net.err.p;
  launch_conv3(s, 16, x0, u, fwd_w(c, k, 0), g, err);  // A1
  launch_conv3(s, 16, u, v, fwd_w(c, k, 1), g, err);   // A2
  launch_conv3(s, 16, v, u, fwd_w(c, k, 2), g, err);   // A3
  launch_conv3(s, 16, u, v, fwd_w(c, k, 3), g, err);   // H = G x0
  launch_conv3(s, 16, v, u, adj_w(c, k, 3), g, err);   // B3
  launch_conv3(s, 16, u, v, adj_w(c, k, 2), g, err);   // B2
  launch_conv3(s, 16, v, u, adj_w(c, k, 1), g, err);   // B1
  launch_conv3(s, 8, u, y, adj_w(c, k, 0), g, err);    // B0 = G^T H, 6 channels
}

// y = G_k^T G_k x0 keeping every activation: act = A1 A2 A3 H B3 B2 B1.
void stack_forward_train(hx_ctx* c, int k, const GridN& g, const __nv_bfloat16* x0,
                         DevBuf<__nv_bfloat16>* act, __nv_bfloat16* y) {
  launch_conv3(c->stream, 16, x0, act[0].p, fwd_w(c, k, 0), g, c->net.err.p);
  for (int l = 1; l < 4; ++l)
    launch_conv3(c->stream, 16, act[l - 1].p, act[l].p, fwd_w(c, k, l), g, c->net.err.p);
  for (int l = 3; l >= 1; --l)
    launch_conv3(c->stream, 16, act[6 - l].p, act[7 - l].p, adj_w(c, k, l), g, c->net.err.p);
  launch_conv3(c->stream, 8, act[6].p, y, adj_w(c, k, 0), g, c->net.err.p);
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
    // E_{l+1}; l = 3: dLoss/dH
    launch_conv3(c->stream, 16, e0, e1, fwd_w(c, k, l), g, c->net.err.p);
    std::swap(e0, e1);
  }
  // forward uses: layer l maps A_l (x0 for l = 0) to A_{l+1} (H for l = 3)
  const __nv_bfloat16* ain[4] = {x0, act[0].p, act[1].p, act[2].p};
  for (int l = 3; l >= 0; --l) {
    launch_conv3_wgrad(c->stream, ain[l], e0, N.part.p, grad + l * LP, true, g);
    if (l > 0) {
      launch_conv3(c->stream, 16, e0, e1, adj_w(c, k, l), g, c->net.err.p);
      std::swap(e0, e1);
    }
  }
}

// z = M^-1 r + s D^-1/2 sum_l R_l^T E_l^T G_l^T G_l E_l R_l (D^-1/2 r / s).
// The mesh-grid passes are fused: the level-1 field is restricted straight
// from BF16(D^-1/2 r) (k_restrict_ys) and the level-1 correction is
// prolongated inside the output kernel, so no FP32 field is stored on the
// mesh's node grid.  `train`
// keeps the activations; q_old: FCG beta reduction (see k_net_output).
// The level-1 field is restricted from ys = BF16(D^-1/2 r): passed in when
// already formed (FCG loops: by the residual update), else formed here.
// T: precision of r, minv, z, q_old (the solver's vectors).
template <typename T>
void precond_z(hx_ctx* c, const T* r, const T* minv, CgState* st, double scale_mul, T* z,
               const T* q_old, bool train, const __nv_bfloat16* ys = nullptr) {
  auto& N = c->net;
  GridN gl[NET_TOP + 1];
  for (int l = 0; l <= NET_TOP; ++l) gl[l] = level_grid(c->g, l);
  if (!ys) {
    const int64_t n = c->g.dofs();
    __nv_bfloat16* y = N.ys.ensure(n + 8);
    launch_dinv_bf16<T>(c->stream, r, minv, y, n);
    ys = y;
  }
  launch_restrict_ys(c->stream, ys, st, scale_mul, N.lv[1].x.p, gl[0], gl[1]);
  if (train) {
    for (int l = 2; l <= NET_TOP; ++l)
      launch_restrict(c->stream, 3, N.lv[l - 1].x.p, N.lv[l].x.p, gl[l - 1], gl[l], false);
    for (int l = NET_TOP; l >= NET_L0; --l) {
      auto& L = N.lv[l];
      launch_lift(c->stream, L.x.p, L.feat.p, L.x0.p, gl[l]);
      stack_forward_train(c, l - NET_L0, gl[l], L.x0.p, L.act, L.y.p);
    }
    // acc_l = E_l^T y_l (network levels) + R^T acc_{l+1}, coarsest first
    for (int l = NET_TOP; l >= NET_L0; --l) {
      auto& L = N.lv[l];
      launch_unlift(c->stream, L.y.p, L.feat.p, L.acc.p, false, nodes_of(gl[l]));
      if (l < NET_TOP)
        launch_prolong(c->stream, N.lv[l + 1].acc.p, L.acc.p, gl[l], gl[l + 1], true);
    }
  } else {
    for (int l = 2; l <= NET_L0; ++l)
      launch_restrict(c->stream, 3, N.lv[l - 1].x.p, N.lv[l].x.p, gl[l - 1], gl[l], false);
    // Each coarser network on its own side stream, the finest on the main
    // one; a side stream also restricts its level's input (after its finer
    // neighbour's, event ev_x) and sums its coarser neighbour's correction
    // into its own (after ev_join of that neighbour), so that only the
    // finest level's transfers stay on the main stream.  Inside a stream
    // capture the events become edges between parallel graph branches.
    HX_CUDA(cudaEventRecord(N.ev_fork, c->stream));
    for (int l = NET_L0 + 1; l <= NET_TOP; ++l) {
      const int side = l - NET_L0 - 1;
      cudaStream_t ss = N.side[side];
      auto& L = N.lv[l];
      HX_CUDA(cudaStreamWaitEvent(ss, side == 0 ? N.ev_fork : N.ev_x[side - 1], 0));
      launch_restrict(ss, 3, N.lv[l - 1].x.p, L.x.p, gl[l - 1], gl[l], false);
      if (l < NET_TOP) HX_CUDA(cudaEventRecord(N.ev_x[side], ss));
      launch_lift(ss, L.x.p, L.feat.p, L.x0.p, gl[l]);
      stack_apply(c, ss, l - NET_L0, gl[l], L.x0.p, L.y.p, L.pp[0].p, L.pp[1].p);
    }
    // corrections, coarsest first: acc_l = E_l^T y_l + R^T acc_{l+1}
    for (int l = NET_TOP; l > NET_L0; --l) {
      const int side = l - NET_L0 - 1;
      cudaStream_t ss = N.side[side];
      auto& L = N.lv[l];
      launch_unlift(ss, L.y.p, L.feat.p, L.acc.p, false, nodes_of(gl[l]));
      if (l < NET_TOP) {
        HX_CUDA(cudaStreamWaitEvent(ss, N.ev_join[side + 1], 0));
        launch_prolong(ss, N.lv[l + 1].acc.p, L.acc.p, gl[l], gl[l + 1], true);
      }
      HX_CUDA(cudaEventRecord(N.ev_join[side], ss));
    }
    auto& L1 = N.lv[NET_L0];
    launch_lift(c->stream, L1.x.p, L1.feat.p, L1.x0.p, gl[NET_L0]);
    stack_apply(c, c->stream, 0, gl[NET_L0], L1.x0.p, L1.y.p, N.tmp[0].p, N.tmp[1].p);
    launch_unlift(c->stream, L1.y.p, L1.feat.p, L1.acc.p, false, nodes_of(gl[NET_L0]));
    if (NET_TOP > NET_L0) {
      HX_CUDA(cudaStreamWaitEvent(c->stream, N.ev_join[0], 0));
      launch_prolong(c->stream, N.lv[NET_L0 + 1].acc.p, L1.acc.p, gl[NET_L0], gl[NET_L0 + 1],
                     true);
    }
  }
  // levels below the networks: acc_l = R^T acc_{l+1}
  for (int l = NET_L0 - 1; l >= 1; --l)
    launch_prolong(c->stream, N.lv[l + 1].acc.p, N.lv[l].acc.p, gl[l], gl[l + 1], false);
  launch_net_output<T>(c->stream, r, minv, N.lv[1].acc.p, gl[0], gl[1], st, scale_mul, z, q_old,
                       c->d_partials.p);
}

// Jacobi scaling and density features of the current operator (after a
// solve set up M^-1 for `fac`).
void net_operator_inputs(hx_ctx* c, const double* fac) {
  auto& N = c->net;
  const int64_t n = c->g.dofs();
  HX_REQUIRE(c->d_minv.n >= (size_t)n, "no Jacobi data: run a solve on this grid first");
  net_buffers(c, false);
  launch_rho_feature(c->stream, fac, N.lv[0].feat.p, c->g);
  for (int l = 1; l <= NET_TOP; ++l)
    launch_restrict(c->stream, 1, N.lv[l - 1].feat.p, N.lv[l].feat.p, level_grid(c->g, l - 1),
                    level_grid(c->g, l), true);
  // private copy: training steps apply the operator long after the caller's call
  double* fb = N.facbuf.ensure(c->g.elems());
  if (fb != fac)
    HX_CUDA(cudaMemcpyAsync(fb, fac, c->g.elems() * sizeof(double), cudaMemcpyDeviceToDevice,
                            c->stream));
  N.fac_last = fb;
  N.prepared_dofs = n;
}

void require_prepared(hx_ctx* c) {
  HX_REQUIRE(c->net.ready, "network not initialised");
  HX_REQUIRE(c->net.fac_last != nullptr && c->net.prepared_dofs == c->g.dofs(),
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

// Host [node][16] (FP32; channels >= NET_IN ignored) -> a device activation
// in half-rows (act16), BF16.
static void upload_act16(hx_ctx* c, const GridN& g, const float* a, __nv_bfloat16* dst) {
  const int64_t nn = (int64_t)g.nx * g.ny * g.nz;
  std::vector<__nv_bfloat16> h((size_t)nn * 16);
  for (int64_t n = 0; n < nn; ++n) {
    const int64_t r = n / g.nx;
    const int x = (int)(n - r * g.nx);
    for (int ch = 0; ch < 16; ++ch)
      h[act16(g, r, x, ch >> 3) + (ch & 7)] =
          __float2bfloat16_rn(ch < NET_IN ? a[n * 16 + ch] : 0.f);
  }
  HX_CUDA(cudaMemcpyAsync(dst, h.data(), h.size() * 2, cudaMemcpyHostToDevice, c->stream));
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
  upload_act16(c, g, x0, bx0.p);
  stack_forward_train(c, 0, g, bx0.p, act, by.p);
  std::vector<__nv_bfloat16> hy((size_t)nn * 8);
  HX_CUDA(cudaMemcpyAsync(hy.data(), by.p, hy.size() * 2, cudaMemcpyDeviceToHost, c->stream));
  upload_act16(c, g, dy, N.da.p);
  HX_CUDA(cudaMemsetAsync(N.grad.p, 0, NET_PARAMS * sizeof(float), c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  stack_backward_train(c, 0, g, bx0.p, act, false);
  HX_CUDA(cudaMemcpyAsync(grads, N.grad.p, NET_PARAMS * sizeof(float), cudaMemcpyDeviceToHost,
                          c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  for (int64_t n = 0; n < nn; ++n)
    for (int ch = 0; ch < 16; ++ch)
      y[n * 16 + ch] = ch < 8 ? __bfloat162float(hy[n * 8 + ch]) : 0.f;
  check_conv_error(c);
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
  double* z = N.z.ensure(n);
  double* q = c->d_q.ensure(n);
  precond_z<double>(c, r, c->d_minv.p, s3, scale_mul, z, nullptr, true);
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
  launch_restrict_dof<double>(c->stream, gvec, c->d_minv.p, s3, s2, mode, scale_mul, N.lv[1].gx.p,
                      level_grid(g, 0), level_grid(g, 1));
  for (int l = 2; l <= NET_TOP; ++l)
    launch_restrict(c->stream, 3, N.lv[l - 1].gx.p, N.lv[l].gx.p, level_grid(g, l - 1),
                    level_grid(g, l), false);
  for (int l = NET_L0; l <= NET_TOP; ++l) {
    const GridN gl = level_grid(g, l);
    launch_lift(c->stream, N.lv[l].gx.p, N.lv[l].feat.p, N.da.p, gl);
    stack_backward_train(c, l - NET_L0, gl, N.lv[l].x0.p, N.lv[l].act, !first);
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
  check_conv_error(c);
  return sum / count;
}

void net_prepare(hx_ctx* c, const double* fac) { net_operator_inputs(c, fac); }

// Failure detection of the tensor-core convolution, without a fault: one CTA
// waits on a barrier nothing arrives on; its bounded wait must run out, set
// the error flag and return.  Then an ordinary convolution on the same
// context must succeed.  Returns whether the timeout was detected.
bool conv_wait_selftest(hx_ctx* c) {
  auto& N = c->net;
  net_alloc_params(c);
  const GridN g{8, 16, 4};
  const size_t a = (size_t)g.nx * g.ny * g.nz * 16;
  DevBuf<__nv_bfloat16> x, y;
  x.ensure(a);
  y.ensure(a);
  HX_CUDA(cudaMemsetAsync(x.p, 0, a * sizeof(__nv_bfloat16), c->stream));
  HX_CUDA(cudaMemsetAsync(N.wf.p, 0, NET_PARAMS * sizeof(__nv_bfloat16), c->stream));
  HX_CUDA(cudaMemsetAsync(N.err.p, 0, sizeof(int), c->stream));
  launch_conv3_selftest(c->stream, x.p, y.p, N.wf.p, N.err.p);
  int e = 0;
  HX_CUDA(cudaMemcpyAsync(&e, N.err.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  HX_CUDA(cudaMemsetAsync(N.err.p, 0, sizeof(int), c->stream));
  // the context stays usable: an ordinary layer runs and reports no error
  launch_conv3(c->stream, 16, x.p, y.p, N.wf.p, g, N.err.p);
  check_conv_error(c);
  if (N.ready) net_pack(c);  // restore the packed weights the test cleared
  HX_CUDA(cudaStreamSynchronize(c->stream));
  return e != 0;
}

// z = P r with the prepared operator (FP64 device vectors, grid numbering).
void net_apply_vec(hx_ctx* c, const double* r, double* z) {
  require_prepared(c);
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
  precond_z<double>(c, r, c->d_minv.p, s3, scale_mul, z, nullptr, false);
  check_conv_error(c);
}

std::function<void()> net_time_body(hx_ctx* c, int which) {
  require_prepared(c);
  auto& N = c->net;
  const Grid g = c->g;
  const int64_t n = g.dofs();
  HX_REQUIRE(c->d_b.n >= (size_t)n, "run a solve before timing the network");
  net_buffers(c, false);
  if (which == 0) {  // one 16 -> 16 layer on the finest network's grid
    const GridN g1 = level_grid(g, NET_L0);
    HX_CUDA(cudaMemsetAsync(N.tmp[0].p, 0, (size_t)nodes_of(g1) * 16 * sizeof(__nv_bfloat16),
                            c->stream));
    return [c, g1] {
      launch_conv3(c->stream, 16, c->net.tmp[0].p, c->net.tmp[1].p, fwd_w(c, 0, 1), g1,
                   c->net.err.p);
    };
  }
  // applied to the last solve's right-hand side b; state slot 3 holds b.M^-1 b
  CgState* s3 = c->d_state.p + 3;
  HX_CUDA(cudaMemsetAsync(s3, 0, sizeof(CgState), c->stream));
  launch_cg_init<double>(c->stream, c->d_b.p, nullptr, c->d_minv.p, c->d_aux1.ensure(n),
                         c->d_aux2.ensure(n), n, s3, c->d_partials.p);
  double* z = N.z.ensure(n);
  // as in the FCG loops: the restriction reads BF16(D^-1/2 b)
  __nv_bfloat16* ys = N.ys.ensure(n + 8);
  launch_dinv_bf16<double>(c->stream, c->d_b.p, c->d_minv.p, ys, n);
  return [c, s3, z, n, ys] {
    const double scale_mul = 1.0 / (double)n;
    precond_z<double>(c, c->d_b.p, c->d_minv.p, s3, scale_mul, z, nullptr, false, ys);
  };
}

// ---------------------------------------------------------------------------
// Flexible CG with the network preconditioner (FP64 vectors and operator,
// BF16 network).  Falls back to Jacobi-PCG from the current iterate when
// FCG breaks down, diverges, or stalls.
// ---------------------------------------------------------------------------
static CgState learned_fcg(hx_ctx* c, const double* fac, const double* b, double* x, bool warm,
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
  // ys = BF16(D^-1/2 r): formed here for the initial residual, then by
  // every residual update
  __nv_bfloat16* ys = N.ys.ensure(n + 8);
  launch_dinv_bf16<double>(c->stream, r, minv, ys, n);
  auto one = [&](double* pin, double* pout) {
    precond_z<double>(c, r, minv, st, scale_mul, z, q, false, ys);
    launch_fcg_step<double>(c->stream, pin, pout, z, x, q, fac, c->d_nmask.p, g, c->K, shift,
                            st, c->d_partials.p);
    launch_cg_update2<double>(c->stream, r, q, minv, n, st, c->d_partials.p, ys);
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
  // One graph, checked between launches for stagnation: no 10% gain on the
  // best residual within max(500, iterations / 4) iterations.  (CG
  // residuals are not monotone and on hard problems halve only every few
  // hundred iterations, so a tighter test would misfire.)
  auto keep_going = [&](const CgState& sv) {
    if (sv.rel_res < 0.9 * best) {
      best = sv.rel_res;
      best_it = sv.iter;
    }
    stalled = !o.learned_no_fallback && sv.iter - best_it > std::max(500, sv.iter / 4);
    return !stalled;
  };
  sf = run_batched(c, 0, reps, body, o.wall_limit_ms, t0, timed_out, 0, keep_going);
  if (sf.status != HX_RUNNING) stalled = false;
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

// ---------------------------------------------------------------------------
// Mixed precision learned FCG.  The FCG iteration (preconditioner, fused
// step, residual update) runs on FP32 vectors and the FP32 operator, with
// FP64 reductions, and accumulates its correction in d32.  Reliable updates
// as in solve_mixed: after each batch (which also ends when the recursive
// residual has dropped by opts.inner_tol since the last replacement, or
// claims convergence) d32 is folded into the FP64 x, the true residual
// b - (K+sI)x is recomputed in FP64 and replaces the FP32 one, and the
// iteration resumes with the same direction: p_old, q_old = K p_old and
// p_old.q_old are kept, so the next flexible-CG coefficient is formed as
// usual; alpha = 0 so the folded step is not applied twice.  Convergence is
// judged only on the FP64 true residual.  Falls back to mixed Jacobi-PCG
// from the current iterate when FCG breaks down or stalls (stagnation is
// measured on the true residual).
// ---------------------------------------------------------------------------
// multigrid: the FP32 V-cycle (hx_gmg.cu) as the variable preconditioner
// in place of the networks; everything else is shared.
static CgState learned_fcg_mixed(hx_ctx* c, const double* fac, const double* b, double* x,
                                 bool warm, double shift, const hx_solve_opts& o, double t0,
                                 bool* timed_out, int* fallback, int* iters_out,
                                 bool multigrid = false) {
  HX_REQUIRE(multigrid || c->net.ready,
             "learned preconditioner requested but no network is loaded");
  auto& N = c->net;
  const Grid& g = c->g;
  const int64_t n = g.dofs(), ne = g.elems();
  if (multigrid) {
    c->gmg.degree = o.mg_smooth_degree > 0 ? o.mg_smooth_degree : GMG_DEFAULT_DEGREE;
    gmg_setup(c, fac, shift);
  } else {
    net_operator_inputs(c, fac);
  }
  float* fac32 = c->d_fac32.ensure(ne);
  float* minv32 = c->d_minv32.ensure(n);
  float* r32 = c->d_r32.ensure(n);
  float* P0 = c->d_p32.ensure(n);
  float* P1 = c->d_p32b.ensure(n);
  float* q32 = c->d_q32.ensure(n);
  float* d32 = c->d_x32.ensure(n);
  float* z32 = N.z32.ensure(n);
  float* s32 = N.s32.ensure(n);  // scratch output of cg_init
  double* q = c->d_q.ensure(n);
  launch_convert<float, double>(c->stream, fac32, fac, ne);
  launch_convert<float, double>(c->stream, minv32, c->d_minv.p, n);
  const ElemCoef<float> K32 = to_float(c->K);
  const float sh32 = (float)shift;
  CgState* so = c->d_state.p;      // FP64 outer: ||b||, true residual
  CgState* si = c->d_state.p + 1;  // FP32 FCG iteration
  const double scale_mul = 1.0 / (double)n;
  *fallback = 0;
  *iters_out = 0;
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
  if (so_h.status != HX_RUNNING || o.max_iter <= 0) return so_h;
  // FP32 iteration state: rz, rr of the replaced residual; no previous
  // direction (p_old = q_old = 0, pq = 0 gives beta = 0, alpha = 0)
  // multigrid drops the residual ~5x per iteration: replace after inner_tol^3
  const double d1 = (o.inner_tol > 0 && o.inner_tol < 1) ? o.inner_tol : 0.1;
  const double delta = multigrid ? d1 * d1 * d1 : d1;
  put_state(c, 1, fresh_state(o.tol, o.max_iter, 1, false, false));
  launch_fill_zero(c->stream, d32, n * sizeof(float));
  launch_fill_zero(c->stream, P1, n * sizeof(float));
  launch_fill_zero(c->stream, q32, n * sizeof(float));
  launch_cg_init<float>(c->stream, r32, nullptr, minv32, r32, s32, n, si, c->d_partials.p);
  CgState st = get_state(c, 1);
  st.bnorm = 1.0;
  st.alpha = 0.0;
  st.beta = 0.0;
  st.pq = 0.0;
  st.aux[1] = delta;
  st.aux[2] = st.rr;
  st.max_iter = o.max_iter;
  put_state(c, 1, st);
  // the V-cycle's kernels run whole after the state has stopped: batches of
  // two iterations for multigrid (tens of iterations per solve)
  const int reps = multigrid ? 1 : std::max(1, auto_batch(g, o.check_every) / 2);
  int parity = 0;  // which P buffer holds p_{k-1}: P1 when parity == 0
  double best = so_h.rel_res;
  int best_it = 0;
  bool stalled = false;
  CgState sf{};
  __nv_bfloat16* ys = multigrid ? nullptr : N.ys.ensure(n + 8);
  for (;;) {
    float* Pin = parity ? P0 : P1;
    float* Pout = parity ? P1 : P0;
    // ys = BF16(D^-1/2 r32) of the (replaced) residual; then every residual
    // update keeps it current
    if (!multigrid) launch_dinv_bf16<float>(c->stream, r32, minv32, ys, n);
    auto one = [&](float* pi, float* po) {
      if (multigrid) {
        gmg_vcycle<float>(c, r32, z32);
        launch_fcg_coeffs<float>(c->stream, z32, q32, r32, n, c->d_partials.p, si);
      } else {
        precond_z<float>(c, r32, minv32, si, scale_mul, z32, q32, false, ys);
      }
      launch_fcg_step<float>(c->stream, pi, po, z32, d32, q32, fac32, c->d_nmask.p, g, K32,
                             sh32, si, c->d_partials.p);
      launch_cg_update2<float>(c->stream, r32, q32, minv32, n, si, c->d_partials.p, ys);
    };
    auto body = [&]() {
      one(Pin, Pout);
      one(Pout, Pin);
    };
    // a batch ends on a reliable-update pause, convergence, failure, or
    // stagnation of the recursive residual (relative to ||b||, as the true
    // one) by the test of solve_learned
    auto keep_going = [&](const CgState& sv) {
      if (sv.rel_res < 0.9 * best) {
        best = sv.rel_res;
        best_it = sv.iter;
      }
      stalled = !o.learned_no_fallback && sv.iter - best_it > std::max(500, sv.iter / 4);
      return !stalled;
    };
    const int it_before = st.iter;
    sf = run_batched(c, 1, reps, body, o.wall_limit_ms, t0, timed_out, 0, keep_going);
    const int done = sf.iter - it_before;
    *iters_out += done;
    float* pk = (done % 2 == 1) ? Pout : Pin;  // p of the last completed iteration
    if (done % 2 == 1) parity ^= 1;
    if (sf.status != HX_ST_BREAKDOWN && done > 0)
      launch_axpy_state<float>(c->stream, d32, d32, pk, n, si, 0);  // pending step
    // fold the FP32 correction into x and replace the residual in FP64
    launch_ir_correct(c->stream, x, d32, n, so);
    launch_fill_zero(c->stream, d32, n * sizeof(float));
    launch_matvec<double>(c->stream, 0, x, q, fac, c->d_nmask.p, g, c->K, shift,
                          c->d_state.p + 3, c->d_partials.p, nullptr);
    launch_ir_residual(c->stream, b, q, r32, n, so, c->d_partials.p);
    so_h = get_state(c, 0);
    so_h.iter = *iters_out;
    if (so_h.status != HX_RUNNING) return so_h;  // converged on the true residual (or non-finite)
    const bool broke = sf.status == HX_ST_BREAKDOWN || sf.status == HX_ST_NONFINITE ||
                       sf.status == HX_ST_DIVERGED;
    if (sf.status != HX_RUNNING) stalled = false;
    if (*timed_out || broke || stalled || *iters_out >= o.max_iter) break;
    // resume: rz, rr of the replaced residual; p_old, q_old, pq kept; alpha = 0
    st = get_state(c, 1);
    launch_cg_init<float>(c->stream, r32, nullptr, minv32, r32, s32, n, si, c->d_partials.p);
    CgState s2 = get_state(c, 1);
    s2.bnorm = 1.0;
    s2.alpha = 0.0;
    s2.beta = st.beta;
    s2.pq = st.pq;
    s2.iter = sf.iter;
    s2.aux[1] = delta;
    s2.aux[2] = s2.rr;
    s2.max_iter = o.max_iter;
    s2.status = HX_RUNNING;
    put_state(c, 1, s2);
    st = s2;
  }
  const bool broke = sf.status == HX_ST_BREAKDOWN || sf.status == HX_ST_NONFINITE ||
                     sf.status == HX_ST_DIVERGED;
  if (*timed_out || o.learned_no_fallback || !(broke || stalled)) {
    so_h.status = broke ? sf.status : HX_ST_MAXITER;
    return so_h;
  }
  // fallback: mixed Jacobi-PCG warm-started from the current iterate
  *fallback = 1;
  hx_solve_opts oj = o;
  oj.max_iter = std::max(1, o.max_iter - *iters_out);
  int inner = 0;
  CgState sj = solve_mixed(c, fac, b, x, true, shift, oj, t0, timed_out, &inner);
  *iters_out += inner;
  return sj;
}

CgState solve_learned(hx_ctx* c, const double* fac, const double* b, double* x, bool warm,
                      double shift, const hx_solve_opts& o, double t0, bool* timed_out,
                      int* fallback, int* iters_out) {
  const CgState s = learned_fcg(c, fac, b, x, warm, shift, o, t0, timed_out, fallback, iters_out);
  check_conv_error(c);
  return s;
}

CgState solve_learned_mixed(hx_ctx* c, const double* fac, const double* b, double* x, bool warm,
                            double shift, const hx_solve_opts& o, double t0, bool* timed_out,
                            int* fallback, int* iters_out) {
  const CgState s =
      learned_fcg_mixed(c, fac, b, x, warm, shift, o, t0, timed_out, fallback, iters_out);
  check_conv_error(c);
  return s;
}

CgState solve_gmg_mixed(hx_ctx* c, const double* fac, const double* b, double* x, bool warm,
                        double shift, const hx_solve_opts& o, double t0, bool* timed_out,
                        int* fallback, int* iters_out) {
  return learned_fcg_mixed(c, fac, b, x, warm, shift, o, t0, timed_out, fallback, iters_out,
                           true);
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
