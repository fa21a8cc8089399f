// hx_gmg.cu -- geometric multigrid on the voxel grid: the robust
// preconditioner that replaces the reference's CPU algebraic multigrid
// (src/Solvers/GPUSolver.jl:168-268 assembles the matrix on the host and
// builds AlgebraicMultigrid's smoothed aggregation; every PCG iteration then
// copies r to the host and z back, :513-516).  Here nothing leaves the GPU
// and no matrix is assembled.
//
// Hierarchy: level l+1 halves every element count of level l (built while
// all three are even); its element factor is the mean of its 8 children and
// its element size doubles, so the coarse operator is the same matrix-free
// structured operator (hx_operator.cu) on the coarse grid, with 8 times the
// finer level's diagonal shift.  A coarse node is
// the fine node at twice its index; it is fixed where that fine node's BC
// bit is set, and nodes without stiffness are held at 0 as on level 0.
// Transfers: trilinear prolongation P and its exact transpose R = P^T
// (full weighting), the kernels of the learned preconditioner's levels.
//
// Levels are added until one has at most GMG_STOP_DOFS DOFs (or an element
// count turns odd).
//
// V-cycle (FP32): on each level Chebyshev smoothing of degree G.degree
// (hx_solve_opts.mg_smooth_degree, default GMG_DEFAULT_DEGREE)
// with Jacobi scaling on [0.05, 1.1] x lambda_max(D^-1 A) (a Lanczos
// estimate from Jacobi-PCG steps at set-up), from zero before the restriction and from the
// prolonged correction after it.  The coarsest level, when it has at most
// GMG_DIRECT_DOFS DOFs, is solved by its dense inverse: assembled from the
// element matrices and inverted by blocked Gauss-Jordan in FP64 at set-up, applied
// as one FP32 matrix-vector product per cycle; a larger coarsest level gets
// GMG_COARSE_ITERS iterations of FP32 Jacobi-PCG on the fused kernels.  The
// cycle is symmetric positive definite up to FP32 rounding (and a PCG coarse
// solve's early stop), which the flexible CG around it absorbs (Notay's FCG,
// the same step kernels as the learned preconditioner).
#include <chrono>
#include <cmath>
#include <limits>
#include <type_traits>
#include <vector>

#include "hx_cnn.h"
#include "hx_solver.h"

namespace hx {

namespace {

constexpr int GMG_COARSE_ITERS = 64;   // PCG iterations on a large coarsest level
constexpr int64_t GMG_STOP_DOFS = 1536;    // coarsen until a level has at most this many DOFs
constexpr int64_t GMG_DIRECT_DOFS = 2048;  // coarsest levels up to this size are solved directly
constexpr float GMG_LO = 0.05f, GMG_HI = 1.1f;  // Chebyshev range / lambda_max
constexpr int GMG_LANCZOS = 12;                  // PCG steps of the lambda_max estimate

__device__ __forceinline__ int64_t gt() { return blockIdx.x * (int64_t)blockDim.x + threadIdx.x; }
__device__ __forceinline__ int64_t gs() { return (int64_t)gridDim.x * blockDim.x; }

// coarse element factor = mean of its 8 children
__global__ void k_coarse_fac(const float* __restrict__ ff, float* __restrict__ fc, Grid gf,
                             Grid gc) {
  const int64_t ne = gc.elems();
  for (int64_t e = gt(); e < ne; e += gs()) {
    const int i = (int)(e % gc.nxe);
    const int64_t t = e / gc.nxe;
    const int j = (int)(t % gc.nye), k = (int)(t / gc.nye);
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int fi = 2 * i + (c & 1), fj = 2 * j + ((c >> 1) & 1), fk = 2 * k + (c >> 2);
      s += ff[((int64_t)fk * gf.nye + fj) * gf.nxe + fi];
    }
    fc[e] = 0.125f * s;
  }
}

// coarse node BC bits = those of the fine node at twice its index
__global__ void k_coarse_bc(const uint8_t* __restrict__ bf, uint8_t* __restrict__ bc, Grid gf,
                            Grid gc) {
  const int64_t nn = gc.nodes();
  for (int64_t n = gt(); n < nn; n += gs()) {
    const int i = (int)(n % gc.nxn);
    const int64_t t = n / gc.nxn;
    const int j = (int)(t % gc.nyn), k = (int)(t / gc.nyn);
    bc[n] = bf[((int64_t)(2 * k) * gf.nyn + 2 * j) * gf.nxn + 2 * i];
  }
}

// first Chebyshev step from x = 0: x = (1/theta) M^-1 b
__global__ void k_cheb_first(const float* __restrict__ b, const float* __restrict__ minv,
                             float* __restrict__ x, float inv_theta, int64_t n) {
  for (int64_t i = gt(); i < n; i += gs()) x[i] = inv_theta * minv[i] * b[i];
}

template <typename TD, typename TS>
__global__ void k_copy_cvt(TD* __restrict__ d, const TS* __restrict__ s, int64_t n) {
  for (int64_t i = gt(); i < n; i += gs()) d[i] = (TD)s[i];
}

// a pseudo-random vector (hash of the index), zero on fixed DOFs: the
// right-hand side of the lambda_max estimate
__global__ void k_rand_vec(float* __restrict__ v, const uint8_t* __restrict__ nmask, int64_t nn) {
  for (int64_t i = gt(); i < 3 * nn; i += gs()) {
    uint32_t h = (uint32_t)i * 2654435761u + 0x9E3779B9u;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    const float u = (float)(h & 0xFFFFFF) / 16777216.f - 0.5f;
    v[i] = ((nmask[i / 3] >> (i % 3)) & 1u) ? u : 0.f;
  }
}

// (alpha, beta, status) of the last PCG step, for the lambda_max estimate
__global__ void k_record_step(const CgState* st, double* out) {
  if (threadIdx.x == 0) {
    out[0] = st->alpha;
    out[1] = st->beta;
    out[2] = (double)st->status;
  }
}

// fresh coarse-solve state (inside a captured cycle: no host round trip)
__global__ void k_coarse_reset(CgState* st, int max_iter, double tol) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    st->iter = 0;
    st->max_iter = max_iter;
    st->tol = tol;
    st->status = HX_RUNNING;
    st->check_every = 1;
    st->explode = 0.0;
    st->div_ratio = 0.0;
    st->keep_best = 0;
    st->alpha = 0.0;
    st->beta = 0.0;
    st->aux[1] = 0.0;
    st->best_rel = INFINITY;
  }
}

// the pending x += alpha p_k of the last coarse PCG iteration, p_k picked
// by the iteration count's parity (iteration k writes p into P[k % 2])
__global__ void k_coarse_finish(float* __restrict__ x, const float* __restrict__ p0,
                                const float* __restrict__ p1, const CgState* st, int64_t n) {
  const int it = st->iter;
  if (st->status == HX_ST_BREAKDOWN || it <= 0) return;
  const float* pk = ((it - 1) % 2 == 0) ? p0 : p1;
  const float a = (float)st->alpha;
  for (int64_t i = gt(); i < n; i += gs()) x[i] += a * pk[i];
}

// flexible-CG coefficients for a preconditioned residual z: beta =
// -(z.q_old) / (p_old.q_old) (st->pq), st->aux[3] = z.r (the step length's
// numerator, used by the flexible-CG step)
template <typename T>
__global__ void k_fcg_coeffs(const T* __restrict__ z, const T* __restrict__ q_old,
                             const T* __restrict__ r, int64_t n, double* partials, CgState* st) {
  if (st->status != HX_RUNNING) return;
  double zq = 0.0, zr = 0.0;
  for (int64_t i = gt(); i < n; i += gs()) {
    zq += (double)z[i] * (double)q_old[i];
    zr += (double)z[i] * (double)r[i];
  }
  double v[2] = {zq, zr};
  if (grid_reduce<2>(v, partials, &st->ticket[TK_AUX2]) && threadIdx.x == 0) {
    const double pq = st->pq;
    st->beta = (pq > 0.0 && isfinite(v[0])) ? -v[0] / pq : 0.0;
    st->aux[3] = v[1];
  }
}

// Dense FP64 operator of a (small) level: every element adds f Ke, its
// 24 x 24 stiffness, at its nodes' DOFs (one thread per element and column:
// the column is Ke applied to a unit vector).  A must be zero on entry.
__global__ void k_dense_assemble(const float* __restrict__ fac, Grid g, ElemCoef<double> K,
                                 double* __restrict__ A, int64_t n) {
  const int64_t ne = g.elems();
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ne * 24;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / 24;
    const int col = (int)(t - e * 24), cc = col / 8, cb = col % 8;
    const int i = (int)(e % g.nxe);
    const int64_t r = e / g.nxe;
    const int j = (int)(r % g.nye), k = (int)(r / g.nye);
    double u[3][8], y[3][8];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int b = 0; b < 8; ++b) u[c][b] = (c == cc && b == cb) ? 1.0 : 0.0;
    elem_apply(K, (double)fac[e], u, y);
    auto dof = [&](int b, int c) -> int64_t {
      const int64_t node = ((int64_t)(k + (b >> 2)) * g.nyn + j + ((b >> 1) & 1)) * g.nxn + i +
                           (b & 1);
      return 3 * node + c;
    };
    const int64_t dc = dof(cb, cc);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int b = 0; b < 8; ++b)
        if (y[c][b] != 0.0) atomicAdd(&A[dof(b, c) * n + dc], y[c][b]);
  }
}

// Fixed DOFs (mask bit clear) get identity rows and columns; free ones the
// shift on the diagonal -- the operator the structured kernels apply.
__global__ void k_dense_mask(double* __restrict__ A, const uint8_t* __restrict__ nmask,
                             double shift, int64_t n) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n * n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / n, j = t - i * n;
    const bool fi = (nmask[i / 3] >> (i % 3)) & 1u, fj = (nmask[j / 3] >> (j % 3)) & 1u;
    if (!fi || !fj)
      A[t] = (i == j) ? 1.0 : 0.0;
    else if (i == j)
      A[t] += shift;
  }
}

// Blocked in-place Gauss-Jordan inversion (no pivoting: the matrix is
// symmetric positive definite), GJB pivots per step.  With K the step's
// block of rows and columns, P = inv(A_KK):
//   A_KJ <- P A_KJ,  A_IJ <- A_IJ - A_IK P A_KJ,  A_IK <- -A_IK P,  A_KK <- P
// (I, J outside K), in three launches: the pivot block's inverse, the row
// panel P A_KJ and a copy of the column panel A_IK into buffers, and the
// update of every other entry from the buffers (so no entry is read after
// another thread rewrote it).
constexpr int GJB = 32;

// A_KK <- inv(A_KK) in shared memory: unblocked Gauss-Jordan, one thread
// per entry (GJB x GJB threads), b <= GJB rows.
__global__ void k_gj_pivot_block(double* __restrict__ A, int64_t n, int64_t k0, int b) {
  __shared__ double P[GJB][GJB + 1];
  const int i = threadIdx.y, j = threadIdx.x;
  const bool in = i < b && j < b;
  P[i][j] = in ? A[(k0 + i) * n + k0 + j] : 0.0;
  __syncthreads();
  for (int k = 0; k < b; ++k) {
    const double inv = 1.0 / P[k][k];
    const double aik = P[i][k], akj = P[k][j], aij = P[i][j];
    double v;
    if (i == k && j == k)
      v = inv;
    else if (i == k)
      v = akj * inv;
    else if (j == k)
      v = -aik * inv;
    else
      v = aij - aik * akj * inv;
    __syncthreads();
    P[i][j] = v;
    __syncthreads();
  }
  if (in) A[(k0 + i) * n + k0 + j] = P[i][j];
}

// rowbuf[m][j] = (P A_KJ)[m][j] for every column j (used for j outside K);
// colbuf[i][m] = A[i][k0 + m] for every row i (used for i outside K).
__global__ void k_gj_panels(const double* __restrict__ A, int64_t n, int64_t k0, int b,
                            double* __restrict__ rowbuf, double* __restrict__ colbuf) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < b * n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = t / n, j = t - m * n;
    double s = 0.0;
    for (int q = 0; q < b; ++q) s += A[(k0 + m) * n + k0 + q] * A[(k0 + q) * n + j];
    rowbuf[m * n + j] = s;
    const int64_t i = t / b, m2 = t - i * b;
    colbuf[i * GJB + m2] = A[i * n + k0 + m2];
  }
}

__global__ void k_gj_update(double* __restrict__ A, int64_t n, int64_t k0, int b,
                            const double* __restrict__ rowbuf, const double* __restrict__ colbuf) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n * n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / n, j = t - i * n;
    const bool iK = i >= k0 && i < k0 + b, jK = j >= k0 && j < k0 + b;
    if (iK) {
      if (!jK) A[t] = rowbuf[(i - k0) * n + j];
    } else if (jK) {
      double s = 0.0;
      for (int m = 0; m < b; ++m) s += colbuf[i * GJB + m] * A[(k0 + m) * n + j];
      A[t] = -s;
    } else {
      double s = A[t];
      for (int m = 0; m < b; ++m) s -= colbuf[i * GJB + m] * rowbuf[m * n + j];
      A[t] = s;
    }
  }
}

template <typename TD>
__global__ void k_cvt_f64(TD* __restrict__ d, const double* __restrict__ s, int64_t n) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    d[t] = (TD)s[t];
}

// x = Ainv b (n x n, FP32): one warp per row, b read through the cache
__global__ void k_dense_gemv(const float* __restrict__ Ainv, const float* __restrict__ b,
                             float* __restrict__ x, int64_t n) {
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= n) return;
  const float* row = Ainv + w * n;
  float s = 0.f;
  for (int64_t j = lane; j < n; j += 32) s = fmaf(row[j], __ldg(&b[j]), s);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) x[w] = s;
}

// Largest eigenvalue of the Lanczos tridiagonal T of a PCG run (alpha_j,
// beta_j its step lengths and direction coefficients): T_jj = 1/alpha_j +
// beta_{j-1}/alpha_{j-1}, T_j,j+1 = sqrt(beta_j)/alpha_j; by bisection on
// the Sturm count, from the Gershgorin bound down.
double lanczos_max(const std::vector<double>& al, const std::vector<double>& be) {
  const size_t k = al.size();
  std::vector<double> d(k), e(k, 0.0);
  for (size_t j = 0; j < k; ++j) {
    d[j] = 1.0 / al[j] + (j > 0 ? be[j - 1] / al[j - 1] : 0.0);
    if (j + 1 < k) e[j] = std::sqrt(std::max(be[j], 0.0)) / al[j];
  }
  double lo = 0.0, hi = 0.0;
  for (size_t j = 0; j < k; ++j)
    hi = std::max(hi, d[j] + std::fabs(e[j]) + (j > 0 ? std::fabs(e[j - 1]) : 0.0));
  // eigenvalues below x: sign changes of the LDL^T pivots of T - x I
  auto below = [&](double x) {
    int cnt = 0;
    double q = 1.0;
    for (size_t j = 0; j < k; ++j) {
      const double off = j > 0 ? e[j - 1] * e[j - 1] : 0.0;
      q = d[j] - x - (j > 0 ? off / q : 0.0);
      if (q == 0.0) q = -1e-300;
      if (q < 0.0) ++cnt;
    }
    return cnt;
  };
  for (int it = 0; it < 100; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (below(mid) >= (int)k) hi = mid; else lo = mid;
  }
  return hi;
}

unsigned gblocks(int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, 256), 16LL * sm_count()));
}

GridN node_grid(const Grid& g) { return GridN{g.nxn, g.nyn, g.nzn}; }

}  // namespace

// ---------------------------------------------------------------------------
// Hierarchy set-up for the factors `fac` (FP64, level 0) with the solve's
// node mask and M^-1 (c->d_nmask, c->d_minv, already set up with `shift`).
// ---------------------------------------------------------------------------
void gmg_setup(hx_ctx* c, const double* fac, double shift) {
  auto& G = c->gmg;
  const auto t_start = std::chrono::steady_clock::now();
  cudaStream_t s = c->stream;
  G.nl = 0;
  Grid g = c->g;
  double h[3] = {c->h[0], c->h[1], c->h[2]};
  for (int l = 0; l < HX_GMG_MAX_LEVELS; ++l) {
    auto& L = G.lv[l];
    L.g = g;
    for (int a = 0; a < 3; ++a) L.h[a] = h[a];
    const int64_t nn = g.nodes(), n = g.dofs(), ne = g.elems();
    L.K = to_float(make_elem_coef(h[0], h[1], h[2], c->nu));
    float* fl = L.fac.ensure(ne);
    uint8_t* bc = L.bc.ensure(nn);
    uint8_t* nm = L.nmask.ensure(nn);
    float* minv = L.minv.ensure(n);
    L.b.ensure(n);
    L.x.ensure(n);
    L.r.ensure(n);
    L.d.ensure(n);
    L.q.ensure(n);
    if (l == 0) {
      k_copy_cvt<float, double><<<gblocks(ne), 256, 0, s>>>(fl, fac, ne);
      HX_CHECK_LAUNCH();
      HX_CUDA(cudaMemcpyAsync(bc, c->d_bcfree.p, nn, cudaMemcpyDeviceToDevice, s));
      HX_CUDA(cudaMemcpyAsync(nm, c->d_nmask.p, nn, cudaMemcpyDeviceToDevice, s));
      k_copy_cvt<float, double><<<gblocks(n), 256, 0, s>>>(minv, c->d_minv.p, n);
      HX_CHECK_LAUNCH();
      L.shift = (float)shift;
    } else {
      const auto& F = G.lv[l - 1];
      k_coarse_fac<<<gblocks(ne), 256, 0, s>>>(F.fac.p, fl, F.g, g);
      HX_CHECK_LAUNCH();
      k_coarse_bc<<<gblocks(nn), 256, 0, s>>>(F.bc.p, bc, F.g, g);
      HX_CHECK_LAUNCH();
      // the fine level's shift s I seen through the transfers: P^T (s I) P
      // has row sums 8 s (trilinear P), so a coarse level carries 8 times
      // its parent's shift on the diagonal.  A shift that regularises a
      // free rigid mode on the mesh then keeps the coarse operators (and
      // the dense coarsest inverse) nonsingular too.
      L.shift = 8.f * F.shift;
      put_state(c, 3, CgState{});
      launch_node_diag<float>(s, fl, bc, nm, minv, g, make_elem_coef(h[0], h[1], h[2], c->nu),
                              c->d_partials.p, c->d_state.p + 3, c->d_scalars.p);
      launch_minv<float>(s, nm, minv, minv, nn, (double)L.shift);
      HX_CUDA(cudaStreamSynchronize(s));  // the pinned state mirror is reused below
    }
    G.nl = l + 1;
    const bool even = g.nxe % 2 == 0 && g.nye % 2 == 0 && g.nze % 2 == 0;
    if (!even || n <= GMG_STOP_DOFS || g.nxe < 4 || g.nye < 4 || g.nze < 4) break;
    Grid gc{};
    gc.nxe = g.nxe / 2;
    gc.nye = g.nye / 2;
    gc.nze = g.nze / 2;
    gc.nxn = gc.nxe + 1;
    gc.nyn = gc.nye + 1;
    gc.nzn = gc.nze + 1;
    g = gc;
    for (int a = 0; a < 3; ++a) h[a] *= 2.0;
  }
  // lambda_max(D^-1 A) of every smoothed level (all but the coarsest), from
  // the Lanczos tridiagonal of GMG_LANCZOS Jacobi-PCG steps on a random
  // right-hand side.  The largest Ritz value converges to lambda_max from
  // below much faster than power iteration; an estimate below lambda_max
  // leaves the top of the spectrum outside the Chebyshev interval, where
  // the smoother is not positive definite.
  G.p0.ensure(G.lv[0].g.dofs());
  G.p1.ensure(G.lv[0].g.dofs());
  for (int l = 0; l + 1 < G.nl; ++l) {
    auto& L = G.lv[l];
    const int64_t nn = L.g.nodes(), n = L.g.dofs();
    CgState* st = c->d_state.p + 3;
    k_rand_vec<<<gblocks(n), 256, 0, s>>>(L.b.p, L.nmask.p, nn);
    HX_CHECK_LAUNCH();
    launch_fill_zero(s, L.x.p, n * sizeof(float));
    put_state(c, 3, fresh_state(0.0, 1 << 30, 1, false, false));
    launch_cg_init<float>(s, L.b.p, nullptr, L.minv.p, L.r.p, G.p1.p, n, st, c->d_partials.p);
    // all steps queued at once; each leaves (alpha, beta, status) in rec
    double* rec = G.lanczos.ensure(3 * GMG_LANCZOS);
    for (int it = 0; it < GMG_LANCZOS; ++it) {
      float* pin = (it % 2 == 0) ? G.p1.p : G.p0.p;
      float* pout = (it % 2 == 0) ? G.p0.p : G.p1.p;
      launch_pcg_step<float>(s, pin, pout, L.r.p, L.minv.p, L.x.p, L.q.p, L.fac.p, L.nmask.p, L.g,
                             L.K, L.shift, st, c->d_partials.p);
      launch_cg_update2<float>(s, L.r.p, L.q.p, L.minv.p, n, st, c->d_partials.p);
      k_record_step<<<1, 32, 0, s>>>(st, rec + 3 * it);
      HX_CHECK_LAUNCH();
    }
    double h[3 * GMG_LANCZOS];
    HX_CUDA(cudaMemcpyAsync(h, rec, sizeof(h), cudaMemcpyDeviceToHost, s));
    HX_CUDA(cudaStreamSynchronize(s));
    std::vector<double> al, be;
    for (int it = 0; it < GMG_LANCZOS; ++it) {
      const double a = h[3 * it], bt = h[3 * it + 1];
      const int stt = (int)h[3 * it + 2];
      if (stt == HX_ST_BREAKDOWN || !(a > 0.0) || !std::isfinite(a)) break;
      al.push_back(a);
      be.push_back(bt);
      if (stt != HX_RUNNING) break;
    }
    L.lmax = al.empty() ? 2.0f : (float)lanczos_max(al, be);
  }
  // Coarsest level: its dense inverse when small enough (blocked
  // Gauss-Jordan in FP64), else a fixed-count FP32 PCG at every cycle.
  {
    auto& L = G.lv[G.nl - 1];
    const int64_t n = L.g.dofs();
    G.direct = n <= GMG_DIRECT_DOFS;
    if (G.direct) {
      const int64_t nn2 = n * n;
      double* A = G.dense.ensure(nn2);
      double* gj = G.gj.ensure(2 * GJB * n);  // row panel [GJB][n], column panel [n][GJB]
      HX_CUDA(cudaMemsetAsync(A, 0, nn2 * sizeof(double), s));
      const ElemCoef<double> K = make_elem_coef(L.h[0], L.h[1], L.h[2], c->nu);
      k_dense_assemble<<<gblocks(L.g.elems() * 24), 256, 0, s>>>(L.fac.p, L.g, K, A, n);
      HX_CHECK_LAUNCH();
      k_dense_mask<<<gblocks(nn2), 256, 0, s>>>(A, L.nmask.p, (double)L.shift, n);
      HX_CHECK_LAUNCH();
      for (int64_t k0 = 0; k0 < n; k0 += GJB) {
        const int b = (int)std::min<int64_t>(GJB, n - k0);
        k_gj_pivot_block<<<1, dim3(GJB, GJB), 0, s>>>(A, n, k0, b);
        HX_CHECK_LAUNCH();
        k_gj_panels<<<gblocks(b * n), 256, 0, s>>>(A, n, k0, b, gj, gj + GJB * n);
        HX_CHECK_LAUNCH();
        k_gj_update<<<gblocks(nn2), 256, 0, s>>>(A, n, k0, b, gj, gj + GJB * n);
        HX_CHECK_LAUNCH();
      }
      k_cvt_f64<float><<<gblocks(nn2), 256, 0, s>>>(G.ainv.ensure(nn2), A, nn2);
      HX_CHECK_LAUNCH();
    }
  }
  // the coarse solve's state: zeroed once, so that its reduction tickets
  // start at 0 (k_coarse_reset renews the other fields every cycle)
  if (!G.coarse_st.p) {
    G.coarse_st.ensure(1);
    HX_CUDA(cudaMemsetAsync(G.coarse_st.p, 0, sizeof(CgState), s));
  }
  G.p0.ensure(G.lv[G.nl - 1].g.dofs());
  G.p1.ensure(G.lv[G.nl - 1].g.dofs());
  G.ready = true;
  HX_CUDA(cudaStreamSynchronize(s));
  G.setup_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() -
                                                          t_start).count();
}

// Chebyshev smoothing of A x = b on level L (c->gmg.degree steps, Jacobi
// scaling on [GMG_LO, GMG_HI] lambda_max): from x = 0 when xzero, else from
// x; leaves r = b - A x in L.r when want_residual.  Three-term form:
//   x_1 = x_0 + (1/theta) M^-1 (b - A x_0),
//   x_{k+1} = x_k + rho_k rho_{k-1} (x_k - x_{k-1}) + (2 rho_k / delta) M^-1 (b - A x_k),
// rho_0 = 1/sigma, rho_k = 1/(2 sigma - rho_{k-1}): each step is one operator
// launch whose epilogue forms x_{k+1} (MODE 5 of the structured kernel).
// x_k and x_{k-1} alternate between x and L.d; the start is chosen so
// that the result lands in x.
static void cheb_smooth(hx_ctx* c, hx_ctx::GmgLevel& L, const float* b, float* x, bool xzero,
                        bool want_residual) {
  cudaStream_t s = c->stream;
  const int64_t n = L.g.dofs();
  const int m = c->gmg.degree;
  const float lmax = L.lmax;
  const float lo = GMG_LO * lmax, hi = GMG_HI * lmax;
  const float theta = 0.5f * (hi + lo), delta = 0.5f * (hi - lo);
  const float sigma = theta / delta;
  float* buf[2] = {x, L.d.p};
  int cur;  // buffer holding x_k
  int k;    // steps done
  if (xzero) {
    cur = (m % 2 == 1) ? 0 : 1;  // x_1 .. x_m alternate, x_m in L.x
    k_cheb_first<<<gblocks(n), 256, 0, s>>>(b, L.minv.p, buf[cur], 1.0f / theta, n);
    HX_CHECK_LAUNCH();
    k = 1;
  } else {
    cur = 0;
    if (m % 2 == 1) {  // an odd count of steps from L.x would end in L.d
      HX_CUDA(cudaMemcpyAsync(L.d.p, x, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
      cur = 1;
    }
    k = 0;
  }
  float rho = 1.0f / sigma;
  for (; k < m; ++k) {
    float omega = 0.f, gamma = 1.0f / theta;
    if (k > 0) {
      const float rho_n = 1.0f / (2.0f * sigma - rho);
      omega = rho_n * rho;
      gamma = 2.0f * rho_n / delta;
      rho = rho_n;
    }
    // after a start from x = 0, x_prev = x_0 = 0
    launch_cheb_step<float>(s, buf[cur], buf[cur ^ 1], xzero && k == 1, b, L.minv.p, omega,
                            gamma, L.fac.p, L.nmask.p, L.g, L.K, L.shift);
    cur ^= 1;
  }
  if (want_residual)
    launch_residual<float>(s, x, b, L.r.p, L.fac.p, L.nmask.p, L.g, L.K, L.shift);
}

// z = V(r): one V-cycle on r (FP64 or FP32 DOF vector of level 0).
// Every launch is on c->stream and needs no host round trip, so the cycle
// can be captured in a CUDA graph.
template <typename T>
void gmg_vcycle(hx_ctx* c, const T* r, T* z) {
  auto& G = c->gmg;
  HX_REQUIRE(G.ready, "multigrid hierarchy not set up");
  cudaStream_t s = c->stream;
  const int nl = G.nl;
  // level 0's right-hand side and solution: r and z themselves in FP32
  // (neither is touched by anything else during the cycle), FP32 copies of
  // FP64 vectors otherwise
  auto& L0 = G.lv[0];
  const int64_t n0 = L0.g.dofs();
  const float* b0;
  float* x0;
  if constexpr (std::is_same<T, float>::value) {
    b0 = r;
    x0 = z;
  } else {
    k_copy_cvt<float, T><<<gblocks(n0), 256, 0, s>>>(L0.b.p, r, n0);
    HX_CHECK_LAUNCH();
    b0 = L0.b.p;
    x0 = L0.x.p;
  }
  auto bx = [&](int l, const float*& b, float*& x) {
    b = l == 0 ? b0 : G.lv[l].b.p;
    x = l == 0 ? x0 : G.lv[l].x.p;
  };
  for (int l = 0; l + 1 < nl; ++l) {
    auto& L = G.lv[l];
    auto& C = G.lv[l + 1];
    const float* b;
    float* x;
    bx(l, b, x);
    cheb_smooth(c, L, b, x, true, true);
    // coarse right-hand side R r, zero on the coarse fixed DOFs
    launch_restrict(s, 3, L.r.p, C.b.p, node_grid(L.g), node_grid(C.g), false, C.nmask.p);
  }
  {
    auto& L = G.lv[nl - 1];
    const int64_t n = L.g.dofs();
    const float* b;
    float* x;
    bx(nl - 1, b, x);
    if (G.direct) {
      // coarsest level (the only one for small grids): its dense inverse
      k_dense_gemv<<<(unsigned)cdiv(n * 32, 256), 256, 0, s>>>(G.ainv.p, b, x, n);
      HX_CHECK_LAUNCH();
    } else {
      // a large coarsest level: fixed-count FP32 Jacobi-PCG from zero
      CgState* st = G.coarse_st.p;
      k_coarse_reset<<<1, 32, 0, s>>>(st, GMG_COARSE_ITERS, 1e-4);
      HX_CHECK_LAUNCH();
      launch_fill_zero(s, x, n * sizeof(float));
      launch_cg_init<float>(s, b, nullptr, L.minv.p, L.r.p, G.p1.p, n, st, c->d_partials.p);
      for (int it = 0; it < GMG_COARSE_ITERS; it += 2) {
        launch_pcg_step<float>(s, G.p1.p, G.p0.p, L.r.p, L.minv.p, x, L.q.p, L.fac.p,
                               L.nmask.p, L.g, L.K, L.shift, st, c->d_partials.p);
        launch_cg_update2<float>(s, L.r.p, L.q.p, L.minv.p, n, st, c->d_partials.p);
        launch_pcg_step<float>(s, G.p0.p, G.p1.p, L.r.p, L.minv.p, x, L.q.p, L.fac.p,
                               L.nmask.p, L.g, L.K, L.shift, st, c->d_partials.p);
        launch_cg_update2<float>(s, L.r.p, L.q.p, L.minv.p, n, st, c->d_partials.p);
      }
      k_coarse_finish<<<gblocks(n), 256, 0, s>>>(x, G.p0.p, G.p1.p, st, n);
      HX_CHECK_LAUNCH();
    }
  }
  for (int l = nl - 2; l >= 0; --l) {
    auto& L = G.lv[l];
    auto& C = G.lv[l + 1];
    const float* b;
    float* x;
    bx(l, b, x);
    // x_l += P x_{l+1}, zero on the fixed DOFs; then post-smoothing from it
    launch_prolong(s, C.x.p, x, node_grid(L.g), node_grid(C.g), true, L.nmask.p);
    cheb_smooth(c, L, b, x, false, false);
  }
  if constexpr (!std::is_same<T, float>::value) {
    k_copy_cvt<T, float><<<gblocks(n0), 256, 0, s>>>(z, L0.x.p, n0);
    HX_CHECK_LAUNCH();
  }
}
template void gmg_vcycle<double>(hx_ctx*, const double*, double*);
template void gmg_vcycle<float>(hx_ctx*, const float*, float*);

template <typename T>
void launch_fcg_coeffs(cudaStream_t s, const T* z, const T* q_old, const T* r, int64_t n,
                       double* partials, CgState* st) {
  k_fcg_coeffs<T><<<gblocks(n), 256, 0, s>>>(z, q_old, r, n, partials, st);
  HX_CHECK_LAUNCH();
}
template void launch_fcg_coeffs<double>(cudaStream_t, const double*, const double*,
                                        const double*, int64_t, double*, CgState*);
template void launch_fcg_coeffs<float>(cudaStream_t, const float*, const float*, const float*,
                                       int64_t, double*, CgState*);

// ---------------------------------------------------------------------------
// FP64 flexible CG preconditioned by the V-cycle (Notay's FCG, one stored
// direction, the step kernels of the learned solve).  Convergence on the
// recursive residual, confirmed on the true one by solve_grid.  With
// keep_best the best iterate is kept, as the reference's failure handling
// needs it.
// ---------------------------------------------------------------------------
CgState solve_gmg(hx_ctx* c, const double* fac, const double* b, double* x, bool warm,
                  double shift, const hx_solve_opts& o, double t0, bool* timed_out,
                  int* iters_out) {
  const Grid& g = c->g;
  const int64_t n = g.dofs();
  c->gmg.degree = o.mg_smooth_degree > 0 ? o.mg_smooth_degree : GMG_DEFAULT_DEGREE;
  gmg_setup(c, fac, shift);
  double* r = c->d_r.ensure(n);
  double* P0 = c->d_p.ensure(n);
  double* P1 = c->d_p2.ensure(n);
  double* q = c->d_q.ensure(n);
  double* z = c->gmg.z.ensure(n);
  double* s64 = c->gmg.s.ensure(n);
  double* xbest = o.keep_best ? c->d_xbest.ensure(n) : nullptr;
  const double* minv = c->d_minv.p;
  CgState* st = c->d_state.p;
  put_state(c, 0, fresh_state(o.tol, o.max_iter, 1, o.divergence_checks != 0, o.keep_best != 0));
  if (warm) {
    launch_matvec<double>(c->stream, 0, x, q, fac, c->d_nmask.p, g, c->K, shift,
                          c->d_state.p + 3, c->d_partials.p, nullptr);
    launch_cg_init<double>(c->stream, b, q, minv, r, s64, n, st, c->d_partials.p);
  } else {
    launch_fill_zero(c->stream, x, n * sizeof(double));
    launch_cg_init<double>(c->stream, b, nullptr, minv, r, s64, n, st, c->d_partials.p);
  }
  // no previous direction: p_old = q_old = 0 and pq = 0 give beta = 0
  launch_fill_zero(c->stream, q, n * sizeof(double));
  launch_fill_zero(c->stream, P1, n * sizeof(double));
  if (xbest)
    HX_CUDA(cudaMemcpyAsync(xbest, x, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  CgState s0 = get_state(c, 0);
  *iters_out = 0;
  if (s0.status != HX_RUNNING || o.max_iter <= 0) return s0;
  s0.pq = 0.0;
  s0.alpha = 0.0;
  s0.beta = 0.0;
  put_state(c, 0, s0);
  auto one = [&](double* pin, double* pout) {
    gmg_vcycle<double>(c, r, z);
    launch_fcg_coeffs<double>(c->stream, z, q, r, n, c->d_partials.p, st);
    launch_fcg_step<double>(c->stream, pin, pout, z, x, q, fac, c->d_nmask.p, g, c->K, shift, st,
                            c->d_partials.p);
    launch_cg_update2<double>(c->stream, r, q, minv, n, st, c->d_partials.p);
    // best-iterate snapshot (the reference's failure handling returns it)
    if (xbest) launch_axpy_state<double>(c->stream, xbest, x, pout, n, st, pout == P0 ? 1 : 2);
  };
  auto body = [&]() {
    one(P1, P0);
    one(P0, P1);
  };
  // a multigrid solve takes tens of iterations and the V-cycle's kernels run
  // whole even after the state has stopped: two iterations per graph launch
  // waste at most one cycle
  const int reps = 1;
  CgState sf = run_batched(c, 0, reps, body, o.wall_limit_ms, t0, timed_out, 0);
  if (sf.status != HX_ST_BREAKDOWN && sf.iter > 0) {
    double* pk = ((sf.iter - 1) % 2 == 0) ? P0 : P1;
    launch_axpy_state<double>(c->stream, x, x, pk, n, st, 0);
  }
  *iters_out = sf.iter;
  return sf;
}

}  // namespace hx
