// hx_filter.cu -- Helmholtz PDE density filter on the structured node grid.
//
// The reference (src/Optimization/GPUHelmholtz.jl:39-229) assembles
// Ae = r^2 Ke + Me element by element with atomics.  On a full structured
// grid of identical box elements the assembled operator is exactly
//   A = r^2 (Sx(x)My(x)Mz + Mx(x)Sy(x)Mz + Mx(x)My(x)Sz) + Mx(x)My(x)Mz
// with S/M the assembled 1D stiffness/mass (tridiagonal; boundary rows carry
// one element).  The matvec applies it separably on a 3x3x3 register window
// that slides along z: 54 + 27 + 12 FMAs per node, no atomics, no stored
// matrix.  ref_compat=1 reproduces the reference element whose top face is
// at z=+dz (src/Core/Element.jl:106-107), i.e. a box 1.5*dz tall.
#include "hx_internal.h"

namespace hx {

FilterCoef make_filter_coef(double dx, double dy, double dz, double radius, int ref_compat) {
  FilterCoef F{};
  const double h[3] = {dx, dy, ref_compat ? 1.5 * dz : dz};
  for (int a = 0; a < 3; ++a) {
    const double s = 1.0 / h[a], m = h[a] / 6.0;
    // row type 0: first node (one element on its +side)
    F.S[a][0][0] = 0;  F.S[a][0][1] = s;       F.S[a][0][2] = -s;
    F.M[a][0][0] = 0;  F.M[a][0][1] = 2 * m;   F.M[a][0][2] = m;
    // row type 1: interior
    F.S[a][1][0] = -s; F.S[a][1][1] = 2 * s;   F.S[a][1][2] = -s;
    F.M[a][1][0] = m;  F.M[a][1][1] = 4 * m;   F.M[a][1][2] = m;
    // row type 2: last node
    F.S[a][2][0] = -s; F.S[a][2][1] = s;       F.S[a][2][2] = 0;
    F.M[a][2][0] = m;  F.M[a][2][1] = 2 * m;   F.M[a][2][2] = 0;
  }
  F.r2 = radius * radius;
  F.vol8 = dx * dy * dz / 8.0;  // the RHS uses the true volume (GPUHelmholtz.jl:175-176)
  return F;
}

namespace {

__device__ __forceinline__ int row_type(int i, int n) {
  return (n == 1) ? 1 : (i == 0 ? 0 : (i == n - 1 ? 2 : 1));
}

constexpr int FB_X = 32, FB_Y = 8;

// y = A x on the node grid; MODE 2 also reduces p.q into the CG state.
template <int MODE>
__global__ void __launch_bounds__(FB_X* FB_Y)
    k_filter_matvec(const double* __restrict__ x, double* __restrict__ y, Grid g, FilterCoef F,
                    int kchunk, CgState* st, double* partials) {
  if (MODE == 2 && st->status != HX_RUNNING) return;
  const int i = blockIdx.x * FB_X + threadIdx.x;
  const int j = blockIdx.y * FB_Y + threadIdx.y;
  const int k0 = blockIdx.z * kchunk, k1 = min(k0 + kchunk, g.nzn);
  const bool act = i < g.nxn && j < g.nyn;
  const int64_t pl = (int64_t)g.nxn * g.nyn;
  const int tx = row_type(i, g.nxn), ty = row_type(j, g.nyn);
  double Sx[3], Mx[3], Sy[3], My[3];
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    Sx[t] = F.S[0][tx][t];
    Mx[t] = F.M[0][tx][t];
    Sy[t] = F.S[1][ty][t];
    My[t] = F.M[1][ty][t];
  }
  auto ld = [&](int a, int b, int k) -> double {
    const int ii = i + a, jj = j + b;
    if (!act || k < 0 || k >= g.nzn || ii < 0 || jj < 0 || ii >= g.nxn || jj >= g.nyn) return 0.0;
    return __ldg(&x[(int64_t)k * pl + (int64_t)jj * g.nxn + ii]);
  };
  double w[3][3][3];  // [a][b][c] for offsets -1..1
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      w[a][b][0] = 0.0;
      w[a][b][1] = ld(a - 1, b - 1, k0 - 1);
      w[a][b][2] = ld(a - 1, b - 1, k0);
    }
  double dsum = 0.0;
  for (int k = k0; k < k1; ++k) {
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        w[a][b][0] = w[a][b][1];
        w[a][b][1] = w[a][b][2];
        w[a][b][2] = ld(a - 1, b - 1, k + 1);
      }
    const int tz = row_type(k, g.nzn);
    const double* Sz = F.S[2][tz];
    const double* Mz = F.M[2][tz];
    double yMM[3], ySM[3], yMS[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double zM[3], zS[3];
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        zM[b] = Mz[0] * w[a][b][0] + Mz[1] * w[a][b][1] + Mz[2] * w[a][b][2];
        zS[b] = Sz[0] * w[a][b][0] + Sz[1] * w[a][b][1] + Sz[2] * w[a][b][2];
      }
      yMM[a] = My[0] * zM[0] + My[1] * zM[1] + My[2] * zM[2];
      ySM[a] = Sy[0] * zM[0] + Sy[1] * zM[1] + Sy[2] * zM[2];
      yMS[a] = My[0] * zS[0] + My[1] * zS[1] + My[2] * zS[2];
    }
    double v = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
      v += F.r2 * (Sx[a] * yMM[a] + Mx[a] * (ySM[a] + yMS[a])) + Mx[a] * yMM[a];
    if (act) {
      y[(int64_t)k * pl + (int64_t)j * g.nxn + i] = v;
      if (MODE != 0) dsum += w[1][1][1] * v;
    }
  }
  if (MODE != 0) {
    double vv[1] = {dsum};
    if (grid_reduce<1>(vv, partials, &st->ticket[TK_MATVEC]) && threadIdx.x == 0 &&
        threadIdx.y == 0) {
      const double pq = vv[0];
      st->pq = pq;
      if (!(pq > 0.0) || !isfinite(pq))
        st->status = HX_ST_BREAKDOWN;
      else
        st->alpha = st->rz / pq;
    }
  }
}

__global__ void k_filter_invdiag(double* __restrict__ invd, Grid g, FilterCoef F) {
  const int64_t nn = g.nodes();
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(n % g.nxn);
    const int64_t r = n / g.nxn;
    const int j = (int)(r % g.nyn), k = (int)(r / g.nyn);
    const int tx = row_type(i, g.nxn), ty = row_type(j, g.nyn), tz = row_type(k, g.nzn);
    const double sx = F.S[0][tx][1], mx = F.M[0][tx][1];
    const double sy = F.S[1][ty][1], my = F.M[1][ty][1];
    const double sz = F.S[2][tz][1], mz = F.M[2][tz][1];
    const double d = F.r2 * (sx * my * mz + mx * sy * mz + mx * my * sz) + mx * my * mz;
    invd[n] = 1.0 / d;
  }
}

// b_n = vol/8 * sum of rho over the (up to 8) elements around node n
// (GPUHelmholtz.jl:39-50 scatters the same sums with atomics).
__global__ void k_filter_rhs(const double* __restrict__ rho, double* __restrict__ b, Grid g,
                             double vol8) {
  const int64_t nn = g.nodes();
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(n % g.nxn);
    const int64_t r = n / g.nxn;
    const int j = (int)(r % g.nyn), k = (int)(r / g.nyn);
    double s = 0.0;
#pragma unroll
    for (int dk = -1; dk <= 0; ++dk)
#pragma unroll
      for (int dj = -1; dj <= 0; ++dj)
#pragma unroll
        for (int di = -1; di <= 0; ++di) {
          const int ei = i + di, ej = j + dj, ek = k + dk;
          if (ei >= 0 && ej >= 0 && ek >= 0 && ei < g.nxe && ej < g.nye && ek < g.nze)
            s += rho[((int64_t)ek * g.nye + ej) * g.nxe + ei];
        }
    b[n] = s * vol8;
  }
}

// element value = mean of its 8 nodal values (GPUHelmholtz.jl:78-89)
__global__ void k_filter_extract(const double* __restrict__ x, double* __restrict__ out, Grid g) {
  const int64_t ne = g.elems();
  const int64_t pl = (int64_t)g.nxn * g.nyn;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % g.nxe);
    const int64_t r = e / g.nxe;
    const int j = (int)(r % g.nye), k = (int)(r / g.nye);
    const int64_t n0 = (int64_t)k * pl + (int64_t)j * g.nxn + i;
    const double s = x[n0] + x[n0 + 1] + x[n0 + g.nxn + 1] + x[n0 + g.nxn] + x[n0 + pl] +
                     x[n0 + pl + 1] + x[n0 + pl + g.nxn + 1] + x[n0 + pl + g.nxn];
    out[e] = s / 8.0;
  }
}

unsigned flat_blocks(int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, 256), 16LL * sm_count()));
}

}  // namespace

void launch_filter_matvec(cudaStream_t s, const double* x, double* y, const Grid& g,
                          const FilterCoef& F, CgState* st, double* partials) {
  const int64_t cols = (int64_t)cdiv(g.nxn, FB_X) * cdiv(g.nyn, FB_Y);
  const int nch = (int)std::max<int64_t>(1, (4LL * sm_count() + cols - 1) / cols);
  const int kc = std::max(4, (int)cdiv(g.nzn, nch));
  const dim3 grid(cdiv(g.nxn, FB_X), cdiv(g.nyn, FB_Y), cdiv(g.nzn, kc));
  const dim3 block(FB_X, FB_Y);
  if (st)
    k_filter_matvec<2><<<grid, block, 0, s>>>(x, y, g, F, kc, st, partials);
  else
    k_filter_matvec<0><<<grid, block, 0, s>>>(x, y, g, F, kc, st, partials);
  HX_CHECK_LAUNCH();
}

void launch_filter_invdiag(cudaStream_t s, double* invd, const Grid& g, const FilterCoef& F) {
  k_filter_invdiag<<<flat_blocks(g.nodes()), 256, 0, s>>>(invd, g, F);
  HX_CHECK_LAUNCH();
}

void launch_filter_rhs(cudaStream_t s, const double* rho, double* b, const Grid& g, double vol8) {
  k_filter_rhs<<<flat_blocks(g.nodes()), 256, 0, s>>>(rho, b, g, vol8);
  HX_CHECK_LAUNCH();
}

void launch_filter_extract(cudaStream_t s, const double* x, double* out, const Grid& g) {
  k_filter_extract<<<flat_blocks(g.elems()), 256, 0, s>>>(x, out, g);
  HX_CHECK_LAUNCH();
}

}  // namespace hx
