// hx_stress.cu -- per-element stress (src/Core/Stress.jl:10-100), element
// strain energy for compliance sensitivities, and the OC bisection.
#include "hx_internal.h"

namespace hx {

namespace {

__device__ __forceinline__ void gather_elem(const double* __restrict__ u, const Grid& g, int64_t e,
                                            double (&ue)[3][8]) {
  const int i = (int)(e % g.nxe);
  const int64_t r = e / g.nxe;
  const int j = (int)(r % g.nye), k = (int)(r / g.nye);
  const int64_t pl = (int64_t)g.nxn * g.nyn;
  const int64_t n0 = (int64_t)k * pl + (int64_t)j * g.nxn + i;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const int64_t n = n0 + (b & 1) + ((b >> 1) & 1) * (int64_t)g.nxn + ((b >> 2) & 1) * pl;
#pragma unroll
    for (int c = 0; c < 3; ++c) ue[c][b] = u[3 * n + c];
  }
}

// Symmetric 3x3 eigen-decomposition by cyclic Jacobi rotations (FP64);
// S = (xx, yy, zz, xy, yz, xz).  Eigenvalues descending; v0 = unit vector
// of the largest, sign fixed so its largest-magnitude component is positive.
__device__ void sym3_eigen(const double S[6], double ev[3], double v0[3]) {
  double a[3][3] = {{S[0], S[3], S[5]}, {S[3], S[1], S[4]}, {S[5], S[4], S[2]}};
  double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 64; ++sweep) {
    const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    const double scale = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off <= 1e-34 * scale || off == 0.0) break;
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int q = p + 1; q < 3; ++q) {
        if (a[p][q] == 0.0) continue;
        const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const double vkp = v[k][p], vkq = v[k][q];
          v[k][p] = c * vkp - s * vkq;
          v[k][q] = s * vkp + c * vkq;
        }
      }
  }
  int idx[3] = {0, 1, 2};
  const double d[3] = {a[0][0], a[1][1], a[2][2]};
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = i + 1; j < 3; ++j)
      if (d[idx[j]] > d[idx[i]]) {
        const int t = idx[i];
        idx[i] = idx[j];
        idx[j] = t;
      }
#pragma unroll
  for (int i = 0; i < 3; ++i) ev[i] = d[idx[i]];
  double w[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) w[i] = v[i][idx[0]];
  const double nrm = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  int big = 0;
#pragma unroll
  for (int i = 1; i < 3; ++i)
    if (fabs(w[i]) > fabs(w[big])) big = i;
  const double sg = (w[big] < 0 ? -1.0 : 1.0) / nrm;
#pragma unroll
  for (int i = 0; i < 3; ++i) v0[i] = w[i] * sg;
}

// Centre-point stress of a box element: dN_b/dx_a = +-1/(4 h_a), so the
// strain components are the first-level Haar differences / (4 h).
__global__ void k_stress(const double* __restrict__ u, const double* __restrict__ dens, double E,
                         double nu, Grid g, double hx, double hy, double hz,
                         double* __restrict__ principal, double* __restrict__ vm,
                         double* __restrict__ voigt, double* __restrict__ l1,
                         double* __restrict__ dir) {
  const int64_t ne = g.elems();
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    double pr[3] = {0, 0, 0}, dv[3] = {0, 0, 0}, sg[6] = {0, 0, 0, 0, 0, 0}, vmv = 0, l1v = 0;
    const double rho = dens[e];
    if (rho > 1e-6) {
      double ue[3][8];
      gather_elem(u, g, e, ue);
#pragma unroll
      for (int c = 0; c < 3; ++c) haar_fwd(ue[c]);
      const double ax = 0.25 / hx, ay = 0.25 / hy, az = 0.25 / hz;
      const double exx = ue[0][1] * ax, eyy = ue[1][2] * ay, ezz = ue[2][4] * az;
      const double gxy = ue[0][2] * ay + ue[1][1] * ax;
      const double gyz = ue[1][4] * az + ue[2][2] * ay;
      const double gxz = ue[0][4] * az + ue[2][1] * ax;
      // material_matrix(E*rho, nu), src/Core/Element.jl:45-62
      const double f = E * rho / ((1.0 + nu) * (1.0 - 2.0 * nu));
      const double c1 = (1.0 - nu) * f, c2 = nu * f, c3 = ((1.0 - 2.0 * nu) / 2.0) * f;
      sg[0] = c1 * exx + c2 * (eyy + ezz);
      sg[1] = c1 * eyy + c2 * (exx + ezz);
      sg[2] = c1 * ezz + c2 * (exx + eyy);
      sg[3] = c3 * gxy;
      sg[4] = c3 * gyz;
      sg[5] = c3 * gxz;
      sym3_eigen(sg, pr, dv);
      // von Mises, src/Core/Stress.jl:52
      vmv = sqrt(0.5 * ((sg[0] - sg[1]) * (sg[0] - sg[1]) + (sg[1] - sg[2]) * (sg[1] - sg[2]) +
                        (sg[2] - sg[0]) * (sg[2] - sg[0])) +
                 3.0 * (sg[3] * sg[3] + sg[4] * sg[4] + sg[5] * sg[5]));
      l1v = fabs(pr[0]) + fabs(pr[1]) + fabs(pr[2]);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      principal[3 * e + i] = pr[i];
      dir[3 * e + i] = dv[i];
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) voigt[6 * e + i] = sg[i];
    vm[e] = vmv;
    l1[e] = l1v;
  }
}

__global__ void k_energy(const double* __restrict__ u, Grid g, ElemCoef<double> K,
                         double* __restrict__ ce) {
  const int64_t ne = g.elems();
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    double ue[3][8];
    gather_elem(u, g, e, ue);
    ce[e] = elem_energy<double>(K, ue);
  }
}

// One bisection step of the OC update (state aux: l1, l2, lmid).
__global__ void k_oc_step(const double* __restrict__ x, const double* __restrict__ dc,
                          const double* __restrict__ dv, int64_t n, double volfrac, double move,
                          double* __restrict__ xnew, CgState* st, double* partials) {
  if (st->status != HX_RUNNING) return;
  const double l1 = st->aux[0], l2 = st->aux[1];
  const double lmid = 0.5 * (l1 + l2);
  double vol = 0.0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const double xe = x[e];
    const double be = sqrt(fmax(-dc[e], 0.0) / (lmid * (dv ? dv[e] : 1.0)));
    double xn = xe * be;
    const double lo = fmax(0.0, xe - move), hi = fmin(1.0, xe + move);
    xn = fmin(fmax(xn, lo), hi);
    xnew[e] = xn;
    vol += xn;
  }
  double v[1] = {vol};
  if (grid_reduce<1>(v, partials, &st->ticket[TK_AUX]) && threadIdx.x == 0) {
    double a = l1, b = l2;
    if (v[0] > volfrac * (double)n)
      a = lmid;
    else
      b = lmid;
    st->aux[0] = a;
    st->aux[1] = b;
    st->aux[2] = lmid;
    st->iter += 1;
    if (!((b - a) / (a + b) > 1e-3)) st->status = HX_ST_CONVERGED;
  }
}

// SIMP: fac = emin + max(rho, 0)^p (e0 - emin).  With u (sensitivity mode):
// out = -p max(rho, 0)^(p-1) (e0 - emin) * ce, ce the unit-modulus element
// energies u_e^T Ke u_e already in `out`.
__global__ void k_simp(const double* __restrict__ rho, double p, double e0, double emin,
                       double* __restrict__ out, int64_t n, int sensitivity) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const double r = fmax(rho[e], 0.0);
    out[e] = sensitivity ? -p * pow(r, p - 1.0) * (e0 - emin) * out[e]
                         : emin + pow(r, p) * (e0 - emin);
  }
}

// p-norm aggregate of the element von Mises stresses, in two passes for
// range safety: pass 0 reduces m = max vm into st->aux[0]; pass 1 reduces
// sum (vm / m)^P into st->aux[1].  sigma_PN = m * aux[1]^(1/P).
__global__ void k_pnorm(const double* __restrict__ vm, int64_t n, double P, int pass,
                        CgState* st, double* partials) {
  const double m = pass ? st->aux[0] : 0.0;
  double acc = 0.0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const double v = vm[e];
    if (pass == 0)
      acc = fmax(acc, v);
    else if (m > 0.0)
      acc += pow(v / m, P);
  }
  double r[1] = {acc};
  if (pass == 0) {
    if (grid_reduce<1, true>(r, partials, &st->ticket[TK_AUX]) && threadIdx.x == 0)
      st->aux[0] = r[0];
  } else {
    if (grid_reduce<1>(r, partials, &st->ticket[TK_AUX2]) && threadIdx.x == 0) st->aux[1] = r[0];
  }
}

unsigned eblocks(int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, 128), 32LL * sm_count()));
}

}  // namespace

void launch_stress(cudaStream_t s, const double* u, const double* dens, double E, double nu,
                   const Grid& g, double hx, double hy, double hz, double* principal, double* vm,
                   double* voigt, double* l1, double* dir) {
  k_stress<<<eblocks(g.elems()), 128, 0, s>>>(u, dens, E, nu, g, hx, hy, hz, principal, vm, voigt,
                                              l1, dir);
  HX_CHECK_LAUNCH();
}

void launch_simp(cudaStream_t s, const double* rho, double p, double e0, double emin, double* out,
                 int64_t n, bool sensitivity) {
  k_simp<<<eblocks(n), 128, 0, s>>>(rho, p, e0, emin, out, n, sensitivity ? 1 : 0);
  HX_CHECK_LAUNCH();
}

void launch_pnorm(cudaStream_t s, const double* vm, int64_t n, double P, CgState* st,
                  double* partials) {
  const unsigned blocks =
      (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, 256), 8LL * sm_count()));
  for (int pass = 0; pass < 2; ++pass) {
    k_pnorm<<<blocks, 256, 0, s>>>(vm, n, P, pass, st, partials);
    HX_CHECK_LAUNCH();
  }
}

void launch_energy(cudaStream_t s, const double* u, const Grid& g, const ElemCoef<double>& K,
                   double* ce) {
  k_energy<<<eblocks(g.elems()), 128, 0, s>>>(u, g, K, ce);
  HX_CHECK_LAUNCH();
}

void launch_oc(cudaStream_t s, const double* x, const double* dc, const double* dv, int64_t n,
               double volfrac, double move, double* xnew, CgState* st, double* partials,
               int max_steps) {
  const unsigned blocks =
      (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, 256), 8LL * sm_count()));
  for (int i = 0; i < max_steps; ++i) {
    k_oc_step<<<blocks, 256, 0, s>>>(x, dc, dv, n, volfrac, move, xnew, st, partials);
    HX_CHECK_LAUNCH();
  }
}

}  // namespace hx
