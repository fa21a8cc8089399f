/*
 * hexat_oracle.c -- CPU FP64 restatement of the HEXA(T) v069 inner solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load this library, and
 * only as the checker or as the timed CPU baseline.  The product (the CUDA
 * library under 2025_12_09_hexat_v069_b200/) never calls into it.
 *
 * PARITY UNPINNED: the reference (a Julia project) ships no tests, golden
 * vectors or fixtures for this path, and Julia is not available to run it.
 * This restatement is pinned instead by independent checks in tests/:
 * a scipy sparse direct solve of the assembled system, the rigid-body null
 * space and rank of Ke, symmetry, the closed-form Kronecker form of Ke,
 * mass conservation of the scalar element matrices (including the reference's
 * 1.5*dz element quirk) and constant-field invariance of the filter.
 *
 * Every function cites the reference file:line it restates, relative to the
 * reference project root (v069_2025_12_09_HEXAS_TOPO_anti_checkerboard/).
 * Connectivity is 0-based int32, row-major nE x 8 (element e, corner c at
 * e*8+c), corner order as src/Core/Element.jl:8-17 NAT_COORDS.  DOFs are
 * interleaved: dof = 3*node + component.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define HXO_API __attribute__((visibility("default")))

/* NAT_COORDS, src/Core/Element.jl:8-17 */
static const double NAT[8][3] = {
    {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
    {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

/* shape_functions, src/Core/Element.jl:23-43 */
static void shape_functions(double xi, double eta, double zeta, double N[8],
                            double dN[8][3]) {
  for (int i = 0; i < 8; ++i) {
    double tx = 1.0 + xi * NAT[i][0];
    double ty = 1.0 + eta * NAT[i][1];
    double tz = 1.0 + zeta * NAT[i][2];
    N[i] = 0.125 * tx * ty * tz;
    dN[i][0] = 0.125 * NAT[i][0] * ty * tz;
    dN[i][1] = 0.125 * tx * NAT[i][1] * tz;
    dN[i][2] = 0.125 * tx * ty * NAT[i][2];
  }
}

/* material_matrix, src/Core/Element.jl:45-62 (Voigt xx,yy,zz,xy,yz,xz) */
HXO_API void hxo_material_matrix(double E, double nu, double D[36]) {
  double f = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
  double c1 = (1.0 - nu) * f, c2 = nu * f, c3 = ((1.0 - 2.0 * nu) / 2.0) * f;
  memset(D, 0, 36 * sizeof(double));
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) D[i * 6 + j] = (i == j) ? c1 : c2;
  D[3 * 6 + 3] = D[4 * 6 + 4] = D[5 * 6 + 5] = c3;
}

static double det3(const double J[3][3]) {
  return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
         J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
         J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}

static void inv3(const double J[3][3], double Ji[3][3]) {
  double d = det3(J);
  Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / d;
  Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / d;
  Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / d;
  Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / d;
  Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / d;
  Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / d;
  Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / d;
  Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / d;
  Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / d;
}

/* dN/dx at (xi,eta,zeta) for an element with corner coordinates X[8][3];
 * returns detJ.  src/Core/Element.jl:72-79 */
static double physical_gradients(const double X[8][3], double xi, double eta,
                                 double zeta, double N[8], double dNdx[8][3]) {
  double dN[8][3], J[3][3] = {{0}}, Ji[3][3];
  shape_functions(xi, eta, zeta, N, dN);
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      for (int i = 0; i < 8; ++i) J[a][b] += dN[i][a] * X[i][b];
  double detJ = det3(J);
  inv3(J, Ji);
  for (int i = 0; i < 8; ++i)
    for (int a = 0; a < 3; ++a) {
      double s = 0;
      for (int b = 0; b < 3; ++b) s += dN[i][b] * Ji[a][b];
      dNdx[i][a] = s;
    }
  return detJ;
}

/* B matrix (6x24), src/Core/Element.jl:81-89 */
static void bmatrix(const double dNdx[8][3], double B[6][24]) {
  memset(B, 0, 6 * 24 * sizeof(double));
  for (int i = 0; i < 8; ++i) {
    int c = 3 * i;
    B[0][c] = dNdx[i][0];
    B[1][c + 1] = dNdx[i][1];
    B[2][c + 2] = dNdx[i][2];
    B[3][c] = dNdx[i][1];
    B[3][c + 1] = dNdx[i][0];
    B[4][c + 1] = dNdx[i][2];
    B[4][c + 2] = dNdx[i][1];
    B[5][c] = dNdx[i][2];
    B[5][c + 2] = dNdx[i][0];
  }
}

/* hex_element_stiffness + get_canonical_stiffness (unit E),
 * src/Core/Element.jl:64-102.  ke is 24x24 row-major. */
HXO_API void hxo_canonical_ke(double dx, double dy, double dz, double nu,
                              double *ke) {
  double X[8][3];
  for (int i = 0; i < 8; ++i) {
    X[i][0] = (NAT[i][0] > 0 ? dx : 0.0) - dx / 2;
    X[i][1] = (NAT[i][1] > 0 ? dy : 0.0) - dy / 2;
    X[i][2] = (NAT[i][2] > 0 ? dz : 0.0) - dz / 2;
  }
  double D[36];
  hxo_material_matrix(1.0, nu, D);
  memset(ke, 0, 576 * sizeof(double));
  const double a = 1.0 / sqrt(3.0);
  const double g[2] = {-a, a};
  for (int p = 0; p < 2; ++p)
    for (int q = 0; q < 2; ++q)
      for (int r = 0; r < 2; ++r) {
        double N[8], dNdx[8][3], B[6][24], DB[6][24];
        double detJ = physical_gradients(X, g[p], g[q], g[r], N, dNdx);
        bmatrix(dNdx, B);
        for (int i = 0; i < 6; ++i)
          for (int j = 0; j < 24; ++j) {
            double s = 0;
            for (int k = 0; k < 6; ++k) s += D[i * 6 + k] * B[k][j];
            DB[i][j] = s;
          }
        for (int i = 0; i < 24; ++i)
          for (int j = 0; j < 24; ++j) {
            double s = 0;
            for (int k = 0; k < 6; ++k) s += B[k][i] * DB[k][j];
            ke[i * 24 + j] += s * detJ;
          }
      }
}

/* get_scalar_canonical_matrices, src/Core/Element.jl:104-125.
 * ref_compat=1 reproduces the reference's top-face z coordinate of +dz
 * (Element.jl:107), i.e. an element 1.5*dz tall; ref_compat=0 uses +dz/2. */
HXO_API void hxo_scalar_ke_me(double dx, double dy, double dz, int ref_compat,
                              double *ke, double *me) {
  double X[8][3];
  for (int i = 0; i < 8; ++i) {
    X[i][0] = NAT[i][0] * dx / 2;
    X[i][1] = NAT[i][1] * dy / 2;
    X[i][2] = NAT[i][2] > 0 ? (ref_compat ? dz : dz / 2) : -dz / 2;
  }
  memset(ke, 0, 64 * sizeof(double));
  memset(me, 0, 64 * sizeof(double));
  const double a = 1.0 / sqrt(3.0);
  const double g[2] = {-a, a};
  for (int p = 0; p < 2; ++p)
    for (int q = 0; q < 2; ++q)
      for (int r = 0; r < 2; ++r) {
        double N[8], dNdx[8][3];
        double w = physical_gradients(X, g[p], g[q], g[r], N, dNdx);
        for (int i = 0; i < 8; ++i)
          for (int j = 0; j < 8; ++j) {
            ke[i * 8 + j] += (dNdx[i][0] * dNdx[j][0] + dNdx[i][1] * dNdx[j][1] +
                              dNdx[i][2] * dNdx[j][2]) * w;
            me[i * 8 + j] += N[i] * N[j] * w;
          }
      }
}

static int omp_threads(int nthreads) {
#ifdef _OPENMP
  return nthreads > 0 ? nthreads : omp_get_max_threads();
#else
  (void)nthreads;
  return 1;
#endif
}

/* apply_stiffness, src/Solvers/CPUSolver.jl:50-94: y = sum_e factor_e*Ke*x_e
 * over elements with factor_e != 0 (the caller encodes the reference's
 * density < min_stiffness_threshold skip as factor 0).  Per-thread full-length
 * accumulators reduced serially, as the reference does. */
HXO_API void hxo_apply_stiffness(int64_t nN, int64_t nE, const int32_t *elem,
                                 const double *ke, const double *factor,
                                 const double *x, double *y, int nthreads) {
  int nt = omp_threads(nthreads);
  int64_t ndof = 3 * nN;
  double *acc = (double *)calloc((size_t)nt * (size_t)ndof, sizeof(double));
#pragma omp parallel num_threads(nt)
  {
#ifdef _OPENMP
    int tid = omp_get_thread_num();
#else
    int tid = 0;
#endif
    double *loc = acc + (size_t)tid * (size_t)ndof;
#pragma omp for schedule(static)
    for (int64_t e = 0; e < nE; ++e) {
      double f = factor[e];
      if (f == 0.0) continue;
      const int32_t *c = elem + 8 * e;
      double ue[24], fe[24];
      for (int i = 0; i < 8; ++i)
        for (int d = 0; d < 3; ++d) ue[3 * i + d] = x[3 * (int64_t)c[i] + d];
      for (int i = 0; i < 24; ++i) {
        double s = 0;
        for (int j = 0; j < 24; ++j) s += ke[i * 24 + j] * ue[j];
        fe[i] = s * f;
      }
      for (int i = 0; i < 8; ++i)
        for (int d = 0; d < 3; ++d) loc[3 * (int64_t)c[i] + d] += fe[3 * i + d];
    }
  }
  memset(y, 0, (size_t)ndof * sizeof(double));
  for (int t = 0; t < nt; ++t) {
    const double *loc = acc + (size_t)t * (size_t)ndof;
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t i = 0; i < ndof; ++i) y[i] += loc[i];
  }
  free(acc);
}

/* compute_diagonal_preconditioner, src/Solvers/CPUSolver.jl:109-148 */
HXO_API void hxo_diagonal(int64_t nN, int64_t nE, const int32_t *elem,
                          const double *ke, const double *factor, double *diag) {
  memset(diag, 0, (size_t)(3 * nN) * sizeof(double));
  for (int64_t e = 0; e < nE; ++e) {
    double f = factor[e];
    if (f == 0.0) continue;
    const int32_t *c = elem + 8 * e;
    for (int i = 0; i < 8; ++i)
      for (int d = 0; d < 3; ++d)
        diag[3 * (int64_t)c[i] + d] += ke[(3 * i + d) * 25] * f;
  }
}

static double dotv(int64_t n, const double *a, const double *b) {
  double s = 0;
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/* Jacobi-preconditioned CG on the free DOFs with diagonal shift,
 * src/Solvers/CPUSolver.jl:150-212 (shift = shift_factor*max(diag_free),
 * diag clamp :170, stop when ||r||/||b|| < tol :191-197).  free_mask[dof]=1
 * for free DOFs.  precond_add=0 clamps the diagonal at the shift
 * (CPUSolver.jl:170); precond_add=1 uses M^-1 = 1/(diag + shift), the GPU
 * path's rule (src/Solvers/GPUSolver.jl:402).  x_inout holds the initial
 * guess when warm != 0 (the GPU
 * path's warm start, src/Solvers/GPUSolver.jl:408-412) and the full-length
 * solution on return (zeros at constrained DOFs).  Returns iterations run;
 * *rel_res gets the final recursive residual ratio.  Returns -1 on
 * breakdown (p.Ap == 0 or NaN, src/Solvers/GPUSolver.jl:462-466). */
HXO_API int hxo_cg_solve(int64_t nN, int64_t nE, const int32_t *elem,
                         const double *ke, const double *factor,
                         const uint8_t *free_mask, const double *f,
                         double *x_inout, int warm, int max_iter, double tol,
                         double shift_factor, int precond_add, int nthreads,
                         double *rel_res, double *shift_out) {
  int64_t ndof = 3 * nN;
  int64_t nf = 0;
  for (int64_t i = 0; i < ndof; ++i) nf += free_mask[i] ? 1 : 0;
  int64_t *fd = (int64_t *)malloc((size_t)(nf ? nf : 1) * sizeof(int64_t));
  nf = 0;
  for (int64_t i = 0; i < ndof; ++i)
    if (free_mask[i]) fd[nf++] = i;
  double *diag = (double *)malloc((size_t)ndof * sizeof(double));
  double *xf = (double *)calloc((size_t)(nf > 0 ? nf : 0) + 1, sizeof(double));
  double *r = (double *)malloc(((size_t)nf + 1) * sizeof(double));
  double *z = (double *)malloc(((size_t)nf + 1) * sizeof(double));
  double *p = (double *)malloc(((size_t)nf + 1) * sizeof(double));
  double *ap = (double *)malloc(((size_t)nf + 1) * sizeof(double));
  double *df = (double *)malloc(((size_t)nf + 1) * sizeof(double));
  const size_t nd = (size_t)(ndof > 0 ? ndof : 1);
  double *full = (double *)calloc(nd, sizeof(double));
  double *yfull = (double *)malloc(nd * sizeof(double));

  hxo_diagonal(nN, nE, elem, ke, factor, diag);
  double maxd = -INFINITY;
  for (int64_t i = 0; i < nf; ++i) {
    df[i] = diag[fd[i]];
    if (df[i] > maxd) maxd = df[i];
  }
  double shift = nf ? shift_factor * maxd : 0.0;
  if (shift_out) *shift_out = shift;
  for (int64_t i = 0; i < nf; ++i) {
    if (precond_add)
      df[i] += shift;
    else if (df[i] <= shift)
      df[i] = shift;
  }

  /* r = f - (K+sI) x0 */
  for (int64_t i = 0; i < nf; ++i) r[i] = f[fd[i]];
  if (warm) {
    for (int64_t i = 0; i < nf; ++i) xf[i] = x_inout[fd[i]];
    for (int64_t i = 0; i < nf; ++i) full[fd[i]] = xf[i];
    hxo_apply_stiffness(nN, nE, elem, ke, factor, full, yfull, nthreads);
    for (int64_t i = 0; i < nf; ++i) r[i] -= yfull[fd[i]] + shift * xf[i];
  }
  double normf = 0;
  for (int64_t i = 0; i < nf; ++i) normf += f[fd[i]] * f[fd[i]];
  normf = sqrt(normf);
  int iters = 0;
  double res = 0.0;
  if (normf == 0.0) {
    memset(x_inout, 0, (size_t)ndof * sizeof(double));
    *rel_res = 0.0;
    goto done;
  }
  for (int64_t i = 0; i < nf; ++i) z[i] = r[i] / df[i];
  memcpy(p, z, (size_t)nf * sizeof(double));
  double rz = dotv(nf, r, z);
  for (int it = 1; it <= max_iter; ++it) {
    for (int64_t i = 0; i < nf; ++i) full[fd[i]] = p[i];
    hxo_apply_stiffness(nN, nE, elem, ke, factor, full, yfull, nthreads);
    for (int64_t i = 0; i < nf; ++i) ap[i] = yfull[fd[i]] + shift * p[i];
    double pap = dotv(nf, p, ap);
    if (pap == 0.0 || isnan(pap)) {
      iters = -1;
      break;
    }
    double alpha = rz / pap;
    for (int64_t i = 0; i < nf; ++i) {
      xf[i] += alpha * p[i];
      r[i] -= alpha * ap[i];
    }
    res = sqrt(dotv(nf, r, r)) / normf;
    iters = it;
    if (res < tol) break;
    for (int64_t i = 0; i < nf; ++i) z[i] = r[i] / df[i];
    double rzn = dotv(nf, r, z);
    double beta = rzn / rz;
    for (int64_t i = 0; i < nf; ++i) p[i] = z[i] + beta * p[i];
    rz = rzn;
  }
  memset(x_inout, 0, (size_t)ndof * sizeof(double));
  for (int64_t i = 0; i < nf; ++i) x_inout[fd[i]] = xf[i];
  *rel_res = res;
done:
  free(fd); free(diag); free(xf); free(r); free(z); free(p); free(ap);
  free(df); free(full); free(yfull);
  return iters;
}

/* Scalar EbE product y = sum_e Ae x_e over all elements (no factor),
 * src/Optimization/GPUHelmholtz.jl:52-76. */
static void scalar_apply(int64_t nN, int64_t nE, const int32_t *elem,
                         const double *ae, const double *x, double *y) {
  memset(y, 0, (size_t)nN * sizeof(double));
  for (int64_t e = 0; e < nE; ++e) {
    const int32_t *c = elem + 8 * e;
    double xe[8];
    for (int i = 0; i < 8; ++i) xe[i] = x[c[i]];
    for (int i = 0; i < 8; ++i) {
      double s = 0;
      for (int j = 0; j < 8; ++j) s += ae[i * 8 + j] * xe[j];
      y[c[i]] += s;
    }
  }
}

/* Helmholtz PDE filter, src/Optimization/GPUHelmholtz.jl:108-229:
 * Ae = radius^2*Ke + Me (:129), diag by element sum (:91-102), RHS
 * b_n = sum_e rho_e*vol/8 (:39-50, :175-177), Jacobi-CG from x=0 with at most
 * max_iter iterations and ||r||/||b|| tested every 10 iterations (:197-223),
 * element value = mean of its 8 nodal values (:78-89).  On a zero RHS the
 * input is returned unchanged (:179-182).  Returns iterations; *rel_res gets
 * the last tested residual ratio. */
HXO_API int hxo_helmholtz_filter(int64_t nN, int64_t nE, const int32_t *elem,
                                 double dx, double dy, double dz, double radius,
                                 int ref_compat, const double *rho, double *out,
                                 double tol, int max_iter, double *rel_res) {
  double ke[64], me[64], ae[64];
  hxo_scalar_ke_me(dx, dy, dz, ref_compat, ke, me);
  for (int i = 0; i < 64; ++i) ae[i] = radius * radius * ke[i] + me[i];
  double *b = (double *)calloc((size_t)nN, sizeof(double));
  double *dg = (double *)calloc((size_t)nN, sizeof(double));
  double *x = (double *)calloc((size_t)nN, sizeof(double));
  double *r = (double *)malloc((size_t)nN * sizeof(double));
  double *z = (double *)malloc((size_t)nN * sizeof(double));
  double *p = (double *)malloc((size_t)nN * sizeof(double));
  double *ap = (double *)malloc((size_t)nN * sizeof(double));
  double vs = dx * dy * dz / 8.0;
  for (int64_t e = 0; e < nE; ++e)
    for (int i = 0; i < 8; ++i) {
      b[elem[8 * e + i]] += rho[e] * vs;
      dg[elem[8 * e + i]] += ae[i * 9];
    }
  double normb = sqrt(dotv(nN, b, b));
  int iters = 0;
  double res = 0.0;
  if (normb == 0.0) {
    memcpy(out, rho, (size_t)nE * sizeof(double));
    *rel_res = 0.0;
    goto done;
  }
  for (int64_t i = 0; i < nN; ++i) {
    r[i] = b[i];
    z[i] = r[i] / dg[i];
    p[i] = z[i];
  }
  double rho_old = dotv(nN, r, z);
  for (int it = 1; it <= max_iter; ++it) {
    iters = it;
    scalar_apply(nN, nE, elem, ae, p, ap);
    double alpha = rho_old / dotv(nN, p, ap);
    for (int64_t i = 0; i < nN; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * ap[i];
    }
    if (it % 10 == 0) {
      res = sqrt(dotv(nN, r, r)) / normb;
      if (res < tol) break;
    }
    for (int64_t i = 0; i < nN; ++i) z[i] = r[i] / dg[i];
    double rho_new = dotv(nN, r, z);
    double beta = rho_new / rho_old;
    for (int64_t i = 0; i < nN; ++i) p[i] = z[i] + beta * p[i];
    rho_old = rho_new;
  }
  for (int64_t e = 0; e < nE; ++e) {
    double s = 0;
    for (int i = 0; i < 8; ++i) s += x[elem[8 * e + i]];
    out[e] = s / 8.0;
  }
  *rel_res = res;
done:
  free(b); free(dg); free(x); free(r); free(z); free(p); free(ap);
  return iters;
}

/* Symmetric 3x3 eigen-decomposition by cyclic Jacobi rotations (FP64).
 * Replaces LAPACK eigen (src/Core/Stress.jl:44).  Eigenvalues sorted
 * descending (Stress.jl:45-47); vec0 = unit eigenvector of the largest, its
 * sign fixed so that its largest-magnitude component is positive (LAPACK's
 * sign is arbitrary, so the reference's direction is defined up to sign). */
HXO_API void hxo_sym3_eigen(const double S[6], double ev[3], double vec0[3]) {
  double a[3][3] = {{S[0], S[3], S[5]}, {S[3], S[1], S[4]}, {S[5], S[4], S[2]}};
  double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    double scale = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off <= 1e-34 * scale || off == 0.0) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (a[p][q] == 0.0) continue;
        double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        double t = (theta >= 0 ? 1.0 : -1.0) /
                   (fabs(theta) + sqrt(theta * theta + 1.0));
        double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {
          double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {
          double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {
          double vkp = v[k][p], vkq = v[k][q];
          v[k][p] = c * vkp - s * vkq;
          v[k][q] = s * vkp + c * vkq;
        }
      }
  }
  int idx[3] = {0, 1, 2};
  double d[3] = {a[0][0], a[1][1], a[2][2]};
  for (int i = 0; i < 3; ++i)
    for (int j = i + 1; j < 3; ++j)
      if (d[idx[j]] > d[idx[i]]) {
        int t = idx[i];
        idx[i] = idx[j];
        idx[j] = t;
      }
  for (int i = 0; i < 3; ++i) ev[i] = d[idx[i]];
  double w[3] = {v[0][idx[0]], v[1][idx[0]], v[2][idx[0]]};
  double nrm = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  int big = 0;
  for (int i = 1; i < 3; ++i)
    if (fabs(w[i]) > fabs(w[big])) big = i;
  double sg = (w[big] < 0 ? -1.0 : 1.0) / nrm;
  for (int i = 0; i < 3; ++i) vec0[i] = w[i] * sg;
}

/* compute_stress_field, src/Core/Stress.jl:10-100.  Centre-point strain of
 * each element with E_local = E*density[e] (:86), von Mises (:52), principal
 * values sorted descending, L1 = sum |principal| (:90), Voigt
 * (xx,yy,zz,xy,yz,xz) (:96); elements with density <= 1e-6 are left 0
 * (:85).  nodes is nN x 3 row-major; outputs: principal[3*e+i], vm[e],
 * voigt[6*e+i], l1[e], dir[3*e+i]. */
HXO_API void hxo_stress(int64_t nN, int64_t nE, const int32_t *elem,
                        const double *nodes, const double *u, double E,
                        double nu, const double *density, double *principal,
                        double *vm, double *voigt, double *l1, double *dir) {
  (void)nN;
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < nE; ++e) {
    for (int i = 0; i < 3; ++i) principal[3 * e + i] = dir[3 * e + i] = 0.0;
    for (int i = 0; i < 6; ++i) voigt[6 * e + i] = 0.0;
    vm[e] = l1[e] = 0.0;
    if (!(density[e] > 1e-6)) continue;
    const int32_t *c = elem + 8 * e;
    double X[8][3], ue[24], N[8], dNdx[8][3], B[6][24], D[36];
    for (int i = 0; i < 8; ++i)
      for (int d = 0; d < 3; ++d) {
        X[i][d] = nodes[3 * (int64_t)c[i] + d];
        ue[3 * i + d] = u[3 * (int64_t)c[i] + d];
      }
    physical_gradients(X, 0.0, 0.0, 0.0, N, dNdx);
    bmatrix(dNdx, B);
    hxo_material_matrix(E * density[e], nu, D);
    double eps[6], sig[6];
    for (int i = 0; i < 6; ++i) {
      double s = 0;
      for (int j = 0; j < 24; ++j) s += B[i][j] * ue[j];
      eps[i] = s;
    }
    for (int i = 0; i < 6; ++i) {
      double s = 0;
      for (int j = 0; j < 6; ++j) s += D[i * 6 + j] * eps[j];
      sig[i] = s;
    }
    /* sym3 storage order: xx, yy, zz, xy, yz, xz */
    double ev[3], v0[3];
    hxo_sym3_eigen(sig, ev, v0);
    double sxx = sig[0], syy = sig[1], szz = sig[2];
    double sxy = sig[3], syz = sig[4], sxz = sig[5];
    vm[e] = sqrt(0.5 * ((sxx - syy) * (sxx - syy) + (syy - szz) * (syy - szz) +
                        (szz - sxx) * (szz - sxx)) +
                 3.0 * (sxy * sxy + syz * syz + sxz * sxz));
    l1[e] = fabs(ev[0]) + fabs(ev[1]) + fabs(ev[2]);
    for (int i = 0; i < 3; ++i) {
      principal[3 * e + i] = ev[i];
      dir[3 * e + i] = v0[i];
    }
    for (int i = 0; i < 6; ++i) voigt[6 * e + i] = sig[i];
  }
}

/* Element strain energy density ce_e = u_e^T Ke u_e (unit modulus).  No
 * reference counterpart: compliance sensitivities of the published OC method
 * (Bendsoe & Sigmund; the "top88"/"top3d" family). */
HXO_API void hxo_element_energy(int64_t nE, const int32_t *elem,
                                const double *ke, const double *u, double *ce) {
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < nE; ++e) {
    const int32_t *c = elem + 8 * e;
    double ue[24];
    for (int i = 0; i < 8; ++i)
      for (int d = 0; d < 3; ++d) ue[3 * i + d] = u[3 * (int64_t)c[i] + d];
    double s = 0;
    for (int i = 0; i < 24; ++i) {
      double t = 0;
      for (int j = 0; j < 24; ++j) t += ke[i * 24 + j] * ue[j];
      s += ue[i] * t;
    }
    ce[e] = s;
  }
}

/* Optimality-criteria update with bisection on the Lagrange multiplier
 * (published OC method; no reference counterpart).  Design variables in
 * [0,1]; x_new = clamp(x*sqrt(max(-dc,0)/(lmid*dv)), x-move, x+move) within
 * [0,1]; bisection from [0, 1e9] until (l2-l1)/(l1+l2) <= 1e-3, keeping
 * l1 = lmid while sum(x_new) > volfrac*nE.  Returns bisection steps. */
HXO_API int hxo_oc_update(int64_t nE, const double *x, const double *dc,
                          const double *dv, double volfrac, double move,
                          double *xnew, double *lambda_out) {
  double l1 = 0.0, l2 = 1e9, target = volfrac * (double)nE;
  int steps = 0;
  double lmid = 0.5 * (l1 + l2);
  while ((l2 - l1) / (l1 + l2) > 1e-3) {
    lmid = 0.5 * (l1 + l2);
    double vol = 0.0;
    for (int64_t e = 0; e < nE; ++e) {
      double be = sqrt(fmax(-dc[e], 0.0) / (lmid * dv[e]));
      double xn = x[e] * be;
      double lo = fmax(0.0, x[e] - move), hi = fmin(1.0, x[e] + move);
      xn = fmin(fmax(xn, lo), hi);
      xnew[e] = xn;
      vol += xn;
    }
    if (vol > target)
      l1 = lmid;
    else
      l2 = lmid;
    ++steps;
  }
  if (lambda_out) *lambda_out = lmid;
  return steps;
}
