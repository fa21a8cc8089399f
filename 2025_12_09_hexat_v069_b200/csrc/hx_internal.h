// hx_internal.h -- host-side internals shared by the library's translation
// units: grid description, device buffers, kernel launchers and the context.
#pragma once
#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_bf16.h>

#include "hx_common.cuh"

#define HX_GMG_MAX_LEVELS 10

namespace hx {

struct Grid {
  int nxe, nye, nze;  // elements per axis
  int nxn, nyn, nzn;  // nodes per axis (elements + 1)
  __host__ __device__ int64_t nodes() const { return (int64_t)nxn * nyn * nzn; }
  __host__ __device__ int64_t elems() const { return (int64_t)nxe * nye * nze; }
  __host__ __device__ int64_t dofs() const { return 3 * nodes(); }
};

// Owning device buffer (grown on demand, never shrunk while a context lives).
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  T* ensure(size_t count) {
    if (count > n) {
      if (p) HX_CUDA(cudaFree(p));
      p = nullptr;
      n = 0;
      HX_CUDA(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
      n = count;
    }
    return p;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// ---- operator (hx_operator.cu) ----
// z-chunk length for `resident` CTAs per SM; CTAs of one launch; the most
// CTAs of any precision (the reduction workspace's size)
int mv_kchunk(const Grid& g, int resident);
size_t mv_num_blocks(const Grid& g, int resident);
size_t mv_max_blocks(const Grid& g);
template <typename T>
void launch_matvec(cudaStream_t s, int mode, const T* x, T* y, const T* fac, const uint8_t* nmask,
                   const Grid& g, const ElemCoef<T>& K, T shift, CgState* st, double* partials,
                   double* out);
// Fused PCG step (see hx_operator.cu): p_out = M^-1 r + beta p_in,
// x += alpha_old p_in (owned nodes), q = mask(K p_out + s p_out),
// st->alpha = rz / (p_out . q).
template <typename T>
void launch_pcg_step(cudaStream_t s, const T* pin, T* pout, const T* r, const T* minv, T* x, T* q,
                     const T* fac, const uint8_t* nmask, const Grid& g, const ElemCoef<T>& K,
                     T shift, CgState* st, double* partials);
// Flexible-CG step: p_out = z + beta p_in, x += alpha_old p_in (owned
// nodes), q = mask(K p_out + s p_out), st->alpha = (z . r) / (p_out . q)
// with z . r in st->aux[3] (the preconditioner's output pass reduces it).
template <typename T>
void launch_fcg_step(cudaStream_t s, const T* pin, T* pout, const T* z, T* x, T* q, const T* fac,
                     const uint8_t* nmask, const Grid& g, const ElemCoef<T>& K, T shift,
                     CgState* st, double* partials);
// Multigrid smoothing (FP32): one Chebyshev step as a three-term recurrence,
// xprev_new <- x + omega (x - xprev_new) + gamma M^-1 (b - (K + sI) x) on the
// free DOFs (0 on the fixed ones; xprev_zero: x_prev = 0, not read); and the
// residual r = mask(b - (K + sI) x).
template <typename T>
void launch_cheb_step(cudaStream_t s, const T* x, T* xprev_new, bool xprev_zero, const T* b,
                      const T* minv, T omega, T gamma, const T* fac, const uint8_t* nmask,
                      const Grid& g, const ElemCoef<T>& K, T shift);
template <typename T>
void launch_residual(cudaStream_t s, const T* x, const T* b, T* r, const T* fac,
                     const uint8_t* nmask, const Grid& g, const ElemCoef<T>& K, T shift);
template <typename T>
void launch_node_diag(cudaStream_t s, const T* fac, const uint8_t* bcfree, uint8_t* nmask, T* diag,
                      const Grid& g, const ElemCoef<double>& K, double* partials, CgState* st,
                      double* out);
template <typename T>
void launch_minv(cudaStream_t s, const uint8_t* nmask, const T* diag, T* minv, int64_t nn,
                 double shift);

// ---- vector kernels (hx_vector.cu) ----
unsigned vec_blocks(int64_t n);
constexpr int VEC_THREADS = 256;
template <typename T>
void launch_cg_init(cudaStream_t s, const T* b, const T* q, const T* minv, T* r, T* p, int64_t n,
                    CgState* st, double* partials);
template <typename T>
void launch_cg_update(cudaStream_t s, T* x, const T* p, T* r, const T* q, const T* minv, int64_t n,
                      CgState* st, double* partials);
template <typename T>
void launch_cg_pupdate(cudaStream_t s, T* p, const T* r, const T* minv, int64_t n, CgState* st);
// ys (optional, n + 8 entries): BF16(D^-1/2 r) of the new residual, the
// learned preconditioner's input
template <typename T>
void launch_cg_update2(cudaStream_t s, T* r, const T* q, const T* minv, int64_t n, CgState* st,
                       double* partials, __nv_bfloat16* ys = nullptr);
template <typename T>
void launch_dinv_bf16(cudaStream_t s, const T* r, const T* minv, __nv_bfloat16* ys, int64_t n);
template <typename T>
void launch_axpy_state(cudaStream_t s, T* dst, const T* x, const T* p, int64_t n,
                       const CgState* st, int when_snap);
void launch_copy_if_snap(cudaStream_t s, double* dst, const double* src, int64_t n, CgState* st);
// out = sum (b - q)^2 over the n entries, and sum b^2
void launch_resid_norm(cudaStream_t s, const double* b, const double* q, int64_t n, CgState* st,
                       double* partials, double* out2);
// b = minv != 0 ? f : 0
template <typename T>
void launch_mask_rhs(cudaStream_t s, const double* f, const T* minv, double* b, int64_t n);
// dot product, deterministic: out = sum a*b
void launch_dot(cudaStream_t s, const double* a, const double* b, int64_t n, CgState* st,
                double* partials, double* out);
// Mixed precision helpers.
// r = b - q (FP64), r32 = r * scale_from_state; also ||r||^2 into st->rr etc.
void launch_ir_residual(cudaStream_t s, const double* b, const double* q, float* r32, int64_t n,
                        CgState* st, double* partials);
void launch_ir_correct(cudaStream_t s, double* x, const float* d32, int64_t n, const CgState* st);
template <typename TD, typename TS>
void launch_convert(cudaStream_t s, TD* dst, const TS* src, int64_t n);
void launch_fill_zero(cudaStream_t s, void* p, size_t bytes);
// fac = density >= thr ? E * density : 0 (Float32 product, as the reference)
void launch_threshold_factor(cudaStream_t s, const float* dens, float thr, float E, double* fac,
                             int64_t n);
// free-DOF bits per node from a column-major nN x 3 bc_indicator
void launch_bc_bits(cudaStream_t s, const float* bc, uint8_t* free_bits, int64_t nn);
// r = a - b
void launch_axpby(cudaStream_t s, double* r, const double* a, const double* b, int64_t n);

// ---- filter (hx_filter.cu) ----
struct FilterCoef {
  // assembled 1D tridiagonal entries per axis: [axis][0=boundary-lo row,
  // 1=interior, 2=boundary-hi row][lo, diag, hi] for S and M
  double S[3][3][3];
  double M[3][3][3];
  double r2;
  double vol8;
};
FilterCoef make_filter_coef(double dx, double dy, double dz, double radius, int ref_compat);
void launch_filter_rhs(cudaStream_t s, const double* rho, double* b, const Grid& g, double vol8);
void launch_filter_invdiag(cudaStream_t s, double* invd, const Grid& g, const FilterCoef& F);
void launch_filter_matvec(cudaStream_t s, const double* x, double* y, const Grid& g,
                          const FilterCoef& F, CgState* st, double* partials);
void launch_filter_extract(cudaStream_t s, const double* x, double* out, const Grid& g);

// ---- stress / OC (hx_stress.cu) ----
void launch_stress(cudaStream_t s, const double* u, const double* dens, double E, double nu,
                   const Grid& g, double hx, double hy, double hz, double* principal, double* vm,
                   double* voigt, double* l1, double* dir);
void launch_energy(cudaStream_t s, const double* u, const Grid& g, const ElemCoef<double>& K,
                   double* ce);
// fac = emin + rho^p (e0 - emin); sensitivity: out = -p rho^(p-1) (e0 - emin) * out
void launch_simp(cudaStream_t s, const double* rho, double p, double e0, double emin, double* out,
                 int64_t n, bool sensitivity);
// sigma_PN = (sum vm^P)^(1/P): st->aux[0] = max vm, st->aux[1] = sum (vm/max)^P
void launch_pnorm(cudaStream_t s, const double* vm, int64_t n, double P, CgState* st,
                  double* partials);
void launch_oc(cudaStream_t s, const double* x, const double* dc, const double* dv, int64_t n,
               double volfrac, double move, double* xnew, CgState* st, double* partials,
               int max_steps);

}  // namespace hx

// ---------------------------------------------------------------------------
// The context behind the opaque hx_ctx handle.
// ---------------------------------------------------------------------------
struct hx_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_in = nullptr;  // orders the stream after the legacy default stream
  // preconditioner, precision and multigrid fallback of the reference-shaped
  // drop-in solves (the reference's "jacobi_amg" by default)
  int32_t dropin_pc = 0, dropin_prec = 0, dropin_fallback = 1;
  std::string err;

  // mesh
  bool has_mesh = false;
  hx::Grid g{};
  double h[3] = {1, 1, 1};
  double E = 1.0, nu = 0.3;
  hx::ElemCoef<double> K{};
  // caller numbering -> grid numbering (empty vectors: identity)
  std::vector<int64_t> node_map;  // caller node -> grid node
  std::vector<int64_t> elem_map;  // caller element -> grid element
  int64_t n_user_nodes = 0, n_user_elem = 0;
  std::vector<uint8_t> present;   // grid node present in the caller's mesh

  // boundary conditions: per grid node free-DOF bits
  std::vector<uint8_t> bcfree;
  bool bc_dirty = true;

  // device buffers
  hx::DevBuf<uint8_t> d_bcfree, d_nmask;
  hx::DevBuf<double> d_f, d_b, d_fac, d_x, d_r, d_p, d_p2, d_q, d_minv, d_xbest;
  hx::DevBuf<double> d_partials, d_scalars;
  hx::DevBuf<hx::CgState> d_state;
  hx::DevBuf<float> d_fac32, d_minv32, d_r32, d_p32, d_p32b, d_q32, d_x32;
  hx::DevBuf<double> d_aux0, d_aux1, d_aux2, d_aux3, d_aux4, d_aux5;
  hx::CgState* h_state = nullptr;  // pinned mirror

  // host<->device staging for F32 callers
  hx::DevBuf<char> d_stage;

  // filter grid and cache (the counterpart of GLOBAL_HELMHOLTZ_CACHE)
  hx::Grid fg{};
  double fh[3] = {1, 1, 1};
  bool filt_ready = false;
  double filt_radius = -1;
  int filt_compat = -1;
  hx::DevBuf<double> f_invd, f_x, f_r, f_p, f_q, f_b, f_rho, f_out;

  // filter kernel coefficients of the last filter call (for timing)
  double f_radius_last = 0;
  int f_compat_last = 0;
  bool f_used = false;

  int64_t launches = 0;  // kernels launched on behalf of this context

  // geometric multigrid hierarchy (hx_gmg.cu): FP32 levels, level 0 = the mesh's grid
  struct GmgLevel {
    hx::Grid g{};
    double h[3] = {1, 1, 1};
    hx::ElemCoef<float> K{};
    float shift = 0.f, lmax = 1.f;  // operator shift; lambda_max(D^-1 A)
    hx::DevBuf<float> fac, minv, b, x, r, d, q;
    hx::DevBuf<uint8_t> bc, nmask;  // BC bits; free-DOF mask (BC and stiffness)
  };
  struct Gmg {
    bool ready = false;
    int nl = 0;
    GmgLevel lv[HX_GMG_MAX_LEVELS];
    hx::DevBuf<hx::CgState> coarse_st;
    hx::DevBuf<float> p0, p1;   // coarse PCG directions
    hx::DevBuf<double> z, s;    // FCG: preconditioned residual, scratch
    // direct coarsest-level solve: dense inverse (FP32, n x n) of the masked
    // coarsest operator, formed in FP64 at set-up
    bool direct = false;
    hx::DevBuf<double> dense, gj;  // FP64 matrix being inverted; pivot row/column buffers
    hx::DevBuf<float> ainv;
    hx::DevBuf<double> lanczos;  // (alpha, beta, status) per step of the lambda_max estimate
    double setup_ms = 0;         // set-up time accumulated over the current solve
    int degree = 2;              // Chebyshev degree per smoothing
  } gmg;

  // lattice origin of the mesh (the minimum node coordinates; 0 for hx_set_grid)
  double origin[3] = {0, 0, 0};

  // webdata export (hx_export.cu): per-block survivor counts and offsets, outputs
  struct Export {
    hx::DevBuf<unsigned long long> counts, offsets;
    hx::DevBuf<float> cent, dens, sl1;
  } exp;

  // density update (hx_update.cu): Float32 fields, FP64 filter buffers
  struct Update {
    hx::DevBuf<float> dens, l1, orig, dc, fout;
    hx::DevBuf<uint8_t> prot;
    hx::DevBuf<double> a, b, c, d;
    hx::DevBuf<unsigned int> hist;
  } upd;

  // convolutional preconditioner networks (see hx_net.cu)
  struct Net {
    bool ready = false;
    int step = 0;  // Adam steps taken
    hx::DevBuf<float> w, m, v, grad, part;
    hx::DevBuf<unsigned char> live;
    hx::DevBuf<__nv_bfloat16> wf, wb, da, db, tmp[2];
    struct Level {  // one node-grid level (0 = the mesh's node grid)
      hx::DevBuf<float> x, acc, gx, feat;  // [node][3] fields, [node] feature
      hx::DevBuf<__nv_bfloat16> x0, y, act[7];  // network input, output, training activations
      hx::DevBuf<__nv_bfloat16> pp[2];          // application ping-pong (levels >= 2)
    } lv[8];
    // side streams and events: the coarser networks run beside the finest;
    // ev_x[i]: side i's level restricted, ev_join[i]: its correction summed
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_x[2] = {nullptr, nullptr}, ev_join[2] = {nullptr, nullptr};
    hx::DevBuf<double> z, scal, facbuf;
    hx::DevBuf<float> z32, s32;  // mixed-precision FCG: preconditioned vector, scratch
    hx::DevBuf<__nv_bfloat16> ys;  // FCG: BF16(D^-1/2 r), n + 8 entries
    hx::DevBuf<int> err;         // set by a conv CTA whose bounded wait ran out
    const double* fac_last = nullptr;  // factors the operator inputs were built for
    int64_t prepared_dofs = -1;        // DOF count of the mesh they were built on
  } net;

  size_t partial_capacity() const { return d_partials.n; }
};
