// hx_vector.cu -- fused Krylov vector kernels with device-side scalars.
//
// One CG iteration of the reference (src/Solvers/GPUSolver.jl:452-526) is
// ~8 broadcast kernels plus 3 cuBLAS dots, each dot a host round trip.  Here
// it is two kernels and no host round trip:
//   PCG step (hx_operator.cu):  p = M^-1 r + beta p_old; x += alpha_old p_old;
//                  q = A p; pq = p.q; alpha = rz/pq
//   k_cg_update2:  r -= alpha q; z = M^-1 r (not stored); rz' = r.z,
//                  rr = r.r; convergence / divergence tests; beta = rz'/rz
// x lags one step behind (x += alpha p happens in the next PCG step); the
// host applies the last step with k_axpy_state once the loop stops.
// The three-kernel form (k_cg_update + k_cg_pupdate around a plain matvec)
// is kept for the Helmholtz filter, whose operator is not fused.
// All reductions are FP64 and deterministic (fixed-order block partials).
#include "hx_internal.h"

namespace hx {

namespace {

template <typename T>
struct Vec2;
template <>
struct Vec2<double> {
  using type = double2;
};
template <>
struct Vec2<float> {
  using type = float2;
};

// 16 bytes of T, loaded and stored as one vector (W entries)
template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
  using type = double2;
  static constexpr int W = 2;
  __device__ static void get(const double2& v, double (&a)[2]) { a[0] = v.x; a[1] = v.y; }
  __device__ static double2 make(const double (&a)[2]) { return make_double2(a[0], a[1]); }
};
template <>
struct Vec16<float> {
  using type = float4;
  static constexpr int W = 4;
  __device__ static void get(const float4& v, float (&a)[4]) {
    a[0] = v.x;
    a[1] = v.y;
    a[2] = v.z;
    a[3] = v.w;
  }
  __device__ static float4 make(const float (&a)[4]) { return make_float4(a[0], a[1], a[2], a[3]); }
};

__device__ __forceinline__ uint32_t bf16x2_bits(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

__device__ __forceinline__ int64_t gtid() {
  return (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
}
__device__ __forceinline__ int64_t gstride() { return (int64_t)gridDim.x * blockDim.x; }

// r = b - q (q may be null), z = M^-1 r, p = z; reduces rz, rr, bb.
template <typename T>
__global__ void k_cg_init(const T* __restrict__ b, const T* __restrict__ q,
                          const T* __restrict__ minv, T* __restrict__ r, T* __restrict__ p,
                          int64_t n, CgState* st, double* partials) {
  double rz = 0, rr = 0, bb = 0;
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const T bi = b[i];
    const T ri = q ? bi - q[i] : bi;
    const T zi = minv[i] * ri;
    r[i] = ri;
    p[i] = zi;
    rz += (double)ri * (double)zi;
    rr += (double)ri * (double)ri;
    bb += (double)bi * (double)bi;
  }
  double v[3] = {rz, rr, bb};
  if (grid_reduce<3>(v, partials, &st->ticket[TK_INIT]) && threadIdx.x == 0) {
    st->rz = v[0];
    st->rr = v[1];
    st->bnorm = sqrt(v[2]);
    st->iter = 0;
    st->best_rel = INFINITY;
    st->snap = 0;
    if (st->bnorm == 0.0) {
      st->rel_res = 0.0;
      st->status = HX_ST_ZERO_RHS;
    } else {
      st->rel_res = sqrt(v[1]) / st->bnorm;
      st->status = isfinite(st->rel_res) ? HX_RUNNING : HX_ST_NONFINITE;
    }
  }
}

// Finalisation shared by the update kernels (runs in one thread).
__device__ __forceinline__ void cg_finish_iteration(CgState* st, double rzn, double rr) {
  st->iter += 1;
  const double rel = sqrt(rr) / st->bnorm;
  st->rr = rr;
  const bool tested = (st->iter % st->check_every) == 0;
  if (tested) st->rel_res = rel;
  int status = HX_RUNNING;
  // Order of tests as src/Solvers/GPUSolver.jl:478-511.
  if (st->div_ratio > 0.0 && st->iter > 50 && rel > st->div_ratio * st->best_rel)
    status = HX_ST_DIVERGED;
  else if (!isfinite(rel))
    status = HX_ST_NONFINITE;
  else if (st->explode > 0.0 && rel > st->explode)
    status = HX_ST_DIVERGED;
  if (status == HX_RUNNING) {
    st->snap = 0;
    if (rel < st->best_rel) {
      st->best_rel = rel;
      if (st->keep_best && rel < 1e-2) st->snap = 1;
    }
    if (tested && rel < st->tol) {
      status = HX_ST_CONVERGED;
      if (st->keep_best) st->snap = 1;
    } else if (st->iter >= st->max_iter) {
      status = HX_ST_MAXITER;
    } else if (st->aux[1] > 0.0) {
      // reliable updates: pause once the recursive residual has dropped by
      // delta since the last FP64 residual replacement
      if (rr > st->aux[2]) st->aux[2] = rr;
      if (rr < st->aux[1] * st->aux[1] * st->aux[2]) status = HX_ST_PAUSED;
    }
    st->beta = rzn / st->rz;
    st->rz = rzn;
  }
  if (!tested && status != HX_RUNNING) st->rel_res = rel;
  st->status = status;
}

template <typename T>
__global__ void k_cg_update(T* __restrict__ x, const T* __restrict__ p, T* __restrict__ r,
                            const T* __restrict__ q, const T* __restrict__ minv, int64_t n,
                            CgState* st, double* partials) {
  if (st->status != HX_RUNNING) return;
  const T alpha = (T)st->alpha;
  double rz = 0, rr = 0;
  using V = typename Vec2<T>::type;
  const int64_t n2 = n >> 1;
  V* x2 = reinterpret_cast<V*>(x);
  V* r2 = reinterpret_cast<V*>(r);
  const V* p2 = reinterpret_cast<const V*>(p);
  const V* q2 = reinterpret_cast<const V*>(q);
  const V* m2 = reinterpret_cast<const V*>(minv);
  for (int64_t i = gtid(); i < n2; i += gstride()) {
    V xv = x2[i], rv = r2[i];
    const V pv = p2[i], qv = q2[i], mv = m2[i];
    xv.x += alpha * pv.x;
    xv.y += alpha * pv.y;
    rv.x -= alpha * qv.x;
    rv.y -= alpha * qv.y;
    x2[i] = xv;
    r2[i] = rv;
    rz += (double)rv.x * (double)(mv.x * rv.x) + (double)rv.y * (double)(mv.y * rv.y);
    rr += (double)rv.x * (double)rv.x + (double)rv.y * (double)rv.y;
  }
  if ((n & 1) && gtid() == 0) {
    const int64_t i = n - 1;
    x[i] += alpha * p[i];
    const T ri = r[i] - alpha * q[i];
    r[i] = ri;
    rz += (double)ri * (double)(minv[i] * ri);
    rr += (double)ri * (double)ri;
  }
  double v[2] = {rz, rr};
  if (grid_reduce<2>(v, partials, &st->ticket[TK_UPDATE]) && threadIdx.x == 0)
    cg_finish_iteration(st, v[0], v[1]);
}

// Second half of a fused PCG iteration: r -= alpha q, dots, tests.  With
// ys: also ys = BF16(D^-1/2 r) of the new residual (the learned
// preconditioner's input, D^-1/2 = sqrt(minv)).  16-byte vector accesses
// (4 FP32 or 2 FP64 entries per thread and step), then a scalar tail.
template <typename T>
__global__ void k_cg_update2(T* __restrict__ r, const T* __restrict__ q,
                             const T* __restrict__ minv, int64_t n, CgState* st,
                             double* partials, __nv_bfloat16* __restrict__ ys) {
  if (st->status != HX_RUNNING) return;
  const T alpha = (T)st->alpha;
  double rz = 0, rr = 0;
  using VT = Vec16<T>;
  using V = typename VT::type;
  constexpr int W = VT::W;
  const int64_t nv = n / W;
  V* rV = reinterpret_cast<V*>(r);
  const V* qV = reinterpret_cast<const V*>(q);
  const V* mV = reinterpret_cast<const V*>(minv);
  for (int64_t i = gtid(); i < nv; i += gstride()) {
    T ra[W], qa[W], ma[W];
    VT::get(rV[i], ra);
    VT::get(qV[i], qa);
    VT::get(mV[i], ma);
    float ya[W];
#pragma unroll
    for (int e = 0; e < W; ++e) {
      ra[e] -= alpha * qa[e];
      ya[e] = dinv_sqrt((float)ma[e]) * (float)ra[e];
      rz += (double)ra[e] * (double)(ma[e] * ra[e]);
      rr += (double)ra[e] * (double)ra[e];
    }
    rV[i] = VT::make(ra);
    if (ys) {
      if constexpr (W == 4)
        reinterpret_cast<uint2*>(ys)[i] =
            make_uint2(bf16x2_bits(ya[0], ya[1]), bf16x2_bits(ya[2], ya[3]));
      else
        reinterpret_cast<uint32_t*>(ys)[i] = bf16x2_bits(ya[0], ya[1]);
    }
  }
  for (int64_t i = nv * W + gtid(); i < n; i += gstride()) {
    const T ri = r[i] - alpha * q[i];
    r[i] = ri;
    if (ys) ys[i] = __float2bfloat16_rn(dinv_sqrt((float)minv[i]) * (float)ri);
    rz += (double)ri * (double)(minv[i] * ri);
    rr += (double)ri * (double)ri;
  }
  double v[2] = {rz, rr};
  if (grid_reduce<2>(v, partials, &st->ticket[TK_UPDATE]) && threadIdx.x == 0)
    cg_finish_iteration(st, v[0], v[1]);
}

// ys = BF16(D^-1/2 r), as k_cg_update2 writes it (for a residual that
// another kernel produced).
template <typename T>
__global__ void k_dinv_bf16(const T* __restrict__ r, const T* __restrict__ minv,
                            __nv_bfloat16* __restrict__ ys, int64_t n) {
  for (int64_t i = gtid(); i < n; i += gstride())
    ys[i] = __float2bfloat16_rn(dinv_sqrt((float)minv[i]) * (float)r[i]);
}

// dst = x + alpha p, with alpha from the state; `when_snap` restricts it to
// iterations flagged as the best so far.
template <typename T>
__global__ void k_axpy_state(T* __restrict__ dst, const T* __restrict__ x,
                             const T* __restrict__ p, int64_t n, const CgState* st,
                             int when_snap) {
  // when_snap 1 / 2: a best-iterate snapshot, taken only if the last
  // iteration asked for one and its direction p_k is the buffer given (P0
  // after iteration k = iter - 1 even, P1 after an odd one).  Launches of a
  // batch that run after the loop stopped then rewrite the same snapshot
  // instead of combining x with an older direction.
  if (when_snap && !(st->snap && ((st->iter - 1) & 1) == when_snap - 1)) return;
  const T a = (T)st->alpha;
  for (int64_t i = gtid(); i < n; i += gstride()) dst[i] = x[i] + a * p[i];
}

template <typename T>
__global__ void k_cg_pupdate(T* __restrict__ p, const T* __restrict__ r,
                             const T* __restrict__ minv, int64_t n, const CgState* st) {
  if (st->status != HX_RUNNING) return;
  const T beta = (T)st->beta;
  using V = typename Vec2<T>::type;
  const int64_t n2 = n >> 1;
  V* p2 = reinterpret_cast<V*>(p);
  const V* r2 = reinterpret_cast<const V*>(r);
  const V* m2 = reinterpret_cast<const V*>(minv);
  for (int64_t i = gtid(); i < n2; i += gstride()) {
    V pv = p2[i];
    const V rv = r2[i], mv = m2[i];
    pv.x = mv.x * rv.x + beta * pv.x;
    pv.y = mv.y * rv.y + beta * pv.y;
    p2[i] = pv;
  }
  if ((n & 1) && gtid() == 0) p[n - 1] = minv[n - 1] * r[n - 1] + beta * p[n - 1];
}

__global__ void k_copy_if_snap(double* __restrict__ dst, const double* __restrict__ src,
                               int64_t n, const CgState* st) {
  if (!st->snap) return;
  for (int64_t i = gtid(); i < n; i += gstride()) dst[i] = src[i];
}

__global__ void k_resid_norm(const double* __restrict__ b, const double* __restrict__ q,
                             int64_t n, CgState* st, double* partials, double* out2) {
  double rr = 0, bb = 0;
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const double bi = b[i], ri = bi - q[i];
    rr += ri * ri;
    bb += bi * bi;
  }
  double v[2] = {rr, bb};
  if (grid_reduce<2>(v, partials, &st->ticket[TK_AUX2]) && threadIdx.x == 0) {
    out2[0] = v[0];
    out2[1] = v[1];
  }
}

template <typename T>
__global__ void k_mask_rhs(const double* __restrict__ f, const T* __restrict__ minv,
                           double* __restrict__ b, int64_t n) {
  for (int64_t i = gtid(); i < n; i += gstride()) b[i] = (minv[i] != T(0)) ? f[i] : 0.0;
}

__global__ void k_dot(const double* __restrict__ a, const double* __restrict__ b, int64_t n,
                      CgState* st, double* partials, double* out) {
  double s = 0;
  for (int64_t i = gtid(); i < n; i += gstride()) s += a[i] * b[i];
  double v[1] = {s};
  if (grid_reduce<1>(v, partials, &st->ticket[TK_AUX2]) && threadIdx.x == 0) out[0] = v[0];
}

// Outer step of mixed-precision refinement: r = b - q in FP64, r32 = r/||b||,
// ||r|| reduced; convergence of the outer loop decided on the true residual.
__global__ void k_ir_residual(const double* __restrict__ b, const double* __restrict__ q,
                              float* __restrict__ r32, int64_t n, CgState* st,
                              double* partials) {
  if (st->status != HX_RUNNING) return;
  const double inv_b = 1.0 / st->bnorm;
  double rr = 0;
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const double ri = b[i] - q[i];
    r32[i] = (float)(ri * inv_b);
    rr += ri * ri;
  }
  double v[1] = {rr};
  if (grid_reduce<1>(v, partials, &st->ticket[TK_UPDATE]) && threadIdx.x == 0) {
    const double rel = sqrt(v[0]) / st->bnorm;
    st->rr = v[0];
    st->rel_res = rel;
    if (!isfinite(rel))
      st->status = HX_ST_NONFINITE;
    else if (rel < st->tol)
      st->status = HX_ST_CONVERGED;
    else if (st->iter >= st->max_iter)
      st->status = HX_ST_MAXITER;
    st->iter += 1;
  }
}

__global__ void k_ir_correct(double* __restrict__ x, const float* __restrict__ d32, int64_t n,
                             const CgState* st) {
  const double sb = st->bnorm;
  for (int64_t i = gtid(); i < n; i += gstride()) x[i] += sb * (double)d32[i];
}

template <typename TD, typename TS>
__global__ void k_convert(TD* __restrict__ dst, const TS* __restrict__ src, int64_t n) {
  for (int64_t i = gtid(); i < n; i += gstride()) dst[i] = (TD)src[i];
}

}  // namespace

unsigned vec_blocks(int64_t n) {
  const int64_t want = cdiv(std::max<int64_t>(n / 2, 1), VEC_THREADS);
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, 8LL * sm_count()));
}

template <typename T>
void launch_cg_init(cudaStream_t s, const T* b, const T* q, const T* minv, T* r, T* p, int64_t n,
                    CgState* st, double* partials) {
  k_cg_init<T><<<vec_blocks(n), VEC_THREADS, 0, s>>>(b, q, minv, r, p, n, st, partials);
  HX_CHECK_LAUNCH();
}

template <typename T>
void launch_cg_update(cudaStream_t s, T* x, const T* p, T* r, const T* q, const T* minv, int64_t n,
                      CgState* st, double* partials) {
  k_cg_update<T><<<vec_blocks(n), VEC_THREADS, 0, s>>>(x, p, r, q, minv, n, st, partials);
  HX_CHECK_LAUNCH();
}

template <typename T>
void launch_cg_pupdate(cudaStream_t s, T* p, const T* r, const T* minv, int64_t n, CgState* st) {
  k_cg_pupdate<T><<<vec_blocks(n), VEC_THREADS, 0, s>>>(p, r, minv, n, st);
  HX_CHECK_LAUNCH();
}

template <typename T>
void launch_cg_update2(cudaStream_t s, T* r, const T* q, const T* minv, int64_t n, CgState* st,
                       double* partials, __nv_bfloat16* ys) {
  k_cg_update2<T><<<vec_blocks(n), VEC_THREADS, 0, s>>>(r, q, minv, n, st, partials, ys);
  HX_CHECK_LAUNCH();
}

template <typename T>
void launch_dinv_bf16(cudaStream_t s, const T* r, const T* minv, __nv_bfloat16* ys, int64_t n) {
  k_dinv_bf16<T><<<vec_blocks(n), VEC_THREADS, 0, s>>>(r, minv, ys, n);
  HX_CHECK_LAUNCH();
}

template <typename T>
void launch_axpy_state(cudaStream_t s, T* dst, const T* x, const T* p, int64_t n,
                       const CgState* st, int when_snap) {
  k_axpy_state<T><<<vec_blocks(n), VEC_THREADS, 0, s>>>(dst, x, p, n, st, when_snap);
  HX_CHECK_LAUNCH();
}

#define HX_INST_CG(T)                                                                         \
  template void launch_cg_init<T>(cudaStream_t, const T*, const T*, const T*, T*, T*, int64_t, \
                                  CgState*, double*);                                         \
  template void launch_cg_update<T>(cudaStream_t, T*, const T*, T*, const T*, const T*,       \
                                    int64_t, CgState*, double*);                              \
  template void launch_cg_pupdate<T>(cudaStream_t, T*, const T*, const T*, int64_t, CgState*); \
  template void launch_cg_update2<T>(cudaStream_t, T*, const T*, const T*, int64_t, CgState*,  \
                                     double*, __nv_bfloat16*);                                 \
  template void launch_dinv_bf16<T>(cudaStream_t, const T*, const T*, __nv_bfloat16*,         \
                                    int64_t);                                                  \
  template void launch_axpy_state<T>(cudaStream_t, T*, const T*, const T*, int64_t,            \
                                     const CgState*, int);
HX_INST_CG(double)
HX_INST_CG(float)

void launch_copy_if_snap(cudaStream_t s, double* dst, const double* src, int64_t n, CgState* st) {
  k_copy_if_snap<<<vec_blocks(n), VEC_THREADS, 0, s>>>(dst, src, n, st);
  HX_CHECK_LAUNCH();
}

void launch_resid_norm(cudaStream_t s, const double* b, const double* q, int64_t n, CgState* st,
                       double* partials, double* out2) {
  k_resid_norm<<<vec_blocks(n), VEC_THREADS, 0, s>>>(b, q, n, st, partials, out2);
  HX_CHECK_LAUNCH();
}

template <typename T>
void launch_mask_rhs(cudaStream_t s, const double* f, const T* minv, double* b, int64_t n) {
  k_mask_rhs<T><<<vec_blocks(n), VEC_THREADS, 0, s>>>(f, minv, b, n);
  HX_CHECK_LAUNCH();
}
template void launch_mask_rhs<double>(cudaStream_t, const double*, const double*, double*,
                                      int64_t);
template void launch_mask_rhs<float>(cudaStream_t, const double*, const float*, double*, int64_t);

void launch_dot(cudaStream_t s, const double* a, const double* b, int64_t n, CgState* st,
                double* partials, double* out) {
  k_dot<<<vec_blocks(n), VEC_THREADS, 0, s>>>(a, b, n, st, partials, out);
  HX_CHECK_LAUNCH();
}

void launch_ir_residual(cudaStream_t s, const double* b, const double* q, float* r32, int64_t n,
                        CgState* st, double* partials) {
  k_ir_residual<<<vec_blocks(n), VEC_THREADS, 0, s>>>(b, q, r32, n, st, partials);
  HX_CHECK_LAUNCH();
}

void launch_ir_correct(cudaStream_t s, double* x, const float* d32, int64_t n,
                       const CgState* st) {
  k_ir_correct<<<vec_blocks(n), VEC_THREADS, 0, s>>>(x, d32, n, st);
  HX_CHECK_LAUNCH();
}

template <typename TD, typename TS>
void launch_convert(cudaStream_t s, TD* dst, const TS* src, int64_t n) {
  k_convert<TD, TS><<<vec_blocks(n), VEC_THREADS, 0, s>>>(dst, src, n);
  HX_CHECK_LAUNCH();
}
template void launch_convert<float, double>(cudaStream_t, float*, const double*, int64_t);
template void launch_convert<double, float>(cudaStream_t, double*, const float*, int64_t);
template void launch_convert<double, double>(cudaStream_t, double*, const double*, int64_t);

__global__ void k_sub(double* __restrict__ r, const double* __restrict__ a,
                      const double* __restrict__ b, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    r[i] = a[i] - b[i];
}
void launch_axpby(cudaStream_t s, double* r, const double* a, const double* b, int64_t n) {
  k_sub<<<vec_blocks(n), VEC_THREADS, 0, s>>>(r, a, b, n);
  HX_CHECK_LAUNCH();
}

// Device-side pruning of the reference's solve entry (src/Solvers/Solver.jl:
// 60-91 with src/Mesh/MeshPruner.jl:18-112): element factor E * density
// where density >= thr (GPUSolver.jl:128,147), else 0; nodes left without
// stiffness are then held at 0 by the node mask, which is what the
// reference's prune-solve-reconstruct returns for them.
__global__ void k_threshold_factor(const float* __restrict__ dens, float thr, float E,
                                   double* __restrict__ fac, int64_t n) {
  for (int64_t e = gtid(); e < n; e += gstride()) {
    const float d = dens[e];
    fac[e] = d >= thr ? (double)(E * d) : 0.0;
  }
}

// Free-DOF bits per node from the reference's bc_indicator (nN x 3 Float32,
// column-major, > 0 = fixed; src/Core/Boundary.jl:135-160).
__global__ void k_bc_bits(const float* __restrict__ bc, uint8_t* __restrict__ free_bits,
                          int64_t nn) {
  for (int64_t i = gtid(); i < nn; i += gstride()) {
    unsigned m = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d)
      if (!(bc[d * nn + i] > 0.0f)) m |= 1u << d;
    free_bits[i] = (uint8_t)m;
  }
}

void launch_threshold_factor(cudaStream_t s, const float* dens, float thr, float E, double* fac,
                             int64_t n) {
  k_threshold_factor<<<vec_blocks(n), VEC_THREADS, 0, s>>>(dens, thr, E, fac, n);
  HX_CHECK_LAUNCH();
}

void launch_bc_bits(cudaStream_t s, const float* bc, uint8_t* free_bits, int64_t nn) {
  k_bc_bits<<<vec_blocks(nn), VEC_THREADS, 0, s>>>(bc, free_bits, nn);
  HX_CHECK_LAUNCH();
}

void launch_fill_zero(cudaStream_t s, void* p, size_t bytes) {
  HX_CUDA(cudaMemsetAsync(p, 0, bytes, s));
}

}  // namespace hx
