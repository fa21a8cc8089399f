// hx_operator.cu -- structured-grid Hex8 stiffness operator K(f) x.
//
// Layout in HBM: node n = i + NXn*(j + NYn*k) (i fastest, src/Mesh/Mesh.jl:
// 114-116), vectors interleaved 3 per node (dof = 3n + c), element
// e = i + NXe*(j + NYe*k) (Mesh.jl:145-156), one factor per element, one
// byte of free-DOF bits per node.
//
// Kernel design (replaces the one-thread-per-element, 24-atomics kernel of
// src/Solvers/GPUSolver.jl:37-79):
//  * a CTA owns a 31 x (BY-1) column of output nodes and marches along z
//    over a chunk of node planes; its 32 x BY threads each own one element
//    column, recomputing the one-element halo in x and y (atomic-free and
//    deterministic);
//  * node planes are staged into shared memory with cp.async (zero-filled
//    outside the grid), double-buffered so the next plane loads while the
//    current element layer computes;
//  * each element product runs in the Haar basis (45 nonzeros, see
//    hx_common.cuh); bottom-corner results meet the carried top-corner
//    results of the layer below in registers, then the four element columns
//    around a node are summed with one warp shuffle (x) and one shared-memory
//    exchange (y);
//  * the epilogue applies the free-DOF mask and the diagonal shift and
//    accumulates p.q for the CG step, reduced deterministically.
#include "hx_internal.h"

namespace hx {

namespace {

constexpr int MV_BX = 32;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

template <int BYTES>
__device__ __forceinline__ void cp_async_zfill(void* sdst, const void* gsrc, bool valid) {
  const unsigned n = valid ? BYTES : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(smem_u32(sdst)),
               "l"(gsrc), "n"(BYTES), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

template <typename T, int BY>
struct MvSmem {
  T xs[2][BY + 1][MV_BX + 1][3];
  T red[BY][MV_BX][3];
};

// Issue the copies of node plane kp (tile incl. one-node halo) into slot.
template <typename T, int BY>
__device__ __forceinline__ void issue_plane(MvSmem<T, BY>& sm, int slot, const T* __restrict__ x,
                                            const Grid& g, int i0, int j0, int kp, int tid) {
  constexpr int ROW = (MV_BX + 1) * 3;
  constexpr int NT = MV_BX * BY;
  const bool kin = kp >= 0 && kp < g.nzn;
  const int64_t base = (int64_t)kp * g.nxn * g.nyn;
  for (int idx = tid; idx < (BY + 1) * ROW; idx += NT) {
    const int b = idx / ROW, rem = idx - b * ROW;
    const int a = rem / 3, c = rem - a * 3;
    const int ii = i0 - 1 + a, jj = j0 - 1 + b;
    const bool ok = kin && ii >= 0 && ii < g.nxn && jj >= 0 && jj < g.nyn;
    const T* src = ok ? x + 3 * (base + (int64_t)jj * g.nxn + ii) + c : x;
    cp_async_zfill<sizeof(T)>(&sm.xs[slot][b][a][c], src, ok);
  }
  cp_async_commit();
}

// MODE 0: y = mask(K x + s x);  MODE 1: also out[0] = sum x.y;
// MODE 2: CG step, st->pq = p.q, st->alpha = rz / pq, breakdown detection.
template <typename T, int BY, int MODE>
__global__ void __launch_bounds__(MV_BX* BY)
    k_matvec_struct(const T* __restrict__ x, T* __restrict__ y, const T* __restrict__ fac,
                    const uint8_t* __restrict__ nmask, Grid g, int kchunk, ElemCoef<T> K,
                    T shift, CgState* st, double* partials, double* out) {
  if (MODE == 2 && st->status != HX_RUNNING) return;
  __shared__ MvSmem<T, BY> sm;
  const int lx = threadIdx.x, ly = threadIdx.y;
  const int tid = lx + MV_BX * ly;
  const int i0 = blockIdx.x * (MV_BX - 1), j0 = blockIdx.y * (BY - 1);
  const int k0 = blockIdx.z * kchunk;
  const int k1 = min(k0 + kchunk, g.nzn);
  const int in = i0 - 1 + lx, jn = j0 - 1 + ly;
  const bool col_ok = in >= 0 && jn >= 0 && in < g.nxe && jn < g.nye;
  const bool out_ok = lx >= 1 && ly >= 1 && in < g.nxn && jn < g.nyn;
  const int64_t nplane = (int64_t)g.nxn * g.nyn;
  const int64_t eplane = (int64_t)g.nxe * g.nye;

  issue_plane<T, BY>(sm, (k0 - 1) & 1, x, g, i0, j0, k0 - 1, tid);
  issue_plane<T, BY>(sm, k0 & 1, x, g, i0, j0, k0, tid);
  cp_async_wait<1>();
  __syncthreads();

  T xb[4][3], acc[4][3];
  {
    const int s = (k0 - 1) & 1;
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        xb[q][c] = sm.xs[s][ly + (q >> 1)][lx + (q & 1)][c];
        acc[q][c] = T(0);
      }
  }
  double dsum = 0.0;

  for (int ke = k0 - 1; ke < k1; ++ke) {
    T f = T(0);
    if (col_ok && ke >= 0 && ke < g.nze) f = fac[(int64_t)ke * eplane + (int64_t)jn * g.nxe + in];
    cp_async_wait<0>();
    __syncthreads();
    // Slot ke&1 (plane ke) is no longer read by anyone: prefetch plane ke+2.
    if (ke + 2 <= k1) issue_plane<T, BY>(sm, ke & 1, x, g, i0, j0, ke + 2, tid);

    const int s = (ke + 1) & 1;
    T u[3][8], xt[4][3];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        xt[q][c] = sm.xs[s][ly + (q >> 1)][lx + (q & 1)][c];
        u[c][q] = xb[q][c];
        u[c][4 + q] = xt[q][c];
      }
    T yv[3][8];
    elem_apply<T>(K, f, u, yv);

    T rowA[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T c0 = acc[0][c] + yv[c][0];
      const T c1 = acc[1][c] + yv[c][1];
      const T c2 = acc[2][c] + yv[c][2];
      const T c3 = acc[3][c] + yv[c][3];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q][c] = yv[c][4 + q];
      // element lx-1 contributes its +x corners to this thread's nodes
      const T l1 = __shfl_up_sync(0xffffffffu, c1, 1);
      const T l3 = __shfl_up_sync(0xffffffffu, c3, 1);
      rowA[c] = c0 + l1;
      sm.red[ly][lx][c] = c2 + l3;
    }
    __syncthreads();
    if (ke >= k0 && out_ok) {
      const int64_t node = (int64_t)ke * nplane + (int64_t)jn * g.nxn + in;
      const unsigned m = nmask ? nmask[node] : 7u;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T v = rowA[c] + sm.red[ly - 1][lx][c];
        const T xv = xb[0][c];
        v = ((m >> c) & 1u) ? v + shift * xv : T(0);
        y[3 * node + c] = v;
        if (MODE != 0) dsum += (double)xv * (double)v;
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int c = 0; c < 3; ++c) xb[q][c] = xt[q][c];
  }

  if (MODE != 0) {
    double v[1] = {dsum};
    if (grid_reduce<1>(v, partials, &st->ticket[TK_MATVEC]) && tid == 0) {
      if (MODE == 1) {
        out[0] = v[0];
      } else {
        const double pq = v[0];
        st->pq = pq;
        if (!(pq > 0.0) || !isfinite(pq)) {
          st->status = HX_ST_BREAKDOWN;
        } else {
          st->alpha = st->rz / pq;
        }
      }
    }
  }
}

// Per-node Jacobi diagonal: diag(n,c) = kd[c] * sum of the factors of the
// (up to 8) elements around n; node mask = fixed-DOF bits of `bcfree`
// cleared where the node carries no stiffness.  Writes diag into `diag`,
// the mask into `nmask`, and reduces the max diagonal over free DOFs.
template <typename T>
__global__ void k_node_diag(const T* __restrict__ fac, const uint8_t* __restrict__ bcfree,
                            uint8_t* __restrict__ nmask, T* __restrict__ diag, Grid g,
                            ElemCoef<double> K, double* partials, CgState* st, double* out) {
  const int64_t nn = (int64_t)g.nxn * g.nyn * g.nzn;
  double mx = 0.0;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(n % g.nxn);
    const int64_t r = n / g.nxn;
    const int j = (int)(r % g.nyn);
    const int k = (int)(r / g.nyn);
    double s = 0.0;
#pragma unroll
    for (int dk = -1; dk <= 0; ++dk)
#pragma unroll
      for (int dj = -1; dj <= 0; ++dj)
#pragma unroll
        for (int di = -1; di <= 0; ++di) {
          const int ei = i + di, ej = j + dj, ek = k + dk;
          if (ei >= 0 && ej >= 0 && ek >= 0 && ei < g.nxe && ej < g.nye && ek < g.nze)
            s += (double)fac[((int64_t)ek * g.nye + ej) * g.nxe + ei];
        }
    const unsigned m = (s > 0.0) ? (bcfree ? bcfree[n] : 7u) : 0u;
    nmask[n] = (uint8_t)m;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double d = K.kd[c] * s;
      diag[3 * n + c] = (T)d;
      if ((m >> c) & 1u) mx = fmax(mx, d);
    }
  }
  double v[1] = {mx};
  if (grid_reduce<1, true>(v, partials, &st->ticket[TK_AUX]) &&
      threadIdx.x == 0)
    out[0] = v[0];
}

// minv = free ? 1/(diag + shift) : 0   (src/Solvers/GPUSolver.jl:402)
template <typename T>
__global__ void k_minv(const uint8_t* __restrict__ nmask, const T* __restrict__ diag,
                       T* __restrict__ minv, int64_t nn, double shift) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * nn;
       i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned m = nmask[i / 3];
    const int c = (int)(i % 3);
    minv[i] = ((m >> c) & 1u) ? (T)(1.0 / ((double)diag[i] + shift)) : T(0);
  }
}

constexpr int MV_BY = 8;

inline dim3 mv_grid(const Grid& g, int kchunk) {
  return dim3(cdiv(g.nxn, MV_BX - 1), cdiv(g.nyn, MV_BY - 1), cdiv(g.nzn, kchunk));
}

}  // namespace

int mv_kchunk(const Grid& g) {
  // Enough CTAs to fill every SM a few times; at least 8 planes per chunk so
  // the recomputed halo layer stays small.
  const int64_t cols = (int64_t)cdiv(g.nxn, MV_BX - 1) * cdiv(g.nyn, MV_BY - 1);
  const int64_t want = 4LL * sm_count();
  int nch = (int)std::max<int64_t>(1, (want + cols - 1) / cols);
  int kc = (int)cdiv(g.nzn, nch);
  if (kc < 8) kc = std::min(8, g.nzn);
  return kc;
}

size_t mv_num_blocks(const Grid& g) {
  const dim3 gr = mv_grid(g, mv_kchunk(g));
  return (size_t)gr.x * gr.y * gr.z;
}

template <typename T>
void launch_matvec(cudaStream_t s, int mode, const T* x, T* y, const T* fac, const uint8_t* nmask,
                   const Grid& g, const ElemCoef<T>& K, T shift, CgState* st, double* partials,
                   double* out) {
  const int kc = mv_kchunk(g);
  const dim3 grid = mv_grid(g, kc);
  const dim3 block(MV_BX, MV_BY);
  switch (mode) {
    case 0:
      k_matvec_struct<T, MV_BY, 0><<<grid, block, 0, s>>>(x, y, fac, nmask, g, kc, K, shift, st,
                                                          partials, out);
      break;
    case 1:
      k_matvec_struct<T, MV_BY, 1><<<grid, block, 0, s>>>(x, y, fac, nmask, g, kc, K, shift, st,
                                                          partials, out);
      break;
    default:
      k_matvec_struct<T, MV_BY, 2><<<grid, block, 0, s>>>(x, y, fac, nmask, g, kc, K, shift, st,
                                                          partials, out);
  }
  HX_CHECK_LAUNCH();
}

template void launch_matvec<double>(cudaStream_t, int, const double*, double*, const double*,
                                    const uint8_t*, const Grid&, const ElemCoef<double>&, double,
                                    CgState*, double*, double*);
template void launch_matvec<float>(cudaStream_t, int, const float*, float*, const float*,
                                   const uint8_t*, const Grid&, const ElemCoef<float>&, float,
                                   CgState*, double*, double*);

template <typename T>
void launch_node_diag(cudaStream_t s, const T* fac, const uint8_t* bcfree, uint8_t* nmask, T* diag,
                      const Grid& g, const ElemCoef<double>& K, double* partials, CgState* st,
                      double* out) {
  const int64_t nn = (int64_t)g.nxn * g.nyn * g.nzn;
  const unsigned blocks = std::min<int64_t>(cdiv(nn, 256), 8LL * sm_count());
  k_node_diag<T><<<blocks, 256, 0, s>>>(fac, bcfree, nmask, diag, g, K, partials, st, out);
  HX_CHECK_LAUNCH();
}
template void launch_node_diag<double>(cudaStream_t, const double*, const uint8_t*, uint8_t*,
                                       double*, const Grid&, const ElemCoef<double>&, double*,
                                       CgState*, double*);
template void launch_node_diag<float>(cudaStream_t, const float*, const uint8_t*, uint8_t*, float*,
                                      const Grid&, const ElemCoef<double>&, double*, CgState*,
                                      double*);

template <typename T>
void launch_minv(cudaStream_t s, const uint8_t* nmask, const T* diag, T* minv, int64_t nn,
                 double shift) {
  const unsigned blocks = std::min<int64_t>(cdiv(3 * nn, 256), 16LL * sm_count());
  k_minv<T><<<blocks, 256, 0, s>>>(nmask, diag, minv, nn, shift);
  HX_CHECK_LAUNCH();
}
template void launch_minv<double>(cudaStream_t, const uint8_t*, const double*, double*, int64_t,
                                  double);
template void launch_minv<float>(cudaStream_t, const uint8_t*, const float*, float*, int64_t,
                                 double);

}  // namespace hx
