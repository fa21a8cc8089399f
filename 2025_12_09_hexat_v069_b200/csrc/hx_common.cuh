// hx_common.cuh -- shared device infrastructure for the HEXA(T) inner-solve
// library: error plumbing, the device-resident Krylov state, deterministic
// block/grid reductions and the Haar-domain Hex8 element operator.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <utility>

#include "../../include/hexat_b200.h"

namespace hx {

// ---------------------------------------------------------------------------
// Host-side error plumbing: every CUDA call is checked; the first failure is
// turned into an hx_status plus a message kept in the context.
// ---------------------------------------------------------------------------
struct Error {
  hx_status status;
  std::string msg;
};

#define HX_CUDA(call)                                                         \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      throw ::hx::Error{e_ == cudaErrorMemoryAllocation ? HX_OOM              \
                                                        : HX_CUDA_ERROR,      \
                        std::string(#call) + ": " + cudaGetErrorString(e_)};  \
    }                                                                         \
  } while (0)

// Kernels launched by this host thread (graph replays are added by the
// graph runner); the C ABI layer attributes the count to a context.
int64_t& launch_counter();

#define HX_CHECK_LAUNCH()            \
  do {                               \
    ++::hx::launch_counter();        \
    HX_CUDA(cudaGetLastError());     \
  } while (0)

#define HX_REQUIRE(cond, msg)                                \
  do {                                                       \
    if (!(cond)) throw ::hx::Error{HX_BAD_ARG, (msg)};       \
  } while (0)

// Programmatic dependent launch.  A kernel launched by launch_pdl may be
// scheduled while the previous kernel on its stream is still running; it
// calls pdl_wait() before its first global memory access, which returns once
// that kernel has completed and its writes are visible (and at once after an
// ordinary launch), and pdl_trigger() to let its own dependent be scheduled.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                Args&&... args) {
  cudaLaunchConfig_t lc{};
  lc.gridDim = grid;
  lc.blockDim = block;
  lc.dynamicSmemBytes = smem;
  lc.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  HX_CUDA(cudaLaunchKernelEx(&lc, kernel, std::forward<Args>(args)...));
}

// ---------------------------------------------------------------------------
// Device-resident Krylov state.  All scalars of a CG run (alpha, beta, dot
// products, residual history, status) live here, so an iteration never
// returns a scalar to the host; the host polls `status` every few
// iterations.  Kernels return immediately once status != HX_RUNNING.
// ---------------------------------------------------------------------------
enum : int {
  HX_RUNNING = 0,
  HX_ST_CONVERGED = 1,
  HX_ST_BREAKDOWN = 2,
  HX_ST_NONFINITE = 3,
  HX_ST_DIVERGED = 4,
  HX_ST_MAXITER = 5,
  HX_ST_ZERO_RHS = 6,
  HX_ST_PAUSED = 7,  // reliable-update point reached (mixed precision)
};

struct CgState {
  double rz;        // r.z of the current iterate
  double pq;        // p.(A p)
  double alpha;     // rz / pq
  double beta;      // rz_new / rz
  double rr;        // r.r
  double bnorm;     // ||b||
  double rel_res;   // ||r|| / ||b|| (recursive residual)
  double best_rel;  // lowest rel_res seen
  double tol;
  double explode;   // status DIVERGED when ||r|| > explode * ||b|| (0: off)
  double div_ratio; // status DIVERGED when rel > div_ratio*best after 50 its (0: off)
  double aux[4];    // derived scalars; CG with reliable updates uses
                    // aux[1] = delta (> 0 enables), aux[2] = max r.r since update
  int iter;         // completed iterations
  int max_iter;
  int status;
  int check_every;  // residual tested when iter % check_every == 0
  int snap;         // 1 when the current iterate is the best so far
  int keep_best;    // maintain the best-iterate flag
  int pad[2];
  unsigned int ticket[8];  // last-block-done counters (one per kernel kind)
};

// Ticket slots (a kernel kind owns one slot; kernels of the same kind never
// overlap on a stream).
enum : int {
  TK_MATVEC = 0,
  TK_UPDATE = 1,
  TK_INIT = 2,
  TK_AUX = 3,
  TK_AUX2 = 4,
};

// ---------------------------------------------------------------------------
// Deterministic reductions.  Per-block partial sums are reduced in a fixed
// shuffle tree; the block partials are written to a scratch array and summed
// in a fixed order by whichever block finishes last.  The result does not
// depend on block scheduling, so repeated runs are bit-identical.
// ---------------------------------------------------------------------------
// D^-1/2 entry from an M^-1 entry: sqrt(m) as m rsqrt(m) (branch-free, a
// few ulp; the fields it scales feed BF16 networks), exactly 0 on fixed
// DOFs (m = 0).  Every pass of the learned preconditioner uses it, so the
// preconditioner stays symmetric.
__device__ __forceinline__ float dinv_sqrt(float m) { return m > 0.f ? m * rsqrtf(m) : 0.f; }

template <int NV>
__device__ __forceinline__ void warp_sum(double (&v)[NV]) {
#pragma unroll
  for (int k = 0; k < NV; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
}

template <int NV>
__device__ __forceinline__ void warp_max(double (&v)[NV]) {
#pragma unroll
  for (int k = 0; k < NV; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      v[k] = fmax(v[k], __shfl_down_sync(0xffffffffu, v[k], o));
}

// Sum over the block; result valid in thread 0.  `red` needs NV*32 doubles.
template <int NV, bool MAX = false>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double* red) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  const int lane = tid & 31, w = tid >> 5, nw = (nthr + 31) >> 5;
  if (MAX) warp_max(v); else warp_sum(v);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) red[k * 32 + w] = v[k];
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = lane < nw ? red[k * 32 + lane] : (MAX ? -INFINITY : 0.0);
    if (MAX) warp_max(v); else warp_sum(v);
  }
}

// Grid-wide deterministic reduction of NV values.  Every block calls it with
// its per-thread contributions.  Returns true in exactly one block (the last
// to finish); in that block thread 0 holds the grid totals in `v`.
template <int NV, bool MAX = false>
__device__ bool grid_reduce(double (&v)[NV], double* partials, unsigned int* ticket) {
  __shared__ double red[NV * 32];
  __shared__ bool last;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  const unsigned nblk = gridDim.x * gridDim.y * gridDim.z;
  const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  block_reduce<NV, MAX>(v, red);
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[(size_t)bid * NV + k] = v[k];
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    last = (t == nblk - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  // four independent running sums per thread (loads in flight together),
  // combined in a fixed order: deterministic for a given grid
  double s4[4][NV];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int k = 0; k < NV; ++k) s4[a][k] = MAX ? -INFINITY : 0.0;
  unsigned b = tid;
  for (; b + 3 * nthr < nblk; b += 4 * nthr)
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int k = 0; k < NV; ++k) {
        const double pv = __ldcg(&partials[(size_t)(b + a * nthr) * NV + k]);
        s4[a][k] = MAX ? fmax(s4[a][k], pv) : s4[a][k] + pv;
      }
  for (; b < nblk; b += nthr)
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      const double pv = __ldcg(&partials[(size_t)b * NV + k]);
      s4[0][k] = MAX ? fmax(s4[0][k], pv) : s4[0][k] + pv;
    }
  double s[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k)
    s[k] = MAX ? fmax(fmax(s4[0][k], s4[1][k]), fmax(s4[2][k], s4[3][k]))
               : (s4[0][k] + s4[1][k]) + (s4[2][k] + s4[3][k]);
  __syncthreads();
  block_reduce<NV, MAX>(s, red);
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = s[k];
    *ticket = 0u;
  }
  return true;
}

// ---------------------------------------------------------------------------
// Hex8 element operator in the per-axis sum/difference ("Haar") basis.
//
// For a rectangular box element with trilinear shape functions and isotropic
// material, 2x2x2 Gauss quadrature integrates the stiffness exactly and every
// 8x8 block of Ke is a sum of Kronecker products of 1D 2x2 matrices (1D
// stiffness S, mass M and the mixed integrals C, C^T).  In the basis
// e_s=(1,1), e_d=(-1,1) along each axis all of these act monomially
// (S e_d = 2/h e_d, M e_s = h/2 e_s, M e_d = h/6 e_d, C e_s = e_d,
// C^T e_d = e_s), so Ke has 45 nonzeros instead of 576 there: 7 diagonal
// entries per component and 4 couplings per component pair.  The element
// product is then: forward butterfly (u -> U, unnormalised), sparse 45-term
// product, scale by the element factor, inverse butterfly.
//
// Nodal values are indexed by corner bits b = bx + 2*by + 4*bz; transformed
// values by sigma bits (bit set = difference along that axis).
// ---------------------------------------------------------------------------
template <typename T>
struct ElemCoef {
  T dg[3][8];   // diagonal of the Haar-domain operator per component
  T lam[3][2];  // lambda * m_k(sigma_k) / 8, k = axis not in the coupled pair
  T mu[3][2];   // mu * m_k(sigma_k) / 8
  T kd[3];      // Ke diagonal entry per component (same at every corner)
};

// Reference corner order (NAT_COORDS) -> corner bits.
__host__ __device__ constexpr int nat_to_bits(int c) {
  return (c == 0) ? 0 : (c == 1) ? 1 : (c == 2) ? 3 : (c == 3) ? 2
       : (c == 4) ? 4 : (c == 5) ? 5 : (c == 6) ? 7 : 6;
}

template <typename T>
__device__ __forceinline__ void haar_fwd(T (&u)[8]) {
#pragma unroll
  for (int bit = 1; bit < 8; bit <<= 1)
#pragma unroll
    for (int b = 0; b < 8; ++b)
      if (!(b & bit)) {
        T s = u[b] + u[b | bit], d = u[b | bit] - u[b];
        u[b] = s;
        u[b | bit] = d;
      }
}

template <typename T>
__device__ __forceinline__ void haar_inv(T (&y)[8]) {
#pragma unroll
  for (int bit = 1; bit < 8; bit <<= 1)
#pragma unroll
    for (int b = 0; b < 8; ++b)
      if (!(b & bit)) {
        T s = y[b], d = y[b | bit];
        y[b] = s - d;
        y[b | bit] = s + d;
      }
}

// Y = Lambda' U in the Haar domain (U already transformed).  Y[c][0] == 0.
template <typename T>
__device__ __forceinline__ void haar_apply(const ElemCoef<T>& K, const T (&U)[3][8],
                                           T (&Y)[3][8]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Y[c][0] = T(0);
#pragma unroll
    for (int s = 1; s < 8; ++s) Y[c][s] = K.dg[c][s] * U[c][s];
  }
#pragma unroll
  for (int pr = 0; pr < 3; ++pr) {
    const int i = (pr == 2) ? 0 : pr;       // pairs (0,1), (1,2), (0,2)
    const int j = (pr == 0) ? 1 : 2;
    const int k = 3 - i - j;
#pragma unroll
    for (int sk = 0; sk < 2; ++sk) {
      const int P = (1 << j) | (sk << k);  // sigma_i = s, sigma_j = d
      const int Q = (1 << i) | (sk << k);  // sigma_i = d, sigma_j = s
      const T l = K.lam[k][sk], m = K.mu[k][sk];
      Y[i][Q] += l * U[j][P];
      Y[i][P] += m * U[j][Q];
      Y[j][P] += l * U[i][Q];
      Y[j][Q] += m * U[i][P];
    }
  }
}

// y = f * Ke * u for one element; u, y indexed [component][corner bits].
template <typename T>
__device__ __forceinline__ void elem_apply(const ElemCoef<T>& K, T f, T (&u)[3][8],
                                           T (&y)[3][8]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) haar_fwd(u[c]);
  haar_apply(K, u, y);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int s = 1; s < 8; ++s) y[c][s] *= f;
    haar_inv(y[c]);
  }
}

// Quadratic form u^T Ke u (unit modulus) for one element.
template <typename T>
__device__ __forceinline__ T elem_energy(const ElemCoef<T>& K, T (&u)[3][8]) {
  T Y[3][8];
#pragma unroll
  for (int c = 0; c < 3; ++c) haar_fwd(u[c]);
  haar_apply(K, u, Y);
  T e = T(0);
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int s = 1; s < 8; ++s) e += u[c][s] * Y[c][s];
  return e;
}

// Host: Haar-domain coefficients of the unit-modulus Ke of a dx*dy*dz box.
ElemCoef<double> make_elem_coef(double dx, double dy, double dz, double nu);
ElemCoef<float> to_float(const ElemCoef<double>& k);

// Launch geometry helpers.
inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

// Number of SMs of the current device (cached per device, thread-safe).
int sm_count();

// Ordinal of the calling thread's current device.
int current_device();

// Runs a per-device set-up step (a kernel attribute such as the dynamic
// shared-memory opt-in, which CUDA keeps per device) once for each device it
// is used on.  Thread-safe: concurrent first calls may both run the step,
// which must therefore be idempotent.  Devices beyond the 64 tracked ones
// run it on every call.
class PerDeviceOnce {
 public:
  template <typename F>
  void run(F&& step) {
    const int dev = current_device();
    const bool tracked = dev >= 0 && dev < 64;
    const uint64_t bit = tracked ? (uint64_t(1) << dev) : 0;
    if (tracked && (done_.load(std::memory_order_acquire) & bit)) return;
    step();
    if (tracked) done_.fetch_or(bit, std::memory_order_acq_rel);
  }

 private:
  std::atomic<uint64_t> done_{0};
};

// Largest grids the structured kernels index: nodes per axis below 2^20, a
// node plane's DOFs plus a margin of 16 node rows (3 * nxn * (nyn + 16),
// the staged halo rows of a CTA) below 2^31, since in-plane offsets are
// 32-bit, and all DOFs below 2^40.  True when nx x ny x nz elements fit.
inline bool grid_extent_ok(int64_t nx, int64_t ny, int64_t nz) {
  if (nx < 1 || ny < 1 || nz < 1) return false;
  if (nx >= (1 << 20) || ny >= (1 << 20) || nz >= (1 << 20)) return false;
  if (3 * (nx + 1) * (ny + 1 + 16) >= (int64_t(1) << 31)) return false;
  return 3 * (nx + 1) * (ny + 1) * (nz + 1) < (int64_t(1) << 40);
}

}  // namespace hx
