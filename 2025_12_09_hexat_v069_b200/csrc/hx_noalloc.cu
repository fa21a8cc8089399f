// hx_noalloc.cu -- K(f)x and x.K(f)x without any device allocation.
//
// Some callers cannot let a library allocate device memory:
//  * cudaMalloc/cudaFree synchronize the device, which stalls every other
//    stream of a caller that keeps several solves or copies in flight;
//  * a host runtime that pools device memory itself (CUDA.jl in the Julia
//    host this library serves) keeps most of the device reserved for its
//    own pool, so a foreign cudaMalloc can fail while the pool has room.
// For them, hx_apply_stiffness_noalloc runs the structured operator kernel
// with its scratch (the reduction's per-CTA partial sums and its
// completion counter) in one statically allocated device array instead of
// context-owned buffers.  The caller passes every input and output as a
// device pointer and the stream to run on.
//
// The array below is loaded with the library: every GPU that loads the
// library holds HX_NOALLOC_SCRATCH_BYTES of device memory until the
// process exits.  All calls on a device share it, so calls that overlap on
// the GPU (different streams, or host threads without ordering) race on it;
// callers must order them, e.g. on one stream.  Each call clears the
// completion counter before its kernel runs; the partial sums are fully
// rewritten by every call, so contents left by the previous call do not
// matter.
#include <mutex>

#include "hx_solver.h"

namespace {

constexpr size_t kStateBytes = 256;  // CgState (ticket counters) rounded up
static_assert(sizeof(hx::CgState) <= kStateBytes, "CgState grew past its scratch slot");
constexpr size_t kScratchBytes = kStateBytes + sizeof(double) * HX_NOALLOC_MAX_BLOCKS;

// The one scratch array.  Its name is a host-side stand-in, not a device
// address: host code must go through cudaGetSymbolAddress (below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device, resolved once
// per device with that device current.
hx_status scratch_address(unsigned char** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return HX_CUDA_ERROR;
  }
  if (dev < 0 || dev >= kMaxDevices) return HX_BAD_ARG;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return HX_CUDA_ERROR;
    }
    g_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_addr[dev];
  return HX_OK;
}

}  // namespace

extern "C" HX_API hx_status hx_apply_stiffness_noalloc(int64_t nx, int64_t ny, int64_t nz,
                                                       double dx, double dy, double dz, double nu,
                                                       const double* x, const double* factor,
                                                       double* y, double* xKx, void* stream) {
  if (!x || !factor || !y || !xKx) return HX_BAD_ARG;
  // Every array is read or written as FP64 words, and the operator stages x
  // in 16-byte chunks: a misaligned pointer is refused here, before anything
  // reaches the GPU, rather than becoming a misaligned-address fault that
  // would end the caller's CUDA context.
  const auto misaligned = [](const void* p, uintptr_t a) {
    return (reinterpret_cast<uintptr_t>(p) & (a - 1)) != 0;
  };
  if (misaligned(x, 16) || misaligned(factor, 8) || misaligned(y, 8) || misaligned(xKx, 8))
    return HX_BAD_ARG;
  if (!hx::grid_extent_ok(nx, ny, nz)) return HX_BAD_ARG;
  if (!(dx > 0 && dy > 0 && dz > 0) || !(nu > -1.0 && nu < 0.5)) return HX_BAD_ARG;
  hx::Grid g{};
  g.nxe = (int)nx;
  g.nye = (int)ny;
  g.nze = (int)nz;
  g.nxn = g.nxe + 1;
  g.nyn = g.nye + 1;
  g.nzn = g.nze + 1;
  // The reduction writes one partial sum per CTA of the operator kernel.
  if (hx::mv_num_blocks(g, 2) > (size_t)HX_NOALLOC_MAX_BLOCKS) return HX_BAD_ARG;  // FP64: 2 CTAs/SM
  unsigned char* base = nullptr;
  const hx_status st = scratch_address(&base);
  if (st != HX_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  hx::CgState* state = reinterpret_cast<hx::CgState*>(base);
  double* partials = reinterpret_cast<double*>(base + kStateBytes);
  try {
    const hx::ElemCoef<double> K = hx::make_elem_coef(dx, dy, dz, nu);
    HX_CUDA(cudaMemsetAsync(state, 0, sizeof(hx::CgState), s));  // completion counter = 0
    hx::launch_matvec<double>(s, 1, x, y, factor, nullptr, g, K, 0.0, state, partials, xKx);
  } catch (hx::Error& e) {
    return e.status;
  }
  return HX_OK;
}
