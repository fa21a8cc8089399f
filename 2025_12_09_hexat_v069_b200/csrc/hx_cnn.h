// hx_cnn.h -- launchers of the convolutional preconditioner network.
#pragma once
#include <cuda_bf16.h>

#include "hx_internal.h"

namespace hx {

struct GridN {  // node grid of the network (nodes per axis)
  int nx, ny, nz;
};

// 16-channel activations are stored in half-rows: channels 8h .. 8h + 7 of
// node (x, y, z) start at element ((r * 2 + h) * nx + x) * 8, r = z * ny + y,
// so that each half of a node row is one contiguous run of 16 nx bytes and a
// convolution's TMA load copies 10 nodes per row request (with [node][16] it
// was one node's 16 bytes per request, and the loads bounded the layer).
// 8-channel tensors (the network output y) are plain [node][8].
__host__ __device__ inline int64_t act16(const GridN& g, int64_t r, int x, int h) {
  return ((r * 2 + h) * g.nx + x) * 8;
}

constexpr int NET_LAYERS = 4;
constexpr int NET_LAYER_PARAMS = 27 * 256;  // weights [27 taps][16 co][16 ci], no bias
constexpr int NET_NET_PARAMS = NET_LAYERS * NET_LAYER_PARAMS;  // one network
constexpr int NET_NETS = 3;        // networks on node-grid levels NET_L0 .. NET_TOP
constexpr int NET_L0 = 2;          // level of the first (finest) network
constexpr int NET_TOP = NET_L0 + NET_NETS - 1;
constexpr int NET_PARAMS = NET_NETS * NET_NET_PARAMS;
constexpr int NET_IN = 6;  // live input channels: D^-1/2 r / s and the same times the density

size_t conv_num_tiles(const GridN& g);
// plain convolution (or, with the packed transposed weights, its transpose)
// on the tcgen05 tensor cores; *err is set when a CTA's bounded wait ran out
void launch_conv3(cudaStream_t s, int cout, const __nv_bfloat16* X, __nv_bfloat16* Y,
                  const __nv_bfloat16* W, const GridN& g, int* err);
// failure-detection self test: one CTA whose wait must run out (8 x 16 x 4 nodes)
void launch_conv3_selftest(cudaStream_t s, const __nv_bfloat16* X, __nv_bfloat16* Y,
                           const __nv_bfloat16* W, int* err);
// grad (+)= dW of one layer from the per-CTA partials
void launch_conv3_wgrad(cudaStream_t s, const __nv_bfloat16* X, const __nv_bfloat16* D,
                        float* part, float* grad, bool accumulate, const GridN& g);
void launch_adam(cudaStream_t s, float* w, float* m, float* v, const float* grad,
                 const unsigned char* live, int n, float lr, int step);
void launch_pack_weights(cudaStream_t s, const float* w, __nv_bfloat16* wf, __nv_bfloat16* wb);
// level-1 field R (k D^-1/2 v) of a DOF vector, D^-1/2 = sqrt(minv) (k by
// mode: 0 network input, 1 energy-loss gradient, 2 residual-loss gradient)
template <typename T>
void launch_restrict_dof(cudaStream_t s, const T* v, const T* minv, const CgState* sst,
                         const CgState* lst, int mode, double scale_mul, float* out,
                         const GridN& gf, const GridN& gc);
// the same field (mode 0) from ys = BF16(D^-1/2 v), n + 8 entries
void launch_restrict_ys(cudaStream_t s, const __nv_bfloat16* ys, const CgState* sst,
                        double scale_mul, float* out, const GridN& gf, const GridN& gc);
// full-weighting restriction fine -> coarse node grid (ch 3 or 1), and its
// transpose; an optional node mask (3 channels: free-DOF bits) zeroes the
// fixed components of the output
void launch_restrict(cudaStream_t s, int ch, const float* in, float* out, const GridN& gf,
                     const GridN& gc, bool normalise, const uint8_t* cmask = nullptr);
void launch_prolong(cudaStream_t s, const float* coarse, float* fine, const GridN& gf,
                    const GridN& gc, bool accumulate, const uint8_t* fmask = nullptr);
// lifting E: [node][3] FP32 -> 16-channel BF16 activation (x, feat * x), and its transpose
void launch_lift(cudaStream_t s, const float* x, const float* feat, __nv_bfloat16* X,
                 const GridN& g);
void launch_unlift(cudaStream_t s, const __nv_bfloat16* Y, const float* feat, float* acc,
                   bool accumulate, int64_t nn);
// partials k_net_output needs (one per block)
size_t net_output_blocks(const GridN& gf);
// z = M^-1 r + s D^-1/2 R^T t  (t: level-1 correction), with the FCG beta from q_old
template <typename T>
void launch_net_output(cudaStream_t s, const T* r, const T* minv, const float* t, const GridN& gf,
                       const GridN& gc, CgState* st, double scale_mul, T* z, const T* q_old,
                       double* partials);
void launch_net_aloss(cudaStream_t s, const double* d, const double* q, const double* e,
                      const double* r, int64_t n, double* partials, CgState* st, double* out);
void launch_rho_feature(cudaStream_t s, const double* fac, float* feat, const Grid& g);

}  // namespace hx
