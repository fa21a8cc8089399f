// hx_cnn.h -- launchers of the convolutional preconditioner network.
#pragma once
#include <cuda_bf16.h>

#include "hx_internal.h"

namespace hx {

struct GridN {  // node grid of the network (nodes per axis)
  int nx, ny, nz;
};

constexpr int NET_LAYERS = 4;
constexpr int NET_LAYER_PARAMS = 27 * 256;  // weights [27 taps][16 co][16 ci], no bias
constexpr int NET_PARAMS = NET_LAYERS * NET_LAYER_PARAMS;
constexpr int NET_IN = 6;  // live input channels: D^-1/2 r / s and the same times the density

size_t conv_num_tiles(const GridN& g);
// plain convolution (or, with the packed transposed weights, its transpose)
void launch_conv3(cudaStream_t s, int cout, const __nv_bfloat16* X, __nv_bfloat16* Y,
                  const __nv_bfloat16* W, const GridN& g);
// grad (+)= dW of one layer from the per-CTA partials
void launch_conv3_wgrad(cudaStream_t s, const __nv_bfloat16* X, const __nv_bfloat16* D,
                        float* part, float* grad, bool accumulate, const GridN& g);
void launch_adam(cudaStream_t s, float* w, float* m, float* v, const float* grad,
                 const unsigned char* live, int n, float lr, int step);
void launch_pack_weights(cudaStream_t s, const float* w, __nv_bfloat16* wf, __nv_bfloat16* wb);
void launch_net_lift(cudaStream_t s, const double* v, const double* dinvs, const float* feat,
                     const CgState* sst, const CgState* lst, int mode, double scale_mul,
                     __nv_bfloat16* X, int64_t nn);
void launch_net_output(cudaStream_t s, const double* r, const double* minv, const double* dinvs,
                       const float* feat, const __nv_bfloat16* Y, CgState* st, double scale_mul,
                       double* z, const double* q_old, double* partials, int64_t nn);
void launch_net_aloss(cudaStream_t s, const double* d, const double* q, const double* e,
                      const double* r, int64_t n, double* partials, CgState* st, double* out);
void launch_sqrt(cudaStream_t s, const double* a, double* b, int64_t n);
void launch_rho_feature(cudaStream_t s, const double* fac, float* feat, const Grid& g);

}  // namespace hx
