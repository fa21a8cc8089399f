// hx_cnn.h -- launchers of the convolutional preconditioner network.
#pragma once
#include <cuda_bf16.h>

#include "hx_internal.h"

namespace hx {

struct GridN {  // node grid of the network (nodes per axis)
  int nx, ny, nz;
};

constexpr int NET_LAYERS = 4;
constexpr int NET_LAYER_PARAMS = 27 * 256 + 16;  // weights [27][16 co][16 ci] + bias[16]
constexpr int NET_PARAMS = NET_LAYERS * NET_LAYER_PARAMS;

size_t conv_num_tiles(const GridN& g);
// epi 0: +bias, ReLU; 1: +bias; 2: * (M > 0) (no bias)
void launch_conv3(cudaStream_t s, int cout, int epi, const __nv_bfloat16* X, __nv_bfloat16* Y,
                  const __nv_bfloat16* W, const float* bias, const __nv_bfloat16* M,
                  const GridN& g);
void launch_conv3_wgrad(cudaStream_t s, const __nv_bfloat16* X, const __nv_bfloat16* D,
                        float* part, float* grad, const GridN& g);
void launch_adam(cudaStream_t s, float* w, float* m, float* v, const float* grad,
                 const unsigned char* live, int n, float lr, int step);
void launch_pack_weights(cudaStream_t s, const float* w, __nv_bfloat16* wf, __nv_bfloat16* wb);
void launch_net_input(cudaStream_t s, const double* r, const double* dinvs, const float* feat,
                      const CgState* st, double scale_mul, __nv_bfloat16* X0, int64_t nn);
void launch_net_output(cudaStream_t s, const double* r, const double* minv, const double* dinvs,
                       const __nv_bfloat16* Y, int ystride, CgState* st, double scale_mul,
                       double* z, const double* q_old, double* partials, int64_t nn);
void launch_sqrt(cudaStream_t s, const double* a, double* b, int64_t n);
void launch_rho_feature(cudaStream_t s, const double* fac, float* feat, const Grid& g);
void launch_net_loss(cudaStream_t s, const double* r, const double* e, const double* dinvs,
                     const __nv_bfloat16* Y, const CgState* st, double scale_mul, double inv_nf,
                     __nv_bfloat16* D, double* partials, CgState* rst, double* out, int64_t nn);

}  // namespace hx
