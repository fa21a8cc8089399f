// hx_cnn.cu -- 3D convolutional preconditioner network on the node grid:
// the weight gradient of the BF16 conv3d layers (3x3x3, 16 channels, no
// bias; the convolution itself is in hx_conv_tc.cu), Adam, the grid
// transfers between levels, and the input/output assembly around a Krylov
// solver.
//
// Activations are channels-last BF16, [node][16] (32 bytes per node, node
// numbering of the grid).  The weight gradient of a layer is a per-CTA
// tensor-core reduction (mma.sync m16n8k16) over a 16 x 8 x 4 node tile:
// the input tile with its one-node halo (18 x 10 x 6 nodes) and the output
// gradient tile are staged with 16-byte cp.async, the 16-byte halves of each
// node XOR-swizzled so that the 8 rows of an ldmatrix hit distinct banks;
// one tap per warp at a time; partials summed across CTAs in a fixed order.
#include <cuda_bf16.h>

#include "hx_cnn.h"

namespace hx {

namespace {

constexpr int TX = 16, TY = 8, TZ = 4;           // output tile
constexpr int HX_ = TX + 2, HY = TY + 2, HZ = TZ + 2;
constexpr int HNODES = HX_ * HY * HZ;             // 1080
constexpr int C = 16;                             // channels per node (storage)
constexpr int NTHREADS = 256;

__device__ __forceinline__ unsigned su32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp16(unsigned dst, const void* src, bool ok) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src),
               "r"(ok ? 16 : 0));
}
__device__ __forceinline__ void cp_commit_wait() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::);
}
__device__ __forceinline__ void ldsm_x4_t(unsigned addr, unsigned (&r)[4]) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(addr));
}
__device__ __forceinline__ void mma16816(float (&d)[4], const unsigned (&a)[4], unsigned b0,
                                         unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// byte offset of 16-byte half `h` of a 32-byte row `row` (XOR swizzle)
__device__ __forceinline__ unsigned swz(int row, int h) {
  return (unsigned)(row * 32 + ((h ^ ((row >> 2) & 1)) << 4));
}

}  // namespace

// ---------------------------------------------------------------------------
// Weight-gradient partials of one CTA tile:
// dW[tap][co][ci] = sum_n D[n, co] X[n + off(tap), ci]
// For a forward use, X is the layer input and D the gradient w.r.t. its
// output; for a transposed use (output = W^T * x') the roles swap: X = the
// gradient w.r.t. the output, D = x'.  Warp w handles taps w, w+8, w+16,
// w+24 over all 512 nodes of the tile; the result goes to part[cta][27*256]
// (FP32), summed later in fixed order.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(NTHREADS) k_conv3_wgrad(const __nv_bfloat16* __restrict__ X,
                                                          const __nv_bfloat16* __restrict__ D,
                                                          float* __restrict__ part, GridN g) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __nv_bfloat16* xs = reinterpret_cast<__nv_bfloat16*>(smraw);
  __nv_bfloat16* ds = xs + HNODES * C;  // [512 nodes][16], swizzled rows
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;
  const unsigned xb = su32(xs), db = su32(ds);
  for (int ch = threadIdx.x; ch < HNODES * 2; ch += NTHREADS) {
    const int node = ch >> 1, h = ch & 1;
    const int hx = node % HX_, r = node / HX_;
    const int hy = r % HY, hz = r / HY;
    const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + hz;
    const bool ok = gx >= 0 && gy >= 0 && gz >= 0 && gx < g.nx && gy < g.ny && gz < g.nz;
    const int64_t go = ok ? act16(g, (int64_t)gz * g.ny + gy, gx, h) : 0;
    cp16(xb + swz(node, h), X + go, ok);
  }
  for (int ch = threadIdx.x; ch < TX * TY * TZ * 2; ch += NTHREADS) {
    const int node = ch >> 1, h = ch & 1;  // node = x + 16 (y + 8 z)
    const int tx = node & 15, ty = (node >> 4) & 7, tz = node >> 7;
    const int gx = x0 + tx, gy = y0 + ty, gz = z0 + tz;
    const bool ok = gx < g.nx && gy < g.ny && gz < g.nz;  // outside: zero gradient
    const int64_t go = ok ? act16(g, (int64_t)gz * g.ny + gy, gx, h) : 0;
    cp16(db + swz(node, h), D + go, ok);
  }
  cp_commit_wait();
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  float* out = part + (size_t)(blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)) *
                          (27 * 256);
  // ldmatrix.trans row addresses: matrix mi = lane/8, row r = lane%8
  const int mi = lane >> 3, rr = lane & 7;
  for (int tap = warp; tap < 27; tap += 8) {
    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};  // M = ci, N = co
    for (int row = 0; row < 32; ++row) {  // 16-node k-steps
      const int ty = row & 7, tz = row >> 3;
      // A = X^T (ci x nodes): matrices (ci 0-7, n 0-7), (ci 8-15, n 0-7),
      // (ci 0-7, n 8-15), (ci 8-15, n 8-15) from X[n][ci] via .trans
      unsigned a[4];
      {
        const int nx_ = ((mi >> 1) << 3) + rr, h = mi & 1;
        const int hx = nx_ + 1 + dx, hy = ty + 1 + dy, hz = tz + 1 + dz;
        ldsm_x4_t(xb + swz((hz * HY + hy) * HX_ + hx, h), a);
      }
      // B = D (nodes x co): matrices (n 0-7, co 0-7), (n 8-15, co 0-7),
      // (n 0-7, co 8-15), (n 8-15, co 8-15) via .trans
      unsigned b[4];
      {
        const int nx_ = ((mi & 1) << 3) + rr, h = mi >> 1;
        ldsm_x4_t(db + swz(nx_ + 16 * (ty + 8 * tz), h), b);
      }
      mma16816(acc[0], a, b[0], b[1]);
      mma16816(acc[1], a, b[2], b[3]);
    }
    // acc[nt]: rows ci = gq (+8), cols co = nt*8 + 2tq (+1)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int ci = gq + hh * 8, co = nt * 8 + 2 * tq;
        out[tap * 256 + co * 16 + ci] = acc[nt][2 * hh];
        out[tap * 256 + (co + 1) * 16 + ci] = acc[nt][2 * hh + 1];
      }
  }
}

// Sum the per-CTA partials in a fixed order: grad[k] (+)= sum_c part[c][k].
__global__ void k_reduce_parts(const float* __restrict__ part, int nparts, int len,
                               float* __restrict__ grad, int accumulate) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= len) return;
  double s = 0.0;
  for (int c = 0; c < nparts; ++c) s += (double)part[(size_t)c * len + k];
  grad[k] = accumulate ? grad[k] + (float)s : (float)s;
}

// Adam step on the FP32 master parameters (weights [27][16][16] per layer,
// concatenated).  `live` masks the parameters that exist (padding channels
// stay zero).
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ grad, const unsigned char* __restrict__ live,
                       int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n || !live[k]) return;
  const float gk = grad[k];
  const float mk = b1 * m[k] + (1.f - b1) * gk;
  const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
  m[k] = mk;
  v[k] = vk;
  w[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
}

// Master FP32 parameters of one layer (W[tap][co][ci], tap = (dz + 1) * 9 +
// s, s = (dy + 1) * 3 + dx + 1) -> the BF16 B operands of the tensor-core
// convolution, in its shared-memory order [s][plane][row][8]: per in-plane
// shift s, 48 rows = the three z-offsets' output channels (row = b * 16 +
// out, b = 1 - dz: dz = +1, 0, -1), plane = which 8 of the 16 reduced
// channels.  wf for the convolution (out = co, reduced over ci) and wb for
// its transpose (tap flipped, out = ci, reduced over co).
__global__ void k_pack_weights(const float* __restrict__ w, __nv_bfloat16* __restrict__ wf,
                               __nv_bfloat16* __restrict__ wb) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 27 * 256) return;
  const int tap = k / 256, co = (k / 16) % 16, ci = k % 16;
  const int dz = tap / 9 - 1, s = tap % 9;
  const __nv_bfloat16 v = __float2bfloat16_rn(w[k]);
  wf[((s * 2 + (ci >> 3)) * 48 + (1 - dz) * 16 + co) * 8 + (ci & 7)] = v;
  // transpose: tap 26 - tap, i.e. dz -> -dz and s -> 8 - s
  wb[(((8 - s) * 2 + (co >> 3)) * 48 + (1 + dz) * 16 + ci) * 8 + (co & 7)] = v;
}

// ---------------------------------------------------------------------------
// Solver <-> network glue (node grid, interleaved FP64 vectors)
// ---------------------------------------------------------------------------
// 1D full-weighting factor of fine offset d = j - 2i (|d| <= 1)
__device__ __forceinline__ float fw(int d) { return d == 0 ? 1.f : 0.5f; }

// Per axis, the coarse nodes i with |f - 2i| <= 1 and their weights
// (floor(f/2), and for odd f also f/2 + 1; weight 0 past the coarse grid).
__device__ __forceinline__ void prolong_axis(int f, int nc, int (&i)[2], float (&w)[2]) {
  if ((f & 1) == 0) {
    i[0] = f >> 1;
    w[0] = 1.f;
    i[1] = 0;
    w[1] = 0.f;
  } else {
    i[0] = f >> 1;
    w[0] = 0.5f;
    i[1] = (f >> 1) + 1;
    w[1] = 0.5f;
    if (i[1] >= nc) {
      i[1] = 0;
      w[1] = 0.f;
    }
  }
  if (i[0] >= nc) {
    i[0] = 0;
    w[0] = 0.f;
  }
}

// Restriction to the next coarser node grid (coarse node i <-> fine node
// 2i), full weighting (1/2, 1, 1/2) per axis, zero outside the grid:
// out[i][c] = sum_d w(d) in[2i + d][c].  With `normalise`, divides by the
// sum of the weights inside the grid (a weighted average; for features).
template <int CH>
__global__ void k_restrict(const float* __restrict__ in, float* __restrict__ out, GridN gf,
                           GridN gc, int normalise, const uint8_t* __restrict__ cmask) {
  pdl_wait();
  pdl_trigger();
  const int64_t nc = (int64_t)gc.nx * gc.ny * gc.nz;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nc;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(n % gc.nx);
    const int64_t t = n / gc.nx;
    const int j = (int)(t % gc.ny), k = (int)(t / gc.ny);
    // the 27 fine neighbours at clamped indices, weight 0 outside the grid:
    // every load is unconditional, so they can all be in flight together
    float acc[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) acc[c] = 0.f;
    float wsum = 0.f;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz) {
      const int fz0 = 2 * k + dz;
      const bool okz = fz0 >= 0 && fz0 < gf.nz;
      const int fz = min(max(fz0, 0), gf.nz - 1);
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy) {
        const int fy0 = 2 * j + dy;
        const bool oky = okz && fy0 >= 0 && fy0 < gf.ny;
        const int fy = min(max(fy0, 0), gf.ny - 1);
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
          const int fx0 = 2 * i + dx;
          const bool ok = oky && fx0 >= 0 && fx0 < gf.nx;
          const int fx = min(max(fx0, 0), gf.nx - 1);
          const float w = ok ? fw(dz) * fw(dy) * fw(dx) : 0.f;
          const int64_t f = ((int64_t)fz * gf.ny + fy) * gf.nx + fx;
#pragma unroll
          for (int c = 0; c < CH; ++c) acc[c] += w * in[f * CH + c];
          wsum += w;
        }
      }
    }
    const float sc = (normalise && wsum > 0.f) ? 1.f / wsum : 1.f;
    // cmask (3 channels): bit c clear -> component c is a fixed DOF, set to 0
    const unsigned m = cmask ? cmask[n] : 0xffu;
#pragma unroll
    for (int c = 0; c < CH; ++c) out[n * CH + c] = ((m >> c) & 1u) ? acc[c] * sc : 0.f;
  }
}

// Coefficient k of the scaled field x = k D^-1/2 v of `mode`:  0: 1/s
// (network input, s the RMS of D^-1/2 r);  1: 2 s / (e.r) (energy-loss
// gradient);  2: 2 s / (r.M^-1 r) (residual-loss gradient).  s from
// sst->rz; e.r from lst->aux[0].
__device__ __forceinline__ double field_coef(const CgState* sst, const CgState* lst, int mode,
                                             double scale_mul) {
  const double s = sqrt(sst->rz * scale_mul);
  if (mode == 0) return 1.0 / fmax(s, 1e-300);
  const double den = (mode == 1) ? lst->aux[0] : sst->rz;
  return den > 0.0 ? 2.0 * s / den : 0.0;
}

// The mesh-grid passes below run one CTA per coarse row: blockIdx.x is a
// chunk of at most ROW_CX coarse x-cells (chunk width from row_chunk), y the
// coarse y-row j, z the coarse z-plane k.  Every global access walks a fine
// row as a contiguous run of DOFs (lane = DOF), so it is coalesced whatever
// the row's alignment.
constexpr int ROW_CX = 256;


// Coarse x-cells per chunk: the coarse row split into near-equal chunks of at
// most ROW_CX cells.
static int row_chunk(int ncx) {
  const int n = (int)cdiv(ncx, ROW_CX);
  return (int)cdiv(ncx, n);
}

// Level-1 field of a DOF vector in one pass: out = R (k D^-1/2 v) with
// D^-1/2 = sqrt(minv) (0 on fixed DOFs), R the full-weighting restriction
// of k_restrict; the scaled field on the mesh's node grid is never stored.
// T: the precision of the solver's vectors; the field is FP32 (it feeds the
// BF16 network), so it is formed in FP32 whatever T is.
//
// Per CTA (coarse row (j, k), cells cx0 .. cx0+w-1, w <= RES_CX): the 9 fine
// rows (2j+dy, 2k+dz), |dy|, |dz| <= 1, of v and minv are staged in shared
// memory with cp.async (every copy of the CTA in flight at once; rows
// outside the grid are read at a clamped index with weight 0), collapsed
// with their y-z weights per fine DOF, then the x weights are applied.
constexpr int RES_CX = 128;

template <typename T>
__device__ __forceinline__ void cp_async_elem(T* sdst, const T* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(
                   (unsigned)__cvta_generic_to_shared(sdst)),
               "l"(gsrc), "n"(sizeof(T)));
}

// Dynamic shared memory of k_restrict_dof for chunk width cxw.
template <typename T>
static size_t restrict_smem(int cxw) {
  const size_t seg = 3 * (2 * (size_t)cxw + 1);  // DOFs per staged row
  return 18 * seg * sizeof(T) + seg * sizeof(float);
}

template <typename T>
__global__ void __launch_bounds__(256)
    k_restrict_dof(const T* __restrict__ v, const T* __restrict__ minv, const CgState* sst,
                   const CgState* lst, int mode, double scale_mul, float* __restrict__ out,
                   GridN gf, GridN gc, int cxw) {
  extern __shared__ __align__(16) unsigned char rsm[];
  const int seg = 3 * (2 * cxw + 1);
  T* sm_m = reinterpret_cast<T*>(rsm);  // [9][seg]
  T* sm_v = sm_m + 9 * seg;             // [9][seg]
  float* srow = reinterpret_cast<float*>(sm_v + 9 * seg);  // [seg]
  const int cx0 = blockIdx.x * cxw, w = min(cxw, gc.nx - cx0);
  const int j = blockIdx.y, k = blockIdx.z;
  // fine nodes 2 cx0 - 1 .. 2 (cx0 + w - 1) + 1, clipped to the grid
  // (at most 2 w + 1 <= 2 cxw + 1 nodes)
  const int fxa = max(2 * cx0 - 1, 0);
  const int fxb = min(2 * (cx0 + w - 1) + 1, gf.nx - 1);
  const int L = 3 * (fxb - fxa + 1);
  float rw[9];
#pragma unroll
  for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy) {
      const int q = (dz + 1) * 3 + (dy + 1);
      const int fz0 = 2 * k + dz, fy0 = 2 * j + dy;
      const bool ok = fz0 >= 0 && fz0 < gf.nz && fy0 >= 0 && fy0 < gf.ny;
      const int fz = min(max(fz0, 0), gf.nz - 1), fy = min(max(fy0, 0), gf.ny - 1);
      const int64_t rb = 3 * (((int64_t)fz * gf.ny + fy) * gf.nx + fxa);
      rw[q] = ok ? fw(dz) * fw(dy) : 0.f;
      for (int dl = threadIdx.x; dl < L; dl += blockDim.x) {
        cp_async_elem(sm_m + q * seg + dl, minv + rb + dl);
        cp_async_elem(sm_v + q * seg + dl, v + rb + dl);
      }
    }
  asm volatile("cp.async.commit_group;\n" ::);
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  for (int dl = threadIdx.x; dl < L; dl += blockDim.x) {
    float acc = 0.f;
#pragma unroll
    for (int q = 0; q < 9; ++q)
      acc += rw[q] * (dinv_sqrt((float)sm_m[q * seg + dl]) * (float)sm_v[q * seg + dl]);
    srow[dl] = acc;
  }
  __syncthreads();
  const float kc = (float)field_coef(sst, lst, mode, scale_mul);
  const int64_t ob = 3 * (((int64_t)k * gc.ny + j) * gc.nx + cx0);
  for (int e = threadIdx.x; e < 3 * w; e += blockDim.x) {
    const int cl = e / 3, c = e - 3 * cl;
    const int fx = 2 * (cx0 + cl);  // the coincident fine node
    const int l = fx - fxa;
    float a = srow[3 * l + c];
    if (fx >= 1) a += 0.5f * srow[3 * (l - 1) + c];
    if (fx + 1 < gf.nx) a += 0.5f * srow[3 * (l + 1) + c];
    out[ob + e] = kc * a;
  }
}

// The same level-1 field from ys = BF16(D^-1/2 v) (k_cg_update2 writes it
// with the residual): out = k R ys.  One CTA per (x-chunk of w <= YS_CX
// coarse cells, block of YS_JB coarse y-rows j0.., segment of kseg coarse
// planes).  Thread t < 3w owns coarse cell cx0 + t/3, component t%3, and
// keeps in registers the sums of its YS_JB coarse rows for two coarse
// planes (k even, k odd) while the CTA marches up the fine planes of its
// segment.  Per fine plane the rows 2j0-1 .. 2j0+2 YS_JB-1 inside the grid
// are staged with 16-byte cp.async chunks into a ring of YS_RING slots
// (planes p+1 .. p+YS_RING-1 in flight while p is used), each row from the
// chunk holding its first entry (a shift of 0-7 entries; the last chunk may
// reach 7 entries past n, so ys holds n + 8 entries).  A thread collapses
// its three fine x-nodes of each staged row (weights 1/2, 1, 1/2), adds
// the value into its coarse rows with the y weights and, per plane, into
// its coarse planes with the z weight; a finished coarse plane is stored.
// Each fine row is read once per segment (the rows shared with the
// neighbouring row blocks and the plane below the segment twice).
constexpr int YS_CX = 85;  // coarse cells per chunk: 3 x 85 = 255 threads
constexpr int YS_JB = 4;
constexpr int YS_NY = 2 * YS_JB + 1;  // staged fine y-rows per plane
constexpr int YS_RING = 4;            // staged planes: the one in use and 3 ahead
constexpr int YS_CPT = (YS_NY * (3 * (2 * YS_CX + 1) / 8 + 3) + 255) / 256;  // chunks per thread

__device__ __forceinline__ float bf16_bits(unsigned short h) { return __uint_as_float((unsigned)h << 16); }

__global__ void __launch_bounds__(256)
    k_restrict_ys(const __nv_bfloat16* __restrict__ ys, const CgState* sst, double scale_mul,
                  float* __restrict__ out, GridN gf, GridN gc, int cxw, int kseg) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ __align__(16) unsigned char rsm[];
  const int seg = 3 * (2 * cxw + 1);
  const int segc = seg / 8 + 3;  // 16-byte chunks per staged row
  uint4* sc = reinterpret_cast<uint4*>(rsm);  // [YS_RING][YS_NY][segc]
  const int cx0 = blockIdx.x * cxw, w = min(cxw, gc.nx - cx0);
  const int j0 = blockIdx.y * YS_JB;
  const int jn = min(YS_JB, gc.ny - j0);  // coarse rows of this block
  const int k0 = blockIdx.z * kseg, k1 = min(k0 + kseg, gc.nz);
  const int fxa = max(2 * cx0 - 1, 0);
  const int fxb = min(2 * (cx0 + w - 1) + 1, gf.nx - 1);
  const int L = 3 * (fxb - fxa + 1);
  const int fy0 = 2 * j0 - 1;  // fine row of staged row 0 (-1 on the first block)
  // fine planes of the segment: 2k0-1 .. 2k1-1, clipped to the grid
  const int pa = max(2 * k0 - 1, 0), pb = min(2 * k1 - 1, gf.nz - 1);
  const int np = pb - pa + 1;
  const uint4* yc = reinterpret_cast<const uint4*>(ys);
  auto row_in = [&](int ry) { return fy0 + ry >= 0 && fy0 + ry < gf.ny; };
  // Staged row ry of plane p starts at entry e(p, ry) = 3 ((p ny + fy0 + ry)
  // nx + fxa); planes are staged in order, so each of this thread's chunks
  // (YS_CPT of them, fixed row and chunk index) keeps e of its row in its
  // next plane and advances it by one plane (PN entries) per staging.
  const int64_t PN = 3LL * gf.ny * gf.nx;
  int s_cu[YS_CPT], s_dst[YS_CPT];
  int64_t s_e[YS_CPT];
#pragma unroll
  for (int i = 0; i < YS_CPT; ++i) {
    const int u = threadIdx.x + i * 256;
    const int ry = u / segc;
    s_cu[i] = (u < YS_NY * segc && row_in(ry)) ? u - ry * segc : -1;  // -1: no chunk
    s_dst[i] = ry * segc + (u - ry * segc);
    s_e[i] = 3 * (((int64_t)pa * gf.ny + fy0 + ry) * gf.nx + fxa);
  }
  auto stage = [&](int slot) {
#pragma unroll
    for (int i = 0; i < YS_CPT; ++i) {
      const int64_t e0 = s_e[i];
      s_e[i] = e0 + PN;
      if (s_cu[i] < 0) continue;
      const int64_t c0 = e0 >> 3;
      if (s_cu[i] < (int)(((e0 + L + 7) >> 3) - c0))
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(
                         (unsigned)__cvta_generic_to_shared(sc + slot * YS_NY * segc + s_dst[i])),
                     "l"(yc + c0 + s_cu[i]));
    }
  };
#pragma unroll
  for (int i = 0; i < YS_RING - 1; ++i) {
    if (i < np) stage(i);
    asm volatile("cp.async.commit_group;\n" ::);
  }
  // lead of staged row ry in plane p: e(p, ry) mod 8 = (lb(p) + ry rs) mod 8,
  // lb advancing by PN mod 8 per plane
  const int rs = (int)((3LL * gf.nx) & 7), pn8 = (int)(PN & 7);
  int lb = (int)((pa * PN + 3 * ((int64_t)fy0 * gf.nx + fxa)) & 7);
  // this thread's coarse cell and component; its fine x-nodes fx-1, fx,
  // fx+1 (a missing neighbour reads the centre with weight 0)
  const int t = threadIdx.x;
  const bool act = t < 3 * w;
  const int cl = act ? t / 3 : 0, c = act ? t - 3 * cl : 0;
  const int fx = 2 * (cx0 + cl);
  const int ic = 3 * (fx - fxa) + c;
  const float wl = fx >= 1 ? 0.5f : 0.f, wr = fx + 1 < gf.nx ? 0.5f : 0.f;
  const int il = fx >= 1 ? ic - 3 : ic, ir = fx + 1 < gf.nx ? ic + 3 : ic;
  const float kc = (float)field_coef(sst, nullptr, 0, scale_mul);
  float accE[YS_JB], accO[YS_JB];  // coarse planes k even / k odd
#pragma unroll
  for (int jj = 0; jj < YS_JB; ++jj) accE[jj] = accO[jj] = 0.f;
  // z step of fine plane p = 2 kp (+1) with its y-collapsed rows vy; lo:
  // sums of coarse plane kp, hi: of kp + 1
  auto zstep = [&](float (&lo)[YS_JB], float (&hi)[YS_JB], const float (&vy)[YS_JB], int kp,
                   bool odd) {
#pragma unroll
    for (int jj = 0; jj < YS_JB; ++jj) {
      if (odd) {
        if (kp >= k0) lo[jj] += 0.5f * vy[jj];
        if (kp + 1 < k1) hi[jj] = 0.5f * vy[jj];
      } else {
        lo[jj] = kp > 0 ? lo[jj] + vy[jj] : vy[jj];
      }
    }
  };
  auto store = [&](const float (&a)[YS_JB], int k) {
    if (!act) return;
#pragma unroll
    for (int jj = 0; jj < YS_JB; ++jj)
      if (jj < jn) out[3 * (((int64_t)k * gc.ny + j0 + jj) * gc.nx + cx0) + t] = kc * a[jj];
  };
  for (int i = 0; i < np; ++i) {
    const int p = pa + i, slot = i % YS_RING;
    asm volatile("cp.async.wait_group %0;\n" ::"n"(YS_RING - 2) : "memory");
    __syncthreads();  // plane p landed for every thread; slot of plane p-1 free
    if (i + YS_RING - 1 < np) stage((i + YS_RING - 1) % YS_RING);
    asm volatile("cp.async.commit_group;\n" ::);
    const unsigned short* sp =
        reinterpret_cast<const unsigned short*>(sc + slot * YS_NY * segc);
    float vy[YS_JB];
#pragma unroll
    for (int jj = 0; jj < YS_JB; ++jj) vy[jj] = 0.f;
#pragma unroll
    for (int ry = 0; ry < YS_NY; ++ry) {
      if (!row_in(ry)) continue;
      const unsigned short* rp = sp + ry * segc * 8 + ((lb + ry * rs) & 7);
      const float xv = bf16_bits(rp[ic]) + wl * bf16_bits(rp[il]) + wr * bf16_bits(rp[ir]);
      // staged row ry is fine row 2 (j0 + jj) + d with d = ry - 1 - 2 jj
#pragma unroll
      for (int jj = 0; jj < YS_JB; ++jj) {
        const int d = ry - 1 - 2 * jj;
        if (d == 0) vy[jj] += xv;
        else if (d == 1 || d == -1) vy[jj] += 0.5f * xv;
      }
    }
    lb = (lb + pn8) & 7;
    const int kp = p >> 1;
    const bool odd = p & 1;
    if ((kp & 1) == 0) zstep(accE, accO, vy, kp, odd);
    else zstep(accO, accE, vy, kp, odd);
    // a coarse plane is complete after its top fine plane 2k+1, or after
    // plane 2k when that is the grid's last
    const int kdone = odd ? kp : (p == gf.nz - 1 ? kp : -1);
    if (kdone >= k0) {
      if ((kdone & 1) == 0) store(accE, kdone);
      else store(accO, kdone);
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// coarse planes per CTA: as many segments as fill one wave of resident CTAs
// (per_sm of them per SM; more segments would leave a partial second wave)
static int ys_kseg(const GridN& gc, int cxw, int per_sm) {
  const int64_t cols = cdiv(gc.nx, cxw) * cdiv(gc.ny, YS_JB);
  const int64_t want = (int64_t)per_sm * sm_count();
  const int64_t segs = std::max<int64_t>(1, std::min<int64_t>(gc.nz, want / cols));
  return (int)cdiv(gc.nz, segs);
}

static size_t restrict_ys_smem(int cxw) {
  const size_t seg = 3 * (2 * (size_t)cxw + 1);
  return (size_t)YS_RING * YS_NY * (seg / 8 + 3) * 16;
}

// Prolongation, the exact transpose of k_restrict (without normalisation):
// fine[j][c] = (accumulate ? fine[j][c] : 0) + sum_{i: |j - 2i| <= 1} w(j - 2i) coarse[i][c].
__global__ void k_prolong(const float* __restrict__ coarse, float* __restrict__ fine, GridN gf,
                          GridN gc, int accumulate, const uint8_t* __restrict__ fmask) {
  pdl_wait();
  pdl_trigger();
  const int64_t nf = (int64_t)gf.nx * gf.ny * gf.nz;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nf;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int fx = (int)(n % gf.nx);
    const int64_t t = n / gf.nx;
    const int fy = (int)(t % gf.ny), fz = (int)(t / gf.ny);
    int ix[2], iy[2], iz[2];
    float wx[2], wy[2], wz[2];
    prolong_axis(fx, gc.nx, ix, wx);
    prolong_axis(fy, gc.ny, iy, wy);
    prolong_axis(fz, gc.nz, iz, wz);
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
    for (int az = 0; az < 2; ++az)
#pragma unroll
      for (int ay = 0; ay < 2; ++ay)
#pragma unroll
        for (int ax = 0; ax < 2; ++ax) {
          // absent neighbours have index 0 and weight 0 (prolong_axis): no branch
          const float w = wz[az] * wy[ay] * wx[ax];
          const int64_t c = ((int64_t)iz[az] * gc.ny + iy[ay]) * gc.nx + ix[ax];
          a0 += w * coarse[3 * c + 0];
          a1 += w * coarse[3 * c + 1];
          a2 += w * coarse[3 * c + 2];
        }
    if (accumulate) {
      a0 += fine[3 * n + 0];
      a1 += fine[3 * n + 1];
      a2 += fine[3 * n + 2];
    }
    // fmask: bit c clear -> component c is a fixed DOF, set to 0
    const unsigned m = fmask ? fmask[n] : 7u;
    fine[3 * n + 0] = (m & 1u) ? a0 : 0.f;
    fine[3 * n + 1] = (m & 2u) ? a1 : 0.f;
    fine[3 * n + 2] = (m & 4u) ? a2 : 0.f;
  }
}

// The lifting E of a nodal field: X[n] = (x (3 ch), feat * x (3 ch), 0 ...) in
// BF16, stored as half-rows (act16).
__global__ void k_lift(const float* __restrict__ x, const float* __restrict__ feat,
                       __nv_bfloat16* __restrict__ X, GridN g) {
  pdl_wait();
  pdl_trigger();
  const int64_t nn = (int64_t)g.nx * g.ny * g.nz;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    __align__(16) __nv_bfloat16 o[16];
    const float fn = feat[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float t = x[3 * n + c];
      o[c] = __float2bfloat16_rn(t);
      o[c + 3] = __float2bfloat16_rn(t * fn);
    }
#pragma unroll
    for (int c = 6; c < 16; ++c) o[c] = __float2bfloat16_rn(0.f);
    const int64_t r = n / g.nx;
    const int xi = (int)(n - r * g.nx);
    *reinterpret_cast<uint4*>(X + act16(g, r, xi, 0)) = *reinterpret_cast<uint4*>(&o[0]);
    *reinterpret_cast<uint4*>(X + act16(g, r, xi, 1)) = *reinterpret_cast<uint4*>(&o[8]);
  }
}

// Its transpose on the network output (6 channels, stride 8):
// acc[n][c] (+)= Y[c] + feat * Y[c + 3].
__global__ void k_unlift(const __nv_bfloat16* __restrict__ Y, const float* __restrict__ feat,
                         float* __restrict__ acc, int accumulate, int64_t nn) {
  pdl_wait();
  pdl_trigger();
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    const uint4 yy = *reinterpret_cast<const uint4*>(Y + n * 8);
    const __nv_bfloat16* y = reinterpret_cast<const __nv_bfloat16*>(&yy);
    const float fn = feat[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float t = __bfloat162float(y[c]) + fn * __bfloat162float(y[c + 3]);
      if (accumulate) t += acc[3 * n + c];
      acc[3 * n + c] = t;
    }
  }
}

// z = M^-1 r + s D^-1/2 (R^T t)  with t the level-1 correction field (FP32
// [node][3]), R^T the prolongation of k_prolong computed on the fly and
// D^-1/2 = sqrt(minv) (masked DOFs have minv = 0).  With q_old: reduces
// z.q_old and z.r, sets the flexible-CG coefficient st->beta = -(z.q_old) /
// (p_old.q_old) (0 without a previous step) and st->aux[3] = z.r (the
// numerator of the step length, see k_struct MODE 4).  T: vector precision.
//
// Per CTA (coarse row (j, k), cells cx0 .. cx0+w-1): the fine nodes
// fx in [2 cx0, 2 (cx0 + w)), fy in {2j, 2j+1}, fz in {2k, 2k+1}.  The
// coarse rows j, j+1 x k, k+1 are first interpolated in y and z into shared
// memory (one row per fine (fy, fz)); each fine DOF then needs two shared
// loads for its x interpolation.
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 6 : 5)
    k_net_output(const T* __restrict__ r, const T* __restrict__ minv, const float* __restrict__ t,
                 GridN gf, GridN gc, int cxw, CgState* st, double scale_mul, T* __restrict__ z,
                 const T* __restrict__ q_old, double* partials) {
  pdl_wait();
  pdl_trigger();
  __shared__ float cyz[4][(ROW_CX + 1) * 3];  // [oy + 2 oz][cell][c]
  if (st->status != HX_RUNNING) return;
  const double s = sqrt(st->rz * scale_mul);
  const int cx0 = blockIdx.x * cxw, w = min(cxw, gc.nx - cx0);
  const int j = blockIdx.y, k = blockIdx.z;
  {
    // cells cx0 .. cx0 + w: the last is the right neighbour of the chunk's
    // last odd fine node (0 past the grid, like rows j+1 and planes k+1)
    const bool jn = j + 1 < gc.ny, kn = k + 1 < gc.nz;
    const int64_t r00 = ((int64_t)k * gc.ny + j) * gc.nx;
    const int64_t r10 = r00 + (jn ? gc.nx : 0);
    const int64_t r01 = r00 + (kn ? (int64_t)gc.nx * gc.ny : 0);
    const int64_t r11 = r01 + (jn ? gc.nx : 0);
    const float wj = jn ? 0.5f : 0.f, wk = kn ? 0.5f : 0.f;
    for (int e = threadIdx.x; e < 3 * (w + 1); e += blockDim.x) {
      const int cl = e / 3, c = e - 3 * cl;
      const int cx = cx0 + cl;
      const float m = cx < gc.nx ? 1.f : 0.f;
      const int64_t o = 3 * (int64_t)min(cx, gc.nx - 1) + c;
      const float t00 = t[3 * r00 + o], t10 = t[3 * r10 + o];
      const float t01 = t[3 * r01 + o], t11 = t[3 * r11 + o];
      cyz[0][e] = m * t00;
      cyz[1][e] = m * (0.5f * t00 + wj * t10);
      cyz[2][e] = m * (0.5f * t00 + wk * t01);
      cyz[3][e] = m * (0.25f * t00 + 0.5f * (wj * t10 + wk * t01) + wj * wk * t11);
    }
  }
  __syncthreads();
  // the (up to) 4 fine rows, each L DOFs: a thread takes the same DOF
  // offset in every row (12 loads in flight); rows past the grid are read at
  // row 0 and not stored
  const int fx0 = 2 * cx0;
  const int L = 3 * (min(2 * (cx0 + w), gf.nx) - fx0);
  // the rows' first DOFs as offsets from row 0's (32-bit: at most a fine
  // plane of DOFs and a row, which the grid extent limit keeps below 2^31),
  // to save registers: 6 CTAs per SM instead of 5 keep more loads in flight
  const int64_t base = 3 * (((int64_t)(2 * k) * gf.ny + 2 * j) * gf.nx + fx0);
  const T* rb = r + base;
  const T* mb = minv + base;
  const T* qb = q_old ? q_old + base : nullptr;
  T* zb = z + base;
  int rowo[4];
  unsigned rowok = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int fy = 2 * j + (q & 1), fz = 2 * k + (q >> 1);
    const bool ok = fy < gf.ny && fz < gf.nz;
    rowok |= (ok ? 1u : 0u) << q;
    rowo[q] = ok ? 3 * ((q >> 1) * gf.ny * gf.nx + (q & 1) * gf.nx) : 0;
  }
  const float sf = (float)s;
  T zq = T(0), zr = T(0);  // per-thread partials in the vectors' precision
  for (int dl = threadIdx.x; dl < L; dl += blockDim.x) {
    const int fl = dl / 3, c = dl - 3 * fl;
    const int ce = 3 * (fl >> 1) + c;
    T mv[4], rv[4], qv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      mv[q] = mb[rowo[q] + dl];
      rv[q] = rb[rowo[q] + dl];
      qv[q] = qb ? qb[rowo[q] + dl] : T(0);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (!((rowok >> q) & 1u)) continue;
      const float a = (fl & 1) ? 0.5f * (cyz[q][ce] + cyz[q][ce + 3]) : cyz[q][ce];
      // the correction is BF16-accurate: formed in FP32
      const T zi = mv[q] * rv[q] + (T)(sf * dinv_sqrt((float)mv[q]) * a);
      zb[rowo[q] + dl] = zi;
      zq += zi * qv[q];
      zr += zi * rv[q];
    }
  }
  if (!q_old) return;
  double v[2] = {(double)zq, (double)zr};
  if (grid_reduce<2>(v, partials, &st->ticket[TK_AUX2]) && threadIdx.x == 0) {
    const double pq = st->pq;
    st->beta = (pq > 0.0 && isfinite(v[0])) ? -v[0] / pq : 0.0;
    st->aux[3] = v[1];
  }
}

// Energy-norm training loss.  With z the preconditioned vector and
// d = z - e:  loss = d.Ad / e.Ae, e.Ae = e.r.  Reduces [d.q, e.r] (q = A d)
// into st->aux[0] = e.r and out[0] = loss.
__global__ void k_net_aloss(const double* __restrict__ d, const double* __restrict__ q,
                            const double* __restrict__ e, const double* __restrict__ r,
                            int64_t n, double* partials, CgState* st, double* out) {
  double dq = 0.0, er = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    dq += d[i] * q[i];
    er += e[i] * r[i];
  }
  double v[2] = {dq, er};
  if (grid_reduce<2>(v, partials, &st->ticket[TK_AUX2]) && threadIdx.x == 0) {
    st->aux[0] = v[1];
    out[0] = v[1] > 0.0 ? v[0] / v[1] : 0.0;
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
static dim3 conv_grid(const GridN& g) {
  return dim3((unsigned)cdiv(g.nx, TX), (unsigned)cdiv(g.ny, TY), (unsigned)cdiv(g.nz, TZ));
}

size_t conv_num_tiles(const GridN& g) {
  const dim3 d = conv_grid(g);
  return (size_t)d.x * d.y * d.z;
}

void launch_conv3_wgrad(cudaStream_t s, const __nv_bfloat16* X, const __nv_bfloat16* D,
                        float* part, float* grad, bool accumulate, const GridN& g) {
  const size_t smem = (HNODES + TX * TY * TZ) * C * sizeof(__nv_bfloat16);
  static PerDeviceOnce cfg;
  cfg.run([&] {
    HX_CUDA(cudaFuncSetAttribute(k_conv3_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  });
  k_conv3_wgrad<<<conv_grid(g), NTHREADS, smem, s>>>(X, D, part, g);
  HX_CHECK_LAUNCH();
  const int len = 27 * 256;
  k_reduce_parts<<<cdiv(len, 256), 256, 0, s>>>(part, (int)conv_num_tiles(g), len, grad,
                                                accumulate ? 1 : 0);
  HX_CHECK_LAUNCH();
}

void launch_adam(cudaStream_t s, float* w, float* m, float* v, const float* grad,
                 const unsigned char* live, int n, float lr, int step) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<cdiv(n, 256), 256, 0, s>>>(w, m, v, grad, live, n, lr, b1, b2, eps, c1, c2);
  HX_CHECK_LAUNCH();
}

void launch_pack_weights(cudaStream_t s, const float* w, __nv_bfloat16* wf, __nv_bfloat16* wb) {
  k_pack_weights<<<cdiv(27 * 256, 256), 256, 0, s>>>(w, wf, wb);
  HX_CHECK_LAUNCH();
}

template <typename T>
void launch_restrict_dof(cudaStream_t s, const T* v, const T* minv, const CgState* sst,
                         const CgState* lst, int mode, double scale_mul, float* out,
                         const GridN& gf, const GridN& gc) {
  static PerDeviceOnce configured;  // per instantiation and device
  configured.run([&] {
    HX_CUDA(cudaFuncSetAttribute(k_restrict_dof<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)restrict_smem<T>(RES_CX)));
  });
  const int cxw = (int)cdiv(gc.nx, cdiv(gc.nx, RES_CX));  // near-equal chunks <= RES_CX
  const dim3 grid((unsigned)cdiv(gc.nx, cxw), (unsigned)gc.ny, (unsigned)gc.nz);
  k_restrict_dof<T><<<grid, 256, restrict_smem<T>(cxw), s>>>(v, minv, sst, lst, mode, scale_mul,
                                                             out, gf, gc, cxw);
  HX_CHECK_LAUNCH();
}
template void launch_restrict_dof<double>(cudaStream_t, const double*, const double*,
                                          const CgState*, const CgState*, int, double, float*,
                                          const GridN&, const GridN&);
template void launch_restrict_dof<float>(cudaStream_t, const float*, const float*, const CgState*,
                                         const CgState*, int, double, float*, const GridN&,
                                         const GridN&);

void launch_restrict_ys(cudaStream_t s, const __nv_bfloat16* ys, const CgState* sst,
                        double scale_mul, float* out, const GridN& gf, const GridN& gc) {
  static PerDeviceOnce configured;
  configured.run([&] {
    HX_CUDA(cudaFuncSetAttribute(k_restrict_ys, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)restrict_ys_smem(YS_CX)));
  });
  const int cxw = (int)cdiv(gc.nx, cdiv(gc.nx, YS_CX));
  int per_sm = 0;
  HX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_restrict_ys, 256,
                                                        restrict_ys_smem(cxw)));
  const int kseg = ys_kseg(gc, cxw, std::max(per_sm, 1));
  const dim3 grid((unsigned)cdiv(gc.nx, cxw), (unsigned)cdiv(gc.ny, YS_JB),
                  (unsigned)cdiv(gc.nz, kseg));
  launch_pdl(k_restrict_ys, grid, 256, restrict_ys_smem(cxw), s, ys, sst, scale_mul, out, gf, gc,
             cxw, kseg);
  HX_CHECK_LAUNCH();
}

void launch_restrict(cudaStream_t s, int ch, const float* in, float* out, const GridN& gf,
                     const GridN& gc, bool normalise, const uint8_t* cmask) {
  const int64_t nc = (int64_t)gc.nx * gc.ny * gc.nz;
  HX_REQUIRE(ch == 3 || !cmask, "a DOF mask needs 3 channels");
  if (ch == 3)
    launch_pdl(k_restrict<3>, vec_blocks(nc), 256, 0, s, in, out, gf, gc, normalise ? 1 : 0, cmask);
  else if (ch == 1)
    launch_pdl(k_restrict<1>, vec_blocks(nc), 256, 0, s, in, out, gf, gc, normalise ? 1 : 0,
               (const uint8_t*)nullptr);
  else
    throw Error{HX_BAD_ARG, "unsupported channel count"};
  HX_CHECK_LAUNCH();
}

void launch_prolong(cudaStream_t s, const float* coarse, float* fine, const GridN& gf,
                    const GridN& gc, bool accumulate, const uint8_t* fmask) {
  const int64_t nf = (int64_t)gf.nx * gf.ny * gf.nz;
  launch_pdl(k_prolong, vec_blocks(nf), 256, 0, s, coarse, fine, gf, gc, accumulate ? 1 : 0, fmask);
  HX_CHECK_LAUNCH();
}

void launch_lift(cudaStream_t s, const float* x, const float* feat, __nv_bfloat16* X,
                 const GridN& g) {
  launch_pdl(k_lift, vec_blocks((int64_t)g.nx * g.ny * g.nz), 256, 0, s, x, feat, X, g);
  HX_CHECK_LAUNCH();
}

void launch_unlift(cudaStream_t s, const __nv_bfloat16* Y, const float* feat, float* acc,
                   bool accumulate, int64_t nn) {
  launch_pdl(k_unlift, vec_blocks(nn), 256, 0, s, Y, feat, acc, accumulate ? 1 : 0, nn);
  HX_CHECK_LAUNCH();
}

template <typename T>
void launch_net_output(cudaStream_t s, const T* r, const T* minv, const float* t, const GridN& gf,
                       const GridN& gc, CgState* st, double scale_mul, T* z, const T* q_old,
                       double* partials) {
  // two block partials per coarse row chunk: `partials` must hold
  // 2 net_output_blocks(gf) values
  const int cxw = row_chunk(gc.nx);
  const dim3 grid((unsigned)cdiv(gc.nx, cxw), (unsigned)gc.ny, (unsigned)gc.nz);
  launch_pdl(k_net_output<T>, grid, 256, 0, s, r, minv, t, gf, gc, cxw, st, scale_mul, z, q_old,
             partials);
  HX_CHECK_LAUNCH();
}

size_t net_output_blocks(const GridN& gf) {
  const GridN gc{(gf.nx - 1) / 2 + 1, (gf.ny - 1) / 2 + 1, (gf.nz - 1) / 2 + 1};
  return (size_t)cdiv(gc.nx, row_chunk(gc.nx)) * gc.ny * gc.nz;
}
template void launch_net_output<double>(cudaStream_t, const double*, const double*, const float*,
                                        const GridN&, const GridN&, CgState*, double, double*,
                                        const double*, double*);
template void launch_net_output<float>(cudaStream_t, const float*, const float*, const float*,
                                       const GridN&, const GridN&, CgState*, double, float*,
                                       const float*, double*);

// Density feature of a node: mean over its elements of (log10 f + 9) / 9,
// clamped to [0, 1] (f = stiffness factor, 1e-9 .. 1 under SIMP).
__global__ void k_rho_feature(const double* __restrict__ fac, float* __restrict__ feat, Grid g) {
  const int64_t nn = g.nodes();
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(n % g.nxn);
    const int64_t rr = n / g.nxn;
    const int j = (int)(rr % g.nyn), k = (int)(rr / g.nyn);
    double s = 0.0;
    int cnt = 0;
    for (int dk = -1; dk <= 0; ++dk)
      for (int dj = -1; dj <= 0; ++dj)
        for (int di = -1; di <= 0; ++di) {
          const int ei = i + di, ej = j + dj, ek = k + dk;
          if (ei < 0 || ej < 0 || ek < 0 || ei >= g.nxe || ej >= g.nye || ek >= g.nze) continue;
          const double f = fac[((int64_t)ek * g.nye + ej) * g.nxe + ei];
          s += fmin(fmax((log10(fmax(f, 1e-12)) + 9.0) / 9.0, 0.0), 1.0);
          ++cnt;
        }
    feat[n] = cnt ? (float)(s / cnt) : 0.f;
  }
}
void launch_rho_feature(cudaStream_t s, const double* fac, float* feat, const Grid& g) {
  k_rho_feature<<<vec_blocks(g.nodes()), 256, 0, s>>>(fac, feat, g);
  HX_CHECK_LAUNCH();
}

void launch_net_aloss(cudaStream_t s, const double* d, const double* q, const double* e,
                      const double* r, int64_t n, double* partials, CgState* st, double* out) {
  k_net_aloss<<<vec_blocks(n), 256, 0, s>>>(d, q, e, r, n, partials, st, out);
  HX_CHECK_LAUNCH();
}

}  // namespace hx
