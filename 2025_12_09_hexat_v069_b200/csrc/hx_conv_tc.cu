// hx_conv_tc.cu -- 3x3x3 conv3d (16 input channels, BF16, no bias) on the
// 5th-generation tensor cores: tcgen05.mma with operands in shared memory,
// staged by TMA, and the FP32 accumulators in tensor memory (TMEM).
//
// Y[n, co] = sum_{tap, ci} X[n + off(tap), ci] * W[tap][co][ci]   (zero padding)
// The transpose (backward-data pass) is the same kernel on the flipped,
// per-tap transposed weights.
//
// One CTA (4 warps) computes an 8 x 16 x TZ node tile (TZ = 4).  Implicit
// GEMM with the z-offset folded into N: for input plane q of the staged
// tile (q = 0 .. TZ + 1) and in-plane shift s = (dy, dx), one MMA of M = 128
// nodes (8 x by 16 y), N = 48 = the output channels of the three z-offsets
// (dz = +1, 0, -1, which send plane q to output slices q - 1, q, q + 1), K
// = 16 input channels.  A tile is (TZ + 2) x 9 such MMAs (plus TZ + 1 that
// start a slice's accumulator) instead of TZ x 27 of N = 16: each N = 16
// MMA costs nearly as much as an N = 48 one (the A operand, 4 KB of shared
// memory, is read either way), so the layer needs about half the tensor
// time.  The accumulators of slices -1 .. TZ + 2 (relative to the tile; the
// outer four are discarded) are 16 TMEM columns each.
//
// Shared-memory layout.  An MMA operand descriptor (no swizzle, K-major)
// addresses 8-row core matrices whose rows are 16 bytes apart; the stride
// between consecutive core matrices (SBO) and between the two 8-channel
// halves of K (LBO) are descriptor fields.  The input tile with its one-node
// halo (10 x 18 x (TZ + 2) nodes) is staged as two planes of 8 channels, 16
// bytes per node, x fastest: node (z, y, x) at ((z * 18 + y) * 10 + x) * 16.  The
// 128 rows of plane q for shift (dy, dx) are then 16 core matrices, one per
// y, of 8 consecutive x: core matrix j starts at node
// (q * 18 + 1 + dy + j) * 10 + 1 + dx, i.e. a fixed start plus j * 160
// bytes (SBO = 160).  Every shift is a start address in the same staged
// tile, so one TMA tile load per plane (box 10 nodes x 8 ch, 18 y, TZ + 2 z
// from the half-row activation tensor, act16 in hx_cnn.h: each row request
// copies 160 contiguous bytes; coordinates outside the grid read as zero)
// stages all the operands.  Row m of the accumulator is node
// (x0 + m % 8, y0 + m / 8).  The weights are staged as [s][plane][48 rows][8]
// (the B operand; k_pack_weights in hx_cnn.cu).
//
// One tile per CTA; with 48 KB of shared memory and 128 TMEM columns 4 CTAs
// share an SM, so the loads of some overlap the MMAs and epilogues of
// others.  (Measured and dropped: the unfolded form, 27 N = 16 MMAs per
// slice, 10.0 us per layer on an 81 x 41 x 41 grid; a persistent kernel
// running all 8 layers of all three networks with grid-wide barriers,
// slower at one CTA per SM, the most a kernel that allocates TMEM gets in
// a cooperative launch.)
// Thread 0 issues the bulk copy of the layer's weights (pre-packed in this
// order) and the tile's TMA loads on one mbarrier, then the 59 MMAs and a
// tcgen05.commit on a second.  Layers are launched as programmatic
// dependents of the preceding kernel: a CTA allocates TMEM, initialises its
// barriers and starts the weight copy while the previous layer finishes,
// and waits for it (griddepcontrol.wait) before loading its tile.  Every wait is bounded (1 s of
// %globaltimer time); on timeout the CTA records it in *err, waits once more
// (bounded) for its own loads or MMAs, frees its TMEM and returns, and the
// host reports the error.  Residual hazard: if that second wait also runs
// out, the CTA returns with its TMA writes or MMAs still in flight, and a
// later CTA on the SM could see its shared memory or TMEM overwritten; the
// error flag has then already failed the call.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "hx_cnn.h"

namespace hx {

namespace {

#ifndef HX_CONV_TZ
#define HX_CONV_TZ 4
#endif
constexpr int TX = 8, TY = 16, TZ = HX_CONV_TZ;
constexpr int BX = TX + 2, BY = TY + 2, BZ = TZ + 2;          // staged box with halo
constexpr int BOX_NODES = BX * BY * BZ;                       // 720
constexpr int PLANE_BYTES = BOX_NODES * 16;                   // 11520
constexpr int X_BYTES = 2 * PLANE_BYTES;                      // 23040: [plane]
constexpr int W_BYTES = 9 * 2 * 48 * 16;                      // 13824: [s][plane][48 rows]
constexpr int SMEM_BYTES = X_BYTES + W_BYTES + 64;            // + barriers, TMEM address
constexpr int NTHREADS = 128;
constexpr int ACC_COLS = (TZ + 4) * 16;                       // slices -1 .. TZ + 2
constexpr int TMEM_COLS = ACC_COLS <= 64 ? 64 : (ACC_COLS <= 128 ? 128 : 256);
constexpr uint32_t TMA_BYTES = (uint32_t)X_BYTES;
// Bounded waits: a wait gives up after WAIT_NS of %globaltimer time or
// WAIT_POLLS polls, whichever comes first (the poll count only backs up the
// clock).
constexpr unsigned long long WAIT_NS = 1000000000ull;  // 1 s
constexpr long long WAIT_POLLS = 1ll << 24;

static_assert(TX == 8 && TX * TY == 128, "a z-slice is 16 core matrices of 8 x-nodes");
static_assert(PLANE_BYTES % 128 == 0, "TMA destinations 128-byte aligned");
static_assert(ACC_COLS <= TMEM_COLS, "accumulators fit the allocation");

// Shared-memory matrix descriptor (tcgen05): no swizzle, K-major.  Fields in
// 16-byte units: start address [0,14), leading byte offset (between the two
// 8-element K halves) [16,30), stride byte offset (between 8-row groups)
// [32,46); version 1 [46,48); base offset 0; layout type 0 (no swizzle).
__host__ __device__ constexpr uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16: D FP32 [4,6) = 1, A BF16 [7,10) = 1,
// B BF16 [10,13) = 1, both K-major, N >> 3 at [17,23), M >> 4 at [24,29).
__host__ __device__ constexpr uint32_t instr_desc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

static_assert(instr_desc(128, 16) == 0x08040490u, "instruction descriptor encoding");
static_assert(instr_desc(128, 48) == 0x080C0490u, "instruction descriptor encoding");
static_assert(smem_desc(0x400, 17280, 160) ==
                  ((1ull << 46) | (10ull << 32) | (1080ull << 16) | 0x40ull),
              "shared-memory descriptor encoding");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t phase) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(done)
      : "r"(bar), "r"(phase)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait; false when the time (or poll) limit was reached
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
  const unsigned long long t0 = global_ns();
  for (long long i = 0; i < WAIT_POLLS; ++i) {
    if (mbar_try_wait(bar, phase)) return true;
    if (global_ns() - t0 > WAIT_NS) return false;
  }
  return false;
}

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int c0, int c1, int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
      : "memory");
}

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace

template <int COUT>
__global__ void __launch_bounds__(NTHREADS) k_conv3_tc(const __grid_constant__ CUtensorMap xmap,
                                                       const __nv_bfloat16* __restrict__ W,
                                                       __nv_bfloat16* __restrict__ Y, GridN g,
                                                       int* __restrict__ err, int selftest) {
  // selftest != 0 (hx_selftest_wait_timeout only): no load is issued, so the
  // load barrier never completes and the bounded wait must run out
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* xs = smem;                        // [plane][720 nodes][16 B]
  unsigned char* ws = smem + X_BYTES;              // [tap][plane][16 co][16 B]
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + X_BYTES + W_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
  int* fail = reinterpret_cast<int*>(bars + 2) + 1;
  const uint32_t load_bar = smem_u32(&bars[0]), mma_bar = smem_u32(&bars[1]);
  const uint32_t xb = smem_u32(xs), wsb = smem_u32(ws);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;

  if (warp == 0) {  // TMEM for the TZ accumulators
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    mbar_init(load_bar, 1);
    mbar_init(mma_bar, 1);
    *fail = 0;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // barriers visible to TMA
    // the layer's weights and the input tile (two 8-channel planes) on one
    // barrier; the weights are not written by the preceding kernel, so
    // their copy starts before the wait for it
    if (!selftest) {
      mbar_expect_tx(load_bar, TMA_BYTES + W_BYTES);
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
          "[%3];" ::"r"(wsb),
          "l"(W), "r"(W_BYTES), "r"(load_bar)
          : "memory");
    }
  }
  // Programmatic dependent launch: the set-up above may overlap the
  // preceding kernel (the previous layer); every access to the activations
  // follows this wait for its completion.  Then this grid lets the next
  // layer's CTAs start their own set-up.
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  if (threadIdx.x == 0 && !selftest)
    for (int h = 0; h < 2; ++h)
      tma_load_4d(xb + (uint32_t)(h * PLANE_BYTES), &xmap, load_bar, (x0 - 1) * 8, h, y0 - 1,
                  z0 - 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (threadIdx.x == 0) {
    if (!mbar_wait(load_bar, 0)) {
      *fail = 1;
      atomicExch(err, 1);
      if (!selftest) mbar_wait(load_bar, 0);  // give the loads in flight another bounded chance
    } else {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // descriptors: a fixed part plus the start address (16-byte units, low
      // bits), so each MMA adds a compile-time offset.  Slice j's accumulator
      // is at column 16 (j + 1); plane q writes slices q - 1 .. q + 1 from
      // column 16 q.  The first write of each slice has the accumulate bit
      // clear: plane 0's first MMA starts slices -1 .. 1, and the first
      // shift of plane q >= 1 is split into N = 32 (slices q - 1, q) and a
      // starting N = 16 (slice q + 1, weight rows 32 .. 47: 512 bytes on).
      const uint64_t a0 = smem_desc(xb, PLANE_BYTES, BX * 16);
      const uint64_t b0 = smem_desc(wsb, 768, 128);
      constexpr uint32_t id48 = instr_desc(128, 48), id32 = instr_desc(128, 32),
                         id16 = instr_desc(128, 16);
#pragma unroll
      for (int q = 0; q < TZ + 2; ++q) {
#pragma unroll
        for (int sh = 0; sh < 9; ++sh) {
          const int dy = sh / 3 - 1, dx = sh % 3 - 1;
          const uint64_t a = a0 + (uint32_t)((q * BY + 1 + dy) * BX + 1 + dx);
          const uint64_t b = b0 + (uint32_t)(sh * 96);  // 1536 bytes per shift
          if (sh == 0 && q > 0) {
            umma_f16(tmem + (uint32_t)(16 * q), a, b, id32, 1u);
            umma_f16(tmem + (uint32_t)(16 * (q + 2)), a, b + 32u, id16, 0u);
          } else {
            umma_f16(tmem + (uint32_t)(16 * q), a, b, id48, (q == 0 && sh == 0) ? 0u : 1u);
          }
        }
      }
      umma_commit(mma_bar);
    }
  }
  __syncthreads();
  bool ok = *fail == 0;
  if (ok && !mbar_wait(mma_bar, 0)) {
    ok = false;
    atomicExch(err, 1);
    // the committed MMAs may still be writing TMEM: give them another
    // bounded wait before the allocation is released below
    mbar_wait(mma_bar, 0);
  }
  if (ok) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int m = warp * 32 + lane;  // accumulator row = TMEM lane
    const int gx = x0 + (m & 7), gy = y0 + (m >> 3);
#pragma unroll
    for (int z = 0; z < TZ; ++z) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(16 * (z + 2)), v);
      const int gz = z0 + z;
      if (gx < g.nx && gy < g.ny && gz < g.nz) {
        const int64_t row = (int64_t)gz * g.ny + gy;
        uint32_t o[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const __nv_bfloat162 h2 = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
          o[i] = *reinterpret_cast<const uint32_t*>(&h2);
        }
        if (COUT == 16) {  // half-rows (act16)
          *reinterpret_cast<uint4*>(Y + act16(g, row, gx, 0)) = make_uint4(o[0], o[1], o[2], o[3]);
          *reinterpret_cast<uint4*>(Y + act16(g, row, gx, 1)) = make_uint4(o[4], o[5], o[6], o[7]);
        } else {
          *reinterpret_cast<uint4*>(Y + (row * g.nx + gx) * 8) = make_uint4(o[0], o[1], o[2], o[3]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS)
                 : "memory");
}

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

// Tensor map of a 16-channel activation in half-rows (act16), viewed as
// [nz][ny][2 halves][8 nx] BF16, with the staging box (10 nodes x 8 ch, one
// half, 18 y, TZ + 2 z): a load of half h lands as the plane [z][y][x][8 ch].
CUtensorMap activation_map(const __nv_bfloat16* X, const GridN& g) {
  auto fn = encode_fn();
  HX_REQUIRE(fn != nullptr, "cuTensorMapEncodeTiled is not available from the driver");
  HX_REQUIRE((reinterpret_cast<uintptr_t>(X) & 15) == 0, "activations must be 16-byte aligned");
  CUtensorMap map;
  const cuuint64_t dims[4] = {(cuuint64_t)g.nx * 8, 2, (cuuint64_t)g.ny, (cuuint64_t)g.nz};
  const cuuint64_t strides[3] = {(cuuint64_t)g.nx * 16, (cuuint64_t)g.nx * 32,
                                 (cuuint64_t)g.nx * g.ny * 32};
  const cuuint32_t box[4] = {BX * 8, 1, BY, BZ};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r =
      fn(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(X), dims, strides,
         box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
         CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  HX_REQUIRE(r == CUDA_SUCCESS, "cuTensorMapEncodeTiled failed");
  return map;
}

}  // namespace

static void conv3_launch(cudaStream_t s, int cout, const __nv_bfloat16* X, __nv_bfloat16* Y,
                         const __nv_bfloat16* W, const GridN& g, int* err, int selftest) {
  HX_REQUIRE(cout == 16 || cout == 8, "unsupported conv configuration");
  HX_REQUIRE(err != nullptr, "conv error flag missing");
  static PerDeviceOnce cfg[2];  // per output width and device
  const int idx = cout == 16 ? 0 : 1;
  cfg[idx].run([&] {
    HX_CUDA(cudaFuncSetAttribute(cout == 16 ? k_conv3_tc<16> : k_conv3_tc<8>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
  });
  const CUtensorMap map = activation_map(X, g);
  const dim3 grid((unsigned)cdiv(g.nx, TX), (unsigned)cdiv(g.ny, TY), (unsigned)cdiv(g.nz, TZ));
  // launched as a programmatic dependent of the preceding kernel on s
  cudaLaunchConfig_t lc{};
  lc.gridDim = grid;
  lc.blockDim = dim3(NTHREADS);
  lc.dynamicSmemBytes = SMEM_BYTES;
  lc.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  if (cout == 16)
    HX_CUDA(cudaLaunchKernelEx(&lc, k_conv3_tc<16>, map, W, Y, g, err, selftest));
  else
    HX_CUDA(cudaLaunchKernelEx(&lc, k_conv3_tc<8>, map, W, Y, g, err, selftest));
  HX_CHECK_LAUNCH();
}

void launch_conv3(cudaStream_t s, int cout, const __nv_bfloat16* X, __nv_bfloat16* Y,
                  const __nv_bfloat16* W, const GridN& g, int* err) {
  conv3_launch(s, cout, X, Y, W, g, err, 0);
}

// One CTA whose load barrier is never armed: its bounded wait runs out, it
// records the error in *err and returns (no load or MMA in flight).
void launch_conv3_selftest(cudaStream_t s, const __nv_bfloat16* X, __nv_bfloat16* Y,
                           const __nv_bfloat16* W, int* err) {
  conv3_launch(s, 16, X, Y, W, GridN{TX, TY, TZ}, err, 1);
}

}  // namespace hx
