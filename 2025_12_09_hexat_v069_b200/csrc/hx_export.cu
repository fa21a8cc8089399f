// hx_export.cu -- the reference's "webdata" result file from device buffers:
// export_binary_for_web (src/IO/Postprocessing.jl:159-262), the file its
// viewers and its checkpoint restart (src/IO/Configuration.jl:31-77) read.
//
// The elements with density >= threshold are compacted on the device in
// element order (the order of the reference's findall): each block owns a
// contiguous range of elements, counts its survivors, and after an
// exclusive scan of the block counts writes them at its offset in order.
// Per survivor: the centroid (the sum of its 8 corner coordinates in
// NAT_COORDS order times 0.125, in Float32, as MeshUtilities.element_centroid
// sums them), the density, and the L1 stress signed by the principal stress
// of largest magnitude (Postprocessing.jl:183-193).  The host writes the
// header, the three arrays and the caller's JSON text.
#include <cstdio>
#include <vector>

#include "hx_solver.h"

namespace hx {

namespace {

constexpr int EXP_THREADS = 256;

// Float32 node coordinate of lattice index i along an axis (generate_mesh:
// (i - 1) * dx with a 1-based i, as a Float32 product), plus the origin.
__device__ __forceinline__ float node_coord(int i, float h, float o) {
  return (float)i * h + o;
}

__device__ __forceinline__ float jsign(float v) {  // Julia sign(): -1, 0, 1 (NaN stays)
  return v > 0.f ? 1.f : (v < 0.f ? -1.f : v);
}

template <typename T>
__global__ void k_survivor_count(const T* __restrict__ dens, float thr, int64_t n, int64_t chunk,
                                 unsigned long long* __restrict__ counts) {
  const int64_t b0 = (int64_t)blockIdx.x * chunk, b1 = min(n, b0 + chunk);
  unsigned long long c = 0;
  for (int64_t e = b0 + threadIdx.x; e < b1; e += blockDim.x) c += (float)dens[e] >= thr ? 1 : 0;
  __shared__ unsigned long long s[EXP_THREADS];
  s[threadIdx.x] = c;
  __syncthreads();
  for (int o = EXP_THREADS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) counts[blockIdx.x] = s[0];
}

// Writes block b's survivors at offsets[b] .. in element order: the block
// walks its range in tiles of EXP_THREADS elements, placing each tile's
// survivors by a block-wide prefix count.
template <typename T>
__global__ void k_survivor_write(const T* __restrict__ dens, const T* __restrict__ l1,
                                 const T* __restrict__ pr, float thr, Grid g, float hx, float hy,
                                 float hz, float ox, float oy, float oz, int64_t chunk,
                                 const unsigned long long* __restrict__ offsets,
                                 float* __restrict__ cent, float* __restrict__ dout,
                                 float* __restrict__ sl1) {
  const int64_t n = g.elems();
  const int64_t b0 = (int64_t)blockIdx.x * chunk, b1 = min(n, b0 + chunk);
  __shared__ int warp_tot[EXP_THREADS / 32];
  unsigned long long base = offsets[blockIdx.x];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int64_t t0 = b0; t0 < b1; t0 += EXP_THREADS) {
    const int64_t e = t0 + threadIdx.x;
    const bool keep = e < b1 && (float)dens[e] >= thr;
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    const int before_in_warp = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) warp_tot[w] = __popc(bal);
    __syncthreads();
    int before = before_in_warp, total = 0;
    for (int k = 0; k < EXP_THREADS / 32; ++k) {
      if (k < w) before += warp_tot[k];
      total += warp_tot[k];
    }
    if (keep) {
      const unsigned long long o = base + (unsigned long long)before;
      const int i = (int)(e % g.nxe);
      const int64_t r = e / g.nxe;
      const int j = (int)(r % g.nye), k = (int)(r / g.nye);
      // corners in NAT_COORDS order: (i,j),(i+1,j),(i+1,j+1),(i,j+1), then z+1
      const float x0 = node_coord(i, hx, ox), x1 = node_coord(i + 1, hx, ox);
      const float y0 = node_coord(j, hy, oy), y1 = node_coord(j + 1, hy, oy);
      const float z0 = node_coord(k, hz, oz), z1 = node_coord(k + 1, hz, oz);
      float cx = 0.f, cy = 0.f, cz = 0.f;
      const float xs[8] = {x0, x1, x1, x0, x0, x1, x1, x0};
      const float ys[8] = {y0, y0, y1, y1, y0, y0, y1, y1};
      const float zs[8] = {z0, z0, z0, z0, z1, z1, z1, z1};
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        cx = __fadd_rn(cx, xs[c]);
        cy = __fadd_rn(cy, ys[c]);
        cz = __fadd_rn(cz, zs[c]);
      }
      cent[3 * o + 0] = __fmul_rn(cx, 0.125f);
      cent[3 * o + 1] = __fmul_rn(cy, 0.125f);
      cent[3 * o + 2] = __fmul_rn(cz, 0.125f);
      dout[o] = (float)dens[e];
      const float s1 = (float)pr[3 * e], s2 = (float)pr[3 * e + 1], s3 = (float)pr[3 * e + 2];
      float amax = fabsf(s1), sg = jsign(s1);
      if (fabsf(s2) > amax) {
        amax = fabsf(s2);
        sg = jsign(s2);
      }
      if (fabsf(s3) > amax) sg = jsign(s3);
      sl1[o] = __fmul_rn((float)l1[e], sg);
    }
    base += (unsigned long long)total;
    __syncthreads();
  }
}

}  // namespace

template <typename T>
hx_status export_webdata(hx_ctx* c, const char* path, const T* dens, const T* l1, const T* pr,
                         float threshold, int iter, float radius, const char* json,
                         int64_t json_len, int64_t* count_out) {
  HX_REQUIRE(path && dens && l1 && pr, "null argument");
  HX_REQUIRE(json_len >= 0 && (json || json_len == 0), "bad JSON buffer");
  HX_REQUIRE(json_len <= 0xFFFFFFFFll, "JSON text longer than the format's 32-bit length");
  const Grid& g = c->g;
  const int64_t n = g.elems();
  const int64_t chunk = 8192;
  const int64_t nblk = (n + chunk - 1) / chunk;
  auto& X = c->exp;
  unsigned long long* cnt = X.counts.ensure(nblk);
  unsigned long long* off = X.offsets.ensure(nblk);
  k_survivor_count<T><<<(unsigned)nblk, EXP_THREADS, 0, c->stream>>>(dens, threshold, n, chunk,
                                                                     cnt);
  HX_CHECK_LAUNCH();
  std::vector<unsigned long long> h(nblk);
  HX_CUDA(cudaMemcpyAsync(h.data(), cnt, nblk * sizeof(unsigned long long),
                          cudaMemcpyDeviceToHost, c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  unsigned long long total = 0;
  for (int64_t b = 0; b < nblk; ++b) {
    const unsigned long long v = h[b];
    h[b] = total;
    total += v;
  }
  if (count_out) *count_out = (int64_t)total;
  if (total == 0) return HX_OK;  // the reference writes no file (Postprocessing.jl:175)
  HX_REQUIRE(total <= 0xFFFFFFFFull, "too many elements for the format's 32-bit count");
  HX_CUDA(cudaMemcpyAsync(off, h.data(), nblk * sizeof(unsigned long long),
                          cudaMemcpyHostToDevice, c->stream));
  float* cent = X.cent.ensure(3 * total);
  float* dout = X.dens.ensure(total);
  float* sl1 = X.sl1.ensure(total);
  k_survivor_write<T><<<(unsigned)nblk, EXP_THREADS, 0, c->stream>>>(
      dens, l1, pr, threshold, g, (float)c->h[0], (float)c->h[1], (float)c->h[2],
      (float)c->origin[0], (float)c->origin[1], (float)c->origin[2], chunk, off, cent, dout, sl1);
  HX_CHECK_LAUNCH();
  std::vector<float> hc(3 * total), hd(total), hs(total);
  HX_CUDA(cudaMemcpyAsync(hc.data(), cent, hc.size() * sizeof(float), cudaMemcpyDeviceToHost,
                          c->stream));
  HX_CUDA(cudaMemcpyAsync(hd.data(), dout, hd.size() * sizeof(float), cudaMemcpyDeviceToHost,
                          c->stream));
  HX_CUDA(cudaMemcpyAsync(hs.data(), sl1, hs.size() * sizeof(float), cudaMemcpyDeviceToHost,
                          c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  FILE* fp = std::fopen(path, "wb");
  HX_REQUIRE(fp != nullptr, std::string("cannot open ") + path + " for writing");
  // header (Postprocessing.jl:239-252): magic "HEXA", version 2, iter,
  // radius, threshold, count, dx, dy, dz; little-endian as written by Julia
  const uint32_t magic = 0x48455841u, version = 2u, count = (uint32_t)total;
  const int32_t it32 = (int32_t)iter;
  const float hdr_f[2] = {radius, threshold};
  const float hs3[3] = {(float)c->h[0], (float)c->h[1], (float)c->h[2]};
  const uint32_t jl = (uint32_t)json_len;
  bool ok = std::fwrite(&magic, 4, 1, fp) == 1 && std::fwrite(&version, 4, 1, fp) == 1 &&
            std::fwrite(&it32, 4, 1, fp) == 1 && std::fwrite(hdr_f, 4, 2, fp) == 2 &&
            std::fwrite(&count, 4, 1, fp) == 1 && std::fwrite(hs3, 4, 3, fp) == 3 &&
            std::fwrite(hc.data(), 4, hc.size(), fp) == hc.size() &&
            std::fwrite(hd.data(), 4, hd.size(), fp) == hd.size() &&
            std::fwrite(hs.data(), 4, hs.size(), fp) == hs.size() &&
            std::fwrite(&jl, 4, 1, fp) == 1 &&
            (jl == 0 || std::fwrite(json, 1, jl, fp) == jl);
  ok = (std::fclose(fp) == 0) && ok;
  HX_REQUIRE(ok, std::string("write to ") + path + " failed");
  return HX_OK;
}

template hx_status export_webdata<double>(hx_ctx*, const char*, const double*, const double*,
                                          const double*, float, int, float, const char*, int64_t,
                                          int64_t*);
template hx_status export_webdata<float>(hx_ctx*, const char*, const float*, const float*,
                                         const float*, float, int, float, const char*, int64_t,
                                         int64_t*);

}  // namespace hx
