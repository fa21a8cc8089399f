// hx_update.cu -- the reference's density update on the GPU:
// TopologyOptimization.update_density! (src/Optimization/TopOpt.jl:139-405),
// and the OC update behind the same signature.
//
// The reference runs every step of the update on host threads in Float32
// except its two Helmholtz filters.  Here the per-element steps are device
// kernels in the same Float32 arithmetic (so, given the same filtered field,
// every density is bit-identical), and the filters are the library's FP64
// Helmholtz CG with the reference element (GPUHelmholtz.apply_gpu_filter!
// semantics: radius and element sizes rounded to Float32, at most 200
// iterations, residual tested every 10).
//
// The reference culls by sorting its candidates (TopOpt.jl:385; Julia's
// default sort is stable, so ties go in element order).  On the device the
// cut is a radix select instead: the 64-bit key (monotone Float32 bits of
// the density, element index) of the k-th weakest candidate is found digit
// by digit from 8 histograms of 256 bins, and every candidate whose key is
// not above it is culled -- the same set the stable sort selects.
#include <chrono>
#include <cmath>

#include "hx_solver.h"

namespace hx {

namespace {

constexpr int UPD_THREADS = 256;

unsigned upd_blocks(int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, UPD_THREADS), 8LL * sm_count()));
}

// Julia's clamp(x, lo, hi) = x > hi ? hi : (x < lo ? lo : x) (NaN passes).
__device__ __forceinline__ float jclamp(float x, float lo, float hi) {
  return x > hi ? hi : (x < lo ? lo : x);
}

// Float32 bits mapped to an unsigned integer with the same order.
__device__ __forceinline__ uint32_t ordered_bits(float v) {
  const uint32_t b = __float_as_uint(v);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ bool is_candidate(float d, bool prot, float min_d, float thr) {
  return !prot && d > min_d && d < thr;
}

// Stress-ratio proposal (TopOpt.jl:262-271) as the filter's FP64 input.
__global__ void k_propose(const float* __restrict__ l1, const uint8_t* __restrict__ prot,
                          const float* __restrict__ orig, float allow, float E, float min_d,
                          float max_d, double* __restrict__ out, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const float v = prot[e] ? orig[e] : jclamp(__fdiv_rn(__fdiv_rn(l1[e], allow), E), min_d, max_d);
    out[e] = (double)v;
  }
}

// Float32 -> FP64 and back (filter input / output).
__global__ void k_f32_to_f64(const float* __restrict__ a, double* __restrict__ b, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x)
    b[e] = (double)a[e];
}
__global__ void k_f64_to_f32(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x)
    b[e] = (float)a[e];
}

// Clamp of the filtered field into the density (TopOpt.jl:327-343) and the
// culling counts (:361-377): largest |change| over unprotected elements;
// active = unprotected above min_d plus protected whose original density is
// above min_d; candidates = unprotected in (min_d, thr).  filt_out (may be
// null) receives the filtered field rounded to Float32.
__global__ void k_clamp_count(const double* __restrict__ filt, const uint8_t* __restrict__ prot,
                              const float* __restrict__ orig, float* __restrict__ dens,
                              float* __restrict__ filt_out, float min_d, float max_d, float thr,
                              int64_t n, double* partials, CgState* st) {
  double cnt[2] = {0.0, 0.0};
  double mx[1] = {0.0};
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const float fe = (float)filt[e];
    if (filt_out) filt_out[e] = fe;
    const bool p = prot[e] != 0;
    if (!p) {
      const float nv = jclamp(fe, min_d, max_d);
      const float diff = fabsf(nv - dens[e]);
      if (diff > (float)mx[0]) mx[0] = (double)diff;
      dens[e] = nv;
      cnt[0] += nv > min_d ? 1.0 : 0.0;
      cnt[1] += is_candidate(nv, false, min_d, thr) ? 1.0 : 0.0;
    } else {
      cnt[0] += orig[e] > min_d ? 1.0 : 0.0;
    }
  }
  const unsigned nblk = gridDim.x;
  if (grid_reduce<2>(cnt, partials, &st->ticket[TK_AUX]) && threadIdx.x == 0) {
    st->aux[0] = cnt[0];
    st->aux[1] = cnt[1];
  }
  if (grid_reduce<1, true>(mx, partials + 2 * (size_t)nblk, &st->ticket[TK_AUX2]) &&
      threadIdx.x == 0)
    st->aux[2] = mx[0];
}

// One radix-select pass: histogram of the 8-bit digit at `shift` of the keys
// (ordered density bits << 32 | element) of the candidates whose digits
// above `shift` equal those of `prefix`.
__global__ void k_key_hist(const float* __restrict__ dens, const uint8_t* __restrict__ prot,
                           float min_d, float thr, unsigned long long prefix, int shift,
                           int64_t n, unsigned int* __restrict__ hist) {
  __shared__ unsigned int h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const float d = dens[e];
    if (!is_candidate(d, prot[e] != 0, min_d, thr)) continue;
    const unsigned long long key = ((unsigned long long)ordered_bits(d) << 32) | (uint64_t)e;
    if (shift < 56 && (key >> (shift + 8)) != (prefix >> (shift + 8))) continue;
    atomicAdd(&h[(key >> shift) & 255u], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (h[i]) atomicAdd(&hist[i], h[i]);
}

// Culling (all candidates, or those with key <= kstar) and the protected
// re-enforce (TopOpt.jl:379-402).
__global__ void k_cull(float* __restrict__ dens, const uint8_t* __restrict__ prot,
                       const float* __restrict__ orig, float min_d, float thr, int select,
                       unsigned long long kstar, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const bool p = prot[e] != 0;
    const float d = dens[e];
    if (is_candidate(d, p, min_d, thr)) {
      const unsigned long long key = ((unsigned long long)ordered_bits(d) << 32) | (uint64_t)e;
      if (!select || key <= kstar) dens[e] = min_d;
    }
    if (p) dens[e] = orig[e];
  }
}

// OC step on the clamped Float32 density: x_new from the FP64 OC bisection,
// clamped to [min_d, max_d]; protected elements keep their original
// density; largest |change| over unprotected elements.
__global__ void k_oc_finish(const double* __restrict__ xnew, const uint8_t* __restrict__ prot,
                            const float* __restrict__ orig, float* __restrict__ dens, float min_d,
                            float max_d, int64_t n, double* partials, CgState* st) {
  double mx[1] = {0.0};
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    if (prot[e]) {
      dens[e] = orig[e];
      continue;
    }
    const float nv = jclamp((float)xnew[e], min_d, max_d);
    const float diff = fabsf(nv - dens[e]);
    if (diff > (float)mx[0]) mx[0] = (double)diff;
    dens[e] = nv;
  }
  if (grid_reduce<1, true>(mx, partials, &st->ticket[TK_AUX2]) && threadIdx.x == 0)
    st->aux[2] = mx[0];
}

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

// Radius schedule of update_density!, TopOpt.jl:216-255, in Julia's types:
// percentages and element sizes Float32, max_domain_dim Float64 (a YAML
// number), so the lengths are Float64; t, the guard 1.2 * mean element size
// and the divisor 2.5 are Float32 (when the guard applies, R_length is the
// Float32 guard and R_effective a Float32 quotient).
void update_radius_schedule(const hx_update_params& p, int it, int n_iter, double* R_length,
                            double* R_effective) {
  const float dx = (float)p.h[0], dy = (float)p.h[1], dz = (float)p.h[2];
  const float avg = (dx + dy + dz) / 3.0f;
  const float ri = (float)p.filter_R_init_perc / 100.0f;
  const float rm = (float)p.filter_R_interm_perc / 100.0f;
  const float rf = (float)p.filter_R_final_perc / 100.0f;
  const float rip = (float)p.filter_R_interm_iter_perc / 100.0f;
  const double Ri = (double)ri * p.max_domain_dim, Rm = (double)rm * p.max_domain_dim,
               Rf = (double)rf * p.max_domain_dim;
  const int iter_interm = std::max(1, (int)std::nearbyint(rip * (float)n_iter));
  const int calc = std::min(it, n_iter);
  double R;
  if (calc <= iter_interm) {
    const float t = iter_interm > 1 ? (float)(calc - 1) / (float)(iter_interm - 1) : 0.0f;
    R = Ri * (double)(1.0f - t) + Rm * (double)t;
  } else {
    const float t =
        n_iter > iter_interm ? (float)(calc - iter_interm) / (float)(n_iter - iter_interm) : 0.0f;
    R = Rm * (double)(1.0f - t) + Rf * (double)t;
  }
  const float safe = 1.2f * avg;
  if (R < (double)safe) {
    *R_length = (double)safe;
    *R_effective = (double)(safe / 2.5f);
  } else {
    *R_length = R;
    *R_effective = R / 2.5;
  }
}

hx_status update_density(hx_ctx* c, float* density, float* l1, const uint8_t* prot, float E,
                         float allow, int it, int n_iter, const float* orig, float min_d,
                         float max_d, const hx_update_params& p, const float* dc,
                         float* filtered_out, hx_update_result* res) {
  HX_REQUIRE(density && l1 && prot && orig, "null argument");
  HX_REQUIRE(p.mode == HX_UPDATE_STRESS_RATIO || p.mode == HX_UPDATE_OC, "unknown update mode");
  HX_REQUIRE(p.mode != HX_UPDATE_OC || dc != nullptr, "the OC update needs the sensitivities");
  HX_REQUIRE(n_iter >= 1, "number_of_iterations must be >= 1");
  HX_REQUIRE(grid_extent_ok(p.nelem[0], p.nelem[1], p.nelem[2]), "bad or too large grid");
  HX_REQUIRE(p.h[0] > 0 && p.h[1] > 0 && p.h[2] > 0, "element size must be positive");
  Grid g{};
  g.nxe = (int)p.nelem[0];
  g.nye = (int)p.nelem[1];
  g.nze = (int)p.nelem[2];
  g.nxn = g.nxe + 1;
  g.nyn = g.nye + 1;
  g.nzn = g.nze + 1;
  const int64_t n = g.elems();
  HX_REQUIRE(n < (int64_t(1) << 32), "too many elements for the culling keys");
  // element sizes and tolerances as the reference's Float32 filter sees them
  const double hf[3] = {(double)(float)p.h[0], (double)(float)p.h[1], (double)(float)p.h[2]};
  const double ftol = (double)(float)p.filter_tolerance;
  ensure_workspace(c);
  const unsigned nb = upd_blocks(n);
  c->d_partials.ensure(std::max<size_t>(c->d_partials.n, 4ull * nb));
  auto& U = c->upd;
  float* d_dens = U.dens.ensure(n);
  float* d_l1 = U.l1.ensure(n);
  float* d_orig = U.orig.ensure(n);
  uint8_t* d_prot = U.prot.ensure(n);
  double* a64 = U.a.ensure(n);
  double* b64 = U.b.ensure(n);
  unsigned int* d_hist = U.hist.ensure(256);
  cudaStream_t s = c->stream;
  HX_CUDA(cudaMemcpyAsync(d_dens, density, n * sizeof(float), cudaMemcpyHostToDevice, s));
  HX_CUDA(cudaMemcpyAsync(d_l1, l1, n * sizeof(float), cudaMemcpyHostToDevice, s));
  HX_CUDA(cudaMemcpyAsync(d_orig, orig, n * sizeof(float), cudaMemcpyHostToDevice, s));
  HX_CUDA(cudaMemcpyAsync(d_prot, prot, n, cudaMemcpyHostToDevice, s));
  hx_update_result R{};
  const float avg = ((float)p.h[0] + (float)p.h[1] + (float)p.h[2]) / 3.0f;

  // 2. optional stress regularisation (TopOpt.jl:176-211), radius ratio * h
  const float ratio = (float)p.stress_regularization_ratio;
  if (ratio > 1.0e-6f) {
    k_f32_to_f64<<<nb, UPD_THREADS, 0, s>>>(d_l1, a64, n);
    HX_CHECK_LAUNCH();
    hx_solve_report fr{};
    const hx_status fs = filter_grid(c, g, hf, a64, b64, (double)(ratio * avg), 1, ftol, 200, &fr);
    if (fs != HX_OK) return fs;
    k_f64_to_f32<<<nb, UPD_THREADS, 0, s>>>(b64, d_l1, n);
    HX_CHECK_LAUNCH();
    HX_CUDA(cudaMemcpyAsync(l1, d_l1, n * sizeof(float), cudaMemcpyDeviceToHost, s));
  }
  // 3. radius schedule and guard
  double R_eff = 0;
  update_radius_schedule(p, it, n_iter, &R.R_length, &R_eff);
  const double radius = (double)(float)R_eff;  // the filter workspace's T(radius)
  // culling threshold (TopOpt.jl:352-358), Float32
  const float fthr = (float)p.final_density_threshold;
  const float thr = it > n_iter ? fthr : fthr * ((float)it / (float)n_iter);
  R.current_threshold = p.mode == HX_UPDATE_OC ? 0.0 : (double)thr;

  hx::CgState st0{};
  put_state(c, 3, st0);
  CgState* st = c->d_state.p + 3;
  if (p.mode == HX_UPDATE_STRESS_RATIO) {
    // 4. stress-ratio proposal; 5. its Helmholtz filter
    k_propose<<<nb, UPD_THREADS, 0, s>>>(d_l1, d_prot, d_orig, allow, E, min_d, max_d, a64, n);
    HX_CHECK_LAUNCH();
    hx_solve_report fr{};
    const double t0 = now_s();
    const hx_status fs = filter_grid(c, g, hf, a64, b64, radius, 1, ftol, 200, &fr);
    R.filter_time = now_s() - t0;
    R.filter_iters = fr.iterations;
    R.filter_res = fr.rel_res;
    if (fs != HX_OK) return fs;
    // 6. clamp, largest change, culling counts
    float* d_fo = filtered_out ? U.fout.ensure(n) : nullptr;
    k_clamp_count<<<nb, UPD_THREADS, 0, s>>>(b64, d_prot, d_orig, d_dens, d_fo, min_d, max_d, thr,
                                            n, c->d_partials.p, st);
    HX_CHECK_LAUNCH();
    const CgState cs = get_state(c, 3);
    const int64_t active = (int64_t)cs.aux[0], ncand = (int64_t)cs.aux[1];
    R.max_change = cs.aux[2];
    // 7. culling: floor(Int, active * max_culling_ratio) in Float32, as Int * Float32
    const float ratio_c = (float)p.max_culling_ratio;
    const int64_t max_allowed = (int64_t)std::floor((float)active * ratio_c);
    // select: 0 = cull every candidate, 1 = only keys <= kstar, 2 = none
    int select = 0;
    unsigned long long kstar = 0;
    if (ncand > max_allowed) {
      if (max_allowed <= 0) {
        select = 2;
      } else {
        select = 1;
        // the max_allowed-th smallest key, 8 bits at a time from the top
        int64_t k = max_allowed;  // 1-based rank still to place within the prefix
        unsigned long long prefix = 0;
        unsigned int h[256];
        for (int shift = 56; shift >= 0; shift -= 8) {
          HX_CUDA(cudaMemsetAsync(d_hist, 0, 256 * sizeof(unsigned int), s));
          k_key_hist<<<nb, UPD_THREADS, 0, s>>>(d_dens, d_prot, min_d, thr, prefix, shift, n,
                                                d_hist);
          HX_CHECK_LAUNCH();
          HX_CUDA(cudaMemcpyAsync(h, d_hist, sizeof(h), cudaMemcpyDeviceToHost, s));
          HX_CUDA(cudaStreamSynchronize(s));
          int64_t acc = 0;
          int digit = 255;
          for (int dgt = 0; dgt < 256; ++dgt) {
            if (acc + (int64_t)h[dgt] >= k) {
              digit = dgt;
              break;
            }
            acc += h[dgt];
          }
          k -= acc;
          prefix |= (unsigned long long)digit << shift;
        }
        kstar = prefix;
      }
    }
    // with nothing to cull, a threshold of -inf leaves only the re-enforce
    k_cull<<<nb, UPD_THREADS, 0, s>>>(d_dens, d_prot, d_orig, min_d, select == 2 ? -INFINITY : thr,
                                      select == 1 ? 1 : 0, kstar, n);
    HX_CHECK_LAUNCH();
    R.culled = (int32_t)(select == 2 ? 0 : (select ? max_allowed : ncand));
    if (filtered_out)
      HX_CUDA(cudaMemcpyAsync(filtered_out, d_fo, n * sizeof(float), cudaMemcpyDeviceToHost, s));
  } else {
    // OC: dc filtered with the same Helmholtz radius, bisection on the
    // volume multiplier with unit volumes (hx_oc_update), clamp, protect
    float* d_dc = U.dc.ensure(n);
    double* x64 = U.c.ensure(n);
    double* xn64 = U.d.ensure(n);
    HX_CUDA(cudaMemcpyAsync(d_dc, dc, n * sizeof(float), cudaMemcpyHostToDevice, s));
    k_f32_to_f64<<<nb, UPD_THREADS, 0, s>>>(d_dc, a64, n);
    HX_CHECK_LAUNCH();
    hx_solve_report fr{};
    const double t0 = now_s();
    const hx_status fs = filter_grid(c, g, hf, a64, b64, radius, 1, ftol, 200, &fr);
    R.filter_time = now_s() - t0;
    R.filter_iters = fr.iterations;
    R.filter_res = fr.rel_res;
    if (fs != HX_OK) return fs;
    if (filtered_out) {
      float* d_fo = U.fout.ensure(n);
      k_f64_to_f32<<<nb, UPD_THREADS, 0, s>>>(b64, d_fo, n);
      HX_CHECK_LAUNCH();
      HX_CUDA(cudaMemcpyAsync(filtered_out, d_fo, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    }
    k_f32_to_f64<<<nb, UPD_THREADS, 0, s>>>(d_dens, x64, n);
    HX_CHECK_LAUNCH();
    hx::CgState so{};
    so.aux[0] = 0.0;
    so.aux[1] = 1e9;
    so.status = HX_RUNNING;
    put_state(c, 3, so);
    launch_oc(s, x64, b64, nullptr, n, p.oc_volfrac, p.oc_move, xn64, st, c->d_partials.p, 100);
    get_state(c, 3);  // the bisection is done (and the pinned state mirror free) before reuse
    put_state(c, 3, CgState{});
    k_oc_finish<<<nb, UPD_THREADS, 0, s>>>(xn64, d_prot, d_orig, d_dens, min_d, max_d, n,
                                          c->d_partials.p, st);
    HX_CHECK_LAUNCH();
    const CgState cs = get_state(c, 3);
    R.max_change = cs.aux[2];
  }
  HX_CUDA(cudaMemcpyAsync(density, d_dens, n * sizeof(float), cudaMemcpyDeviceToHost, s));
  HX_CUDA(cudaStreamSynchronize(s));
  if (res) *res = R;
  return HX_OK;
}

}  // namespace hx
