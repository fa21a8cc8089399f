// hx_api.cu -- the C ABI (include/hexat_b200.h): argument checking, mapping
// between the caller's numbering/dtype and the device grid layout, and the
// reference-shaped drop-in entry points.
#include <chrono>
#include <cmath>
#include <cstring>
#include <new>

#include "hx_solver.h"

using hx::DevBuf;
using hx::Grid;

namespace {

double now_ms() {
  using namespace std::chrono;
  return std::chrono::duration<double, std::milli>(steady_clock::now().time_since_epoch())
      .count();
}

template <typename F>
hx_status guard(hx_ctx* c, F&& f) {
  if (!c) return HX_BAD_ARG;
  const int64_t l0 = hx::launch_counter();
  struct Count {
    hx_ctx* c;
    int64_t l0;
    ~Count() { c->launches += hx::launch_counter() - l0; }
  } count{c, l0};
  try {
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) {
      c->err = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
      return HX_CUDA_ERROR;
    }
    // The context's stream does not synchronise with the legacy default
    // stream by itself; every call first waits for the work queued there
    // (device inputs written by, e.g., PyTorch's default stream).
    e = cudaEventRecord(c->ev_in, cudaStreamLegacy);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->ev_in, 0);
    if (e != cudaSuccess) {
      c->err = std::string("ordering after the default stream: ") + cudaGetErrorString(e);
      return HX_CUDA_ERROR;
    }
    hx_status s = f();
    if (s == HX_OK) c->err.clear();
    return s;
  } catch (hx::Error& e) {
    c->err = e.msg;
    return e.status;
  } catch (std::bad_alloc&) {
    c->err = "host allocation failed";
    return HX_OOM;
  } catch (std::exception& e) {
    c->err = e.what();
    return HX_BAD_ARG;
  }
}

void set_grid_impl(hx_ctx* c, int64_t nx, int64_t ny, int64_t nz, double dx, double dy,
                   double dz) {
  HX_REQUIRE(nx >= 1 && ny >= 1 && nz >= 1, "grid needs at least one element per axis");
  HX_REQUIRE(hx::grid_extent_ok(nx, ny, nz),
             "grid too large (axes below 2^20 nodes, 3 x nodes per z-plane below 2^31, "
             "DOFs below 2^40)");
  HX_REQUIRE(dx > 0 && dy > 0 && dz > 0, "element size must be positive");
  c->g.nxe = (int)nx;
  c->g.nye = (int)ny;
  c->g.nze = (int)nz;
  c->g.nxn = (int)nx + 1;
  c->g.nyn = (int)ny + 1;
  c->g.nzn = (int)nz + 1;
  c->h[0] = dx;
  c->h[1] = dy;
  c->h[2] = dz;
  c->K = hx::make_elem_coef(dx, dy, dz, c->nu);
  c->has_mesh = true;
  c->origin[0] = c->origin[1] = c->origin[2] = 0.0;
  c->node_map.clear();
  c->elem_map.clear();
  c->present.clear();
  c->n_user_nodes = c->g.nodes();
  c->n_user_elem = c->g.elems();
  c->bcfree.assign(c->g.nodes(), 7);
  c->bc_dirty = true;
}

bool identity(const hx_ctx* c) { return c->node_map.empty(); }

// Lattice detection for reference-layout meshes (see hx_set_mesh in the
// header).  Throws HX_BAD_ARG for meshes that are not on a lattice.
void set_mesh_impl(hx_ctx* c, const float* nodes, int64_t nN, const int64_t* el, int64_t nE) {
  HX_REQUIRE(nodes && el && nN >= 8 && nE >= 1, "empty mesh");
  auto X = [&](int64_t n, int d) { return (double)nodes[d * nN + n]; };
  auto C = [&](int64_t e, int k) { return el[k * nE + e] - 1; };
  for (int k = 0; k < 8; ++k) HX_REQUIRE(C(0, k) >= 0 && C(0, k) < nN, "element 1 out of range");
  // element size from the first element (src/Solvers/GPUSolver.jl:136-143)
  auto dist = [&](int64_t a, int64_t b) {
    double s = 0;
    for (int d = 0; d < 3; ++d) s += (X(b, d) - X(a, d)) * (X(b, d) - X(a, d));
    return std::sqrt(s);
  };
  const double dx = dist(C(0, 0), C(0, 1)), dy = dist(C(0, 0), C(0, 3)),
               dz = dist(C(0, 0), C(0, 4));
  HX_REQUIRE(dx > 0 && dy > 0 && dz > 0, "degenerate first element");
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t n = 0; n < nN; ++n)
    for (int d = 0; d < 3; ++d) {
      mn[d] = std::min(mn[d], X(n, d));
      mx[d] = std::max(mx[d], X(n, d));
    }
  const double h[3] = {dx, dy, dz};
  int64_t dims[3];
  for (int d = 0; d < 3; ++d) {
    dims[d] = (int64_t)std::llround((mx[d] - mn[d]) / h[d]);
    HX_REQUIRE(dims[d] >= 1, "mesh is flat along an axis");
  }
  HX_REQUIRE(hx::grid_extent_ok(dims[0], dims[1], dims[2]), "mesh bounding grid too large");
  // node -> lattice position
  Grid g{};
  g.nxe = (int)dims[0];
  g.nye = (int)dims[1];
  g.nze = (int)dims[2];
  g.nxn = g.nxe + 1;
  g.nyn = g.nye + 1;
  g.nzn = g.nze + 1;
  std::vector<int64_t> nmap(nN);
  std::vector<uint8_t> present(g.nodes(), 0);
  bool ident = (nN == g.nodes());
  for (int64_t n = 0; n < nN; ++n) {
    int64_t ijk[3];
    for (int d = 0; d < 3; ++d) {
      const double t = (X(n, d) - mn[d]) / h[d];
      ijk[d] = (int64_t)std::llround(t);
      HX_REQUIRE(std::fabs(t - (double)ijk[d]) < 1e-3,
                 "mesh nodes are not on a lattice (unstructured meshes are not supported)");
    }
    const int64_t gid = ijk[0] + g.nxn * (ijk[1] + (int64_t)g.nyn * ijk[2]);
    HX_REQUIRE(!present[gid], "two nodes share a lattice position");
    present[gid] = 1;
    nmap[n] = gid;
    if (gid != n) ident = false;
  }
  // elements -> grid elements, checking the canonical corner pattern
  static const int bits[8] = {0, 1, 3, 2, 4, 5, 7, 6};
  std::vector<int64_t> emap(nE);
  std::vector<uint8_t> eseen(g.elems(), 0);
  if (nE != g.elems()) ident = false;
  const int64_t pl = (int64_t)g.nxn * g.nyn;
  for (int64_t e = 0; e < nE; ++e) {
    const int64_t n0 = C(e, 0);
    HX_REQUIRE(n0 >= 0 && n0 < nN, "element connectivity out of range");
    const int64_t g0 = nmap[n0];
    const int64_t i = g0 % g.nxn, j = (g0 / g.nxn) % g.nyn, k = g0 / pl;
    HX_REQUIRE(i < g.nxe && j < g.nye && k < g.nze, "element not on the lattice");
    for (int c = 0; c < 8; ++c) {
      const int64_t nc = C(e, c);
      HX_REQUIRE(nc >= 0 && nc < nN, "element connectivity out of range");
      const int b = bits[c];
      const int64_t want = g0 + (b & 1) + ((b >> 1) & 1) * (int64_t)g.nxn + ((b >> 2) & 1) * pl;
      HX_REQUIRE(nmap[nc] == want,
                 "element corners do not follow the structured Hex8 pattern "
                 "(unstructured meshes are not supported)");
    }
    const int64_t ge = i + g.nxe * (j + (int64_t)g.nye * k);
    HX_REQUIRE(!eseen[ge], "duplicate element");
    eseen[ge] = 1;
    emap[e] = ge;
    if (ge != e) ident = false;
  }
  set_grid_impl(c, g.nxe, g.nye, g.nze, dx, dy, dz);
  for (int d = 0; d < 3; ++d) c->origin[d] = mn[d];
  if (!ident) {
    c->node_map = std::move(nmap);
    c->elem_map = std::move(emap);
    c->present = std::move(present);
    c->n_user_nodes = nN;
    c->n_user_elem = nE;
    // lattice points without a caller node are held fixed
    for (int64_t n = 0; n < c->g.nodes(); ++n)
      if (!c->present[n]) c->bcfree[n] = 0;
  }
}

// ---- dtype / numbering conversion ----------------------------------------
double load_val(int32_t dt, const void* p, int64_t i) {
  return dt == HX_F64 ? ((const double*)p)[i] : (double)((const float*)p)[i];
}
void store_val(int32_t dt, void* p, int64_t i, double v) {
  if (dt == HX_F64)
    ((double*)p)[i] = v;
  else
    ((float*)p)[i] = (float)v;
}

void check_dtype(int32_t dt) { HX_REQUIRE(dt == HX_F32 || dt == HX_F64, "dtype must be HX_F32 or HX_F64"); }

// Caller array (len_user entries of width w per item) -> grid FP64 device
// array (len_grid items); map == empty means identity.
void upload(hx_ctx* c, int32_t dt, const void* host, const std::vector<int64_t>& map,
            int64_t n_user, int64_t n_grid, int w, double* dev) {
  if (map.empty()) {
    const size_t cnt = (size_t)n_grid * w;
    if (dt == HX_F64) {
      HX_CUDA(cudaMemcpyAsync(dev, host, cnt * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    } else {
      float* st = (float*)c->d_stage.ensure(cnt * sizeof(float));
      HX_CUDA(cudaMemcpyAsync(st, host, cnt * sizeof(float), cudaMemcpyHostToDevice, c->stream));
      hx::launch_convert<double, float>(c->stream, dev, st, (int64_t)cnt);
    }
    return;
  }
  std::vector<double> tmp((size_t)n_grid * w, 0.0);
  for (int64_t i = 0; i < n_user; ++i)
    for (int k = 0; k < w; ++k) tmp[(size_t)map[i] * w + k] = load_val(dt, host, i * w + k);
  HX_CUDA(cudaMemcpyAsync(dev, tmp.data(), tmp.size() * sizeof(double), cudaMemcpyHostToDevice,
                          c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
}

void download(hx_ctx* c, int32_t dt, const double* dev, const std::vector<int64_t>& map,
              int64_t n_user, int64_t n_grid, int w, void* host) {
  if (map.empty()) {
    const size_t cnt = (size_t)n_grid * w;
    if (dt == HX_F64) {
      HX_CUDA(cudaMemcpyAsync(host, dev, cnt * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    } else {
      float* st = (float*)c->d_stage.ensure(cnt * sizeof(float));
      hx::launch_convert<float, double>(c->stream, st, dev, (int64_t)cnt);
      HX_CUDA(cudaMemcpyAsync(host, st, cnt * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    }
    HX_CUDA(cudaStreamSynchronize(c->stream));
    return;
  }
  std::vector<double> tmp((size_t)n_grid * w);
  HX_CUDA(cudaMemcpyAsync(tmp.data(), dev, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost,
                          c->stream));
  HX_CUDA(cudaStreamSynchronize(c->stream));
  for (int64_t i = 0; i < n_user; ++i)
    for (int k = 0; k < w; ++k) store_val(dt, host, i * w + k, tmp[(size_t)map[i] * w + k]);
}

void up_nodes3(hx_ctx* c, int32_t dt, const void* h, double* d) {
  upload(c, dt, h, c->node_map, c->n_user_nodes, c->g.nodes(), 3, d);
}
void down_nodes3(hx_ctx* c, int32_t dt, const double* d, void* h) {
  download(c, dt, d, c->node_map, c->n_user_nodes, c->g.nodes(), 3, h);
}
void up_elems(hx_ctx* c, int32_t dt, const void* h, double* d, int w = 1) {
  upload(c, dt, h, c->elem_map, c->n_user_elem, c->g.elems(), w, d);
}
void down_elems(hx_ctx* c, int32_t dt, const double* d, void* h, int w = 1) {
  download(c, dt, d, c->elem_map, c->n_user_elem, c->g.elems(), w, h);
}

void need_mesh(const hx_ctx* c) {
  HX_REQUIRE(c->has_mesh, "no mesh: call hx_set_grid or hx_set_mesh first");
}

void need_grid_numbering(hx_ctx* c) {
  need_mesh(c);
  HX_REQUIRE(identity(c), "device-array entry points need a grid mesh (hx_set_grid)");
}

hx_solve_opts sanitize(const hx_solve_opts* o) {
  hx_solve_opts r;
  hx_default_opts(&r);
  if (o) r = *o;
  HX_REQUIRE(r.max_iter >= 0, "max_iter must be >= 0");
  HX_REQUIRE(r.tol > 0 && std::isfinite(r.tol), "tol must be positive");
  HX_REQUIRE(r.shift_factor >= 0 && std::isfinite(r.shift_factor), "shift_factor must be >= 0");
  HX_REQUIRE(r.precision >= HX_PREC_FP64 && r.precision <= HX_PREC_MIXED32,
             "unsupported precision");
  HX_REQUIRE(r.mg_smooth_degree >= 0 && r.mg_smooth_degree <= 8,
             "mg_smooth_degree must be 0 (default) .. 8");
  return r;
}

}  // namespace

extern "C" {

HX_API const char* hx_status_string(int32_t s) {
  switch (s) {
    case HX_OK: return "ok";
    case HX_NOT_CONVERGED: return "not converged";
    case HX_STALLED: return "stalled";
    case HX_BREAKDOWN: return "breakdown";
    case HX_NONFINITE: return "non-finite residual";
    case HX_OOM: return "out of memory";
    case HX_BAD_ARG: return "bad argument";
    case HX_CUDA_ERROR: return "CUDA error";
    case HX_NO_DEVICE: return "no CUDA device";
    case HX_DIVERGED: return "diverged";
    default: return "unknown status";
  }
}

HX_API hx_status hx_get_stream(const hx_ctx* c, void** stream) {
  if (!c || !stream) return HX_BAD_ARG;
  *stream = (void*)c->stream;
  return HX_OK;
}

HX_API int64_t hx_kernel_launches(const hx_ctx* c) { return c ? c->launches : 0; }

HX_API hx_status hx_time_kernel(hx_ctx* c, int32_t kernel, int32_t reps, double* avg_ms) {
  return guard(c, [&] { return hx::time_kernel(c, kernel, reps, avg_ms); });
}

HX_API void hx_default_opts(hx_solve_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->precision = HX_PREC_FP64;
  o->preconditioner = HX_PC_JACOBI;
  o->tol = 1e-6;
  o->max_iter = 40000;  // src/Solvers/GPUSolver.jl:614
  o->shift_factor = 0.0;
  o->inner_tol = 0.1;  // mixed: replace the FP32 residual after a 10x drop
  o->max_refine = 30;
  o->verify_true_residual = 1;
}

HX_API hx_status hx_create(hx_ctx** out, int32_t device) {
  if (!out) return HX_BAD_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return HX_NO_DEVICE;
  }
  if (device < 0 || device >= n) return HX_BAD_ARG;
  hx_ctx* c = new (std::nothrow) hx_ctx();
  if (!c) return HX_OOM;
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_in, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return HX_CUDA_ERROR;
  }
  *out = c;
  return HX_OK;
}

HX_API void hx_destroy(hx_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->h_state) cudaFreeHost(c->h_state);
  for (int i = 0; i < 2; ++i) {
    if (c->net.side[i]) cudaStreamDestroy(c->net.side[i]);
    if (c->net.ev_join[i]) cudaEventDestroy(c->net.ev_join[i]);
    if (c->net.ev_x[i]) cudaEventDestroy(c->net.ev_x[i]);
  }
  if (c->net.ev_fork) cudaEventDestroy(c->net.ev_fork);
  if (c->ev_in) cudaEventDestroy(c->ev_in);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

HX_API const char* hx_last_error(const hx_ctx* c) { return c ? c->err.c_str() : "null context"; }

HX_API hx_status hx_set_grid(hx_ctx* c, int64_t nx, int64_t ny, int64_t nz, double dx, double dy,
                             double dz) {
  return guard(c, [&] {
    set_grid_impl(c, nx, ny, nz, dx, dy, dz);
    return HX_OK;
  });
}

HX_API hx_status hx_set_mesh(hx_ctx* c, const float* nodes, int64_t nN, const int64_t* el,
                             int64_t nE) {
  return guard(c, [&] {
    set_mesh_impl(c, nodes, nN, el, nE);
    return HX_OK;
  });
}

HX_API hx_status hx_set_material(hx_ctx* c, double E, double nu) {
  return guard(c, [&] {
    HX_REQUIRE(E > 0 && std::isfinite(E), "E must be positive");
    HX_REQUIRE(nu > -1.0 && nu < 0.5, "nu must lie in (-1, 0.5)");
    c->E = E;
    c->nu = nu;
    c->K = hx::make_elem_coef(c->h[0], c->h[1], c->h[2], nu);
    return HX_OK;
  });
}

HX_API hx_status hx_set_bc(hx_ctx* c, const float* bc, int64_t nN) {
  return guard(c, [&] {
    need_mesh(c);
    HX_REQUIRE(bc != nullptr, "bc_indicator is null");
    HX_REQUIRE(nN == c->n_user_nodes, "bc_indicator has the wrong number of nodes");
    std::vector<uint8_t> fr(c->g.nodes(), identity(c) ? 7 : 0);
    for (int64_t n = 0; n < nN; ++n) {
      uint8_t m = 0;
      for (int d = 0; d < 3; ++d)
        if (!(bc[d * nN + n] > 0.0f)) m |= (uint8_t)(1u << d);
      fr[identity(c) ? n : c->node_map[n]] = m;
    }
    c->bcfree = std::move(fr);
    c->bc_dirty = true;
    return HX_OK;
  });
}

HX_API hx_status hx_get_grid(const hx_ctx* c, int64_t dims[3], double h[3]) {
  if (!c || !dims || !h) return HX_BAD_ARG;
  if (!c->has_mesh) return HX_BAD_ARG;
  dims[0] = c->g.nxe;
  dims[1] = c->g.nye;
  dims[2] = c->g.nze;
  for (int a = 0; a < 3; ++a) h[a] = c->h[a];
  return HX_OK;
}

HX_API hx_status hx_apply_stiffness(hx_ctx* c, int32_t dt, const void* x, const void* factor,
                                    void* y) {
  return guard(c, [&] {
    need_mesh(c);
    check_dtype(dt);
    HX_REQUIRE(x && factor && y, "null argument");
    hx::ensure_workspace(c);
    const int64_t n = c->g.dofs();
    double* dx_ = c->d_x.ensure(n);
    double* dq = c->d_q.ensure(n);
    double* df = c->d_fac.ensure(c->g.elems());
    up_nodes3(c, dt, x, dx_);
    if (!identity(c)) HX_CUDA(cudaMemsetAsync(df, 0, c->g.elems() * sizeof(double), c->stream));
    up_elems(c, dt, factor, df);
    hx::launch_matvec<double>(c->stream, 0, dx_, dq, df, nullptr, c->g, c->K, 0.0,
                              c->d_state.p + 3, c->d_partials.p, nullptr);
    down_nodes3(c, dt, dq, y);
    return HX_OK;
  });
}

HX_API hx_status hx_diagonal(hx_ctx* c, int32_t dt, const void* factor, void* diag) {
  return guard(c, [&] {
    need_mesh(c);
    check_dtype(dt);
    HX_REQUIRE(factor && diag, "null argument");
    hx::ensure_workspace(c);
    double* df = c->d_fac.ensure(c->g.elems());
    double* dd = c->d_q.ensure(c->g.dofs());
    uint8_t* nm = c->d_nmask.ensure(c->g.nodes());
    up_elems(c, dt, factor, df);
    HX_CUDA(cudaMemsetAsync(c->d_state.p + 3, 0, sizeof(hx::CgState), c->stream));
    hx::launch_node_diag<double>(c->stream, df, nullptr, nm, dd, c->g, c->K, c->d_partials.p,
                                 c->d_state.p + 3, c->d_scalars.p);
    down_nodes3(c, dt, dd, diag);
    return HX_OK;
  });
}

struct EventTimer {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t s;
  explicit EventTimer(cudaStream_t st) : s(st) {
    HX_CUDA(cudaEventCreate(&a));
    HX_CUDA(cudaEventCreate(&b));
    HX_CUDA(cudaEventRecord(a, s));
  }
  double stop() {
    HX_CUDA(cudaEventRecord(b, s));
    HX_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    HX_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms;
  }
  ~EventTimer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

HX_API hx_status hx_solve(hx_ctx* c, int32_t dt, const void* f, const void* factor, void* u,
                          const hx_solve_opts* opts, hx_solve_report* rep) {
  return guard(c, [&] {
    const double t0 = now_ms();
    const int64_t l0 = hx::launch_counter();
    EventTimer ev(c->stream);
    need_mesh(c);
    check_dtype(dt);
    HX_REQUIRE(f && factor && u, "null argument");
    hx_solve_opts o = sanitize(opts);
    hx::ensure_workspace(c);
    const int64_t n = c->g.dofs();
    double* df = c->d_f.ensure(n);
    double* dfac = c->d_fac.ensure(c->g.elems());
    double* du = c->d_x.ensure(n);
    up_nodes3(c, dt, f, df);
    if (!identity(c)) HX_CUDA(cudaMemsetAsync(dfac, 0, c->g.elems() * sizeof(double), c->stream));
    up_elems(c, dt, factor, dfac);
    if (o.warm_start) up_nodes3(c, dt, u, du);
    hx_solve_report R{};
    hx_status s = hx::solve_grid(c, df, dfac, du, o, &R);
    down_nodes3(c, dt, du, u);
    R.time_device_ms = ev.stop();
    R.time_total_ms = now_ms() - t0;
    R.kernel_launches = (double)(hx::launch_counter() - l0);
    if (rep) *rep = R;
    return s;
  });
}

HX_API hx_status hx_solve_device(hx_ctx* c, const double* f, const double* fac, double* u,
                                 const hx_solve_opts* opts, hx_solve_report* rep) {
  return guard(c, [&] {
    need_mesh(c);
    HX_REQUIRE(f && fac && u, "null argument");
    // the vector kernels access u two doubles at a time, the operator stages
    // it in 16-byte chunks
    HX_REQUIRE(((uintptr_t)u & 15u) == 0, "u_dev must be 16-byte aligned");
    hx_solve_opts o = sanitize(opts);
    const int64_t l0 = hx::launch_counter();
    EventTimer ev(c->stream);
    // keep an internal copy of the factors (kernel timing reuses it)
    double* dfac = c->d_fac.ensure(c->g.elems());
    if (dfac != fac)
      HX_CUDA(cudaMemcpyAsync(dfac, fac, c->g.elems() * sizeof(double), cudaMemcpyDeviceToDevice,
                              c->stream));
    hx_solve_report R{};
    hx_status s = hx::solve_grid(c, f, dfac, u, o, &R);
    R.time_device_ms = ev.stop();
    R.kernel_launches = (double)(hx::launch_counter() - l0);
    if (rep) *rep = R;
    return s;
  });
}

// Name of the preconditioner that finished a drop-in solve (the reference
// returns "Jacobi" or "AMG"; the multigrid preconditioner replaces AMG).
static const char* dropin_prec_name(int32_t pc, const hx_solve_report& R) {
  if (R.zero_rhs) return "None";
  if (pc == HX_PC_MULTIGRID) return "GMG";
  if (pc == HX_PC_LEARNED) return R.fallback_used ? "Jacobi" : "Learned";
  return R.fallback_used ? "GMG" : "Jacobi";
}

HX_API hx_status hx_set_dropin_solver(hx_ctx* c, int32_t preconditioner, int32_t precision,
                                      int32_t multigrid_fallback) {
  return guard(c, [&] {
    HX_REQUIRE(preconditioner == HX_PC_JACOBI || preconditioner == HX_PC_LEARNED ||
                   preconditioner == HX_PC_MULTIGRID,
               "drop-in preconditioner must be Jacobi, learned or multigrid");
    HX_REQUIRE(precision == HX_PREC_FP64 || precision == HX_PREC_MIXED32, "unsupported precision");
    c->dropin_pc = preconditioner;
    c->dropin_prec = precision;
    c->dropin_fallback = multigrid_fallback != 0;
    return HX_OK;
  });
}

HX_API hx_status hx_solve_system_gpu(hx_ctx* c, const float* nodes, int64_t nN,
                                     const int64_t* elements, int64_t nE, float E, float nu,
                                     const float* bc_indicator, const float* f,
                                     const float* density, int32_t max_iter, double tol,
                                     float shift_factor, float min_stiffness_threshold,
                                     const float* u_guess, float* x_full, double* final_rel_res,
                                     char* prec_name, int32_t prec_name_cap) {
  return guard(c, [&] {
    HX_REQUIRE(nodes && elements && bc_indicator && f && density && x_full,
               "null argument");
    set_mesh_impl(c, nodes, nN, elements, nE);
    HX_REQUIRE(E > 0 && nu > -1 && nu < 0.5, "bad material");
    c->E = E;
    c->nu = nu;
    c->K = hx::make_elem_coef(c->h[0], c->h[1], c->h[2], nu);
    // bc
    {
      std::vector<uint8_t> fr(c->g.nodes(), identity(c) ? 7 : 0);
      for (int64_t n = 0; n < nN; ++n) {
        uint8_t m = 0;
        for (int d = 0; d < 3; ++d)
          if (!(bc_indicator[d * nN + n] > 0.0f)) m |= (uint8_t)(1u << d);
        fr[identity(c) ? n : c->node_map[n]] = m;
      }
      c->bcfree = std::move(fr);
      c->bc_dirty = true;
    }
    // active elements and factors (src/Solvers/GPUSolver.jl:128,147)
    std::vector<float> fac(nE);
    int64_t nact = 0;
    for (int64_t e = 0; e < nE; ++e) {
      const bool act = density[e] >= min_stiffness_threshold;
      fac[e] = act ? E * density[e] : 0.0f;
      nact += act;
    }
    HX_REQUIRE(nact > 0, "no active elements (threshold too high)");
    hx_solve_opts o;
    hx_default_opts(&o);
    o.tol = tol;
    o.max_iter = max_iter;
    o.shift_factor = shift_factor;
    o.warm_start = u_guess != nullptr;
    o.ref_retry = 1;
    o.keep_best = 1;
    o.divergence_checks = 1;
    // hx_set_dropin_solver; by default the reference's "jacobi_amg"
    // (configs/default.yaml:191): multigrid takes over from a failed Jacobi
    // attempt
    o.preconditioner = c->dropin_pc;
    o.precision = c->dropin_prec;
    o.multigrid_fallback = c->dropin_fallback;
    std::vector<float> u(3 * nN, 0.0f);
    if (u_guess) std::memcpy(u.data(), u_guess, u.size() * sizeof(float));
    hx_solve_report R{};
    hx::ensure_workspace(c);
    const int64_t n = c->g.dofs();
    double* df = c->d_f.ensure(n);
    double* dfac = c->d_fac.ensure(c->g.elems());
    double* du = c->d_x.ensure(n);
    up_nodes3(c, HX_F32, f, df);
    if (!identity(c)) HX_CUDA(cudaMemsetAsync(dfac, 0, c->g.elems() * sizeof(double), c->stream));
    up_elems(c, HX_F32, fac.data(), dfac);
    if (o.warm_start) up_nodes3(c, HX_F32, u.data(), du);
    hx_status s = hx::solve_grid(c, df, dfac, du, o, &R);
    down_nodes3(c, HX_F32, du, x_full);
    if (final_rel_res) *final_rel_res = R.rel_res;
    if (prec_name && prec_name_cap > 0) {
      const char* nm = dropin_prec_name(c->dropin_pc, R);
      std::strncpy(prec_name, nm, (size_t)prec_name_cap - 1);
      prec_name[prec_name_cap - 1] = '\0';
    }
    // The reference warns and returns its best iterate when every attempt
    // fails; the status carries that outcome here.
    return s;
  });
}

HX_API hx_status hx_solve_system_grid(hx_ctx* c, int64_t nx, int64_t ny, int64_t nz, double dx,
                                      double dy, double dz, float E, float nu,
                                      const float* bc_indicator, const float* f,
                                      const float* density, int32_t max_iter, double tol,
                                      float shift_factor, float min_stiffness_threshold,
                                      const float* u_guess, float* x_full,
                                      double* final_rel_res, char* prec_name,
                                      int32_t prec_name_cap) {
  return guard(c, [&] {
    HX_REQUIRE(bc_indicator && f && density && x_full, "null argument");
    HX_REQUIRE(E > 0 && nu > -1 && nu < 0.5, "bad material");
    set_grid_impl(c, nx, ny, nz, dx, dy, dz);
    c->E = E;
    c->nu = nu;
    c->K = hx::make_elem_coef(c->h[0], c->h[1], c->h[2], nu);
    hx::ensure_workspace(c);
    const int64_t nn = c->g.nodes(), ne = c->g.elems(), n = c->g.dofs();
    // every per-element and per-node step on the device: the host only copies
    float* st = (float*)c->d_stage.ensure(std::max<int64_t>(3 * nn, ne) * sizeof(float));
    HX_CUDA(cudaMemcpyAsync(st, bc_indicator, 3 * nn * sizeof(float), cudaMemcpyHostToDevice,
                            c->stream));
    hx::launch_bc_bits(c->stream, st, c->d_bcfree.ensure(nn), nn);
    c->bc_dirty = false;  // the device mask is current; the host copy is not used
    double* dfac = c->d_fac.ensure(ne);
    HX_CUDA(cudaMemcpyAsync(st, density, ne * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    hx::launch_threshold_factor(c->stream, st, min_stiffness_threshold, E, dfac, ne);
    double* df = c->d_f.ensure(n);
    double* du = c->d_x.ensure(n);
    HX_CUDA(cudaMemcpyAsync(st, f, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    hx::launch_convert<double, float>(c->stream, df, st, n);
    if (u_guess) {
      HX_CUDA(cudaMemcpyAsync(st, u_guess, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
      hx::launch_convert<double, float>(c->stream, du, st, n);
    }
    hx_solve_opts o;
    hx_default_opts(&o);
    o.tol = tol;
    o.max_iter = max_iter;
    o.shift_factor = shift_factor;
    o.warm_start = u_guess != nullptr;
    o.ref_retry = 1;
    o.keep_best = 1;
    o.divergence_checks = 1;
    // hx_set_dropin_solver; by default the reference's "jacobi_amg"
    // (configs/default.yaml:191): multigrid takes over from a failed Jacobi
    // attempt
    o.preconditioner = c->dropin_pc;
    o.precision = c->dropin_prec;
    o.multigrid_fallback = c->dropin_fallback;
    hx_solve_report R{};
    hx_status s = hx::solve_grid(c, df, dfac, du, o, &R);
    float* so = (float*)c->d_stage.ensure(n * sizeof(float));
    hx::launch_convert<float, double>(c->stream, so, du, n);
    HX_CUDA(cudaMemcpyAsync(x_full, so, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    HX_CUDA(cudaStreamSynchronize(c->stream));
    if (final_rel_res) *final_rel_res = R.rel_res;
    if (prec_name && prec_name_cap > 0) {
      const char* nm = dropin_prec_name(c->dropin_pc, R);
      std::strncpy(prec_name, nm, (size_t)prec_name_cap - 1);
      prec_name[prec_name_cap - 1] = '\0';
    }
    return s;
  });
}

HX_API hx_status hx_export_webdata(hx_ctx* c, const char* path, int32_t dt, const void* density,
                                   const void* l1, const void* principal, float threshold,
                                   int32_t iter, float radius, const char* json, int64_t json_len,
                                   int64_t* count) {
  return guard(c, [&] {
    need_mesh(c);
    check_dtype(dt);
    HX_REQUIRE(density && l1 && principal, "null argument");
    HX_REQUIRE(identity(c), "the export needs the mesh in grid numbering (generate_mesh order)");
    hx::ensure_workspace(c);
    const int64_t ne = c->g.elems();
    double* dd = c->d_aux0.ensure(ne);
    double* dl = c->d_aux1.ensure(ne);
    double* dp = c->d_aux2.ensure(3 * ne);
    up_elems(c, dt, density, dd);
    up_elems(c, dt, l1, dl);
    up_elems(c, dt, principal, dp, 3);
    return hx::export_webdata<double>(c, path, dd, dl, dp, threshold, iter, radius, json,
                                      json_len, count);
  });
}

HX_API hx_status hx_export_webdata_device(hx_ctx* c, const char* path, const double* density,
                                          const double* l1, const double* principal,
                                          float threshold, int32_t iter, float radius,
                                          const char* json, int64_t json_len, int64_t* count) {
  return guard(c, [&] {
    need_grid_numbering(c);
    HX_REQUIRE(density && l1 && principal, "null argument");
    return hx::export_webdata<double>(c, path, density, l1, principal, threshold, iter, radius,
                                      json, json_len, count);
  });
}

HX_API hx_status hx_filter(hx_ctx* c, int32_t dt, const void* rho, void* out, double radius,
                           int32_t ref_compat, double tol, int32_t max_iter,
                           hx_solve_report* rep) {
  return guard(c, [&] {
    need_mesh(c);
    check_dtype(dt);
    HX_REQUIRE(rho && out, "null argument");
    hx::ensure_workspace(c);
    const int64_t ne = c->g.elems();
    double* drho = c->f_rho.ensure(ne);
    double* dout = c->f_out.ensure(ne);
    if (!identity(c)) HX_CUDA(cudaMemsetAsync(drho, 0, ne * sizeof(double), c->stream));
    up_elems(c, dt, rho, drho);
    hx_status s = hx::filter_grid(c, c->g, c->h, drho, dout, radius, ref_compat, tol, max_iter,
                                  rep);
    down_elems(c, dt, dout, out);
    return s;
  });
}

HX_API hx_status hx_filter_device(hx_ctx* c, const double* rho, double* out, double radius,
                                  int32_t ref_compat, double tol, int32_t max_iter,
                                  hx_solve_report* rep) {
  return guard(c, [&] {
    need_mesh(c);
    HX_REQUIRE(rho && out, "null argument");
    return hx::filter_grid(c, c->g, c->h, rho, out, radius, ref_compat, tol, max_iter, rep);
  });
}

HX_API hx_status hx_apply_gpu_filter(hx_ctx* c, const float* density, int64_t nx, int64_t ny,
                                     int64_t nz, double dx, double dy, double dz, double radius,
                                     double tol, int32_t ref_compat, float* filtered,
                                     double* time_s, int32_t* iters, double* res) {
  return guard(c, [&] {
    HX_REQUIRE(density && filtered, "null argument");
    HX_REQUIRE(nx >= 1 && ny >= 1 && nz >= 1 && dx > 0 && dy > 0 && dz > 0, "bad grid");
    HX_REQUIRE(hx::grid_extent_ok(nx, ny, nz), "grid too large");
    Grid g{};
    g.nxe = (int)nx;
    g.nye = (int)ny;
    g.nze = (int)nz;
    g.nxn = g.nxe + 1;
    g.nyn = g.nye + 1;
    g.nzn = g.nze + 1;
    const double h[3] = {dx, dy, dz};
    hx::ensure_workspace(c);
    const int64_t ne = g.elems();
    double* drho = c->f_rho.ensure(ne);
    double* dout = c->f_out.ensure(ne);
    {
      float* st = (float*)c->d_stage.ensure(ne * sizeof(float));
      HX_CUDA(cudaMemcpyAsync(st, density, ne * sizeof(float), cudaMemcpyHostToDevice, c->stream));
      hx::launch_convert<double, float>(c->stream, drho, st, ne);
    }
    hx_solve_report R{};
    hx_status s = hx::filter_grid(c, g, h, drho, dout, radius, ref_compat, tol, 200, &R);
    {
      float* st = (float*)c->d_stage.ensure(ne * sizeof(float));
      hx::launch_convert<float, double>(c->stream, st, dout, ne);
      HX_CUDA(cudaMemcpyAsync(filtered, st, ne * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
      HX_CUDA(cudaStreamSynchronize(c->stream));
    }
    if (time_s) *time_s = R.time_solve_ms / 1000.0;
    if (iters) *iters = R.iterations;
    if (res) *res = R.rel_res;
    return s;
  });
}

HX_API hx_status hx_stress(hx_ctx* c, int32_t dt, const void* u, const void* density, double E,
                           double nu, void* principal, void* vm, void* voigt, void* l1,
                           void* dir) {
  return guard(c, [&] {
    need_mesh(c);
    check_dtype(dt);
    HX_REQUIRE(u && density && principal && vm && voigt && l1 && dir, "null argument");
    hx::ensure_workspace(c);
    const int64_t ne = c->g.elems(), n = c->g.dofs();
    double* du = c->d_x.ensure(n);
    double* dd = c->d_fac.ensure(ne);
    double* pr = c->d_aux0.ensure(3 * ne);
    double* vmv = c->d_aux1.ensure(ne);
    double* vo = c->d_aux2.ensure(6 * ne);
    double* l1v = c->d_aux3.ensure(ne);
    double* dv = c->d_aux4.ensure(3 * ne);
    up_nodes3(c, dt, u, du);
    if (!identity(c)) HX_CUDA(cudaMemsetAsync(dd, 0, ne * sizeof(double), c->stream));
    up_elems(c, dt, density, dd);
    hx::launch_stress(c->stream, du, dd, E, nu, c->g, c->h[0], c->h[1], c->h[2], pr, vmv, vo,
                      l1v, dv);
    down_elems(c, dt, pr, principal, 3);
    down_elems(c, dt, vmv, vm);
    down_elems(c, dt, vo, voigt, 6);
    down_elems(c, dt, l1v, l1);
    down_elems(c, dt, dv, dir, 3);
    return HX_OK;
  });
}

HX_API hx_status hx_stress_pnorm(hx_ctx* c, int32_t dt, const void* u, const void* density,
                                 double E, double nu, double P, double* pnorm, double* vmax) {
  return guard(c, [&] {
    need_mesh(c);
    check_dtype(dt);
    HX_REQUIRE(u && density && pnorm, "null argument");
    HX_REQUIRE(P >= 1.0 && std::isfinite(P), "P must be >= 1");
    hx::ensure_workspace(c);
    const int64_t ne = c->g.elems(), n = c->g.dofs();
    double* du = c->d_x.ensure(n);
    double* dd = c->d_fac.ensure(ne);
    double* pr = c->d_aux0.ensure(3 * ne);
    double* vmv = c->d_aux1.ensure(ne);
    double* vo = c->d_aux2.ensure(6 * ne);
    double* l1v = c->d_aux3.ensure(ne);
    double* dv = c->d_aux4.ensure(3 * ne);
    up_nodes3(c, dt, u, du);
    if (!identity(c)) HX_CUDA(cudaMemsetAsync(dd, 0, ne * sizeof(double), c->stream));
    up_elems(c, dt, density, dd);
    hx::launch_stress(c->stream, du, dd, E, nu, c->g, c->h[0], c->h[1], c->h[2], pr, vmv, vo,
                      l1v, dv);
    hx::put_state(c, 3, hx::CgState{});
    hx::launch_pnorm(c->stream, vmv, ne, P, c->d_state.p + 3, c->d_partials.p);
    const hx::CgState st = hx::get_state(c, 3);
    *pnorm = st.aux[0] > 0.0 ? st.aux[0] * std::pow(st.aux[1], 1.0 / P) : 0.0;
    if (vmax) *vmax = st.aux[0];
    return HX_OK;
  });
}

HX_API hx_status hx_compute_stress_field(hx_ctx* c, const float* nodes, int64_t nN,
                                         const int64_t* elements, int64_t nE, const float* U,
                                         float E, float nu, const float* density,
                                         float* principal, float* vm, float* voigt, float* l1,
                                         float* dir) {
  hx_status s = hx_set_mesh(c, nodes, nN, elements, nE);
  if (s != HX_OK) return s;
  return hx_stress(c, HX_F32, U, density, E, nu, principal, vm, voigt, l1, dir);
}

HX_API hx_status hx_compliance(hx_ctx* c, int32_t dt, const void* f, const void* u, double* out) {
  return guard(c, [&] {
    need_mesh(c);
    check_dtype(dt);
    HX_REQUIRE(f && u && out, "null argument");
    hx::ensure_workspace(c);
    const int64_t n = c->g.dofs();
    double* a = c->d_f.ensure(n);
    double* b = c->d_x.ensure(n);
    up_nodes3(c, dt, f, a);
    up_nodes3(c, dt, u, b);
    HX_CUDA(cudaMemsetAsync(c->d_state.p + 3, 0, sizeof(hx::CgState), c->stream));
    hx::launch_dot(c->stream, a, b, n, c->d_state.p + 3, c->d_partials.p, c->d_scalars.p);
    HX_CUDA(cudaMemcpyAsync(out, c->d_scalars.p, sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    HX_CUDA(cudaStreamSynchronize(c->stream));
    return HX_OK;
  });
}

HX_API hx_status hx_element_energy(hx_ctx* c, int32_t dt, const void* u, void* ce) {
  return guard(c, [&] {
    need_mesh(c);
    check_dtype(dt);
    HX_REQUIRE(u && ce, "null argument");
    hx::ensure_workspace(c);
    const int64_t n = c->g.dofs(), ne = c->g.elems();
    double* du = c->d_x.ensure(n);
    double* de = c->d_aux1.ensure(ne);
    up_nodes3(c, dt, u, du);
    hx::launch_energy(c->stream, du, c->g, c->K, de);
    down_elems(c, dt, de, ce);
    return HX_OK;
  });
}

HX_API hx_status hx_oc_update(hx_ctx* c, int32_t dt, const void* x, const void* dc,
                              const void* dv, double volfrac, double move, void* xnew,
                              double* lambda, int32_t* steps) {
  return guard(c, [&] {
    need_mesh(c);
    check_dtype(dt);
    HX_REQUIRE(x && dc && dv && xnew, "null argument");
    HX_REQUIRE(volfrac > 0 && volfrac <= 1, "volfrac must lie in (0, 1]");
    HX_REQUIRE(move > 0, "move must be positive");
    hx::ensure_workspace(c);
    const int64_t ne = c->n_user_elem;
    double* dx_ = c->d_aux0.ensure(ne);
    double* ddc = c->d_aux1.ensure(ne);
    double* ddv = c->d_aux2.ensure(ne);
    double* dxn = c->d_aux3.ensure(ne);
    static const std::vector<int64_t> none;
    upload(c, dt, x, none, ne, ne, 1, dx_);
    upload(c, dt, dc, none, ne, ne, 1, ddc);
    upload(c, dt, dv, none, ne, ne, 1, ddv);
    hx::CgState s{};
    s.aux[0] = 0.0;
    s.aux[1] = 1e9;
    s.status = hx::HX_RUNNING;
    c->h_state[3] = s;
    HX_CUDA(cudaMemcpyAsync(c->d_state.p + 3, c->h_state + 3, sizeof(s), cudaMemcpyHostToDevice,
                            c->stream));
    hx::launch_oc(c->stream, dx_, ddc, ddv, ne, volfrac, move, dxn, c->d_state.p + 3,
                  c->d_partials.p, 100);
    HX_CUDA(cudaMemcpyAsync(c->h_state + 3, c->d_state.p + 3, sizeof(s), cudaMemcpyDeviceToHost,
                            c->stream));
    download(c, dt, dxn, none, ne, ne, 1, xnew);
    if (lambda) *lambda = c->h_state[3].aux[2];
    if (steps) *steps = c->h_state[3].iter;
    return HX_OK;
  });
}

HX_API void hx_default_update_params(hx_update_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->h[0] = p->h[1] = p->h[2] = 1.0;
  p->filter_tolerance = 1e-5;             // src/Optimization/TopOpt.jl:169
  p->filter_R_interm_iter_perc = 50.0;    // :220
  p->final_density_threshold = 0.95;      // :351
  p->max_culling_ratio = 0.1;             // :352
  p->mode = HX_UPDATE_STRESS_RATIO;
  p->oc_volfrac = 0.3;
  p->oc_move = 0.2;
}

HX_API hx_status hx_update_density(hx_ctx* c, float* density, float* l1,
                                   const uint8_t* prot, float E, float allow, int32_t iter,
                                   int32_t n_iter, const float* orig, float min_d, float max_d,
                                   const hx_update_params* params, const float* dc,
                                   float* filtered_out, hx_update_result* result) {
  return guard(c, [&] {
    HX_REQUIRE(params != nullptr, "params is null");
    return hx::update_density(c, density, l1, prot, E, allow, iter, n_iter, orig, min_d, max_d,
                              *params, dc, filtered_out, result);
  });
}

// ---- device-resident pieces of the optimisation loop (grid numbering) ----

HX_API hx_status hx_simp_device(hx_ctx* c, const double* rho, double p, double e0, double emin,
                                double* fac) {
  return guard(c, [&] {
    need_grid_numbering(c);
    HX_REQUIRE(rho && fac, "null argument");
    HX_REQUIRE(p >= 1.0 && e0 > emin && emin >= 0.0, "bad SIMP parameters");
    hx::launch_simp(c->stream, rho, p, e0, emin, fac, c->g.elems(), false);
    HX_CUDA(cudaStreamSynchronize(c->stream));
    return HX_OK;
  });
}

HX_API hx_status hx_sensitivity_device(hx_ctx* c, const double* rho, const double* u, double p,
                                       double e0, double emin, double* dc) {
  return guard(c, [&] {
    need_grid_numbering(c);
    HX_REQUIRE(rho && u && dc, "null argument");
    HX_REQUIRE(p >= 1.0 && e0 > emin && emin >= 0.0, "bad SIMP parameters");
    hx::launch_energy(c->stream, u, c->g, c->K, dc);
    hx::launch_simp(c->stream, rho, p, e0, emin, dc, c->g.elems(), true);
    HX_CUDA(cudaStreamSynchronize(c->stream));
    return HX_OK;
  });
}

HX_API hx_status hx_compliance_device(hx_ctx* c, const double* f, const double* u, double* out) {
  return guard(c, [&] {
    need_grid_numbering(c);
    HX_REQUIRE(f && u && out, "null argument");
    hx::ensure_workspace(c);
    hx::put_state(c, 3, hx::CgState{});
    hx::launch_dot(c->stream, f, u, c->g.dofs(), c->d_state.p + 3, c->d_partials.p,
                   c->d_scalars.p);
    HX_CUDA(cudaMemcpyAsync(out, c->d_scalars.p, sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    HX_CUDA(cudaStreamSynchronize(c->stream));
    return HX_OK;
  });
}

HX_API hx_status hx_oc_update_device(hx_ctx* c, const double* x, const double* dc,
                                     const double* dv, double volfrac, double move, double* xnew,
                                     double* lambda, int32_t* steps) {
  return guard(c, [&] {
    need_grid_numbering(c);
    HX_REQUIRE(x && dc && xnew, "null argument");
    HX_REQUIRE(volfrac > 0 && volfrac <= 1, "volfrac must lie in (0, 1]");
    HX_REQUIRE(move > 0, "move must be positive");
    hx::ensure_workspace(c);
    hx::CgState s{};
    s.aux[0] = 0.0;
    s.aux[1] = 1e9;
    s.status = hx::HX_RUNNING;
    hx::put_state(c, 3, s);
    hx::launch_oc(c->stream, x, dc, dv, c->g.elems(), volfrac, move, xnew, c->d_state.p + 3,
                  c->d_partials.p, 100);
    const hx::CgState r = hx::get_state(c, 3);
    if (lambda) *lambda = r.aux[2];
    if (steps) *steps = r.iter;
    return HX_OK;
  });
}

HX_API hx_status hx_net_init(hx_ctx* c, uint64_t seed) {
  return guard(c, [&] {
    hx::net_init(c, seed);
    return HX_OK;
  });
}

HX_API hx_status hx_net_set_params(hx_ctx* c, const float* params) {
  return guard(c, [&] {
    HX_REQUIRE(params, "null argument");
    hx::net_set_params(c, params);
    return HX_OK;
  });
}

HX_API hx_status hx_net_get_params(hx_ctx* c, float* params) {
  return guard(c, [&] {
    HX_REQUIRE(params, "null argument");
    hx::net_get_params(c, params);
    return HX_OK;
  });
}

HX_API hx_status hx_net_forward_backward(hx_ctx* c, int32_t nx, int32_t ny, int32_t nz,
                                         const float* x0, const float* dy, float* y,
                                         float* grads) {
  return guard(c, [&] {
    HX_REQUIRE(x0 && dy && y && grads, "null argument");
    hx::net_forward_backward(c, nx, ny, nz, x0, dy, y, grads);
    return HX_OK;
  });
}

HX_API hx_status hx_net_prepare(hx_ctx* c, const double* fac) {
  return guard(c, [&] {
    need_mesh(c);
    HX_REQUIRE(fac, "null argument");
    hx::ensure_workspace(c);
    if (c->bc_dirty) hx::upload_bc(c);
    double shift = 0;
    hx::jacobi_setup_public(c, fac, 0.0, &shift);
    hx::net_prepare(c, fac);
    HX_CUDA(cudaStreamSynchronize(c->stream));
    return HX_OK;
  });
}

HX_API hx_status hx_selftest_wait_timeout(hx_ctx* c, int32_t* detected) {
  return guard(c, [&] {
    HX_REQUIRE(detected != nullptr, "null argument");
    *detected = hx::conv_wait_selftest(c) ? 1 : 0;
    return HX_OK;
  });
}

HX_API hx_status hx_net_apply(hx_ctx* c, const double* r, double* z) {
  return guard(c, [&] {
    need_mesh(c);
    HX_REQUIRE(r && z, "null argument");
    hx::net_apply_vec(c, r, z);
    return HX_OK;
  });
}

HX_API hx_status hx_gmg_apply(hx_ctx* c, const double* r, double* z) {
  return guard(c, [&] {
    need_mesh(c);
    HX_REQUIRE(r && z, "null argument");
    HX_REQUIRE(c->gmg.ready && c->gmg.nl > 0 && c->gmg.lv[0].g.nodes() == c->g.nodes(),
               "no multigrid hierarchy for this grid: run a multigrid solve first");
    hx::gmg_vcycle<double>(c, r, z);
    HX_CUDA(cudaStreamSynchronize(c->stream));
    return HX_OK;
  });
}

HX_API hx_status hx_net_train_step(hx_ctx* c, const double* r, const double* e, double lr,
                                   int32_t loss_kind, double* loss) {
  return hx_net_train_batch(c, &r, e ? &e : nullptr, 1, lr, loss_kind, loss);
}

HX_API hx_status hx_net_train_batch(hx_ctx* c, const double* const* r, const double* const* e,
                                    int32_t count, double lr, int32_t loss_kind, double* loss) {
  return guard(c, [&] {
    need_mesh(c);
    HX_REQUIRE(r != nullptr && count >= 1, "null argument or empty batch");
    for (int i = 0; i < count; ++i) HX_REQUIRE(r[i] != nullptr, "null residual");
    HX_REQUIRE(lr > 0, "lr must be positive");
    HX_REQUIRE(loss_kind == 0 || loss_kind == 1, "loss_kind must be 0 or 1");
    if (loss_kind == 0) {
      HX_REQUIRE(e != nullptr, "the energy loss needs the errors");
      for (int i = 0; i < count; ++i) HX_REQUIRE(e[i] != nullptr, "null error");
    }
    const double l = hx::net_train_step(c, r, e, count, lr, loss_kind);
    if (loss) *loss = l;
    return HX_OK;
  });
}

HX_API hx_status hx_pcg_snapshots(hx_ctx* c, const double* f, const double* fac, int32_t every,
                                  int32_t count, double tol, double* snaps, int32_t* taken) {
  return guard(c, [&] {
    need_mesh(c);
    HX_REQUIRE(f && fac && snaps && count >= 1 && tol > 0, "bad argument");
    const int t = hx::pcg_snapshots(c, f, fac, every, count, tol, snaps);
    if (taken) *taken = t;
    return HX_OK;
  });
}

HX_API hx_status hx_residual_device(hx_ctx* c, const double* f, const double* fac,
                                    const double* x, double* r) {
  return guard(c, [&] {
    need_mesh(c);
    HX_REQUIRE(f && fac && x && r, "null argument");
    HX_REQUIRE(((uintptr_t)x & 7u) == 0, "x_dev must be 8-byte aligned");
    hx::ensure_workspace(c);
    if (c->bc_dirty) hx::upload_bc(c);
    const int64_t n = c->g.dofs();
    // the operator stages x in 16-byte chunks: an x that is only 8-byte
    // aligned (a row of a snapshot matrix with an odd row length) is copied
    if (((uintptr_t)x & 15u) != 0) {
      double* xa = c->d_aux3.ensure(n);
      HX_CUDA(cudaMemcpyAsync(xa, x, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
      x = xa;
    }
    double shift = 0;
    hx::jacobi_setup_public(c, fac, 0.0, &shift);
    double* q = c->d_q.ensure(n);
    hx::launch_matvec<double>(c->stream, 0, x, q, fac, c->d_nmask.p, c->g, c->K, 0.0,
                              c->d_state.p + 3, c->d_partials.p, nullptr);
    double* b = c->d_b.ensure(n);
    hx::launch_mask_rhs<double>(c->stream, f, c->d_minv.p, b, n);
    hx::launch_axpby(c->stream, r, b, q, n);
    HX_CUDA(cudaStreamSynchronize(c->stream));
    return HX_OK;
  });
}

}  // extern "C"
