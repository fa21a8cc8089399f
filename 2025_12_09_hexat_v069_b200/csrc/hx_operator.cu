// hx_operator.cu -- structured-grid Hex8 stiffness operator K(f) x, alone or
// fused with the CG direction/solution updates.
//
// Layout in HBM: node n = i + NXn*(j + NYn*k) (i fastest, src/Mesh/Mesh.jl:
// 13-15), vectors interleaved 3 per node (dof = 3n + c), element
// e = i + NXe*(j + NYe*k) (the element loop of Mesh.jl:44-55), one factor
// per element, one byte of free-DOF bits per node.
//
// Kernel design (replaces the one-thread-per-element, 24-atomics kernel of
// src/Solvers/GPUSolver.jl:37-79 and the broadcast kernels around it):
//  * a CTA owns a 31 x (BY-1) column of output nodes and marches along z
//    over a chunk of node planes; its 32 x BY threads each own one element
//    column, recomputing the one-element halo in x and y (atomic-free and
//    deterministic);
//  * node planes (tile + one-node halo) are staged into shared memory with
//    cp.async into a ring of PF+1 slots: planes k+3 .. k+PF are in flight
//    while plane k+2 is transformed in place and planes k, k+1 feed the
//    element products (PF = mv_prefetch<T>, planes requested ahead);
//  * the element product runs in the per-axis sum/difference (Haar) basis
//    (45 nonzeros, see hx_common.cuh), one displacement component at a
//    time to bound register pressure; the top-face outputs are carried in
//    the Haar domain until the layer above adds its bottom face;
//  * the four element columns around a node are summed with one warp
//    shuffle (x) and one shared-memory exchange (y);
//  * FUSED (the PCG step): the staged plane holds p_old, r, M^-1 and x
//    (the FCG step: p_old, z and x); the in-place transform forms
//    p = M^-1 r + beta p_old (p = z + beta p_old), and for owned nodes
//    stores p and updates x += alpha_old p_old.  p ping-pongs between two
//    buffers so neighbouring CTAs never read a value another CTA rewrote.
//    The epilogue applies the free-DOF mask and the shift and reduces p.q
//    deterministically into the CG state (alpha = rz / pq).
#include <type_traits>

#include "hx_internal.h"

namespace hx {

namespace {

constexpr int MV_BX = 32;
constexpr int MV_BY = 8;
// CTAs per SM (the __launch_bounds__ minimum): FP32 instantiations fit 80
// registers and three CTAs' rings in shared memory (3% faster than two at
// C1); FP64 ones need 128 registers.
template <typename T>
constexpr int mv_resident() { return sizeof(T) == 4 ? 3 : 2; }

// Planes requested ahead of the layer being computed (>= 3).  A deeper ring
// keeps more bytes in flight per SM: FP32 runs 2% faster at depth 5 than 3
// at 320x160x160; the FP64 fused ring at depth 4 (106 KB) drops to one CTA
// per SM and runs 50% slower, so FP64 stays at 3.
#ifndef HX_PF32
#define HX_PF32 5
#endif
#ifndef HX_PF64
#define HX_PF64 3
#endif
template <typename T>
constexpr int mv_prefetch() { return sizeof(T) == 4 ? HX_PF32 : HX_PF64; }

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

// 16-byte asynchronous copy global -> shared; only the first `bytes`
// (0..16) are read, the rest of the 16 are zero-filled.
__device__ __forceinline__ void cp_async16(unsigned sdst, const void* gsrc, unsigned bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sdst), "l"(gsrc),
               "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Staging geometry.  A staged row is the 33 nodes i0-1 .. i0+31 of one
// node row, 99 contiguous values of an interleaved vector.  It is copied in
// 16-byte chunks (V values) starting at the 16-byte boundary at or below its
// first value, so a row takes CPR chunks and sits in shared memory with a
// lead of (first value's index) mod V values, which depends on the row and
// the plane.  Lanes then read node a, component c of row b at
// b*RS + lead_b + 3a + c: a stride of 3 words (FP32) or 3 doublewords
// (FP64) across a warp, free of bank conflicts.
template <typename T>
struct Stage {
  static constexpr int V = 16 / (int)sizeof(T);                // values per chunk
  static constexpr int ROWV = 3 * (MV_BX + 1);                 // 99 values per row
  static constexpr int CPR = (ROWV + V - 1 + V - 1) / V;       // chunks per row
  static constexpr int RS = CPR * V;                           // row stride (values)
  static_assert(RS >= ROWV + V - 1, "a row with any lead fits its staged chunks");
};

// Shared-memory layout (dynamic): rows of interleaved values (see Stage).
template <typename T, int BY, bool FUSED>
struct OpSmem {
  static constexpr int PLANE = (BY + 1) * Stage<T>::RS;
  static_assert((PLANE * sizeof(T)) % 16 == 0, "planes keep 16-byte chunk alignment");
  static constexpr int PF = mv_prefetch<T>();
  static constexpr int NP = PF + 1;             // slots: k, k+1, k+2, k+3 .. k+PF
  static constexpr int NR = FUSED ? PF - 1 : 1;  // slots: k+2 .. k+PF
  static_assert(PF >= 3, "the ring needs planes k .. k+3");
  T p[NP][PLANE];   // x or p
  T r[NR][PLANE];   // r (FUSED)
  T m[NR][PLANE];   // M^-1, or z in MODE 4 (FUSED)
  T x[NR][PLANE];   // x (FUSED)
  T red[BY][3][MV_BX];  // y-direction partials
};

template <typename T>
struct OpArgs {
  const T* pin;   // vector to multiply (MODE 0-2) or p_old (FUSED)
  const T* r;     // MODE 3: residual; MODE 5, 6: right-hand side b
  const T* minv;  // MODE 3, 5: Jacobi inverse diagonal; MODE 4: preconditioned z
  T* x;           // FUSED: solution (x += alpha_old p_old on owned nodes); MODE 5:
                  // x_prev in, x_new out
  T* pout;        // FUSED: new direction p
  T* q;           // output K p (masked, shifted)
  const T* fac;
  const uint8_t* nmask;
  Grid g;
  int kchunk;
  ElemCoef<T> K;
  T shift;
  T omega, gamma;  // MODE 5: recurrence coefficients
  int xprev_zero;  // MODE 5: x_prev = 0 (not read)
  CgState* st;
  double* partials;
  double* out;
};

// 2D sum/difference transform of a node-plane face: v = corners (bx + 2by)
// -> P = coefficients (sigma_x + 2 sigma_y).
template <typename T>
__device__ __forceinline__ void face_fwd(const T (&v)[4], T (&P)[4]) {
  const T e0s = v[0] + v[1], e0d = v[1] - v[0], e1s = v[2] + v[3], e1d = v[3] - v[2];
  P[0] = e0s + e1s;
  P[1] = e0d + e1d;
  P[2] = e1s - e0s;
  P[3] = e1d - e0d;
}

// Component C of f * Lambda U: the diagonal part plus the couplings with
// the other two components (see haar_apply in hx_common.cuh).
template <typename T, int C>
__device__ __forceinline__ void lambda_row(const ElemCoef<T>& K, const T (&U)[3][8], T (&Y)[8]) {
  Y[0] = T(0);
#pragma unroll
  for (int s = 1; s < 8; ++s) Y[s] = K.dg[C][s] * U[C][s];
#pragma unroll
  for (int t = 1; t <= 2; ++t) {
    const int o = (C + t) % 3;
    const int k = 3 - C - o;
#pragma unroll
    for (int sk = 0; sk < 2; ++sk) {
      const int P = (1 << o) | (sk << k);  // sigma_C = s, sigma_o = d
      const int Q = (1 << C) | (sk << k);  // sigma_C = d, sigma_o = s
      Y[Q] += K.lam[k][sk] * U[o][P];
      Y[P] += K.mu[k][sk] * U[o][Q];
    }
  }
}

// MODE 0: q = mask(K x + s x);  MODE 1: also out[0] = x.q;
// MODE 5: Chebyshev step of the multigrid smoother as a three-term
//         recurrence on x: x_new = x + omega (x - x_prev) + gamma M^-1 (b - A x)
//         with A x = mask(K x + s x); x_prev (A.x) is overwritten by x_new
//         (each node's x_prev is read and written by its owner only; the
//         staged x, read by the neighbours, is not written).
// MODE 6: residual r = mask(b - K x - s x) into A.q;
// MODE 2: CG matvec, st->pq = p.q, st->alpha = rz / pq, breakdown test;
// MODE 3: fused PCG step (see file header), then as MODE 2;
// MODE 4: flexible-CG step: p = z + beta p_old (z from a variable
//         preconditioner), x += alpha_old p_old, q = K p; alpha = z.r / p.q
//         with z.r from the preconditioner's output pass (st->aux[3]); p.r
//         = z.r + beta p_old.r and the previous step length makes p_old.r
//         vanish, so r is not staged.
template <typename T, int BY, int MODE, int MINB>
__global__ void __launch_bounds__(MV_BX* BY, MINB) k_struct(OpArgs<T> A) {
  constexpr bool FUSED = MODE == 3 || MODE == 4;
  constexpr bool DOT = MODE >= 1 && MODE <= 4;  // reduces p.q / x.q
  constexpr int NT = MV_BX * BY;
  constexpr int V = Stage<T>::V;
  constexpr int CPR = Stage<T>::CPR;
  constexpr int RS = Stage<T>::RS;
  constexpr int NCH = (BY + 1) * CPR;          // chunks per staged plane
  constexpr int NCT = (NCH + NT - 1) / NT;     // chunks per thread
  constexpr int PF = OpSmem<T, BY, FUSED>::PF;
  constexpr int NP = OpSmem<T, BY, FUSED>::NP;
  constexpr int NR = OpSmem<T, BY, FUSED>::NR;
  using VecT = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  if (MODE >= 2 && MODE <= 4 && A.st->status != HX_RUNNING) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  OpSmem<T, BY, FUSED>& sm = *reinterpret_cast<OpSmem<T, BY, FUSED>*>(smraw);
  const Grid g = A.g;
  const int lx = threadIdx.x, ly = threadIdx.y;
  const int tid = lx + MV_BX * ly;
  const int i0 = blockIdx.x * (MV_BX - 1), j0 = blockIdx.y * (BY - 1);
  const int k0 = blockIdx.z * A.kchunk;
  const int k1 = min(k0 + A.kchunk, g.nzn);
  const int in = i0 - 1 + lx, jn = j0 - 1 + ly;
  const bool col_ok = in >= 0 && jn >= 0 && in < g.nxe && jn < g.nye;
  const bool out_ok = lx >= 1 && ly >= 1 && in < g.nxn && jn < g.nyn;
  const int64_t nplane = (int64_t)g.nxn * g.nyn;
  const int64_t eplane = (int64_t)g.nxe * g.nye;
  const int64_t ndof = 3 * nplane * g.nzn;
  T alpha_old = T(0), beta_old = T(0);
  if (FUSED) {
    alpha_old = (T)A.st->alpha;
    beta_old = (T)A.st->beta;
  }

  // Chunk assignment, the same for every plane: this thread copies (and, in
  // the fused modes, transforms) chunks tid, tid + NT, ... of the plane.
  // row_off = first staged value of the chunk's row, relative to the plane's
  // first value 3 * kp * nplane (32-bit: the grid extent check bounds it);
  // a row's owned nodes i0 .. i0+30 (inside the grid) are the own_len values
  // from row_off + 3; halo rows own none (bit q of own_rows clear).
  int row_off[NCT];
  int cbase[NCT];  // shared-memory offset of the chunk: its row's start + ccv
  int ccv[NCT];    // offset of the chunk within its row (values)
  unsigned own_rows = 0;
  const int own_len = 3 * (min(i0 + MV_BX - 1, g.nxn) - i0);
#pragma unroll
  for (int q = 0; q < NCT; ++q) {
    const int ch = min(tid + q * NT, NCH - 1);
    const int b = ch / CPR, cc = ch - b * CPR;
    const int jj = j0 - 1 + b;
    row_off[q] = 3 * (jj * g.nxn + i0 - 1);
    if (b >= 1 && b <= BY - 1 && jj < g.nyn) own_rows |= 1u << q;
    ccv[q] = cc * V;
    cbase[q] = b * RS + ccv[q];
  }
  // The first staged value of a chunk's row in plane kp has global index
  // o = 3 nplane kp + row_off; the chunk's first value is o rounded down to
  // a multiple of V plus ccv.
  const int64_t P3 = 3 * nplane;

  // One commit group per call, empty for planes past k1, so that the
  // wait counts below hold to the end of the chunk.  Chunks outside the
  // vectors (planes k0-1 < 0 or nzn, rows before the first value) are
  // zero-filled; a chunk reaching past the last value copies only its part
  // inside.  Other values outside the grid (halo nodes beyond a row's end,
  // halo rows beyond the plane) are copied as they lie in memory: they only
  // feed element columns with factor 0, whose products are zero.
  auto issue = [&](int kp, int slp, int slr) {
    if (kp > k1) {
      cp_async_commit();
      return;
    }
    const bool kin = kp >= 0 && kp < g.nzn;
    const unsigned sp = smem_u32(&sm.p[slp][0]);
    const unsigned sr = smem_u32(&sm.r[FUSED ? slr : 0][0]);
    const unsigned smv = smem_u32(&sm.m[FUSED ? slr : 0][0]);
    const unsigned sx = smem_u32(&sm.x[FUSED ? slr : 0][0]);
#pragma unroll
    for (int q = 0; q < NCT; ++q) {
      if (q == NCT - 1 && tid + q * NT >= NCH) continue;
      const int64_t o = (int64_t)kp * P3 + row_off[q];
      const int64_t s = o - (o & (V - 1)) + ccv[q];
      const int64_t left = ndof - s;
      const unsigned bytes =
          (kin && s >= 0 && left > 0) ? (unsigned)((left < V ? left : (int64_t)V) * sizeof(T)) : 0u;
      const int64_t gi = bytes ? s : 0;
      const unsigned so = (unsigned)cbase[q] * (unsigned)sizeof(T);
      cp_async16(sp + so, A.pin + gi, bytes);
      if (FUSED) {
        if (MODE == 3) cp_async16(sr + so, A.r + gi, bytes);
        cp_async16(smv + so, A.minv + gi, bytes);
        cp_async16(sx + so, A.x + gi, bytes);
      }
    }
    cp_async_commit();
  };

  // FUSED: p = M^-1 r + beta p_old (MODE 4: z + beta p_old) in place, chunk
  // by chunk; the values of owned nodes of owned planes are stored to p and
  // advance x with the old direction (16-byte stores where a whole chunk is
  // owned).
  auto transform = [&](int kp, int slp, int slr) {
    if (!FUSED) return;
    const bool kown = kp >= k0 && kp < k1;
    T* ps = &sm.p[slp][0];
    const T* rs = &sm.r[slr][0];
    const T* ms = &sm.m[slr][0];
    const T* xs = &sm.x[slr][0];
#pragma unroll
    for (int q = 0; q < NCT; ++q) {
      if (q == NCT - 1 && tid + q * NT >= NCH) continue;
      const int64_t ob = (int64_t)kp * P3 + row_off[q];
      const int o = cbase[q];
      T pnew[V], xv[V];
      {
        const VecT pv = *reinterpret_cast<const VecT*>(ps + o);
        const VecT mv = *reinterpret_cast<const VecT*>(ms + o);
        const VecT xw = *reinterpret_cast<const VecT*>(xs + o);
        const T* pa = reinterpret_cast<const T*>(&pv);
        const T* ma = reinterpret_cast<const T*>(&mv);
        const T* xa = reinterpret_cast<const T*>(&xw);
        VecT rv{};
        if (MODE == 3) rv = *reinterpret_cast<const VecT*>(rs + o);
        const T* ra = reinterpret_cast<const T*>(&rv);
#pragma unroll
        for (int t = 0; t < V; ++t) {
          pnew[t] = (MODE == 4 ? ma[t] : ma[t] * ra[t]) + beta_old * pa[t];
          xv[t] = xa[t] + alpha_old * pa[t];
        }
      }
      *reinterpret_cast<VecT*>(ps + o) = *reinterpret_cast<const VecT*>(pnew);
      if (!kown || !((own_rows >> q) & 1u)) continue;
      const int64_t s = ob - (ob & (V - 1)) + ccv[q];
      const int64_t lo = ob + 3, hi = lo + own_len;
      if (s >= lo && s + V <= hi) {
        *reinterpret_cast<VecT*>(A.pout + s) = *reinterpret_cast<const VecT*>(pnew);
        *reinterpret_cast<VecT*>(A.x + s) = *reinterpret_cast<const VecT*>(xv);
      } else if (s + V > lo && s < hi) {
#pragma unroll
        for (int t = 0; t < V; ++t)
          if (s + t >= lo && s + t < hi) {
            A.pout[s + t] = pnew[t];
            A.x[s + t] = xv[t];
          }
      }
    }
  };

  // Shared-memory offsets of this thread's nodes (lx, ly) and (lx, ly + 1)
  // in a plane: row start + the row's lead in that plane (see Stage) + 3 lx.
  // The leads of planes ke and ke + 1 advance by 3 nplane mod V per plane.
  const int rowA = 3 * (jn * g.nxn + i0 - 1), rowB = rowA + 3 * g.nxn;
  const int p3m = (int)(P3 & (V - 1));
  int lA0 = (int)(((int64_t)(k0 - 1) * P3 + rowA) & (V - 1));
  int lB0 = (int)(((int64_t)(k0 - 1) * P3 + rowB) & (V - 1));
  int lA1 = (lA0 + p3m) & (V - 1), lB1 = (lB0 + p3m) & (V - 1);
  const int baseA = ly * RS + 3 * lx, baseB = (ly + 1) * RS + 3 * lx;
  // the four corners (bx + 2 by) of component c of the element face
  auto face = [&](const T* ps, int a, int b, int c, T (&v)[4]) {
    v[0] = ps[a + c];
    v[1] = ps[a + 3 + c];
    v[2] = ps[b + c];
    v[3] = ps[b + 3 + c];
  };

  // Ring slots: plane kp sits in slot (kp - k0 + 1) mod NP of the p ring
  // and mod NR of the r / M^-1 / x ring.
  // prologue: planes k0-1 .. k0+PF-3 requested (one group each); k0-1 and
  // k0 staged and transformed; then k0+PF-2 into the r/M^-1/x slot of k0-1
#pragma unroll
  for (int d = 0; d <= PF - 2; ++d) issue(k0 - 1 + d, d, d % NR);
  cp_async_wait<PF - 3>();
  __syncthreads();
  transform(k0 - 1, 0, 0);
  transform(k0, 1, 1 % NR);
  __syncthreads();
  issue(k0 + PF - 2, PF - 1, (PF - 1) % NR);
  // slots of iteration it = ke - k0 + 1: planes ke (c0), ke+1 (c1), ke+2
  // (c2, r2: transformed), ke+PF (cm = slot of ke-1, r1: issued)
  int c0 = 0, c1 = 1, c2 = 2, cm = NP - 1, r2 = 2 % NR, r1 = 1 % NR;
  auto step = [](int v, int n) { return v + 1 == n ? 0 : v + 1; };
  T Ytp[3][4];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int q = 0; q < 4; ++q) Ytp[c][q] = T(0);
  double dsum = 0.0;

  // The element factor and the node mask are plain loads.  In FP32 both are
  // fetched one plane ahead so that their latency overlaps a plane of work;
  // in FP64 the extra live registers would spill (128-register bound), so
  // they are loaded where they are used (so is the face carry below).
  constexpr bool PREFETCH = sizeof(T) == 4;
  auto load_fac = [&](int ke) -> T {
    return (col_ok && ke >= 0 && ke < g.nze) ? A.fac[(int64_t)ke * eplane + (int64_t)jn * g.nxe + in]
                                             : T(0);
  };
  auto load_mask = [&](int kn) -> unsigned {
    if (!A.nmask || !out_ok || kn < k0 || kn >= k1) return 7u;
    return A.nmask[(int64_t)kn * nplane + (int64_t)jn * g.nxn + in];
  };
  T f_next = PREFETCH ? load_fac(k0 - 1) : T(0);
  unsigned m_next = PREFETCH ? load_mask(k0) : 7u;
  // FP32 also carries each plane's face transform from the layer it tops to
  // the layer it bottoms (the plane is not modified in between)
  T Pcarry[3][4];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int q = 0; q < 4; ++q) Pcarry[c][q] = T(0);

  for (int ke = k0 - 1; ke < k1; ++ke) {
    T f;
    unsigned m_pre = 7u;
    if (PREFETCH) {
      f = f_next;
      f_next = load_fac(ke + 1);
      if (ke >= k0) {
        m_pre = m_next;
        m_next = load_mask(ke + 1);
      }
    } else {
      f = load_fac(ke);
    }
    cp_async_wait<PF - 3>();  // groups up to ke+2 complete
    __syncthreads();  // A: planes ke, ke+1 ready; ke+2 landed; ke-1 and red consumed
    if (ke + 2 <= k1) transform(ke + 2, c2, r2);
    issue(ke + PF, cm, r1);  // into the slot of plane ke-1

    const T* pl0 = &sm.p[c0][0];
    const T* pl1 = &sm.p[c1][0];
    const int a0 = baseA + lA0, a1 = baseA + lA1, b1 = baseB + lB1;
    T U[3][8];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T v[4], Pb[4], Pt[4];
      if (PREFETCH && ke > k0 - 1) {  // this plane's face transform, from the layer below
#pragma unroll
        for (int q = 0; q < 4; ++q) Pb[q] = Pcarry[c][q];
      } else {
        face(pl0, a0, baseB + lB0, c, v);
        face_fwd(v, Pb);
      }
      face(pl1, a1, b1, c, v);
      face_fwd(v, Pt);
      if constexpr (sizeof(T) == 4) {  // packed pairs: (q, q + 1)
#pragma unroll
        for (int q = 0; q < 4; q += 2) {
          if (PREFETCH) {
            Pcarry[c][q] = Pt[q];
            Pcarry[c][q + 1] = Pt[q + 1];
          }
          const float2 b = make_float2(Pb[q], Pb[q + 1]), t = make_float2(Pt[q], Pt[q + 1]);
          const float2 su = __fadd2_rn(b, t);
          const float2 di = __ffma2_rn(make_float2(-1.f, -1.f), b, t);
          U[c][q] = su.x;
          U[c][q + 1] = su.y;
          U[c][q + 4] = di.x;
          U[c][q + 5] = di.y;
        }
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (PREFETCH) Pcarry[c][q] = Pt[q];
          U[c][q] = Pb[q] + Pt[q];
          U[c][q + 4] = Pt[q] - Pb[q];
        }
      }
    }
    T rowS[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T Y[8];
      if (c == 0) lambda_row<T, 0>(A.K, U, Y);
      else if (c == 1) lambda_row<T, 1>(A.K, U, Y);
      else lambda_row<T, 2>(A.K, U, Y);
      T F[4];
      // bottom face: f (Y_s - Y_d) plus the layer below's top face; top
      // face: f (Y_s + Y_d), carried to the layer above.  FP32 forms the sum
      // and difference first and works in packed pairs (q, q + 1); in FP64
      // that order needs more live registers than the 128-register bound.
      if constexpr (sizeof(T) == 4) {
        const float2 f2 = make_float2(f, f);
#pragma unroll
        for (int q = 0; q < 4; q += 2) {
          const float2 ys = make_float2(Y[q], Y[q + 1]), yd = make_float2(Y[q + 4], Y[q + 5]);
          const float2 di = __ffma2_rn(make_float2(-1.f, -1.f), yd, ys);
          const float2 Fq = __ffma2_rn(f2, di, make_float2(Ytp[c][q], Ytp[c][q + 1]));
          const float2 nt = __fmul2_rn(f2, __fadd2_rn(ys, yd));
          F[q] = Fq.x;
          F[q + 1] = Fq.y;
          Ytp[c][q] = nt.x;
          Ytp[c][q + 1] = nt.y;
        }
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const T ys = Y[q] * f, yd = Y[q + 4] * f;
          F[q] = (ys - yd) + Ytp[c][q];
          Ytp[c][q] = ys + yd;
        }
      }
      const T as = F[0] - F[2], ad = F[1] - F[3], bs = F[0] + F[2], bd = F[1] + F[3];
      const T c0 = as - ad, c1 = as + ad, c2 = bs - bd, c3 = bs + bd;
      // element lx-1 contributes its +x corners to this thread's nodes
      const T l1 = __shfl_up_sync(0xffffffffu, c1, 1);
      const T l3 = __shfl_up_sync(0xffffffffu, c3, 1);
      rowS[c] = c0 + l1;
      sm.red[ly][c][lx] = c2 + l3;
    }
    __syncthreads();  // B: red of this layer visible
    if (ke >= k0 && out_ok) {
      // this node's p.q in T (3 terms), accumulated in FP64 across planes
      T pdot = T(0);
      const int64_t node = (int64_t)ke * nplane + (int64_t)jn * g.nxn + in;
      const unsigned m = PREFETCH ? m_pre : (A.nmask ? A.nmask[node] : 7u);
      const T* own = pl0 + a0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T v = rowS[c] + sm.red[ly - 1][c][lx];
        const T xv = own[c];
        const bool fr = (m >> c) & 1u;
        v = fr ? v + A.shift * xv : T(0);
        const int64_t dof = 3 * node + c;
        if (MODE == 5) {
          // x_prev: read, or 0 (the step after a start from x = 0), or
          // unused (the first step: omega = 0)
          const T xp = A.xprev_zero ? T(0) : (A.omega != T(0) ? A.x[dof] : xv);
          A.x[dof] = fr ? xv + A.omega * (xv - xp) + A.gamma * A.minv[dof] * (A.r[dof] - v)
                        : T(0);
        } else if (MODE == 6) {
          A.q[dof] = fr ? A.r[dof] - v : T(0);
        } else {
          A.q[dof] = v;
        }
        if (DOT) pdot = fma(xv, v, pdot);
      }
      if (DOT) dsum += (double)pdot;
    }
    c0 = step(c0, NP);
    c1 = step(c1, NP);
    c2 = step(c2, NP);
    cm = step(cm, NP);
    r2 = step(r2, NR);
    r1 = step(r1, NR);
    lA0 = lA1;
    lB0 = lB1;
    lA1 = (lA1 + p3m) & (V - 1);
    lB1 = (lB1 + p3m) & (V - 1);
  }

  if (MODE == 4) {
    double v[1] = {dsum};
    if (grid_reduce<1>(v, A.partials, &A.st->ticket[TK_MATVEC]) && tid == 0) {
      const double pq = v[0], zr = A.st->aux[3];
      A.st->pq = pq;
      if (!(pq > 0.0) || !isfinite(pq) || !isfinite(zr))
        A.st->status = HX_ST_BREAKDOWN;
      else
        A.st->alpha = zr / pq;
    }
  } else if (DOT) {
    double v[1] = {dsum};
    if (grid_reduce<1>(v, A.partials, &A.st->ticket[TK_MATVEC]) && tid == 0) {
      if (MODE == 1) {
        A.out[0] = v[0];
      } else {
        const double pq = v[0];
        A.st->pq = pq;
        if (!(pq > 0.0) || !isfinite(pq))
          A.st->status = HX_ST_BREAKDOWN;
        else
          A.st->alpha = A.st->rz / pq;
      }
    }
  }
}

// Per-node Jacobi diagonal: diag(n,c) = kd[c] * sum of the factors of the
// (up to 8) elements around n; node mask = free-DOF bits of `bcfree`
// cleared where the node carries no stiffness.  Writes diag into `diag`,
// the mask into `nmask`, and reduces the max diagonal over free DOFs.
template <typename T>
__global__ void k_node_diag(const T* __restrict__ fac, const uint8_t* __restrict__ bcfree,
                            uint8_t* __restrict__ nmask, T* __restrict__ diag, Grid g,
                            ElemCoef<double> K, double* partials, CgState* st, double* out) {
  const int64_t nn = (int64_t)g.nxn * g.nyn * g.nzn;
  double mx = 0.0;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(n % g.nxn);
    const int64_t r = n / g.nxn;
    const int j = (int)(r % g.nyn);
    const int k = (int)(r / g.nyn);
    double s = 0.0;
#pragma unroll
    for (int dk = -1; dk <= 0; ++dk)
#pragma unroll
      for (int dj = -1; dj <= 0; ++dj)
#pragma unroll
        for (int di = -1; di <= 0; ++di) {
          const int ei = i + di, ej = j + dj, ek = k + dk;
          if (ei >= 0 && ej >= 0 && ek >= 0 && ei < g.nxe && ej < g.nye && ek < g.nze)
            s += (double)fac[((int64_t)ek * g.nye + ej) * g.nxe + ei];
        }
    const unsigned m = (s > 0.0) ? (bcfree ? bcfree[n] : 7u) : 0u;
    nmask[n] = (uint8_t)m;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double d = K.kd[c] * s;
      diag[3 * n + c] = (T)d;
      if ((m >> c) & 1u) mx = fmax(mx, d);
    }
  }
  double v[1] = {mx};
  if (grid_reduce<1, true>(v, partials, &st->ticket[TK_AUX]) && threadIdx.x == 0) out[0] = v[0];
}

// minv = free ? 1/(diag + shift) : 0   (src/Solvers/GPUSolver.jl:402)
template <typename T>
__global__ void k_minv(const uint8_t* __restrict__ nmask, const T* __restrict__ diag,
                       T* __restrict__ minv, int64_t nn, double shift) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * nn;
       i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned m = nmask[i / 3];
    const int c = (int)(i % 3);
    minv[i] = ((m >> c) & 1u) ? (T)(1.0 / ((double)diag[i] + shift)) : T(0);
  }
}

inline dim3 mv_grid(const Grid& g, int kchunk) {
  return dim3(cdiv(g.nxn, MV_BX - 1), cdiv(g.nyn, MV_BY - 1), cdiv(g.nzn, kchunk));
}

template <typename T, int MODE>
void launch_struct(cudaStream_t s, const OpArgs<T>& a) {
  constexpr bool FUSED = MODE == 3 || MODE == 4;
  constexpr int MINB = mv_resident<T>();
  const size_t smem = sizeof(OpSmem<T, MV_BY, FUSED>);
  static PerDeviceOnce configured;  // per instantiation and device
  configured.run([&] {
    HX_CUDA(cudaFuncSetAttribute(k_struct<T, MV_BY, MODE, MINB>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  });
  k_struct<T, MV_BY, MODE, MINB><<<mv_grid(a.g, a.kchunk), dim3(MV_BX, MV_BY), smem, s>>>(a);
  HX_CHECK_LAUNCH();
}

}  // namespace

int mv_kchunk(const Grid& g, int resident) {
  // Node planes per CTA: the chunk length kc (at least 8, so the two staged
  // halo planes stay a small share) that minimises (waves of resident CTAs)
  // x (planes each CTA stages, kc + 2).  A last wave that fills few SMs
  // costs as much as a full one; ties go to the longer chunk.
  const int64_t cols = (int64_t)cdiv(g.nxn, MV_BX - 1) * cdiv(g.nyn, MV_BY - 1);
  const int64_t slots = (int64_t)resident * sm_count();
  int best_kc = g.nzn;
  int64_t best = INT64_MAX;
  for (int kc = std::min(8, g.nzn); kc <= g.nzn; ++kc) {
    const int64_t waves = cdiv(cols * cdiv(g.nzn, kc), slots);
    const int64_t cost = waves * (kc + 2);
    if (cost <= best) {
      best = cost;
      best_kc = kc;
    }
  }
  return best_kc;
}

size_t mv_num_blocks(const Grid& g, int resident) {
  const dim3 gr = mv_grid(g, mv_kchunk(g, resident));
  return (size_t)gr.x * gr.y * gr.z;
}

size_t mv_max_blocks(const Grid& g) {
  return std::max(mv_num_blocks(g, mv_resident<float>()), mv_num_blocks(g, mv_resident<double>()));
}

template <typename T>
void launch_matvec(cudaStream_t s, int mode, const T* x, T* y, const T* fac, const uint8_t* nmask,
                   const Grid& g, const ElemCoef<T>& K, T shift, CgState* st, double* partials,
                   double* out) {
  OpArgs<T> a{};
  a.pin = x;
  a.q = y;
  a.fac = fac;
  a.nmask = nmask;
  a.g = g;
  a.kchunk = mv_kchunk(g, mv_resident<T>());
  a.K = K;
  a.shift = shift;
  a.st = st;
  a.partials = partials;
  a.out = out;
  if (mode == 0)
    launch_struct<T, 0>(s, a);
  else if (mode == 1)
    launch_struct<T, 1>(s, a);
  else
    launch_struct<T, 2>(s, a);
}

template <typename T>
void launch_cheb_step(cudaStream_t s, const T* x, T* xprev_new, bool xprev_zero, const T* b,
                      const T* minv, T omega, T gamma, const T* fac, const uint8_t* nmask,
                      const Grid& g, const ElemCoef<T>& K, T shift) {
  OpArgs<T> a{};
  a.pin = x;
  a.x = xprev_new;
  a.xprev_zero = xprev_zero ? 1 : 0;
  a.r = b;
  a.minv = minv;
  a.omega = omega;
  a.gamma = gamma;
  a.fac = fac;
  a.nmask = nmask;
  a.g = g;
  a.kchunk = mv_kchunk(g, mv_resident<T>());
  a.K = K;
  a.shift = shift;
  launch_struct<T, 5>(s, a);
}
template void launch_cheb_step<float>(cudaStream_t, const float*, float*, bool, const float*,
                                      const float*, float, float, const float*, const uint8_t*,
                                      const Grid&, const ElemCoef<float>&, float);

template <typename T>
void launch_residual(cudaStream_t s, const T* x, const T* b, T* r, const T* fac,
                     const uint8_t* nmask, const Grid& g, const ElemCoef<T>& K, T shift) {
  OpArgs<T> a{};
  a.pin = x;
  a.r = b;
  a.q = r;
  a.fac = fac;
  a.nmask = nmask;
  a.g = g;
  a.kchunk = mv_kchunk(g, mv_resident<T>());
  a.K = K;
  a.shift = shift;
  launch_struct<T, 6>(s, a);
}
template void launch_residual<float>(cudaStream_t, const float*, const float*, float*,
                                     const float*, const uint8_t*, const Grid&,
                                     const ElemCoef<float>&, float);

template <typename T>
void launch_pcg_step(cudaStream_t s, const T* pin, T* pout, const T* r, const T* minv, T* x, T* q,
                     const T* fac, const uint8_t* nmask, const Grid& g, const ElemCoef<T>& K,
                     T shift, CgState* st, double* partials) {
  OpArgs<T> a{};
  a.pin = pin;
  a.pout = pout;
  a.r = r;
  a.minv = minv;
  a.x = x;
  a.q = q;
  a.fac = fac;
  a.nmask = nmask;
  a.g = g;
  a.kchunk = mv_kchunk(g, mv_resident<T>());
  a.K = K;
  a.shift = shift;
  a.st = st;
  a.partials = partials;
  launch_struct<T, 3>(s, a);
}

template <typename T>
void launch_fcg_step(cudaStream_t s, const T* pin, T* pout, const T* z, T* x, T* q, const T* fac,
                     const uint8_t* nmask, const Grid& g, const ElemCoef<T>& K, T shift,
                     CgState* st, double* partials) {
  OpArgs<T> a{};
  a.pin = pin;
  a.pout = pout;
  a.minv = z;
  a.x = x;
  a.q = q;
  a.fac = fac;
  a.nmask = nmask;
  a.g = g;
  a.kchunk = mv_kchunk(g, mv_resident<T>());
  a.K = K;
  a.shift = shift;
  a.st = st;
  a.partials = partials;
  launch_struct<T, 4>(s, a);
}
template void launch_fcg_step<double>(cudaStream_t, const double*, double*, const double*,
                                      double*, double*, const double*, const uint8_t*,
                                      const Grid&, const ElemCoef<double>&, double, CgState*,
                                      double*);
template void launch_fcg_step<float>(cudaStream_t, const float*, float*, const float*, float*,
                                     float*, const float*, const uint8_t*, const Grid&,
                                     const ElemCoef<float>&, float, CgState*, double*);

template void launch_matvec<double>(cudaStream_t, int, const double*, double*, const double*,
                                    const uint8_t*, const Grid&, const ElemCoef<double>&, double,
                                    CgState*, double*, double*);
template void launch_matvec<float>(cudaStream_t, int, const float*, float*, const float*,
                                   const uint8_t*, const Grid&, const ElemCoef<float>&, float,
                                   CgState*, double*, double*);
template void launch_pcg_step<double>(cudaStream_t, const double*, double*, const double*,
                                      const double*, double*, double*, const double*,
                                      const uint8_t*, const Grid&, const ElemCoef<double>&,
                                      double, CgState*, double*);
template void launch_pcg_step<float>(cudaStream_t, const float*, float*, const float*,
                                     const float*, float*, float*, const float*, const uint8_t*,
                                     const Grid&, const ElemCoef<float>&, float, CgState*,
                                     double*);

template <typename T>
void launch_node_diag(cudaStream_t s, const T* fac, const uint8_t* bcfree, uint8_t* nmask, T* diag,
                      const Grid& g, const ElemCoef<double>& K, double* partials, CgState* st,
                      double* out) {
  const int64_t nn = (int64_t)g.nxn * g.nyn * g.nzn;
  const unsigned blocks = std::min<int64_t>(cdiv(nn, 256), 8LL * sm_count());
  k_node_diag<T><<<blocks, 256, 0, s>>>(fac, bcfree, nmask, diag, g, K, partials, st, out);
  HX_CHECK_LAUNCH();
}
template void launch_node_diag<double>(cudaStream_t, const double*, const uint8_t*, uint8_t*,
                                       double*, const Grid&, const ElemCoef<double>&, double*,
                                       CgState*, double*);
template void launch_node_diag<float>(cudaStream_t, const float*, const uint8_t*, uint8_t*, float*,
                                      const Grid&, const ElemCoef<double>&, double*, CgState*,
                                      double*);

template <typename T>
void launch_minv(cudaStream_t s, const uint8_t* nmask, const T* diag, T* minv, int64_t nn,
                 double shift) {
  const unsigned blocks = std::min<int64_t>(cdiv(3 * nn, 256), 16LL * sm_count());
  k_minv<T><<<blocks, 256, 0, s>>>(nmask, diag, minv, nn, shift);
  HX_CHECK_LAUNCH();
}
template void launch_minv<double>(cudaStream_t, const uint8_t*, const double*, double*, int64_t,
                                  double);
template void launch_minv<float>(cudaStream_t, const uint8_t*, const float*, float*, int64_t,
                                 double);

}  // namespace hx
