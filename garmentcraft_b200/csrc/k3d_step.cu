// The implicit backward-Euler step on the device: one persistent cooperative
// kernel per substep.
//
//   build (elements)  -> per-corner force/Hv/diag records, operator records
//   build (points)    -> rhs b, block-Jacobi inverse, contact set
//   PCG (implizit.rs:370-426), up to two passes with the release test
//   (implizit.rs:908-943), then friction and integration (:957-1014).
//
// Every phase is a grid-stride loop over elements or points, separated by a
// grid barrier. Sums are deterministic: points gather their incident element
// corners in a fixed order (no float atomics), and grid reductions add the
// per-block partials in block order. The barrier waits are bounded by a
// wall-clock limit; on expiry the kernel records K3D_TIMEOUT and every block
// returns.
#include <cfloat>
#include <cstdint>

#include "k3d_device.cuh"
#include "k3d_step.h"

namespace k3d {

// ------------------------------------------------------------ barrier + reductions
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed_i32(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

constexpr uint64_t kBarrierLimitNs = 4000000000ull;  // 4 s per barrier wait
// The FP32 operator resolves the relative residual (P^-1 norm) to about
// 1e-6 on stiff cloth; below that the directions lose conjugacy and a solve
// can diverge. The mixed form never asks for less.
constexpr double kMixedTolFloor = 1e-6;
// Reliable updates of the mixed form: the true residual replaces the
// recursive one once r.z has fallen by kReliable since the last update, or
// grown by kGrow (then the direction restarts).
constexpr double kReliable = 1e-2;
constexpr double kGrow = 1e2;
constexpr int kMaxRed = 4;

struct Shared {
  double red[kMaxRed][32];
  double res[kMaxRed];
  unsigned epoch;  // barriers passed in this launch
  unsigned rbuf;   // reductions done in this launch (partials buffer parity)
  int err;
};

__device__ __forceinline__ unsigned atom_add_release(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// Block sum of NV values in a fixed order (warp xor tree, then the warps in
// order); the result is in v in every thread.
template <int NV>
__device__ __forceinline__ void block_sum(Shared& sh, double (&v)[NV]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sh.red[k][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = 0.0;
      for (int w = 0; w < nw; ++w) t += sh.red[k][w];
      sh.res[k] = t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = sh.res[k];
  __syncthreads();
}

// Grid barrier: every block adds one to a counter that starts at zero in
// each launch; barrier k of the launch is passed when the counter reaches
// k * gridDim.x. With NV > 0 it also sums NV doubles over the grid: each
// block writes its partials before arriving and, once through, adds all
// blocks' partials in block order itself, so every block holds the same
// bits. Partials alternate between two buffers (a block can only reuse a
// buffer after every block has passed the barrier that follows the reads).
// The wait gives up after kBarrierLimitNs or when another block has recorded
// an error; the return value is false then and the caller leaves the kernel.
template <int NV>
__device__ bool grid_sync(const StepArgs& a, Shared& sh, double (&v)[NV > 0 ? NV : 1]) {
  SyncState* s = a.sync;
  const unsigned buf = sh.rbuf & 1u;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if constexpr (NV > 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double x = v[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) sh.red[k][warp] = x;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if constexpr (NV > 0) {
      const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
      for (int k = 0; k < NV; ++k) {
        double t = 0.0;
        for (int w = 0; w < nw; ++w) t += sh.red[k][w];
        a.partials[(buf * kMaxRed + k) * gridDim.x + blockIdx.x] = t;
      }
      sh.rbuf += 1;  // every thread read the parity at entry, before the barrier above
    }
    const unsigned target = (sh.epoch + 1) * gridDim.x;
    atom_add_release(&s->count, 1u);
    const uint64_t t0 = globaltimer();
    int err = 0;
    while (int(ld_acquire_u32(&s->count) - target) < 0) {
      if ((err = ld_relaxed_i32(&s->error)) != 0) break;
      if (globaltimer() - t0 > kBarrierLimitNs) {
        atomicCAS(&s->error, 0, K3D_STATUS_TIMEOUT);
        err = K3D_STATUS_TIMEOUT;
        break;
      }
    }
    sh.err = err;
    sh.epoch += 1;
  }
  __syncthreads();
  if (sh.err != 0) return false;
  if constexpr (NV > 0) {
    // warp 0 adds the block partials in block order (fixed per lane, then a
    // fixed xor tree): every block gets the same bits
    if (warp == 0) {
#pragma unroll
      for (int k = 0; k < NV; ++k) {
        double x = 0.0;
        for (unsigned b = lane; b < gridDim.x; b += 32) x += __ldcg(&a.partials[(buf * kMaxRed + k) * gridDim.x + b]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sh.res[k] = x;
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = sh.res[k];
  }
  return true;
}

// Grid-wide maximum of one non-negative double (bit pattern order equals
// value order for non-negative doubles, so an integer atomicMax is exact).
__device__ bool grid_max(const StepArgs& a, Shared& sh, double (&v)[1]) {
  double x = v[0];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
  if ((threadIdx.x & 31) == 0 && x > 0.0)
    atomicMax(reinterpret_cast<unsigned long long*>(&a.stat_rest_max[1]), (unsigned long long)__double_as_longlong(x));
  double none[1] = {0.0};
  if (!grid_sync<0>(a, sh, none)) return false;
  v[0] = __longlong_as_double((long long)__ldcg(reinterpret_cast<const unsigned long long*>(&a.stat_rest_max[1])));
  return true;
}

__device__ __forceinline__ bool barrier(const StepArgs& a, Shared& sh) {
  double none[1] = {0.0};
  return grid_sync<0>(a, sh, none);
}

#define K3D_FOR(i, n) \
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < (n); i += int64_t(gridDim.x) * blockDim.x)

// ------------------------------------------------------------ typed views
// Per point the CG direction c and the filtered preconditioned residual
// w = S P^-1 r, side by side so an element reads both with one gather.
template <typename R>
struct CW {
  R4<R> c, w;
};

// The next direction c' = w + beta c (implizit.rs:421: S(z + beta c) with c
// already in the filtered space). One helper for the element and the point
// phase, so both hold the same bits.
__device__ __forceinline__ float fmar(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmar(double a, double b, double c) { return __fma_rn(a, b, c); }
template <typename R>
__device__ __forceinline__ R4<R> next_dir(const CW<R>& q, R beta) {
  return {fmar(beta, q.c.x, q.w.x), fmar(beta, q.c.y, q.w.y), fmar(beta, q.c.z, q.w.z), R(0)};
}

template <typename R>
struct View {
  CW<R>* cw;
  R *r, *z, *ap, *pinv, *nrm, *md;
  R4<R>*m_f1w, *m_f2w, *m_kgB;
  const R4<R>*m_rin, *m_kgA;
  R4<R>* b_grad;
  R4<R>* s_dq;
  R* s_k;
  R4<R>* slot;
  __device__ explicit View(const StepArgs& a)
      : cw((CW<R>*)a.c), r((R*)a.r), z((R*)a.z), ap((R*)a.ap), pinv((R*)a.pinv), nrm((R*)a.nrm), md((R*)a.md),
        m_f1w((R4<R>*)a.m_f1w), m_f2w((R4<R>*)a.m_f2w), m_kgB((R4<R>*)a.m_kgB),
        m_rin((const R4<R>*)a.m_rin), m_kgA((const R4<R>*)a.m_kgA), b_grad((R4<R>*)a.b_grad),
        s_dq((R4<R>*)a.s_dq), s_k((R*)a.s_k), slot((R4<R>*)a.slot) {}
};

__device__ __forceinline__ double4 ldg4(const double4* p) {
  const double2 lo = __ldg(reinterpret_cast<const double2*>(p)), hi = __ldg(reinterpret_cast<const double2*>(p) + 1);
  return make_double4(lo.x, lo.y, hi.x, hi.y);
}

__device__ __forceinline__ MembranC membran_c(const StepArgs& a, int64_t t) {
  const double4 r = ldg4(&a.m_r[t]), b = ldg4(&a.m_basis[t]), m = ldg4(&a.m_mat[t]);
  MembranC o;
  o.r[0] = r.x;
  o.r[1] = r.y;
  o.r[2] = r.z;
  o.r[3] = r.w;
  o.kx = b.x;
  o.ky = b.y;
  o.sx = b.z;
  o.sy = b.w;
  o.fl = m.x;
  o.ek = m.y;
  o.es = m.z;
  o.g = m.w;
  return o;
}

// ------------------------------------------------------------ build: elements
// implizit.rs:725-844 and kontinuum.rs, in FP64. Writes, per element corner,
// the contribution to (f - h H v) and, if asked, to the load, plus the
// membrane diagonal blocks; and the per-step operator records in precision R.
template <typename R>
__device__ void build_elements(const StepArgs& a, const View<R>& vw) {
  const double h = a.h;
  K3D_FOR(t, a.nt) {
    const uint4 id = __ldg(&a.m_idx[t]);
    const MembranC m = membran_c(a, t);
    const D3 p0 = ld3(a.x, id.x), p1 = ld3(a.x, id.y), p2 = ld3(a.x, id.z);
    const D3 e1 = p1 - p0, e2 = p2 - p0;
    const D3 f1 = e1 * m.r[0] + e2 * m.r[2];
    const D3 f2 = e1 * m.r[1] + e2 * m.r[3];
    D3 ba, bb, bc;
    basis3(m, ba, bb, bc);
    const D3 g = d3(dot(f1, f1), dot(f2, f2), 2.0 * dot(f1, f2));
    const D3 e = d3(0.5 * (dot(ba, g) - 1.0), 0.5 * (dot(bb, g) - 1.0), 0.5 * dot(bc, g));
    const D3 du = du_dg(m, ba, bb, bc, e);
    D3 F[3];
    kraefte(m.r, f1, f2, du, F);
    const D3 dz = du_dg(m, ba, bb, bc, d3(fmax(e.x, 0.0), fmax(e.y, 0.0), e.z));
    const D3 w = psd2(dz.x, dz.y, dz.z);
    double kg[6];
    kg_sym(m, kg);
    // H v (FP64) with the same record the operator uses
    R4<double> rf1 = {f1.x, f1.y, f1.z, w.x}, rf2 = {f2.x, f2.y, f2.z, w.y};
    R4<double> rr = {m.r[0], m.r[1], m.r[2], m.r[3]};
    R4<double> ka = {kg[0], kg[1], kg[2], kg[3]}, kb = {kg[4], kg[5], w.z, 0.0};
    R4<double> vv[3], hv[3];
    const uint32_t ids[3] = {id.x, id.y, id.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      D3 q = ld3(a.v, ids[k]);
      vv[k] = {q.x, q.y, q.z, 0.0};
    }
    membran_hv<double>(rf1, rf2, rr, ka, kb, vv, hv);
#pragma unroll
    for (int k = 0; k < 3; ++k)
      a.m_bc[3 * t + k] = make_double4(F[k].x - hv[k].x * h, F[k].y - hv[k].y * h, F[k].z - hv[k].z * h, 0.0);
    if (a.need_load) {
      D3 L[3];
      kraefte(m.r, f1, f2, dz, L);
#pragma unroll
      for (int k = 0; k < 3; ++k) a.m_lc[3 * t + k] = make_double4(L[k].x, L[k].y, L[k].z, 0.0);
    }
    // diagonal blocks J_k^T kg J_k + s_kk I (kontinuum.rs:675-708)
    const D3 k1 = coef1(m.r), k2 = coef2(m.r);
    const double c1[3] = {k1.x, k1.y, k1.z}, c2[3] = {k2.x, k2.y, k2.z};
    const double K[3][3] = {{kg[0], kg[3], kg[4]}, {kg[3], kg[1], kg[5]}, {kg[4], kg[5], kg[2]}};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const D3 j[3] = {f1 * (2.0 * c1[k]), f2 * (2.0 * c2[k]), f1 * (2.0 * c2[k]) + f2 * (2.0 * c1[k])};
      D3 u[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) u[i] = j[0] * K[i][0] + j[1] * K[i][1] + j[2] * K[i][2];
      const double s = 2.0 * (w.x * c1[k] * c1[k] + w.y * c2[k] * c2[k] + 2.0 * w.z * c1[k] * c2[k]);
      double* dc = a.m_dc + 8 * (3 * t + k);
      dc[0] = j[0].x * u[0].x + j[1].x * u[1].x + j[2].x * u[2].x + s;
      dc[1] = j[0].y * u[0].y + j[1].y * u[1].y + j[2].y * u[2].y + s;
      dc[2] = j[0].z * u[0].z + j[1].z * u[1].z + j[2].z * u[2].z + s;
      dc[3] = j[0].x * u[0].y + j[1].x * u[1].y + j[2].x * u[2].y;
      dc[4] = j[0].x * u[0].z + j[1].x * u[1].z + j[2].x * u[2].z;
      dc[5] = j[0].y * u[0].z + j[1].y * u[1].z + j[2].y * u[2].z;
    }
    vw.m_f1w[t] = {R(f1.x), R(f1.y), R(f1.z), R(w.x)};
    vw.m_f2w[t] = {R(f2.x), R(f2.y), R(f2.z), R(w.y)};
    vw.m_kgB[t] = {R(kg[4]), R(kg[5]), R(w.z), R(0)};
    if (a.m_f1w64) {
      static_cast<R4<double>*>(a.m_f1w64)[t] = rf1;
      static_cast<R4<double>*>(a.m_f2w64)[t] = rf2;
      static_cast<R4<double>*>(a.m_kgB64)[t] = kb;
    }
  }
  K3D_FOR(b, a.nb) {
    const uint4 id = __ldg(&a.b_idx[b]);
    const double2 kr = __ldg(&a.b_kr[b]);
    const uint32_t ids[4] = {id.x, id.y, id.z, id.w};
    D3 gr[4];
    double theta = 0.0;
    if (!dieder(ld3(a.x, id.x), ld3(a.x, id.y), ld3(a.x, id.z), ld3(a.x, id.w), theta, gr)) {
      theta = 0.0;
#pragma unroll
      for (int q = 0; q < 4; ++q) gr[q] = d3(0, 0, 0);
    }
    const double fehler = winkel_fehler(theta, kr.y);
    double gv = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) gv += dot(gr[q], ld3(a.v, ids[q]));
    const double sb = -kr.x * fehler - h * (kr.x * gv);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      a.b_bc[4 * b + q] = make_double4(gr[q].x * sb, gr[q].y * sb, gr[q].z * sb, 0.0);
      vw.b_grad[4 * b + q] = {R(gr[q].x), R(gr[q].y), R(gr[q].z), R(kr.x)};
      if (a.b_grad64) static_cast<R4<double>*>(a.b_grad64)[4 * b + q] = {gr[q].x, gr[q].y, gr[q].z, kr.x};
    }
  }
  K3D_FOR(s, a.ns) {
    const uint4 id = __ldg(&a.s_idx[s]);
    const double2 kl = a.s_kl[s];
    const double k = kl.x;
    const D3 d = ld3(a.x, id.y) - ld3(a.x, id.x);
    D3 F, n;
    double quer;
    bool zug = false;
    if (id.z == 0) {  // pattern edge with its own stiffness (implizit.rs:742-752)
      const double l = fmax(norm(d), 1e-12);
      n = d * (1.0 / l);
      F = n * (k * (l - kl.y));
      quer = fmax(1.0 - kl.y / l, 0.0);
      zug = l > kl.y;
    } else {  // seam spring (implizit.rs:763-771)
      const double l = norm(d);
      const double l0 = isfinite(kl.y) ? kl.y : l;
      if (l0 > 0.0 && l > 1e-12) {
        F = d * (k * (l - l0) / l);
        n = d * (1.0 / l);
        quer = fmax(1.0 - l0 / l, 0.0);
      } else {
        F = d * k;
        n = d3(0, 0, 0);
        quer = 1.0;
      }
    }
    // H v with d = v_i - v_j (implizit.rs:193-197); end i gets +, end j gets -
    const D3 dv = ld3(a.v, id.x) - ld3(a.v, id.y);
    const D3 bd = (n * (dot(n, dv) * (1.0 - quer)) + dv * quer) * k;
    a.s_bc[s] = make_double4(F.x - bd.x * h, F.y - bd.y * h, F.z - bd.z * h, 0.0);
    if (a.need_load) a.s_lc[s] = zug ? make_double4(F.x, F.y, F.z, 0.0) : make_double4(0, 0, 0, 0);
    vw.s_dq[s] = {R(n.x), R(n.y), R(n.z), R(quer)};
    vw.s_k[s] = R(k);
    if (a.s_dq64) {
      static_cast<R4<double>*>(a.s_dq64)[s] = {n.x, n.y, n.z, quer};
      static_cast<double*>(a.s_k64)[s] = k;
    }
  }
}

// ------------------------------------------------------------ build: points
// implizit.rs:722-723 (gravity, damping), :872-894 (contacts, rhs, pinv).
template <typename R>
__device__ void build_points(const StepArgs& a, const View<R>& vw, double& held) {
  const double h = a.h, h2 = a.h * a.h;
  held = 0.0;
  K3D_FOR(i, a.n) {
    const double m = a.masse[i];
    const D3 vi = ld3(a.v, uint32_t(i));
    D3 acc = d3(a.g[0] * m, a.g[1] * m, a.g[2] * m) - vi * (a.daempf * m);
    D3 load = d3(a.g[0] * m, a.g[1] * m, a.g[2] * m);
    double D[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t e = __ldg(&a.off_t[i]); e < __ldg(&a.off_t[i + 1]); ++e) {
      const uint32_t q = __ldg(&a.ent_t[e]);
      const double4 bc = a.m_bc[q];
      acc = acc + d3(bc.x, bc.y, bc.z);
      const double* dc = a.m_dc + 8 * size_t(q);
#pragma unroll
      for (int k = 0; k < 6; ++k) D[k] += dc[k];
      if (a.need_load) {
        const double4 lc = a.m_lc[q];
        load = load + d3(lc.x, lc.y, lc.z);
      }
    }
    for (uint32_t e = __ldg(&a.off_b[i]); e < __ldg(&a.off_b[i + 1]); ++e) {
      const uint32_t q = __ldg(&a.ent_b[e]);
      const double4 bc = a.b_bc[q];
      acc = acc + d3(bc.x, bc.y, bc.z);
      const R4<R> gq = vw.b_grad[q];
      const double gx = gq.x, gy = gq.y, gz = gq.z, k = gq.w;
      D[0] += k * gx * gx;
      D[1] += k * gy * gy;
      D[2] += k * gz * gz;
      D[3] += k * gx * gy;
      D[4] += k * gx * gz;
      D[5] += k * gy * gz;
    }
    for (uint32_t e = __ldg(&a.off_s[i]); e < __ldg(&a.off_s[i + 1]); ++e) {
      const uint32_t q = __ldg(&a.ent_s[e]);
      const uint32_t s = q >> 1;
      const double sg = (q & 1u) ? -1.0 : 1.0;
      const double4 bc = a.s_bc[s];
      acc = acc + d3(bc.x, bc.y, bc.z) * sg;
      if (a.need_load) {
        const double4 lc = a.s_lc[s];
        load = load + d3(lc.x, lc.y, lc.z) * sg;
      }
      const R4<R> dq = vw.s_dq[s];
      const double k = vw.s_k[s], nx = dq.x, ny = dq.y, nz = dq.z, qu = dq.w;
      const double kn = k * (1.0 - qu), kq = k * qu;
      D[0] += kq + kn * nx * nx;
      D[1] += kq + kn * ny * ny;
      D[2] += kq + kn * nz * nz;
      D[3] += kn * nx * ny;
      D[4] += kn * nx * nz;
      D[5] += kn * ny * nz;
    }
    st3(a.b, uint32_t(i), acc * h);
    if (a.need_load) st3(a.load, uint32_t(i), load);
    const double mdi = m * (1.0 + h * a.daempf);
    double A[6] = {mdi + h2 * D[0], mdi + h2 * D[1], mdi + h2 * D[2], h2 * D[3], h2 * D[4], h2 * D[5]};
    double P[6];
    m3_inv_sym(A, P);
#pragma unroll
    for (int k = 0; k < 6; ++k) vw.pinv[6 * i + k] = R(P[k]);
    vw.md[i] = R(mdi);
    // contact set: the last body that reports a contact wins (implizit.rs:873-883)
    D3 nrm = d3(0, 0, 0);
    double vn_soll = 0.0;
    D3 vb = d3(0, 0, 0);
    bool fest = false;
    if (a.frei[i]) {
      const D3 xi = ld3(a.x, uint32_t(i));
      for (int kb = 0; kb < a.n_bodies; ++kb) {
        D3 nn;
        double tiefe;
        if (kontakt(a.bodies[kb], xi, a.kabst[i] + a.kontakt_rand, nn, tiefe)) {
          const D3 bv = d3(a.bodies[kb].vel[0], a.bodies[kb].vel[1], a.bodies[kb].vel[2]);
          nrm = nn;
          vn_soll = (tiefe - a.kontakt_rand) / h + dot(bv, nn);
          vb = bv;
          fest = true;
        }
      }
    }
    st3(a.nrm_d, uint32_t(i), nrm);
    vw.nrm[3 * i] = R(nrm.x);
    vw.nrm[3 * i + 1] = R(nrm.y);
    vw.nrm[3 * i + 2] = R(nrm.z);
    a.vn_soll[i] = vn_soll;
    st3(a.vk, uint32_t(i), vb);
    a.fnk[i] = 0.0;
    if (fest) held += 1.0;
    if (a.first_step) st3(a.dv, uint32_t(i), d3(a.g[0] * h, a.g[1] * h, a.g[2] * h));
  }
}

// ------------------------------------------------------------ operator A p
// Per element: the corner products H_e p with p = w + beta c at its points
// (implizit.rs:185-221), written to the corners' slots (rank * np + point).
template <typename R>
__device__ void apply_elements(const StepArgs& a, const View<R>& vw, R beta) {
  K3D_FOR(t, a.nt) {
    const uint4 id = __ldg(&a.m_idx[t]);
    const uint4 ps = __ldg(&a.m_pos[t]);
    const R4<R> d[3] = {next_dir<R>(vw.cw[id.x], beta), next_dir<R>(vw.cw[id.y], beta),
                        next_dir<R>(vw.cw[id.z], beta)};
    R4<R> out[3];
    membran_hv<R>(vw.m_f1w[t], vw.m_f2w[t], vw.m_rin[t], vw.m_kgA[t], vw.m_kgB[t], d, out);
    vw.slot[ps.x] = out[0];
    vw.slot[ps.y] = out[1];
    vw.slot[ps.z] = out[2];
  }
  K3D_FOR(b, a.nb) {
    const uint4 id = __ldg(&a.b_idx[b]);
    const uint4 ps = __ldg(&a.b_pos[b]);
    const R4<R> g0 = vw.b_grad[4 * b], g1 = vw.b_grad[4 * b + 1], g2 = vw.b_grad[4 * b + 2], g3 = vw.b_grad[4 * b + 3];
    const R4<R> c0 = next_dir<R>(vw.cw[id.x], beta), c1 = next_dir<R>(vw.cw[id.y], beta),
                c2 = next_dir<R>(vw.cw[id.z], beta), c3 = next_dir<R>(vw.cw[id.w], beta);
    // the four gradients sum to zero (the angle does not change under a
    // translation), so only differences to point 0 enter
    const R gp = g1.x * (c1.x - c0.x) + g1.y * (c1.y - c0.y) + g1.z * (c1.z - c0.z) + g2.x * (c2.x - c0.x) +
                 g2.y * (c2.y - c0.y) + g2.z * (c2.z - c0.z) + g3.x * (c3.x - c0.x) + g3.y * (c3.y - c0.y) +
                 g3.z * (c3.z - c0.z);
    const R s = g0.w * gp;
    vw.slot[ps.x] = {g0.x * s, g0.y * s, g0.z * s, R(0)};
    vw.slot[ps.y] = {g1.x * s, g1.y * s, g1.z * s, R(0)};
    vw.slot[ps.z] = {g2.x * s, g2.y * s, g2.z * s, R(0)};
    vw.slot[ps.w] = {g3.x * s, g3.y * s, g3.z * s, R(0)};
  }
  K3D_FOR(s, a.ns) {
    const uint4 id = __ldg(&a.s_idx[s]);
    const uint2 ps = __ldg(&a.s_pos[s]);
    const R4<R> dq = vw.s_dq[s];
    const R k = vw.s_k[s];
    const R4<R> ci = next_dir<R>(vw.cw[id.x], beta), cj = next_dir<R>(vw.cw[id.y], beta);
    const R dx = ci.x - cj.x, dy = ci.y - cj.y, dz = ci.z - cj.z;
    const R nd = (dq.x * dx + dq.y * dy + dq.z * dz) * (R(1) - dq.w);
    const R ox = k * (dq.x * nd + dx * dq.w), oy = k * (dq.y * nd + dy * dq.w), oz = k * (dq.z * nd + dz * dq.w);
    vw.slot[ps.x] = {ox, oy, oz, R(0)};
    vw.slot[ps.y] = {-ox, -oy, -oz, R(0)};
  }
}

// The operator in FP64 applied to dv, from the FP64 record copies: the
// residuals of the mixed form (start, reliable updates, release test).
__device__ __noinline__ void apply_dv64(const StepArgs& a) {
  const R4<double>* f1w = static_cast<const R4<double>*>(a.m_f1w64);
  const R4<double>* f2w = static_cast<const R4<double>*>(a.m_f2w64);
  const R4<double>* kgB = static_cast<const R4<double>*>(a.m_kgB64);
  const R4<double>* rin = static_cast<const R4<double>*>(a.m_rin64);
  const R4<double>* kgA = static_cast<const R4<double>*>(a.m_kgA64);
  const R4<double>* grad = static_cast<const R4<double>*>(a.b_grad64);
  const R4<double>* sdq = static_cast<const R4<double>*>(a.s_dq64);
  const double* sk = static_cast<const double*>(a.s_k64);
  R4<double>* slot = static_cast<R4<double>*>(a.slot64);
  auto dvp = [&](uint32_t i) -> R4<double> {
    const D3 d = ld3(a.dv, i);
    return {d.x, d.y, d.z, 0.0};
  };
  K3D_FOR(t, a.nt) {
    const uint4 id = __ldg(&a.m_idx[t]);
    const uint4 ps = __ldg(&a.m_pos[t]);
    const R4<double> d[3] = {dvp(id.x), dvp(id.y), dvp(id.z)};
    R4<double> out[3];
    membran_hv<double>(f1w[t], f2w[t], rin[t], kgA[t], kgB[t], d, out);
    slot[ps.x] = out[0];
    slot[ps.y] = out[1];
    slot[ps.z] = out[2];
  }
  K3D_FOR(b, a.nb) {
    const uint4 id = __ldg(&a.b_idx[b]);
    const uint4 ps = __ldg(&a.b_pos[b]);
    const R4<double> g0 = grad[4 * b], g1 = grad[4 * b + 1], g2 = grad[4 * b + 2], g3 = grad[4 * b + 3];
    const R4<double> c0 = dvp(id.x), c1 = dvp(id.y), c2 = dvp(id.z), c3 = dvp(id.w);
    const double gp = g1.x * (c1.x - c0.x) + g1.y * (c1.y - c0.y) + g1.z * (c1.z - c0.z) + g2.x * (c2.x - c0.x) +
                      g2.y * (c2.y - c0.y) + g2.z * (c2.z - c0.z) + g3.x * (c3.x - c0.x) + g3.y * (c3.y - c0.y) +
                      g3.z * (c3.z - c0.z);
    const double sc = g0.w * gp;
    slot[ps.x] = {g0.x * sc, g0.y * sc, g0.z * sc, 0.0};
    slot[ps.y] = {g1.x * sc, g1.y * sc, g1.z * sc, 0.0};
    slot[ps.z] = {g2.x * sc, g2.y * sc, g2.z * sc, 0.0};
    slot[ps.w] = {g3.x * sc, g3.y * sc, g3.z * sc, 0.0};
  }
  K3D_FOR(s, a.ns) {
    const uint4 id = __ldg(&a.s_idx[s]);
    const uint2 ps = __ldg(&a.s_pos[s]);
    const R4<double> dq = sdq[s];
    const double k = sk[s];
    const R4<double> ci = dvp(id.x), cj = dvp(id.y);
    const double dx = ci.x - cj.x, dy = ci.y - cj.y, dz = ci.z - cj.z;
    const double nd = (dq.x * dx + dq.y * dy + dq.z * dz) * (1.0 - dq.w);
    const double ox = k * (dq.x * nd + dx * dq.w), oy = k * (dq.y * nd + dy * dq.w), oz = k * (dq.z * nd + dz * dq.w);
    slot[ps.x] = {ox, oy, oz, 0.0};
    slot[ps.y] = {-ox, -oy, -oz, 0.0};
  }
}

// (A dv)_i in FP64 from the slots of apply_dv64.
__device__ __noinline__ D3 a_dv64(const StepArgs& a, int64_t i) {
  const R4<double>* sl = static_cast<const R4<double>*>(a.slot64) + i;
  double x = 0, y = 0, z = 0;
  const uint32_t cnt = __ldg(&a.cnt_v[i]);
#pragma unroll 6
  for (uint32_t k = 0; k < cnt; ++k) {
    const R4<double> o = sl[size_t(k) * a.np];
    x += o.x;
    y += o.y;
    z += o.z;
  }
  const double h2 = a.h * a.h, md = a.masse[i] * (1.0 + a.h * a.daempf);
  const D3 d = ld3(a.dv, uint32_t(i));
  return d3(md * d.x + h2 * x, md * d.y + h2 * y, md * d.z + h2 * z);
}

// H p at point i: the sum of its corner slots, rank by rank (coalesced over
// consecutive points).
template <typename R>
__device__ __forceinline__ void gather_h(const StepArgs& a, const View<R>& vw, int64_t i, R& hx, R& hy, R& hz) {
  R x = 0, y = 0, z = 0;
  const uint32_t cnt = __ldg(&a.cnt_v[i]);
  const R4<R>* sl = vw.slot + i;
#pragma unroll 6
  for (uint32_t k = 0; k < cnt; ++k) {
    const R4<R> o = sl[size_t(k) * a.np];
    x += o.x;
    y += o.y;
    z += o.z;
  }
  hx = x;
  hy = y;
  hz = z;
}

template <typename R>
__device__ __forceinline__ void filt(const R* nrm, int64_t i, R& x, R& y, R& z) {
  const R nx = nrm[3 * i], ny = nrm[3 * i + 1], nz = nrm[3 * i + 2];
  const R d = x * nx + y * ny + z * nz;
  x -= nx * d;
  y -= ny * d;
  z -= nz * d;
}

template <typename R>
__device__ __forceinline__ void pmul(const R* P, int64_t i, R x, R y, R z, R& ox, R& oy, R& oz) {
  const R p0 = P[6 * i], p1 = P[6 * i + 1], p2 = P[6 * i + 2], p3 = P[6 * i + 3], p4 = P[6 * i + 4],
          p5 = P[6 * i + 5];
  ox = p0 * x + p3 * y + p4 * z;
  oy = p3 * x + p1 * y + p5 * z;
  oz = p4 * x + p5 * y + p2 * z;
}

// w = (R) dv, c = 0: the next element pass with beta = 0 applies A to dv.
template <typename R>
__device__ void dv_to_w(const StepArgs& a, const View<R>& vw) {
  K3D_FOR(i, a.n) {
    const D3 d = ld3(a.dv, uint32_t(i));
    vw.cw[i].w = {R(d.x), R(d.y), R(d.z), R(0)};
    vw.cw[i].c = {R(0), R(0), R(0), R(0)};
  }
}

// ------------------------------------------------------------ assembled A
// A = M(1+hc) + h^2 H as 3x3 blocks (implizit.rs:185-229 written out per
// point pair), from the FP64 records of this step. Each block adds its
// contributions in the fixed order of its list, so the assembly is
// deterministic. Membrane block (a, b): J_a^T kg J_b + s_ab I with the rows
// of J_k = (2 c1_k f1, 2 c2_k f2, 2 c2_k f1 + 2 c1_k f2) and s_ab the
// geometric term (kontinuum.rs:616-708); bend block: k g_a g_b^T; spring
// block: +-k (n n^T (1 - q) + q I).
template <typename R>
__global__ void __launch_bounds__(kBlock) assemble_kernel(const __grid_constant__ StepArgs a) {
  const bool own = sizeof(R) == 8;
  const R4<double>* f1w = static_cast<const R4<double>*>(own ? a.m_f1w : a.m_f1w64);
  const R4<double>* f2w = static_cast<const R4<double>*>(own ? a.m_f2w : a.m_f2w64);
  const R4<double>* kgB = static_cast<const R4<double>*>(own ? a.m_kgB : a.m_kgB64);
  const R4<double>* rin = static_cast<const R4<double>*>(own ? a.m_rin : a.m_rin64);
  const R4<double>* kgA = static_cast<const R4<double>*>(own ? a.m_kgA : a.m_kgA64);
  const R4<double>* grad = static_cast<const R4<double>*>(own ? a.b_grad : a.b_grad64);
  const R4<double>* sdq = static_cast<const R4<double>*>(own ? a.s_dq : a.s_dq64);
  const double* sk = static_cast<const double*>(own ? a.s_k : a.s_k64);
  R* bm = static_cast<R*>(a.bmat);
  const double h2 = a.h * a.h;
  K3D_FOR(sid, a.bplane) {
    const int64_t i = sid % a.np, k = sid / a.np;
    if (i >= a.n || k >= int64_t(__ldg(&a.row_cnt[i]))) continue;
    double B[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t e = __ldg(&a.ctr_off[sid]); e < __ldg(&a.ctr_off[sid + 1]); ++e) {
      const uint32_t code = __ldg(&a.ctr[e]);
      const uint32_t ty = code >> 30, ca = (code >> 28) & 3u, cb = (code >> 26) & 3u, id = code & 0x3ffffffu;
      if (ty == 0) {
        const R4<double> F1 = f1w[id], F2 = f2w[id], KB = kgB[id], RI = rin[id], KA = kgA[id];
        const double c1[3] = {-(RI.x + RI.z), RI.x, RI.z}, c2[3] = {-(RI.y + RI.w), RI.y, RI.w};
        const D3 f1 = d3(F1.x, F1.y, F1.z), f2 = d3(F2.x, F2.y, F2.z);
        const D3 ja[3] = {f1 * (2.0 * c1[ca]), f2 * (2.0 * c2[ca]), f1 * (2.0 * c2[ca]) + f2 * (2.0 * c1[ca])};
        const D3 jb[3] = {f1 * (2.0 * c1[cb]), f2 * (2.0 * c2[cb]), f1 * (2.0 * c2[cb]) + f2 * (2.0 * c1[cb])};
        const double K[3][3] = {{KA.x, KA.w, KB.x}, {KA.w, KA.y, KB.y}, {KB.x, KB.y, KA.z}};
        D3 u[3];  // u_p = sum_q K[p][q] jb_q
#pragma unroll
        for (int pp = 0; pp < 3; ++pp) u[pp] = jb[0] * K[pp][0] + jb[1] * K[pp][1] + jb[2] * K[pp][2];
        const double sab =
            2.0 * (F1.w * c1[ca] * c1[cb] + F2.w * c2[ca] * c2[cb] + KB.z * (c1[ca] * c2[cb] + c2[ca] * c1[cb]));
        double H[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int pp = 0; pp < 3; ++pp) {
          H[0] += ja[pp].x * u[pp].x;
          H[1] += ja[pp].x * u[pp].y;
          H[2] += ja[pp].x * u[pp].z;
          H[3] += ja[pp].y * u[pp].x;
          H[4] += ja[pp].y * u[pp].y;
          H[5] += ja[pp].y * u[pp].z;
          H[6] += ja[pp].z * u[pp].x;
          H[7] += ja[pp].z * u[pp].y;
          H[8] += ja[pp].z * u[pp].z;
        }
        H[0] += sab;
        H[4] += sab;
        H[8] += sab;
#pragma unroll
        for (int q = 0; q < 9; ++q) B[q] += h2 * H[q];
      } else if (ty == 1) {
        const R4<double> ga = grad[4 * size_t(id) + ca], gb = grad[4 * size_t(id) + cb];
        const double kk = h2 * ga.w;
        const double gav[3] = {ga.x, ga.y, ga.z}, gbv[3] = {gb.x, gb.y, gb.z};
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) B[3 * r + c] += kk * gav[r] * gbv[c];
      } else {
        const R4<double> dq = sdq[id];
        const double kk = h2 * sk[id] * (ca == cb ? 1.0 : -1.0);
        const double nv[3] = {dq.x, dq.y, dq.z};
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) B[3 * r + c] += kk * (nv[r] * nv[c] * (1.0 - dq.w) + (r == c ? dq.w : 0.0));
      }
    }
    if (int64_t(__ldg(&a.col[sid])) == i) {
      const double md = a.masse[i] * (1.0 + a.h * a.daempf);
      B[0] += md;
      B[4] += md;
      B[8] += md;
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) bm[q * a.bplane + sid] = R(B[q]);
  }
}

// (A p)_i = sum over the row's blocks of B p_col, p = w + beta c from `buf`.
template <typename R>
__device__ __forceinline__ void bsr_row(const StepArgs& a, const CW<R>* buf, int64_t i, R beta, R& ox, R& oy,
                                        R& oz) {
  const R* bm = static_cast<const R*>(a.bmat);
  const int64_t P = a.bplane;
  R x = 0, y = 0, z = 0;
  const uint32_t cnt = __ldg(&a.row_cnt[i]);
#pragma unroll 2
  for (uint32_t k = 0; k < cnt; ++k) {
    const int64_t sid = int64_t(k) * a.np + i;
    const uint32_t j = __ldg(&a.col[sid]);
    const R4<R> pj = next_dir<R>(buf[j], beta);
    x += bm[sid] * pj.x + bm[P + sid] * pj.y + bm[2 * P + sid] * pj.z;
    y += bm[3 * P + sid] * pj.x + bm[4 * P + sid] * pj.y + bm[5 * P + sid] * pj.z;
    z += bm[6 * P + sid] * pj.x + bm[7 * P + sid] * pj.y + bm[8 * P + sid] * pj.z;
  }
  ox = x;
  oy = y;
  oz = z;
}

// ------------------------------------------------------------ PCG
// implizit.rs:370-426 with the assembled A, two grid syncs per iteration:
//   points: c = w + beta c (neighbours' from one (c, w) buffer, own written to
//           the other), ap = S A c, c.ap                            -> sum
//   points: dv += alpha c, r -= alpha ap, z = P r, w = S z, r.z       -> sum
// The mixed form takes its residuals (start, reliable updates) from the FP64
// operator. Returns false on a barrier error.
template <typename R>
__device__ bool pcg(const StepArgs& a, const View<R>& vw, Shared& sh, int64_t& iters, bool& unconverged,
                    bool& breakdown, double& rest) {
  CW<R>* cur = static_cast<CW<R>*>(a.c);
  CW<R>* nxt = static_cast<CW<R>*>(a.cw2);
  const bool hi = a.m_f1w64 != nullptr;
  // start: pinned points 0, held points get their normal target
  K3D_FOR(i, a.n) {
    D3 d = ld3(a.dv, uint32_t(i));
    if (!a.frei[i]) {
      d = d3(0, 0, 0);
    } else {
      const D3 n = ld3(a.nrm_d, uint32_t(i));
      if (n.x != 0.0 || n.y != 0.0 || n.z != 0.0) {
        const double soll = a.vn_soll[i] - dot(ld3(a.v, uint32_t(i)), n);
        d = (d - n * dot(d, n)) + n * soll;
      }
    }
    st3(a.dv, uint32_t(i), d);
    cur[i].w = {R(d.x), R(d.y), R(d.z), R(0)};
    cur[i].c = {R(0), R(0), R(0), R(0)};
  }
  if (!barrier(a, sh)) return false;
  if (hi) {
    apply_dv64(a);
    if (!barrier(a, sh)) return false;
  }
  double red[2] = {0.0, 0.0};
  K3D_FOR(i, a.n) {
    R rx = 0, ry = 0, rz = 0, zx = 0, zy = 0, zz = 0, cx = 0, cy = 0, cz = 0;
    if (a.frei[i]) {
      const D3 b = ld3(a.b, uint32_t(i));
      D3 ad;
      if (hi) {
        ad = a_dv64(a, i);
      } else {
        R hx, hy, hz;
        bsr_row<R>(a, cur, i, R(0), hx, hy, hz);
        ad = d3(double(hx), double(hy), double(hz));
      }
      const D3 n = ld3(a.nrm_d, uint32_t(i));
      D3 rd = b - ad;
      rd = rd - n * dot(rd, n);
      rx = R(rd.x);
      ry = R(rd.y);
      rz = R(rd.z);
      R fx = R(b.x), fy = R(b.y), fz = R(b.z);
      filt<R>(vw.nrm, i, fx, fy, fz);
      R px, py, pz;
      pmul<R>(vw.pinv, i, fx, fy, fz, px, py, pz);
      red[1] += double(fx) * double(px) + double(fy) * double(py) + double(fz) * double(pz);
      pmul<R>(vw.pinv, i, rx, ry, rz, zx, zy, zz);
      cx = zx;
      cy = zy;
      cz = zz;
      filt<R>(vw.nrm, i, cx, cy, cz);
      red[0] += double(rx) * double(cx) + double(ry) * double(cy) + double(rz) * double(cz);
    }
    vw.r[3 * i] = rx;
    vw.r[3 * i + 1] = ry;
    vw.r[3 * i + 2] = rz;
    nxt[i].w = {cx, cy, cz, R(0)};  // the first direction: w + 0 c
    nxt[i].c = {R(0), R(0), R(0), R(0)};
  }
  if (!grid_sync<2>(a, sh, red)) return false;
  {
    CW<R>* t = cur;
    cur = nxt;
    nxt = t;
  }
  double delta = red[0];
  const double bb = red[1];
  const double tol = sizeof(R) == 4 ? fmax(a.tol, kMixedTolFloor) : a.tol;
  const double ziel = fmax(tol * tol * fmax(bb, delta), a.boden);
  int64_t it = 0;
  double beta = 0.0, delta_ref = delta;
  breakdown = false;
  while (delta > ziel && it < a.cg_max) {
    const R rb = R(beta);
    // ca = c.Ac and, for the FP32 operator, cm = c.M(1+hc)c: the Hessian part
    // is positive semi-definite, so c.Ac >= cm holds exactly; an FP32 product
    // that falls far below it has lost the direction and the solve stops
    // there as at a breakdown (the FP64 form keeps the reference's test only).
    double ca[2] = {0.0, 0.0};
    K3D_FOR(i, a.n) {
      const R4<R> ci = next_dir<R>(cur[i], rb);
      nxt[i].c = ci;
      R ax = 0, ay = 0, az = 0;
      if (a.frei[i]) {
        bsr_row<R>(a, cur, i, rb, ax, ay, az);
        filt<R>(vw.nrm, i, ax, ay, az);
        if (sizeof(R) == 4) {
          const double m = double(vw.md[i]);
          ca[1] += m * (double(ci.x) * double(ci.x) + double(ci.y) * double(ci.y) + double(ci.z) * double(ci.z));
        }
      }
      vw.ap[3 * i] = ax;
      vw.ap[3 * i + 1] = ay;
      vw.ap[3 * i + 2] = az;
      ca[0] += double(ci.x) * double(ax) + double(ci.y) * double(ay) + double(ci.z) * double(az);
    }
    if (sizeof(R) == 4) {
      if (!grid_sync<2>(a, sh, ca)) return false;
    } else {
      double c1[1] = {ca[0]};
      if (!grid_sync<1>(a, sh, c1)) return false;
      ca[0] = c1[0];
    }
    if (ca[0] <= DBL_MIN || !isfinite(ca[0]) || (sizeof(R) == 4 && ca[0] < 0.5 * ca[1])) {
      breakdown = true;
      break;
    }
    const double alpha = delta / ca[0];
    double rzs[1] = {0.0};
    K3D_FOR(i, a.n) {
      const R4<R> ci = nxt[i].c;
      D3 d = ld3(a.dv, uint32_t(i));
      d = d + d3(double(ci.x), double(ci.y), double(ci.z)) * alpha;
      st3(a.dv, uint32_t(i), d);
      const R rx = R(double(vw.r[3 * i]) - alpha * double(vw.ap[3 * i]));
      const R ry = R(double(vw.r[3 * i + 1]) - alpha * double(vw.ap[3 * i + 1]));
      const R rzz = R(double(vw.r[3 * i + 2]) - alpha * double(vw.ap[3 * i + 2]));
      vw.r[3 * i] = rx;
      vw.r[3 * i + 1] = ry;
      vw.r[3 * i + 2] = rzz;
      R zx, zy, zz;
      pmul<R>(vw.pinv, i, rx, ry, rzz, zx, zy, zz);
      if (!a.frei[i]) zx = zy = zz = 0;
      R wx = zx, wy = zy, wz = zz;
      filt<R>(vw.nrm, i, wx, wy, wz);
      nxt[i].w = {wx, wy, wz, R(0)};
      rzs[0] += double(rx) * double(zx) + double(ry) * double(zy) + double(rzz) * double(zz);
    }
    if (!grid_sync<1>(a, sh, rzs)) return false;
    double beta_next = rzs[0] / delta;
    const double delta_prev = delta;
    delta = rzs[0];
    if (hi && (delta < kReliable * delta_ref || delta > kGrow * delta_ref)) {
      // reliable update: replace the recursive FP32 residual by the true one,
      // S (b - A dv) with the FP64 operator; restart the direction if the
      // residual grew
      const bool restart = delta > kGrow * delta_ref;
      apply_dv64(a);
      if (!barrier(a, sh)) return false;
      double rz2[1] = {0.0};
      K3D_FOR(i, a.n) {
        R rx = 0, ry = 0, rz = 0, zx = 0, zy = 0, zz = 0, wx = 0, wy = 0, wz = 0;
        if (a.frei[i]) {
          const D3 n = ld3(a.nrm_d, uint32_t(i));
          D3 rd = ld3(a.b, uint32_t(i)) - a_dv64(a, i);
          rd = rd - n * dot(rd, n);
          rx = R(rd.x);
          ry = R(rd.y);
          rz = R(rd.z);
          pmul<R>(vw.pinv, i, rx, ry, rz, zx, zy, zz);
          wx = zx;
          wy = zy;
          wz = zz;
          filt<R>(vw.nrm, i, wx, wy, wz);
          rz2[0] += double(rx) * double(zx) + double(ry) * double(zy) + double(rz) * double(zz);
        }
        vw.r[3 * i] = rx;
        vw.r[3 * i + 1] = ry;
        vw.r[3 * i + 2] = rz;
        nxt[i].w = {wx, wy, wz, R(0)};
      }
      if (!grid_sync<1>(a, sh, rz2)) return false;
      delta = rz2[0];
      beta_next = restart ? 0.0 : delta / delta_prev;
      delta_ref = delta;
    }
    beta = beta_next;
    {
      CW<R>* t = cur;
      cur = nxt;
      nxt = t;
    }
    ++it;
  }
  iters = it;
  unconverged = delta > ziel;
  rest = sqrt(delta / fmax(bb, a.boden));
  return true;
}

// ------------------------------------------------------------ release pass
// implizit.rs:924-942: normal force from the residual A dv - b along the
// contact normal; a held point that pulls on the body is released.
template <typename R>
__device__ bool release(const StepArgs& a, const View<R>& vw, Shared& sh, double& released) {
  const bool hi = a.m_f1w64 != nullptr;
  if (hi)
    apply_dv64(a);
  else
    dv_to_w<R>(a, vw);
  if (!barrier(a, sh)) return false;
  double cnt[1] = {0.0};
  K3D_FOR(i, a.n) {
    const D3 n = ld3(a.nrm_d, uint32_t(i));
    if (n.x == 0.0 && n.y == 0.0 && n.z == 0.0) continue;
    const D3 b = ld3(a.b, uint32_t(i));
    D3 rest;
    if (hi) {
      rest = a_dv64(a, i) - b;
    } else {
      R hx, hy, hz;
      bsr_row<R>(a, vw.cw, i, R(0), hx, hy, hz);
      rest = d3(double(hx), double(hy), double(hz)) - b;
    }
    const double fn = dot(rest, n) / a.h;
    if (fn < 0.0) {
      st3(a.nrm_d, uint32_t(i), d3(0, 0, 0));
      vw.nrm[3 * i] = vw.nrm[3 * i + 1] = vw.nrm[3 * i + 2] = R(0);
      cnt[0] += 1.0;
    } else {
      a.fnk[i] = fn;
    }
  }
  if (!grid_sync<1>(a, sh, cnt)) return false;
  released = cnt[0];
  return true;
}

// ------------------------------------------------------------ friction + integration
// implizit.rs:957-1013 (no mesh bodies: the segment check does not apply).
__device__ void integrate(const StepArgs& a, double (&cnt)[3]) {
  const double h = a.h;
  K3D_FOR(i, a.n) {
    if (!a.frei[i]) continue;
    D3 v = ld3(a.v, uint32_t(i)) + ld3(a.dv, uint32_t(i));
    const D3 n = ld3(a.nrm_d, uint32_t(i));
    if (n.x != 0.0 || n.y != 0.0 || n.z != 0.0) {
      cnt[0] += 1.0;
      const D3 vb = ld3(a.vk, uint32_t(i));
      const D3 rel = v - vb;
      const D3 t = rel - n * dot(rel, n);
      const double lt = norm(t);
      const double normal = a.normal_aus_last ? fmax(-dot(ld3(a.load, uint32_t(i)), n), 0.0) : a.fnk[i];
      const double grenze = a.reib[i] * normal * h * a.w[i];
      if (lt <= grenze) {
        cnt[1] += 1.0;
        v = v - t;
      } else if (lt > 0.0) {
        v = v - t * (grenze / lt);
      }
    }
    D3 x = ld3(a.x, uint32_t(i)) + v * h;
    for (int kb = 0; kb < a.n_bodies; ++kb) {
      D3 nn;
      double tiefe;
      if (kontakt(a.bodies[kb], x, a.kabst[i], nn, tiefe)) {
        x = x + nn * tiefe;
        const D3 bv = d3(a.bodies[kb].vel[0], a.bodies[kb].vel[1], a.bodies[kb].vel[2]);
        const double vn = dot(v - bv, nn);
        if (vn < 0.0) v = v - nn * vn;
      }
    }
    if (!(isfinite(x.x) && isfinite(x.y) && isfinite(x.z) && isfinite(v.x) && isfinite(v.y) && isfinite(v.z)))
      cnt[2] += 1.0;
    st3(a.x, uint32_t(i), x);
    st3(a.v, uint32_t(i), v);
  }
}

// ------------------------------------------------------------ kernels
// Build (elements): an ordinary grid-stride launch at full occupancy.
template <typename R>
__global__ void __launch_bounds__(kBlock) build_elements_kernel(const __grid_constant__ StepArgs a) {
  const View<R> vw(a);
  build_elements<R>(a, vw);
}

// Build (points): rhs, preconditioner, contact set; counts held points.
template <typename R>
__global__ void __launch_bounds__(kBlock) build_points_kernel(const __grid_constant__ StepArgs a) {
  __shared__ double red[32];
  const View<R> vw(a);
  double held = 0.0;
  build_points<R>(a, vw, held);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) held += __shfl_xor_sync(0xffffffffu, held, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = held;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t += red[w];
    if (t > 0.0) atomicAdd(reinterpret_cast<unsigned long long*>(&a.stats[ST_HELD]), (unsigned long long)t);
  }
}

// PCG with the release test (persistent, cooperative): MODE_STEP runs up to
// two solves with a release pass after each, MODE_SOLVE one solve. One block
// of 512 threads per SM in both precisions: the iteration is bound by the two
// grid barriers, whose cost grows with the number of arriving blocks, and the
// 128 registers a thread gets at this shape keep the FP32 form free of spills.
template <typename R>
__global__ void __launch_bounds__(kSolveBlock, 1) solve_kernel(const __grid_constant__ StepArgs a) {
  __shared__ Shared sh;
  if (threadIdx.x == 0) {
    sh.epoch = 0;
    sh.rbuf = 0;
    sh.err = 0;
  }
  __syncthreads();
  const View<R> vw(a);
  const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
  const bool any_held = a.stats[ST_HELD] > 0;
  int64_t iters = 0;
  bool unconv = false, brk = false;
  double rest = 0.0;
  for (int pass = 0; pass < 2; ++pass) {
    if (!pcg<R>(a, vw, sh, iters, unconv, brk, rest)) return;
    double dvm[1] = {0.0};
    K3D_FOR(i, a.n) {
      const D3 d = ld3(a.dv, uint32_t(i));
      dvm[0] = fmax(dvm[0], fmax(fabs(d.x), fmax(fabs(d.y), fabs(d.z))));
    }
    if (!grid_max(a, sh, dvm)) return;
    if (lead) {
      a.stats[ST_CG_ITERATIONS] += iters;
      a.stats[ST_SOLVES] += 1;
      if (unconv) a.stats[ST_UNCONVERGED] += 1;
      if (brk) a.stats[ST_BREAKDOWNS] += 1;
      a.stat_rest_max[0] = fmax(a.stat_rest_max[0], rest);
      a.stats[ST_LAST_ITERATIONS] = iters;
    }
    if (a.mode == MODE_SOLVE) return;
    if (!any_held) break;
    double rel = 0.0;
    if (!release<R>(a, vw, sh, rel)) return;
    if (lead) a.stats[ST_RELEASED] += int64_t(rel);
    if (rel == 0.0) break;
  }
}

// Friction and integration; counts contacts, sticking and non-finite points.
__global__ void __launch_bounds__(kBlock) integrate_kernel(const __grid_constant__ StepArgs a) {
  __shared__ double red[3][32];
  double cnt[3] = {0.0, 0.0, 0.0};
  integrate(a, cnt);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double x = cnt[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int slot[3] = {ST_CONTACTS, ST_STICKING, ST_NONFINITE};
    for (int k = 0; k < 3; ++k) {
      double t = 0.0;
      for (int w = 0; w < int(blockDim.x >> 5); ++w) t += red[k][w];
      if (t > 0.0) atomicAdd(reinterpret_cast<unsigned long long*>(&a.stats[slot[k]]), (unsigned long long)t);
    }
  }
}

// Probes: c = p (or v), then the element products, then per point
// A c (MODE_OPERATOR), A c - b (MODE_RESIDUAL) or f = b/h + h H v (MODE_SYSTEM).
template <typename R>
__global__ void __launch_bounds__(kBlock) probe_load_kernel(const __grid_constant__ StepArgs a) {
  const View<R> vw(a);
  const double* src = a.mode == MODE_SYSTEM ? a.v : a.p_in;
  K3D_FOR(i, a.n) {
    const D3 q = ld3(src, uint32_t(i));
    vw.cw[i].w = {R(q.x), R(q.y), R(q.z), R(0)};
    vw.cw[i].c = {R(0), R(0), R(0), R(0)};
  }
}
template <typename R>
__global__ void __launch_bounds__(kBlock) apply_kernel(const __grid_constant__ StepArgs a) {
  const View<R> vw(a);
  apply_elements<R>(a, vw, R(0));
}
template <typename R>
__global__ void __launch_bounds__(kBlock) probe_out_kernel(const __grid_constant__ StepArgs a) {
  const View<R> vw(a);
  const double h2 = a.h * a.h;
  K3D_FOR(i, a.n) {
    R hx, hy, hz;
    gather_h<R>(a, vw, i, hx, hy, hz);
    const D3 b = ld3(a.b, uint32_t(i));
    if (a.mode == MODE_SYSTEM) {
      st3(a.p_out, uint32_t(i), b * (1.0 / a.h) + d3(double(hx), double(hy), double(hz)) * a.h);
      continue;
    }
    const R4<R> ci = vw.cw[i].w;
    const R m = vw.md[i];
    D3 o = d3(double(m * ci.x + R(h2) * hx), double(m * ci.y + R(h2) * hy), double(m * ci.z + R(h2) * hz));
    if (a.mode == MODE_RESIDUAL) o = o - b;
    st3(a.p_out, uint32_t(i), o);
  }
}

// ------------------------------------------------------------ launch
template <typename R>
struct Kernels {
  static void* be() { return (void*)build_elements_kernel<R>; }
  static void* bp() { return (void*)build_points_kernel<R>; }
  static void* sv() { return (void*)solve_kernel<R>; }
  static void* pl() { return (void*)probe_load_kernel<R>; }
  static void* ap() { return (void*)apply_kernel<R>; }
  static void* po() { return (void*)probe_out_kernel<R>; }
  static void* as() { return (void*)assemble_kernel<R>; }
};

static int g_solve_blocks[2] = {0, 0};
static int g_sms = 0;

int step_grid_blocks(int precision, int device) {
  const int idx = precision == 0 ? 0 : 1;
  if (g_solve_blocks[idx] > 0) return g_solve_blocks[idx];
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return -1;
  g_sms = prop.multiProcessorCount;
  int per_sm = 0;
  const void* fn = idx == 0 ? Kernels<double>::sv() : Kernels<float>::sv();
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kSolveBlock, 0) != cudaSuccess || per_sm < 1)
    return -1;
  g_solve_blocks[idx] = prop.multiProcessorCount * per_sm;
  return g_solve_blocks[idx];
}

static cudaError_t plain(const void* fn, const StepArgs& a, int64_t work, cudaStream_t st) {
  int64_t blocks = (work + kBlock - 1) / kBlock;
  const int64_t cap = int64_t(g_sms > 0 ? g_sms : 148) * 16;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  void* args[] = {(void*)&a};
  return cudaLaunchKernel(fn, dim3(unsigned(blocks)), dim3(kBlock), args, 0, st);
}

static cudaError_t cooperative(const void* fn, const StepArgs& a, int blocks, cudaStream_t st) {
  void* args[] = {(void*)&a};
  return cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(kSolveBlock), args, 0, st);
}

template <typename R>
static cudaError_t launch_t(const StepArgs& a, int blocks, cudaStream_t st, int& launched) {
  cudaError_t e;
  const int64_t elems = a.nt > a.nb ? (a.nt > a.ns ? a.nt : a.ns) : (a.nb > a.ns ? a.nb : a.ns);
  if ((e = cudaMemsetAsync(&a.sync->count, 0, sizeof(unsigned), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(&a.stats[ST_HELD], 0, sizeof(long long), st)) != cudaSuccess) return e;
  if ((e = plain(Kernels<R>::be(), a, elems, st)) != cudaSuccess) return e;
  if ((e = plain(Kernels<R>::bp(), a, a.n, st)) != cudaSuccess) return e;
  launched = 2;
  if (a.mode == MODE_SYSTEM && !a.p_out) return cudaSuccess;
  if (a.mode == MODE_OPERATOR || a.mode == MODE_RESIDUAL || a.mode == MODE_SYSTEM) {
    if ((e = plain(Kernels<R>::pl(), a, a.n, st)) != cudaSuccess) return e;
    if ((e = plain(Kernels<R>::ap(), a, elems, st)) != cudaSuccess) return e;
    if ((e = plain(Kernels<R>::po(), a, a.n, st)) != cudaSuccess) return e;
    launched += 3;
    return cudaSuccess;
  }
  if (a.ev_solve0 && (e = cudaEventRecord(a.ev_solve0, st)) != cudaSuccess) return e;
  if ((e = plain(Kernels<R>::as(), a, a.bplane, st)) != cudaSuccess) return e;
  launched += 1;
  if ((e = cooperative(Kernels<R>::sv(), a, blocks, st)) != cudaSuccess) return e;
  if (a.ev_solve1 && (e = cudaEventRecord(a.ev_solve1, st)) != cudaSuccess) return e;
  launched += 1;
  if (a.mode == MODE_STEP) {
    if ((e = plain((const void*)integrate_kernel, a, a.n, st)) != cudaSuccess) return e;
    launched += 1;
  }
  return cudaSuccess;
}

cudaError_t launch_step(const StepArgs& a, int precision, int blocks, cudaStream_t stream, int& launched) {
  launched = 0;
  return precision == 0 ? launch_t<double>(a, blocks, stream, launched) : launch_t<float>(a, blocks, stream, launched);
}

}  // namespace k3d
