// Shared device views and helpers of the step kernels (internal to the
// library): the typed view of the step's arrays, the (c, w) pair of the CG
// and the per-point helpers used by both the build and the solve kernels.
#pragma once
#include <cstdint>

#include "k3d_device.cuh"
#include "k3d_step.h"

namespace k3d {

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

// Springs of self-collision (proximity pairs, then the push springs of
// penetration regions; up to five points each) at point i in FP64
// (implizit.rs:214-220, 267-276): over
// the point's incidence entries, B times the sum over the pair's other side
// of om (p_i - p_r) with om = -g_q g_r > 0. `dg` (if given) receives
// sum om B, the springs' part of the diagonal block (xx, yy, zz, xy, xz, yz).
template <typename P>
__device__ __forceinline__ D3 feder_hp64(const StepArgs& a, int64_t i, P&& p, double* dg) {
  D3 out = d3(0.0, 0.0, 0.0);
  const D3 pi = p(uint32_t(i));
  for (uint32_t e = a.sc_off[i]; e < a.sc_off[i + 1]; ++e) {
    const uint32_t ent = a.sc_ent[e], q = ent >> 3, k = ent & 7u;
    const uint4 id = a.sc_idx[q];
    const double4 g4 = a.sc_w[q];
    const double g[5] = {g4.x, g4.y, g4.z, g4.w, a.sc_g5[q]};
    const uint32_t ix[5] = {id.x, id.y, id.z, id.w, a.sc_x5[q]};
    const double gk = g[k];
    D3 sm = d3(0.0, 0.0, 0.0);
    double so = 0.0;
#pragma unroll
    for (int r = 0; r < 5; ++r)
      if ((gk > 0.0 && g[r] < 0.0) || (gk < 0.0 && g[r] > 0.0)) {
        const double om = -gk * g[r];
        sm = sm + (pi - p(ix[r])) * om;
        so += om;
      }
    const double4 b0 = a.sc_b0[q], b1 = a.sc_b1[q];
    out = out + d3(b0.x * sm.x + b0.w * sm.y + b1.x * sm.z, b0.w * sm.x + b0.y * sm.y + b1.y * sm.z,
                   b1.x * sm.x + b1.y * sm.y + b0.z * sm.z);
    if (dg) {
      dg[0] += so * b0.x;
      dg[1] += so * b0.y;
      dg[2] += so * b0.z;
      dg[3] += so * b0.w;
      dg[4] += so * b1.x;
      dg[5] += so * b1.y;
    }
  }
  return out;
}

}  // namespace k3d
