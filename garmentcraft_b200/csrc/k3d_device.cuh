// Device-side data layout and element math of the implicit cloth step.
//
// Layout in HBM (structure of arrays; N points, T membranes, B bending
// constraints, S springs = stiff pattern edges + seams):
//   per point   x, v, dv, b, v_koerper: double[3N]      (streamed per point)
//               r, z, ap: R[3N]; pinv: R[6N] (symmetric); normal: R[3N]
//               c (CG direction, gathered by elements): R4[N]
//   per membrane  idx uint4, r4/basis/mat double4 (scene constants),
//                 f1w/f2w/rin/kgA/kgB R4 (operator record, rebuilt per step)
//   per bend      idx uint4, (k, rest) double2, grad R4[4] (grad[0].w = k)
//   per spring    idx uint4 (i, j, kind), (k, rest) double2, (dir, quer) R4
//   per point CSR of incident (membrane, corner), (bend, corner), (spring, end)
// The element math mirrors sim/src/kontinuum.rs, sim/src/cpu.rs:279-307 and
// sim/src/implizit.rs:725-844 in FP64.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "k3d_netz.cuh"
#include "k3d_vec.cuh"

namespace k3d {

// Body descriptor as the kernel reads it (k3d_body, plus the substep offset).
struct Body {
  int art;
  int dims[3];
  double punkt[3], achse[3], radius, vel[3], ursprung[3], spacing;
  const float* sdf;  // device copy of the grid
  int inst;          // the instance (independent drape) it acts on, -1 = every instance
  const netz::Dev* netz;  // mesh body: the mesh's tables (device)
};
constexpr int kMaxBodies = 64;

// Contact query, sim/src/koerper.rs:69-91 for the cylinder and the mesh (the
// exact nearest point within max(search depth, distance), koerper.rs:80-87);
// the SDF grid is a trilinear interpolant of node values (value and
// gradient), no contact outside the grid. vk: the body's velocity at the
// contact (a mesh with a velocity field: at the nearest point).
__device__ inline bool kontakt(const Body& k, D3 x, double abstand, D3& normale, double& tiefe);
__device__ inline bool kontakt_v(const Body& k, D3 x, double abstand, D3& normale, double& tiefe, D3& vk) {
  vk = d3(k.vel[0], k.vel[1], k.vel[2]);
  if (k.art == 2) {
    netz::Treffer t;
    const D3 xl = x - d3(k.punkt[0], k.punkt[1], k.punkt[2]);
    if (!netz::naechster(*k.netz, xl, fmax(k.netz->suchtiefe, abstand), t)) return false;
    tiefe = abstand - t.abstand;
    if (!(tiefe > 0.0)) return false;
    normale = t.normale;
    vk = netz::geschwindigkeit_an(*k.netz, t.dreieck, t.punkt, vk);
    return true;
  }
  return kontakt(k, x, abstand, normale, tiefe);
}
__device__ inline bool kontakt(const Body& k, D3 x, double abstand, D3& normale, double& tiefe) {
  if (k.art == 2) {
    D3 vk;
    return kontakt_v(k, x, abstand, normale, tiefe, vk);
  }
  if (k.art == 0) {
    D3 ax = d3(k.achse[0], k.achse[1], k.achse[2]);
    D3 a = ax * (1.0 / norm(ax));
    D3 d = x - d3(k.punkt[0], k.punkt[1], k.punkt[2]);
    D3 quer = d - a * dot(d, a);
    double r = norm(quer);
    tiefe = k.radius + abstand - r;
    if (tiefe <= 0.0 || r < 1e-12) return false;
    normale = quer * (1.0 / r);
    return true;
  }
  double u[3] = {(x.x - k.punkt[0] - k.ursprung[0]) / k.spacing, (x.y - k.punkt[1] - k.ursprung[1]) / k.spacing,
                 (x.z - k.punkt[2] - k.ursprung[2]) / k.spacing};
  int64_t ii[3];
  double t[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double fl = floor(u[a]);
    if (!(fl >= 0.0) || !(fl < double(k.dims[a] - 1))) return false;
    ii[a] = int64_t(fl);
    t[a] = u[a] - fl;
  }
  const int64_t sx = 1, sy = k.dims[0], sz = int64_t(k.dims[0]) * k.dims[1];
  const float* g = k.sdf + ii[2] * sz + ii[1] * sy + ii[0];
  double c000 = g[0], c100 = g[sx], c010 = g[sy], c110 = g[sx + sy];
  double c001 = g[sz], c101 = g[sz + sx], c011 = g[sz + sy], c111 = g[sz + sx + sy];
  double tx = t[0], ty = t[1], tz = t[2];
  double c00 = c000 + (c100 - c000) * tx, c10 = c010 + (c110 - c010) * tx;
  double c01 = c001 + (c101 - c001) * tx, c11 = c011 + (c111 - c011) * tx;
  double c0 = c00 + (c10 - c00) * ty, c1 = c01 + (c11 - c01) * ty;
  double wert = c0 + (c1 - c0) * tz;
  double d00 = c100 - c000, d10 = c110 - c010, d01 = c101 - c001, d11 = c111 - c011;
  double e0 = d00 + (d10 - d00) * ty, e1 = d01 + (d11 - d01) * ty;
  double gx = (e0 + (e1 - e0) * tz) / k.spacing;
  double f0 = c10 - c00, f1 = c11 - c01;
  double gy = (f0 + (f1 - f0) * tz) / k.spacing;
  double gz = (c1 - c0) / k.spacing;
  tiefe = abstand - wert;
  if (tiefe <= 0.0) return false;
  D3 gr = d3(gx, gy, gz);
  double gl = norm(gr);
  if (gl < 1e-12) return false;
  normale = gr * (1.0 / gl);
  return true;
}

// ---------------------------------------------------------------- membrane (FP64)
// Scene constants of one membrane: ruhe_inv (r0..r3), basis (kette, schuss),
// mat (flaeche, E_warp, E_weft, G).
struct MembranC {
  double r[4];
  double kx, ky, sx, sy;
  double fl, ek, es, g;
};
__device__ __forceinline__ void basis3(const MembranC& m, D3& a, D3& b, D3& c) {
  a = d3(m.kx * m.kx, m.ky * m.ky, m.kx * m.ky);                      // kontinuum.rs:143-145
  b = d3(m.sx * m.sx, m.sy * m.sy, m.sx * m.sy);
  c = d3(m.kx * m.sx, m.ky * m.sy, 0.5 * (m.kx * m.sy + m.ky * m.sx));  // :147-150
}
__device__ __forceinline__ D3 coef1(const double* r) { return d3(-(r[0] + r[2]), r[0], r[2]); }  // :302-305
__device__ __forceinline__ D3 coef2(const double* r) { return d3(-(r[1] + r[3]), r[1], r[3]); }  // :308-312

// kontinuum.rs:158-177 (nearest PSD matrix of a symmetric 2x2)
__device__ inline D3 psd2(double a, double b, double c) {
  double m = 0.5 * (a + b), d = 0.5 * (a - b);
  double r = sqrt(d * d + c * c);
  if (m - r >= 0.0) return d3(a, b, c);
  double lmax = m + r;
  if (!(lmax > 0.0)) return d3(0, 0, 0);
  double u0 = lmax - b, u1 = c;
  double n2 = u0 * u0 + u1 * u1;
  if (!(n2 > 0.0)) return d3(0, 0, 0);
  double f = lmax / n2;
  return d3(f * u0 * u0, f * u1 * u1, f * u0 * u1);
}

// dU/dg for a strain vector e (kontinuum.rs:376-386)
__device__ __forceinline__ D3 du_dg(const MembranC& m, D3 a, D3 b, D3 c, D3 e) {
  double ka = 0.5 * m.ek * e.x, kb = 0.5 * m.es * e.y, kc = 2.0 * m.g * e.z;
  return d3(m.fl * (ka * a.x + kb * b.x + kc * c.x), m.fl * (ka * a.y + kb * b.y + kc * c.y),
            m.fl * (ka * a.z + kb * b.z + kc * c.z));
}
// -J_k^T d per vertex (kontinuum.rs:504-520)
__device__ __forceinline__ void kraefte(const double* r, D3 f1, D3 f2, D3 d, D3 out[3]) {
  D3 k1 = coef1(r), k2 = coef2(r);
  const double c1[3] = {k1.x, k1.y, k1.z}, c2[3] = {k2.x, k2.y, k2.z};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double s1 = 2.0 * (d.x * c1[k] + d.z * c2[k]);
    double s2 = 2.0 * (d.y * c2[k] + d.z * c1[k]);
    out[k] = d3(-(s1 * f1.x + s2 * f2.x), -(s1 * f1.y + s2 * f2.y), -(s1 * f1.z + s2 * f2.z));
  }
}
// kg = d2U/dg2 as a symmetric 3x3 (kontinuum.rs:391-406): (00, 11, 22, 01, 02, 12)
__device__ __forceinline__ void kg_sym(const MembranC& m, double kg[6]) {
  D3 a, b, c;
  basis3(m, a, b, c);
  const D3 v[3] = {a, b, c};
  const double wt[3] = {0.25 * m.ek, 0.25 * m.es, m.g};
  for (int q = 0; q < 6; ++q) kg[q] = 0.0;
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    double s = m.fl * wt[t];
    kg[0] += s * v[t].x * v[t].x;
    kg[1] += s * v[t].y * v[t].y;
    kg[2] += s * v[t].z * v[t].z;
    kg[3] += s * v[t].x * v[t].y;
    kg[4] += s * v[t].x * v[t].z;
    kg[5] += s * v[t].y * v[t].z;
  }
}

// Hessian-vector product of one membrane (kontinuum.rs:616-664) in the
// operator precision R, from the per-step record: f1, f2, w=(w11,w22,w12),
// rest coefficients r0..r3 and the assembled kg. The corner coefficients sum
// to zero (c1[0] = -(c1[1] + c1[2]), the same for c2), so the product only
// sees the differences d1 - d0 and d2 - d0: a motion common to the three
// points cancels before any rounding.
template <typename R>
__device__ __forceinline__ void membran_hv(const R4<R>& f1w, const R4<R>& f2w, const R4<R>& rin,
                                           const R4<R>& kgA, const R4<R>& kgB, const R4<R> d[3], R4<R> out[3]) {
  const R c1[3] = {-(rin.x + rin.z), rin.x, rin.z};
  const R c2[3] = {-(rin.y + rin.w), rin.y, rin.w};
  const R e1x = d[1].x - d[0].x, e1y = d[1].y - d[0].y, e1z = d[1].z - d[0].z;
  const R e2x = d[2].x - d[0].x, e2y = d[2].y - d[0].y, e2z = d[2].z - d[0].z;
  const R a1 = f1w.x * e1x + f1w.y * e1y + f1w.z * e1z, b1 = f2w.x * e1x + f2w.y * e1y + f2w.z * e1z;
  const R a2 = f1w.x * e2x + f1w.y * e2y + f1w.z * e2z, b2 = f2w.x * e2x + f2w.y * e2y + f2w.z * e2z;
  const R q0 = R(2) * (c1[1] * a1 + c1[2] * a2);
  const R q1 = R(2) * (c2[1] * b1 + c2[2] * b2);
  const R q2 = R(2) * (c2[1] * a1 + c1[1] * b1 + c2[2] * a2 + c1[2] * b2);
  const R t1x = c1[1] * e1x + c1[2] * e2x, t1y = c1[1] * e1y + c1[2] * e2y, t1z = c1[1] * e1z + c1[2] * e2z;
  const R t2x = c2[1] * e1x + c2[2] * e2x, t2y = c2[1] * e1y + c2[2] * e2y, t2z = c2[1] * e1z + c2[2] * e2z;
  // w = kg q; kgA = (00, 11, 22, 01), kgB = (02, 12, w12, -)
  const R w0 = kgA.x * q0 + kgA.w * q1 + kgB.x * q2;
  const R w1 = kgA.w * q0 + kgA.y * q1 + kgB.y * q2;
  const R w2 = kgB.x * q0 + kgB.y * q1 + kgA.z * q2;
  const R w11 = f1w.w, w22 = f2w.w, w12 = kgB.z;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    R s1 = R(2) * (c1[k] * w0 + c2[k] * w2);
    R s2 = R(2) * (c2[k] * w1 + c1[k] * w2);
    R pa = R(2) * (w11 * c1[k] + w12 * c2[k]);
    R qa = R(2) * (w12 * c1[k] + w22 * c2[k]);
    out[k].x = s1 * f1w.x + s2 * f2w.x + pa * t1x + qa * t2x;
    out[k].y = s1 * f1w.y + s2 * f2w.y + pa * t1y + qa * t2y;
    out[k].z = s1 * f1w.z + s2 * f2w.z + pa * t1z + qa * t2z;
    out[k].w = 0;
  }
}

// ---------------------------------------------------------------- dihedral (FP64)
// cpu.rs:288-307 (Bridson et al. 2003)
__device__ inline bool dieder(D3 x0, D3 x1, D3 x2, D3 x3, double& theta, D3 g[4]) {
  D3 e = x1 - x0;
  double le = norm(e);
  D3 n1 = cross(x2 - x0, x2 - x1);
  D3 n2 = cross(x3 - x1, x3 - x0);
  double q1 = dot(n1, n1), q2 = dot(n2, n2);
  if (le < 1e-12 || q1 < 1e-30 || q2 < 1e-30) return false;
  D3 m1 = n1 * (1.0 / sqrt(q1)), m2 = n2 * (1.0 / sqrt(q2));
  theta = atan2(dot(cross(m1, m2), e * (1.0 / le)), dot(m1, m2));
  g[2] = n1 * (-le / q1);
  g[3] = n2 * (-le / q2);
  g[0] = (n1 * (dot(x2 - x1, e) / le / q1) + n2 * (dot(x3 - x1, e) / le / q2)) * -1.0;
  g[1] = n1 * (dot(x2 - x0, e) / le / q1) + n2 * (dot(x3 - x0, e) / le / q2);
  return true;
}
// cpu.rs:279-282; rint is not used because Rust rounds halves away from zero
__device__ __forceinline__ double winkel_fehler(double theta, double ruhe) {
  const double tau = 6.283185307179586476925286766559;
  double d = theta - ruhe;
  return d - tau * round(d / tau);
}

// implizit.rs:444-453, for a symmetric block (00, 11, 22, 01, 02, 12);
// returns the symmetric inverse in the same order.
__device__ __forceinline__ void m3_inv_sym(const double m[6], double o[6]) {
  double a = m[0], b = m[3], c = m[4], e = m[1], f = m[5], i = m[2];
  double d = b, g = c, h = f;
  double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
  double s = 1.0 / det;
  o[0] = (e * i - f * h) * s;
  o[1] = (a * i - c * g) * s;
  o[2] = (a * e - b * d) * s;
  o[3] = (c * h - b * i) * s;
  o[4] = (b * f - c * e) * s;
  o[5] = (c * d - a * f) * s;
}

}  // namespace k3d
