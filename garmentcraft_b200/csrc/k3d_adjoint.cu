// The adjoint of one implicit substep on the device. The reference has no
// adjoint; this differentiates the device's own forward (k3d_build.cu,
// k3d_step.cu: implizit.rs:663-1013 restated) with every discrete decision of
// the recorded substep frozen: the contact set of the last solve and after
// the release pass (a second release pass ends the loop: the points it
// releases keep their constraint in dv but get no friction), stick or slip,
// and which bodies pushed a point out after the move.
//
// Forward, decisions frozen (h = substep, u = v + dv):
//   S (A dv - b) = 0 and n.dv = vn_soll - v.n on held points,
//   A = M(1 + hc) + h^2 H(x), b = h (f(x, v) - h H(x) v),
//   v1 = v + dv, friction on held points -> v2, x1 = x + h v2, push-outs.
// Backward, with Phi = b - A dv at fixed dv:
//   push-outs, integration, friction per point -> dv_bar, rho_bar (slip: the
//     friction bound depends on the normal force n.(A dv - b)/h)
//   g = dv_bar + A rho_bar; adjoint PCG S A S lam = S g (zero target)
//   mu = lam - rho_bar; v_bar += M mu - A mu
//   held points: zeta = n.(g - A lam) enters through the constraint's target
//     and, with lam (n.rho) and the friction terms, through the normal n(x)
//   elements: x_bar, theta_bar += grad of mu.Phi, by forward-mode dual
//     numbers: one thread per (element, direction).
// Compiled without FMA contraction like the build, so that the replayed
// contact queries round exactly as the forward did.
#include <cfloat>
#include <cstdint>

#include "k3d_adjoint.h"
#include "k3d_step_common.cuh"

namespace k3d {
namespace {

// ------------------------------------------------------------ dual numbers
struct Du {
  double v, d;  // value, one directional derivative
};
__device__ __forceinline__ Du du(double v, double d = 0.0) { return {v, d}; }
__device__ __forceinline__ Du operator+(Du a, Du b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Du operator-(Du a, Du b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Du operator-(Du a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Du operator*(Du a, Du b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Du operator/(Du a, Du b) {
  const double q = a.v / b.v;
  return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Du operator-(Du a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ Du operator-(double a, Du b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Du operator*(Du a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Du operator*(double a, Du b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Du dsqrt(Du a) {
  const double s = sqrt(a.v);
  return {s, s > 0.0 ? a.d / (2.0 * s) : 0.0};
}
__device__ __forceinline__ Du datan2(Du y, Du x) {
  const double r2 = x.v * x.v + y.v * y.v;
  return {atan2(y.v, x.v), r2 > 0.0 ? (x.v * y.d - y.v * x.d) / r2 : 0.0};
}
__device__ __forceinline__ Du dmax0(Du a) { return a.v > 0.0 ? a : du(0.0); }
__device__ __forceinline__ Du dmax(Du a, double b) { return a.v > b ? a : du(b); }

struct U3 {
  Du x, y, z;
};
__device__ __forceinline__ U3 u3(Du x, Du y, Du z) { return {x, y, z}; }
__device__ __forceinline__ U3 operator+(U3 a, U3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ U3 operator-(U3 a, U3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ U3 operator*(U3 a, Du s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ U3 operator*(U3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ Du dot(U3 a, U3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ Du dot(U3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ U3 cross(U3 a, U3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ Du norm(U3 a) { return dsqrt(dot(a, a)); }

// kontinuum.rs:158-177, as the build evaluates it
__device__ U3 psd2(Du a, Du b, Du c) {
  const Du m = 0.5 * (a + b), d = 0.5 * (a - b);
  const Du r = dsqrt(d * d + c * c);
  if (m.v - r.v >= 0.0) return {a, b, c};
  const Du lmax = m + r;
  if (!(lmax.v > 0.0)) return {du(0), du(0), du(0)};
  const Du u0 = lmax - b, u1 = c;
  const Du n2 = u0 * u0 + u1 * u1;
  if (!(n2.v > 0.0)) return {du(0), du(0), du(0)};
  const Du f = lmax / n2;
  return {f * u0 * u0, f * u1 * u1, f * u0 * u1};
}

// h mu.f - h^2 mu.(H u) of one membrane (kontinuum.rs:504-520 forces,
// :584-591 geometric stress, :616-664 product), as the build and the
// operator evaluate them, with dual inputs.
__device__ Du membran_phi(U3 f1, U3 f2, const double r[4], Du kx, Du ky, Du sx, Du sy, double fl, Du ek, Du es,
                          Du g, const D3 mu[3], const D3 u[3], double h) {
  const U3 ba = u3(kx * kx, ky * ky, kx * ky), bb = u3(sx * sx, sy * sy, sx * sy);
  const U3 bc = u3(kx * sx, ky * sy, 0.5 * (kx * sy + ky * sx));
  const U3 gv = u3(dot(f1, f1), dot(f2, f2), 2.0 * dot(f1, f2));
  const U3 e = u3(0.5 * (dot(ba, gv) - 1.0), 0.5 * (dot(bb, gv) - 1.0), 0.5 * dot(bc, gv));
  auto dudg = [&](U3 q) -> U3 {
    const Du ka = 0.5 * ek * q.x, kb = 0.5 * es * q.y, kc = 2.0 * g * q.z;
    return u3(fl * (ka * ba.x + kb * bb.x + kc * bc.x), fl * (ka * ba.y + kb * bb.y + kc * bc.y),
              fl * (ka * ba.z + kb * bb.z + kc * bc.z));
  };
  const double c1[3] = {-(r[0] + r[2]), r[0], r[2]}, c2[3] = {-(r[1] + r[3]), r[1], r[3]};
  const U3 dU = dudg(e);
  Du phi = du(0.0);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const Du s1 = 2.0 * (dU.x * c1[k] + dU.z * c2[k]);
    const Du s2 = 2.0 * (dU.y * c2[k] + dU.z * c1[k]);
    const U3 F = (f1 * s1 + f2 * s2) * -1.0;
    phi = phi + h * dot(F, mu[k]);
  }
  const U3 dz = dudg(u3(dmax0(e.x), dmax0(e.y), e.z));
  const U3 w = psd2(dz.x, dz.y, dz.z);
  // kg (00, 11, 22, 01, 02, 12)
  Du kg[6] = {du(0), du(0), du(0), du(0), du(0), du(0)};
  const U3 vv[3] = {ba, bb, bc};
  const Du wt[3] = {0.25 * ek, 0.25 * es, g};
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    const Du s = fl * wt[t];
    kg[0] = kg[0] + s * vv[t].x * vv[t].x;
    kg[1] = kg[1] + s * vv[t].y * vv[t].y;
    kg[2] = kg[2] + s * vv[t].z * vv[t].z;
    kg[3] = kg[3] + s * vv[t].x * vv[t].y;
    kg[4] = kg[4] + s * vv[t].x * vv[t].z;
    kg[5] = kg[5] + s * vv[t].y * vv[t].z;
  }
  const D3 e1 = u[1] - u[0], e2 = u[2] - u[0];
  const Du a1 = dot(f1, e1), b1 = dot(f2, e1), a2 = dot(f1, e2), b2 = dot(f2, e2);
  const Du q0 = 2.0 * (c1[1] * a1 + c1[2] * a2);
  const Du q1 = 2.0 * (c2[1] * b1 + c2[2] * b2);
  const Du q2 = 2.0 * (c2[1] * a1 + c1[1] * b1 + c2[2] * a2 + c1[2] * b2);
  const D3 t1 = e1 * c1[1] + e2 * c1[2], t2 = e1 * c2[1] + e2 * c2[2];
  const Du w0 = kg[0] * q0 + kg[3] * q1 + kg[4] * q2;
  const Du w1 = kg[3] * q0 + kg[1] * q1 + kg[5] * q2;
  const Du w2 = kg[4] * q0 + kg[5] * q1 + kg[2] * q2;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const Du s1 = 2.0 * (c1[k] * w0 + c2[k] * w2);
    const Du s2 = 2.0 * (c2[k] * w1 + c1[k] * w2);
    const Du pa = 2.0 * (w.x * c1[k] + w.z * c2[k]);
    const Du qa = 2.0 * (w.z * c1[k] + w.y * c2[k]);
    const U3 hu = f1 * s1 + f2 * s2 + u3(pa * t1.x, pa * t1.y, pa * t1.z) + u3(qa * t2.x, qa * t2.y, qa * t2.z);
    phi = phi - (h * h) * dot(hu, mu[k]);
  }
  return phi;
}

// The same for one hinge: force -k err(theta) grad theta (implizit.rs:774-796),
// product k g (g.u) (:198-203), dihedral angle and gradients of cpu.rs:288-307.
__device__ Du biegung_phi(const U3 p[4], Du k, double ruhe, const D3 mu[4], const D3 u[4], double h) {
  const U3 e = p[1] - p[0];
  const Du le = norm(e);
  const U3 n1 = cross(p[2] - p[0], p[2] - p[1]);
  const U3 n2 = cross(p[3] - p[1], p[3] - p[0]);
  const Du q1 = dot(n1, n1), q2 = dot(n2, n2);
  if (le.v < 1e-12 || q1.v < 1e-30 || q2.v < 1e-30) return du(0.0);
  const U3 m1 = n1 * (du(1.0) / dsqrt(q1)), m2 = n2 * (du(1.0) / dsqrt(q2));
  const Du theta = datan2(dot(cross(m1, m2), e * (du(1.0) / le)), dot(m1, m2));
  U3 gr[4];
  gr[2] = n1 * ((-le) / q1);
  gr[3] = n2 * ((-le) / q2);
  gr[0] = (n1 * (dot(p[2] - p[1], e) / le / q1) + n2 * (dot(p[3] - p[1], e) / le / q2)) * -1.0;
  gr[1] = n1 * (dot(p[2] - p[0], e) / le / q1) + n2 * (dot(p[3] - p[0], e) / le / q2);
  const double tau = 6.283185307179586476925286766559;
  const Du dd = theta - ruhe;
  const Du fehler = dd - tau * round(dd.v / tau);
  Du gu = du(0.0), gm = du(0.0);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    gu = gu + dot(gr[q], u[q]);
    gm = gm + dot(gr[q], mu[q]);
  }
  return gm * (-(h * k * fehler) - (h * h) * k * gu);
}

// One pattern edge (art 0) or seam (art 1) from i to j (implizit.rs:742-771,
// product :193-197).
__device__ Du feder_phi(int art, U3 xi, U3 xj, double k, double l0, D3 mui, D3 muj, D3 ui, D3 uj, double h) {
  const U3 d = xj - xi;
  U3 F, r;
  Du quer;
  if (art == 0) {
    const Du l = dmax(norm(d), 1e-12);
    r = d * (du(1.0) / l);
    F = r * (k * (l - l0));
    quer = dmax(1.0 - du(l0) / l, 0.0);
  } else {
    const Du l = norm(d);
    const Du L0 = isfinite(l0) ? du(l0) : l;
    if (L0.v > 0.0 && l.v > 1e-12) {
      F = d * (k * (l - L0) / l);
      r = d * (du(1.0) / l);
      quer = dmax(1.0 - L0 / l, 0.0);
    } else {
      F = d * k;
      r = u3(du(0), du(0), du(0));
      quer = du(1.0);
    }
  }
  const D3 dv = ui - uj, dm = mui - muj;
  const U3 bd = (r * (dot(r, dv) * (1.0 - quer)) + u3(quer * dv.x, quer * dv.y, quer * dv.z)) * k;
  return h * dot(F, dm) - (h * h) * dot(bd, dm);
}

// ------------------------------------------------------------ contact derivatives
// The contact query of k3d_device.cuh (cylinder: koerper.rs:69-91; trilinear
// SDF grid) with the x-derivatives of its normal (J[a][c] = d n_a / d x_c)
// and depth. The trilinear interpolant has zero second derivatives along the
// axes; its mixed ones give the normal's derivative (I - n n^T) H / |grad|.
__device__ bool kontakt_abl(const Body& k, D3 x, double abstand, D3& n, double& tiefe, double J[3][3], D3& dt) {
  if (k.art == 0) {
    const D3 ax = d3(k.achse[0], k.achse[1], k.achse[2]);
    const D3 a = ax * (1.0 / norm(ax));
    const D3 d = x - d3(k.punkt[0], k.punkt[1], k.punkt[2]);
    const D3 quer = d - a * dot(d, a);
    const double r = norm(quer);
    tiefe = k.radius + abstand - r;
    if (tiefe <= 0.0 || r < 1e-12) return false;
    n = quer * (1.0 / r);
    const double av[3] = {a.x, a.y, a.z}, nv[3] = {n.x, n.y, n.z};
    for (int p = 0; p < 3; ++p)
      for (int c = 0; c < 3; ++c) J[p][c] = ((p == c ? 1.0 : 0.0) - av[p] * av[c] - nv[p] * nv[c]) / r;
    dt = n * -1.0;
    return true;
  }
  const double u[3] = {(x.x - k.punkt[0] - k.ursprung[0]) / k.spacing, (x.y - k.punkt[1] - k.ursprung[1]) / k.spacing,
                       (x.z - k.punkt[2] - k.ursprung[2]) / k.spacing};
  int64_t ii[3];
  double t[3];
  for (int a = 0; a < 3; ++a) {
    const double fl = floor(u[a]);
    if (!(fl >= 0.0) || !(fl < double(k.dims[a] - 1))) return false;
    ii[a] = int64_t(fl);
    t[a] = u[a] - fl;
  }
  const int64_t sx = 1, sy = k.dims[0], sz = int64_t(k.dims[0]) * k.dims[1];
  const float* g = k.sdf + ii[2] * sz + ii[1] * sy + ii[0];
  const double c000 = g[0], c100 = g[sx], c010 = g[sy], c110 = g[sx + sy];
  const double c001 = g[sz], c101 = g[sz + sx], c011 = g[sz + sy], c111 = g[sz + sx + sy];
  const double tx = t[0], ty = t[1], tz = t[2];
  const double c00 = c000 + (c100 - c000) * tx, c10 = c010 + (c110 - c010) * tx;
  const double c01 = c001 + (c101 - c001) * tx, c11 = c011 + (c111 - c011) * tx;
  const double c0 = c00 + (c10 - c00) * ty, c1 = c01 + (c11 - c01) * ty;
  const double wert = c0 + (c1 - c0) * tz;
  const double d00 = c100 - c000, d10 = c110 - c010, d01 = c101 - c001, d11 = c111 - c011;
  const double e0 = d00 + (d10 - d00) * ty, e1 = d01 + (d11 - d01) * ty;
  const double gx = (e0 + (e1 - e0) * tz) / k.spacing;
  const double f0 = c10 - c00, f1 = c11 - c01;
  const double gy = (f0 + (f1 - f0) * tz) / k.spacing;
  const double gz = (c1 - c0) / k.spacing;
  tiefe = abstand - wert;
  if (tiefe <= 0.0) return false;
  const D3 gr = d3(gx, gy, gz);
  const double gl = norm(gr);
  if (gl < 1e-12) return false;
  n = gr * (1.0 / gl);
  const double s2 = k.spacing * k.spacing;
  const double hxy = ((d10 - d00) + ((d11 - d01) - (d10 - d00)) * tz) / s2;
  const double hxz = (e1 - e0) / s2;
  const double hyz = (f1 - f0) / s2;
  const double H[3][3] = {{0.0, hxy, hxz}, {hxy, 0.0, hyz}, {hxz, hyz, 0.0}};
  const double nv[3] = {n.x, n.y, n.z};
  for (int p = 0; p < 3; ++p)
    for (int c = 0; c < 3; ++c) {
      double s = 0.0;
      for (int q = 0; q < 3; ++q) s += ((p == q ? 1.0 : 0.0) - nv[p] * nv[q]) * H[q][c];
      J[p][c] = s / gl;
    }
  dt = gr * -1.0;
  return true;
}
__device__ __forceinline__ D3 jt_mal(const double J[3][3], D3 v) {  // J^T v
  return d3(J[0][0] * v.x + J[1][0] * v.y + J[2][0] * v.z, J[0][1] * v.x + J[1][1] * v.y + J[2][1] * v.z,
            J[0][2] * v.x + J[1][2] * v.y + J[2][2] * v.z);
}
__device__ __forceinline__ bool body_acts(const StepArgs& a, int kb, int64_t i) {
  const int inst = a.pinst ? int(a.pinst[i]) : 0;
  return !(a.bodies[kb].inst >= 0 && a.bodies[kb].inst != inst);
}
__device__ __forceinline__ D3 body_vel(const Body& b) { return d3(b.vel[0], b.vel[1], b.vel[2]); }

// ------------------------------------------------------------ point stages
// The contact set of the last solve: points released before it lose their normal.
__global__ void __launch_bounds__(kBlock) adj_final_set_kernel(const __grid_constant__ StepArgs a,
                                                                const __grid_constant__ AdjArgs j) {
  double* nrm = static_cast<double*>(a.nrm);
  K3D_FOR(i, a.n) {
    if (j.flags[i] & 9u) continue;
    st3(a.nrm_d, uint32_t(i), d3(0, 0, 0));
    nrm[3 * i] = nrm[3 * i + 1] = nrm[3 * i + 2] = 0.0;
  }
}

// y = A x on the assembled FP64 blocks
__global__ void __launch_bounds__(kBlock) adj_spmv_kernel(const __grid_constant__ StepArgs a, const double* x,
                                                           double* y) {
  const R4<double>* b4 = static_cast<const R4<double>*>(a.bmat);
  const double* b1 = static_cast<const double*>(a.bmat) + 8 * a.bplane;
  const int64_t P = a.bplane;
  K3D_FOR(i, a.n) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    const uint32_t cnt = a.row_cnt[i];
    for (uint32_t k = 0; k < cnt; ++k) {
      const int64_t sid = int64_t(k) * a.np + i;
      const D3 p = ld3(x, a.col[sid]);
      const R4<double> u = b4[sid], v = b4[P + sid];
      sx += u.x * p.x + u.y * p.y + u.z * p.z;
      sy += u.w * p.x + v.x * p.y + v.y * p.z;
      sz += v.z * p.x + v.w * p.y + b1[sid] * p.z;
    }
    st3(y, uint32_t(i), d3(sx, sy, sz));
  }
}

// Push-outs, integration and friction backwards (implizit.rs:957-1013).
__global__ void __launch_bounds__(kBlock) adj_integrate_kernel(const __grid_constant__ StepArgs a,
                                                                const __grid_constant__ AdjArgs j) {
  const double h = a.h;
  K3D_FOR(i, a.n) {
    const uint32_t ui = uint32_t(i);
    const D3 xq = ld3(j.xq, ui), vq = ld3(j.vq, ui);
    const D3 z = d3(0, 0, 0);
    if (!a.frei[i]) {
      st3(j.xa, ui, xq);
      st3(j.va, ui, vq);
      st3(j.gq, ui, z);
      st3(j.rq, ui, z);
      st3(j.nq, ui, z);
      continue;
    }
    const uint32_t fl = j.flags[i];
    const D3 x = ld3(j.x, ui), v = ld3(j.v, ui), dv = ld3(j.dv, ui);
    const D3 v1 = v + dv;
    D3 v2 = v1, n = z, vb = z, rel = z, t = z;
    double lt = 0.0, grenze = 0.0;
    const bool held = (fl & 1u) != 0u;
    if (held) {
      n = ld3(a.nrm_d, ui);
      vb = ld3(a.vk, ui);
      rel = v1 - vb;
      t = rel - n * dot(rel, n);
      lt = norm(t);
      grenze = a.reib[i] * j.fn[i] * h * a.w[i];
      if (fl & 2u)
        v2 = v1 - t;
      else if (fl & 4u)
        v2 = v1 - t * (grenze / lt);
    }
    const D3 x1 = x + v2 * h;
    D3 xb = xq, vbq = vq;
    const int nb = a.n_bodies < kMaxAdjointBodies ? a.n_bodies : kMaxAdjointBodies;
    for (int kb = nb - 1; kb >= 0; --kb) {
      if (!(fl & (1u << (4 + 2 * kb)))) continue;
      D3 xs = x1, vs = v2;  // the state before body kb's push-out
      for (int q = 0; q < kb; ++q) {
        if (!(fl & (1u << (4 + 2 * q)))) continue;
        D3 nn;
        double ti;
        kontakt(a.bodies[q], xs, a.kabst[i], nn, ti);
        xs = xs + nn * ti;
        if (fl & (1u << (5 + 2 * q))) vs = vs - nn * dot(vs - body_vel(a.bodies[q]), nn);
      }
      D3 n2, gt;
      double t2, J[3][3];
      if (!kontakt_abl(a.bodies[kb], xs, a.kabst[i], n2, t2, J, gt)) continue;
      D3 nbar = xb * t2;
      const double tbar = dot(xb, n2);
      if (fl & (1u << (5 + 2 * kb))) {
        const D3 vr = vs - body_vel(a.bodies[kb]);
        nbar = nbar - (vbq * dot(n2, vr) + vr * dot(n2, vbq));
        vbq = vbq - n2 * dot(n2, vbq);
      }
      xb = xb + jt_mal(J, nbar) + gt * tbar;
    }
    st3(j.xa, ui, xb);
    const D3 v2b = vbq + xb * h;
    D3 v1b = v2b, nq = z, rq = z;
    if (held && (fl & 2u)) {
      v1b = n * dot(n, v2b);
      nq = v2b * dot(n, rel) + rel * dot(n, v2b);
    } else if (held && (fl & 4u)) {
      const double sk = grenze / lt;
      const D3 th = t * (1.0 / lt);
      const D3 q = (v2b - th * dot(th, v2b)) * sk;
      v1b = v2b - (q - n * dot(n, q));
      nq = q * dot(n, rel) + rel * dot(n, q);
      const double gb = -dot(v2b, th) * a.reib[i] * a.w[i];
      rq = n * gb;
      const D3 rho = ld3(j.adv, ui) - ld3(a.b, ui);
      nq = nq + rho * gb;
    }
    st3(j.va, ui, v1b);
    st3(j.gq, ui, v1b);
    st3(j.rq, ui, rq);
    st3(j.nq, ui, nq);
  }
}

__global__ void __launch_bounds__(kBlock) adj_rhs_kernel(const __grid_constant__ StepArgs a,
                                                          const __grid_constant__ AdjArgs j) {
  K3D_FOR(i, 3 * a.n) j.gg[i] = j.gq[i] + j.arq[i];
}

// After the adjoint solve: mu, the damping and H v terms of v_bar, and for
// held points the constraint target and the normal's dependence on x.
__global__ void __launch_bounds__(kBlock) adj_points_kernel(const __grid_constant__ StepArgs a,
                                                             const __grid_constant__ AdjArgs j) {
  const double h = a.h;
  K3D_FOR(i, a.n) {
    const uint32_t ui = uint32_t(i);
    const D3 lam = ld3(j.lam, ui), rq = ld3(j.rq, ui), alam = ld3(j.alam, ui), arq = ld3(j.arq, ui);
    const D3 mu = lam - rq;
    D3 vo = ld3(j.va, ui) + mu * a.masse[i] - (alam - arq);
    D3 xo = ld3(j.xa, ui);
    if (a.frei[i] && (j.flags[i] & 9u)) {  // held in the last solve
      const D3 n = ld3(a.nrm_d, ui);
      const D3 x = ld3(j.x, ui), v = ld3(j.v, ui), dv = ld3(j.dv, ui);
      const double zeta = dot(n, ld3(j.gg, ui) - alam);
      vo = vo - n * zeta;
      const D3 rho = ld3(j.adv, ui) - ld3(a.b, ui);
      const D3 nbar = ld3(j.nq, ui) + lam * dot(n, rho) - dv * zeta + (ld3(a.vk, ui) - v) * zeta;
      // the build's contact: the last body in contact (implizit.rs:873-883)
      double J[3][3], Jl[3][3];
      D3 nn, gt, gtl = d3(0, 0, 0);
      double ti;
      bool hat = false;
      for (int kb = 0; kb < a.n_bodies; ++kb) {
        if (!body_acts(a, kb, i)) continue;
        if (kontakt_abl(a.bodies[kb], x, a.kabst[i] + a.kontakt_rand, nn, ti, J, gt)) {
          for (int p = 0; p < 3; ++p)
            for (int c = 0; c < 3; ++c) Jl[p][c] = J[p][c];
          gtl = gt;
          hat = true;
        }
      }
      if (hat) xo = xo + gtl * (zeta / h) + jt_mal(Jl, nbar);
    }
    st3(j.mu, ui, mu);
    st3(j.xa, ui, xo);
    st3(j.va, ui, vo);
  }
}

// ------------------------------------------------------------ element stages
// Directions per membrane: 0-5 the components of f1, f2; 6-8 E_warp, E_weft,
// G; 9 a rotation of the grain basis in the rest plane.
__global__ void __launch_bounds__(kBlock) adj_membran_kernel(const __grid_constant__ StepArgs a,
                                                              const __grid_constant__ AdjArgs j) {
  const double h = a.h;
  K3D_FOR(q, 10 * a.nt) {
    const int64_t t = q % a.nt;
    const int dir = int(q / a.nt);
    const uint4 id = __ldg(&a.m_idx[t]);
    const MembranC m = membran_c(a, t);
    const uint32_t ids[3] = {id.x, id.y, id.z};
    const D3 p0 = ld3(j.x, id.x), p1 = ld3(j.x, id.y), p2 = ld3(j.x, id.z);
    const D3 e1 = p1 - p0, e2 = p2 - p0;
    const D3 f1 = e1 * m.r[0] + e2 * m.r[2];
    const D3 f2 = e1 * m.r[1] + e2 * m.r[3];
    D3 mu[3], u[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      mu[k] = ld3(j.mu, ids[k]);
      u[k] = ld3(j.v, ids[k]) + ld3(j.dv, ids[k]);
    }
    const U3 F1 = u3(du(f1.x, dir == 0), du(f1.y, dir == 1), du(f1.z, dir == 2));
    const U3 F2 = u3(du(f2.x, dir == 3), du(f2.y, dir == 4), du(f2.z, dir == 5));
    const bool rot = dir == 9;
    const Du kx = du(m.kx, rot ? -m.ky : 0.0), ky = du(m.ky, rot ? m.kx : 0.0);
    const Du sx = du(m.sx, rot ? -m.sy : 0.0), sy = du(m.sy, rot ? m.sx : 0.0);
    const Du phi = membran_phi(F1, F2, m.r, kx, ky, sx, sy, m.fl, du(m.ek, dir == 6), du(m.es, dir == 7),
                               du(m.g, dir == 8), mu, u, h);
    j.om[q] = phi.d;
  }
}
// Directions per hinge: 0-11 the coordinates of its four points, 12 k.
__global__ void __launch_bounds__(kBlock) adj_biegung_kernel(const __grid_constant__ StepArgs a,
                                                              const __grid_constant__ AdjArgs j) {
  const double h = a.h;
  K3D_FOR(q, 13 * a.nb) {
    const int64_t b = q % a.nb;
    const int dir = int(q / a.nb);
    const uint4 id = __ldg(&a.b_idx[b]);
    const double2 kr = __ldg(&a.b_kr[b]);
    const uint32_t ids[4] = {id.x, id.y, id.z, id.w};
    U3 p[4];
    D3 mu[4], u[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const D3 x = ld3(j.x, ids[k]);
      p[k] = u3(du(x.x, dir == 3 * k), du(x.y, dir == 3 * k + 1), du(x.z, dir == 3 * k + 2));
      mu[k] = ld3(j.mu, ids[k]);
      u[k] = ld3(j.v, ids[k]) + ld3(j.dv, ids[k]);
    }
    j.ob[q] = biegung_phi(p, du(kr.x, dir == 12), kr.y, mu, u, h).d;
  }
}
// Directions per spring: 0-2 the coordinates of end i, 3-5 those of end j.
__global__ void __launch_bounds__(kBlock) adj_feder_kernel(const __grid_constant__ StepArgs a,
                                                            const __grid_constant__ AdjArgs j) {
  const double h = a.h;
  K3D_FOR(q, 6 * a.ns) {
    const int64_t s = q % a.ns;
    const int dir = int(q / a.ns);
    const uint4 id = __ldg(&a.s_idx[s]);
    const double2 kl = a.s_kl[s];
    const D3 xi = ld3(j.x, id.x), xj = ld3(j.x, id.y);
    const U3 Xi = u3(du(xi.x, dir == 0), du(xi.y, dir == 1), du(xi.z, dir == 2));
    const U3 Xj = u3(du(xj.x, dir == 3), du(xj.y, dir == 4), du(xj.z, dir == 5));
    const D3 ui = ld3(j.v, id.x) + ld3(j.dv, id.x), uj = ld3(j.v, id.y) + ld3(j.dv, id.y);
    j.os[q] = feder_phi(id.z == 0 ? 0 : 1, Xi, Xj, kl.x, kl.y, ld3(j.mu, id.x), ld3(j.mu, id.y), ui, uj, h).d;
  }
}

// Per point: the element derivatives of its corners, in the build's corner
// order (deterministic); out: the cotangents of the substep's input x, v.
__global__ void __launch_bounds__(kBlock) adj_gather_kernel(const __grid_constant__ StepArgs a,
                                                             const __grid_constant__ AdjArgs j) {
  const int64_t T = a.nt, B = a.nb, S = a.ns;
  K3D_FOR(i, a.n) {
    const uint32_t ui = uint32_t(i);
    D3 g = ld3(j.xa, ui);
    for (uint32_t e = a.off_t[i]; e < a.off_t[i + 1]; ++e) {
      const uint32_t q = a.ent_t[e], t = q / 3u, k = q % 3u;
      const double4 r = a.m_r[t];
      const double c1 = k == 0 ? -(r.x + r.z) : (k == 1 ? r.x : r.z);
      const double c2 = k == 0 ? -(r.y + r.w) : (k == 1 ? r.y : r.w);
      g = g + d3(j.om[t], j.om[T + t], j.om[2 * T + t]) * c1 + d3(j.om[3 * T + t], j.om[4 * T + t], j.om[5 * T + t]) * c2;
    }
    for (uint32_t e = a.off_b[i]; e < a.off_b[i + 1]; ++e) {
      const uint32_t q = a.ent_b[e], b = q / 4u, k = q % 4u;
      g = g + d3(j.ob[(3 * k) * B + b], j.ob[(3 * k + 1) * B + b], j.ob[(3 * k + 2) * B + b]);
    }
    for (uint32_t e = a.off_s[i]; e < a.off_s[i + 1]; ++e) {
      const uint32_t q = a.ent_s[e], s = q >> 1, end = q & 1u;
      g = g + d3(j.os[(3 * end) * S + s], j.os[(3 * end + 1) * S + s], j.os[(3 * end + 2) * S + s]);
    }
    st3(j.xq, ui, g);
    st3(j.vq, ui, ld3(j.va, ui));
  }
}

__global__ void __launch_bounds__(kBlock) adj_params_kernel(const __grid_constant__ StepArgs a,
                                                             const __grid_constant__ AdjArgs j) {
  K3D_FOR(q, 4 * a.nt) j.acc_m[q] += j.om[6 * a.nt + q];
  K3D_FOR(b, a.nb) j.acc_b[b] += j.ob[12 * a.nb + b];
}

int g_sms = 0;

cudaError_t grid(const void* fn, void** args, int64_t work, cudaStream_t st) {
  if (g_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) g_sms = 148;
  }
  int64_t blocks = (work + kBlock - 1) / kBlock;
  const int64_t cap = int64_t(g_sms) * 16;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return cudaLaunchKernel(fn, dim3(unsigned(blocks)), dim3(kBlock), args, 0, st);
}

}  // namespace

cudaError_t launch_adjoint_step(const StepArgs& a0, const AdjArgs& j, int blocks, cudaStream_t st, int& launched) {
  StepArgs a = a0;
  a.first_step = 0;
  a.need_load = 0;
  a.adjoint = 0;
  a.rec_flags = nullptr;
  a.stats = j.stats;
  a.stat_rest_max = j.rest;
  a.dv = j.lam;
  const BuildKernels K = build_kernels(0);
  const int64_t elems = a.nt > a.nb ? (a.nt > a.ns ? a.nt : a.ns) : (a.nb > a.ns ? a.nb : a.ns);
  cudaError_t e;
  launched = 0;
  void* a1[] = {(void*)&a};
  void* a2[] = {(void*)&a, (void*)&j};
  auto run1 = [&](const void* fn, int64_t work) {
    ++launched;
    return grid(fn, a1, work, st);
  };
  auto run2 = [&](const void* fn, int64_t work) {
    ++launched;
    return grid(fn, a2, work, st);
  };
  auto spmv = [&](const double* x, double* y) {
    void* as[] = {(void*)&a, (void*)&x, (void*)&y};
    ++launched;
    return grid((const void*)adj_spmv_kernel, as, a.n, st);
  };
  // the system at the recorded input state, with the final contact set
  if ((e = run1(K.elements, elems)) != cudaSuccess) return e;
  if ((e = run1(K.points, a.n)) != cudaSuccess) return e;
  if ((e = run1(K.assemble, a.bplane)) != cudaSuccess) return e;
  if ((e = run2((const void*)adj_final_set_kernel, a.n)) != cudaSuccess) return e;
  // rho = A dv - b; the point stages backwards; g = dv_bar + A rho_bar
  if ((e = spmv(j.dv, j.adv)) != cudaSuccess) return e;
  if ((e = run2((const void*)adj_integrate_kernel, a.n)) != cudaSuccess) return e;
  if ((e = spmv(j.rq, j.arq)) != cudaSuccess) return e;
  if ((e = run2((const void*)adj_rhs_kernel, 3 * a.n)) != cudaSuccess) return e;
  // S A S lam = S g
  StepArgs s = a;
  s.b = j.gg;
  s.adjoint = 1;
  if ((e = launch_pcg64(s, blocks, st)) != cudaSuccess) return e;
  ++launched;
  if ((e = spmv(j.lam, j.alam)) != cudaSuccess) return e;
  if ((e = run2((const void*)adj_points_kernel, a.n)) != cudaSuccess) return e;
  if (a.nt > 0 && (e = run2((const void*)adj_membran_kernel, 10 * a.nt)) != cudaSuccess) return e;
  if (a.nb > 0 && (e = run2((const void*)adj_biegung_kernel, 13 * a.nb)) != cudaSuccess) return e;
  if (a.ns > 0 && (e = run2((const void*)adj_feder_kernel, 6 * a.ns)) != cudaSuccess) return e;
  if ((e = run2((const void*)adj_gather_kernel, a.n)) != cudaSuccess) return e;
  if ((e = run2((const void*)adj_params_kernel, 4 * a.nt > a.nb ? 4 * a.nt : a.nb)) != cudaSuccess) return e;
  return cudaSuccess;
}

}  // namespace k3d
