// The per-step build of the implicit system on the device, and the kernels
// around the PCG launch: element and point build (implizit.rs:663-896), the
// assembled block operator, the probes (ImplizitCg::operator / system_fuer)
// and friction and integration (implizit.rs:957-1014).
//
// This file is compiled without fused multiply-add contraction: every
// product and sum rounds on its own, as in the reference's Rust (which never
// fuses). The projection of the geometric stress (kontinuum.rs:158-177)
// subtracts nearly equal numbers when one normal strain is clamped and the
// shear is small; a one-ulp difference in its inputs then shows as a 1e-3
// relative difference in the element's tangent, so the build has to round
// exactly like the reference.
#include <cfloat>
#include <cstdint>

#include "k3d_step_common.cuh"

namespace k3d {

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
    if (a.sc_off) {  // proximity springs: force, -h H v, diagonal (implizit.rs:798-805, 887-894)
      for (uint32_t e = a.sc_off[i]; e < a.sc_off[i + 1]; ++e) {
        const uint32_t ent = a.sc_ent[e];
        const double4 kf = a.sc_kf[ent >> 3];
        const double4 g4 = a.sc_w[ent >> 3];
        const uint32_t k = ent & 7u;
        const double g = k == 0 ? g4.x : k == 1 ? g4.y : k == 2 ? g4.z : k == 3 ? g4.w : a.sc_g5[ent >> 3];
        acc = acc + d3(kf.x, kf.y, kf.z) * g;
      }
      const D3 hv = feder_hp64(a, i, [&](uint32_t j) { return ld3(a.v, j); }, D);
      acc = acc - hv * h;
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
      const int inst = a.pinst ? int(a.pinst[i]) : 0;
      for (int kb = 0; kb < a.n_bodies; ++kb) {
        if (a.bodies[kb].inst >= 0 && a.bodies[kb].inst != inst) continue;
        D3 nn, bv;
        double tiefe;
        if (kontakt_v(a.bodies[kb], xi, a.kabst[i] + a.kontakt_rand, nn, tiefe, bv)) {
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
    // the block as two 4-vectors (m00 m01 m02 m10), (m11 m12 m20 m21) and m22
    R4<R>* b4 = reinterpret_cast<R4<R>*>(bm);
    b4[sid] = R4<R>{R(B[0]), R(B[1]), R(B[2]), R(B[3])};
    b4[a.bplane + sid] = R4<R>{R(B[4]), R(B[5]), R(B[6]), R(B[7])};
    bm[8 * a.bplane + sid] = R(B[8]);
  }
}

// (A p)_i = sum over the row's blocks of B p_col, p = w + beta c from `buf`.

// ------------------------------------------------------------ friction + integration
// implizit.rs:957-1013: friction, the new position, the segment check against
// mesh bodies (entry point pushed out by the collision distance, the impact's
// normal velocity removed and Coulomb on the impact), the push-out.
__device__ void integrate(const StepArgs& a, double (&cnt)[4]) {
  const double h = a.h;
  K3D_FOR(i, a.n) {
    if (!a.frei[i]) {
      if (a.rec_flags) a.rec_flags[i] = 0u;
      continue;
    }
    uint32_t fl = 0u;
    D3 v = ld3(a.v, uint32_t(i)) + ld3(a.dv, uint32_t(i));
    const D3 n = ld3(a.nrm_d, uint32_t(i));
    if (n.x != 0.0 || n.y != 0.0 || n.z != 0.0) {
      fl |= 1u;
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
        fl |= 2u;
      } else if (lt > 0.0) {
        v = v - t * (grenze / lt);
        fl |= 4u;
      }
    }
    const D3 alt = ld3(a.x, uint32_t(i));
    D3 x = alt + v * h;
    const int inst = a.pinst ? int(a.pinst[i]) : 0;
    if (a.durchstoss_pruefen) {
      for (int kb = 0; kb < a.n_bodies; ++kb) {
        const Body& k = a.bodies[kb];
        if (k.art != 2 || (k.inst >= 0 && k.inst != inst)) continue;
        const D3 vers = d3(k.punkt[0], k.punkt[1], k.punkt[2]);
        D3 pl, nk;
        uint32_t t;
        if (netz::durchstoss(*k.netz, alt - vers, x - vers, pl, nk, t)) {
          cnt[3] += 1.0;
          x = (pl + vers) + nk * a.kabst[i];
          const D3 vk = netz::geschwindigkeit_an(*k.netz, t, pl, d3(k.vel[0], k.vel[1], k.vel[2]));
          const D3 rel = v - vk;
          const double vn = dot(rel, nk);
          if (vn < 0.0) {
            D3 tt = rel - nk * vn;
            const double lt = norm(tt);
            const double grenze = a.reib[i] * -vn;
            tt = lt <= grenze ? d3(0.0, 0.0, 0.0) : tt * (1.0 - grenze / lt);
            v = vk + tt;
          }
        }
      }
    }
    for (int kb = 0; kb < a.n_bodies; ++kb) {
      if (a.bodies[kb].inst >= 0 && a.bodies[kb].inst != inst) continue;
      D3 nn, bv;
      double tiefe;
      if (kontakt_v(a.bodies[kb], x, a.kabst[i], nn, tiefe, bv)) {
        x = x + nn * tiefe;
        const double vn = dot(v - bv, nn);
        if (vn < 0.0) v = v - nn * vn;
        if (kb < kMaxAdjointBodies) fl |= (1u << (4 + 2 * kb)) | (vn < 0.0 ? 1u << (5 + 2 * kb) : 0u);
      }
    }
    if (a.rec_flags) a.rec_flags[i] = fl | (a.rec_flags[i] & 8u);
    if (!(isfinite(x.x) && isfinite(x.y) && isfinite(x.z) && isfinite(v.x) && isfinite(v.y) && isfinite(v.z)))
      cnt[2] += 1.0;
    st3(a.x, uint32_t(i), x);
    st3(a.v, uint32_t(i), v);
  }
}


// ------------------------------------------------------------ body points against cloth triangles
// netzkoerper.rs:612-735 for mesh body kb: per cloth triangle the deepest
// stab of a body point (its line p + t n through the triangle at
// -tief < t < -1e-9; the first of equal depth in the point grid's order),
// then the triangles with a stab lifted in triangle order on one thread.
__global__ void __launch_bounds__(kBlock) kp_such_kernel(const __grid_constant__ StepArgs a, int kb) {
  if (a.kp_ctl[2]) return;
  const Body& k = a.bodies[kb];
  const netz::Dev& g = *k.netz;
  const double tief = a.kp_tief, band = -1e-9, rand = fmax(tief, band);
  const D3 vers = d3(k.punkt[0], k.punkt[1], k.punkt[2]);
  K3D_FOR(t, a.kp_nt) {
    const uint4 tr = a.kp_tri[t];
    if (k.inst >= 0 && a.pinst && int(a.pinst[tr.x]) != k.inst) continue;
    const D3 p0 = ld3(a.x, tr.x), p1 = ld3(a.x, tr.y), p2 = ld3(a.x, tr.z);
    D3 lo = d3(fmin(fmin(p0.x, p1.x), p2.x), fmin(fmin(p0.y, p1.y), p2.y), fmin(fmin(p0.z, p1.z), p2.z));
    D3 hi = d3(fmax(fmax(p0.x, p1.x), p2.x), fmax(fmax(p0.y, p1.y), p2.y), fmax(fmax(p0.z, p1.z), p2.z));
    lo = (lo - vers) - d3(rand, rand, rand);
    hi = (hi - vers) + d3(rand, rand, rand);
    const D3 e1 = p1 - p0, e2 = p2 - p0;
    int r0[3], r1[3];
    if (!netz::bereich(g, lo, hi, r0, r1)) continue;
    bool hat = false;
    double dbest = 0.0;
    D3 nb = d3(0, 0, 0), bb = d3(0, 0, 0);
    uint32_t kir = 0;
    for (int kz = r0[2]; kz <= r1[2]; ++kz)
      for (int ky = r0[1]; ky <= r1[1]; ++ky)
        for (int kx = r0[0]; kx <= r1[0]; ++kx) {
          const int64_t z = (int64_t(kz) * g.zy + ky) * g.zx + kx;
          for (uint32_t e = g.pg_anf[z]; e < g.pg_anf[z + 1]; ++e) {
            const uint32_t q = g.pg_ein[e];
            const D3 p = netz::punkt(g, q) + vers;
            const D3 n = netz::ld4(g.pn[q]);
            const D3 pv = cross(n, e2);
            const double det = dot(e1, pv);
            if (fabs(det) < 1e-18) continue;
            const D3 tv = p - p0;
            const double bu = dot(tv, pv) / det;
            if (!(bu >= 0.0 && bu <= 1.0)) continue;
            const D3 qv = cross(tv, e1);
            const double bv = dot(n, qv) / det;
            if (bv < 0.0 || bu + bv > 1.0) continue;
            const double tt = dot(e2, qv) / det;
            if (tt > -tief && tt < band && (!hat || -tt > dbest)) {
              hat = true;
              dbest = -tt;
              nb = n;
              bb = d3(1.0 - bu - bv, bu, bv);
              kir = q;
            }
          }
        }
    if (hat) {
      a.kp_a[t] = make_double4(dbest, nb.x, nb.y, nb.z);
      a.kp_b[t] = make_double4(bb.x, bb.y, bb.z, double(kir));
      a.kp_list[atomicAdd(&a.kp_ctl[0], 1u)] = uint32_t(t);
    }
  }
}
constexpr uint32_t kKpSort = 4096;
__global__ void __launch_bounds__(1024) kp_anwenden_kernel(const __grid_constant__ StepArgs a, int kb) {
  __shared__ uint32_t sh[kKpSort];
  if (a.kp_ctl[2]) return;
  const uint32_t m = a.kp_ctl[0] < a.kp_nt ? a.kp_ctl[0] : uint32_t(a.kp_nt);
  uint32_t* list = a.kp_list;
  // the listed triangles in ascending order
  if (m > 1 && m <= kKpSort) {
    uint32_t p2 = 1;
    while (p2 < m) p2 <<= 1;
    for (uint32_t i = threadIdx.x; i < p2; i += blockDim.x) sh[i] = i < m ? list[i] : 0xffffffffu;
    __syncthreads();
    for (uint32_t s = 2; s <= p2; s <<= 1)
      for (uint32_t j = s >> 1; j > 0; j >>= 1) {
        for (uint32_t i = threadIdx.x; i < p2; i += blockDim.x) {
          const uint32_t o = i ^ j;
          if (o > i) {
            const bool auf = (i & s) == 0;
            const uint32_t x = sh[i], y = sh[o];
            if ((x > y) == auf) sh[i] = y, sh[o] = x;
          }
        }
        __syncthreads();
      }
    list = sh;
  } else if (m > kKpSort && threadIdx.x == 0) {  // insertion by Ciura's gaps on one thread
    const uint32_t gaps[8] = {701u, 301u, 132u, 57u, 23u, 10u, 4u, 1u};
    for (int gi = 0; gi < 8; ++gi)
      for (uint32_t i = gaps[gi]; i < m; ++i) {
        const uint32_t key = list[i];
        uint32_t j = i;
        while (j >= gaps[gi] && list[j - gaps[gi]] > key) {
          list[j] = list[j - gaps[gi]];
          j -= gaps[gi];
        }
        list[j] = key;
      }
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const Body& k = a.bodies[kb];
  const netz::Dev& g = *k.netz;
  const D3 starr = d3(k.vel[0], k.vel[1], k.vel[2]);
  unsigned zahl = 0;
  for (uint32_t q = 0; q < m; ++q) {
    const uint32_t t = list[q];
    const double4 A = a.kp_a[t], B = a.kp_b[t];
    const uint4 tr = a.kp_tri[t];
    const uint32_t idx[3] = {tr.x, tr.y, tr.z};
    const double bary[3] = {B.x, B.y, B.z}, gew[3] = {a.w[tr.x], a.w[tr.y], a.w[tr.z]};
    double nenner = -0.0;
    for (int j = 0; j < 3; ++j) nenner += bary[j] * bary[j] * gew[j];
    if (nenner <= 0.0) continue;
    const D3 n = d3(A.y, A.z, A.w);
    const D3 vk = g.pv ? ld3(g.pv, uint32_t(B.w)) : starr;
    D3 vq = d3(0.0, 0.0, 0.0);
    for (int j = 0; j < 3; ++j) vq = vq + ld3(a.v, idx[j]) * bary[j];
    vq = vq - vk;
    const double vn = fmin(dot(vq, n), 0.0);
    for (int j = 0; j < 3; ++j) {
      const double f = bary[j] * gew[j] / nenner;
      st3(a.x, idx[j], ld3(a.x, idx[j]) + n * (f * A.x));
      st3(a.v, idx[j], ld3(a.v, idx[j]) - n * (f * vn));
    }
    ++zahl;
  }
  a.kp_ctl[1] += zahl;
  a.kp_ctl[0] = 0u;
  if (zahl) atomicAdd(reinterpret_cast<unsigned long long*>(&a.stats[ST_BODY_POINTS]), (unsigned long long)zahl);
}
// end of a pass: stop when it corrected nothing (implizit.rs:1023-1025)
__global__ void kp_ende_kernel(const __grid_constant__ StepArgs a) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  if (!a.kp_ctl[2] && a.kp_ctl[1] == 0u) a.kp_ctl[2] = 1u;
  a.kp_ctl[1] = 0u;
}

cudaError_t launch_koerperpunkte(const StepArgs& a, cudaStream_t st, int& launched) {
  if (a.kp_passes <= 0 || a.kp_nt <= 0) return cudaSuccess;
  cudaError_t e;
  if ((e = cudaMemsetAsync(a.kp_ctl, 0, 4 * sizeof(unsigned), st)) != cudaSuccess) return e;
  int64_t b = (a.kp_nt + kBlock - 1) / kBlock;
  const unsigned grid = unsigned(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
  for (int pass = 0; pass < a.kp_passes; ++pass) {
    for (int kb = 0; kb < a.n_bodies; ++kb) {
      if (a.bodies[kb].art != 2) continue;
      kp_such_kernel<<<grid, kBlock, 0, st>>>(a, kb);
      kp_anwenden_kernel<<<1, 1024, 0, st>>>(a, kb);
      launched += 2;
    }
    kp_ende_kernel<<<1, 32, 0, st>>>(a);
    launched += 1;
  }
  return cudaGetLastError();
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

__global__ void __launch_bounds__(kBlock) integrate_kernel(const __grid_constant__ StepArgs a) {
  __shared__ double red[4][32];
  double cnt[4] = {0.0, 0.0, 0.0, 0.0};
  integrate(a, cnt);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double x = cnt[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int slot[4] = {ST_CONTACTS, ST_STICKING, ST_NONFINITE, ST_PENETRATIONS};
    for (int k = 0; k < 4; ++k) {
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
    if (a.sc_off) {
      const D3 sp = feder_hp64(
          a, i,
          [&](uint32_t j) {
            const R4<R> c = vw.cw[j].w;
            return d3(double(c.x), double(c.y), double(c.z));
          },
          nullptr);
      hx += R(sp.x);
      hy += R(sp.y);
      hz += R(sp.z);
    }
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


template <typename R>
static BuildKernels kernels_t() {
  BuildKernels k;
  k.elements = (const void*)build_elements_kernel<R>;
  k.points = (const void*)build_points_kernel<R>;
  k.assemble = (const void*)assemble_kernel<R>;
  k.probe_load = (const void*)probe_load_kernel<R>;
  k.probe_apply = (const void*)apply_kernel<R>;
  k.probe_out = (const void*)probe_out_kernel<R>;
  k.integrate = (const void*)integrate_kernel;
  return k;
}

BuildKernels build_kernels(int precision) { return precision == 0 ? kernels_t<double>() : kernels_t<float>(); }

}  // namespace k3d
