// ORACLE (test infrastructure). FP64 CPU adjoint of one implicit substep
// (ImplizitCg::schritt, implizit.rs:899-1038), the check for the device
// adjoint. The reference has no adjoint; this is derived from the forward
// restatement in implizit.cpp with every discrete decision of the recorded
// substep frozen: the contact set of the last solve and after the release
// pass (a second release pass ends the loop, so points it releases keep
// their constraint in dv but get no friction), stick or slip, and which
// bodies pushed a point out. Element and contact derivatives are taken
// by central differences of this oracle's own element and contact functions
// (local to one element or point, so they are well conditioned), which keeps
// the check independent of the device's forward-mode derivatives.
//
// Forward substep with the decisions frozen (h = substep, u = v + dv):
//   S (A dv - b) = 0, (I - S) dv = n (vn_soll - v.n) on held points,
//   A = M(1 + hc) + h^2 H(x), b = h (f(x, v) - h H(x) v)
//   v1 = v + dv; friction on held points; x1 = x + h v2; push-outs.
// Backward, with Phi = b - A dv (dv fixed):
//   g = dv_bar + A rho_bar                 (rho = A dv - b, from slipping points)
//   S A S lam = S g, lam in range(S)       (adjoint PCG on the filtered system)
//   mu = lam - rho_bar
//   v_bar += M mu - A mu,  x_bar, theta_bar += grad of mu.Phi
//   held points: zeta = n.(g - A lam); the constraint and the normal's
//   dependence on x add zeta and n_bar terms.
#include <algorithm>
#include <cfloat>

#include "oracle.hpp"

namespace orc {
namespace {

// h mu.f_e - h^2 mu.(H_e u) of one membrane
double phi_membran(const Membran& m, const std::array<V3, 3>& p, const std::array<V3, 3>& mu,
                   const std::array<V3, 3>& u, double h) {
  auto F = membran_krafte(m, p);
  auto hu = membran_mal_h_aus(m, membran_hessen(m, p), u);
  double s = 0.0;
  for (int k = 0; k < 3; ++k) s += h * dot(mu[k], F[k]) - h * h * dot(mu[k], hu[k]);
  return s;
}
// the same for one hinge (implizit.rs:774-796 force, :198-203 product)
double phi_biegung(const std::array<V3, 4>& p, double k, double ruhe, const std::array<V3, 4>& mu,
                   const std::array<V3, 4>& u, double h) {
  double theta = 0.0;
  std::array<V3, 4> gr{};
  if (!dieder(p, theta, gr)) return 0.0;
  double fehler = winkel_fehler(theta, ruhe);
  double gu = 0.0;
  for (int m = 0; m < 4; ++m) gu += dot(gr[m], u[m]);
  double s = 0.0;
  for (int m = 0; m < 4; ++m) s += h * dot(mu[m], mul(gr[m], -k * fehler)) - h * h * dot(mu[m], mul(gr[m], k * gu));
  return s;
}
// one pattern edge (art 0) or seam (art 1) between i and j (implizit.rs:742-771)
double phi_feder(int art, V3 xi, V3 xj, double k, double l0, V3 mui, V3 muj, V3 ui, V3 uj, double h) {
  V3 d = sub(xj, xi);
  V3 fi, r;
  double quer;
  if (art == 0) {
    double l = std::max(norm(d), 1e-12);
    r = mul(d, 1.0 / l);
    fi = mul(r, k * (l - l0));
    quer = std::max(1.0 - l0 / l, 0.0);
  } else {
    double l = norm(d);
    if (!std::isfinite(l0)) l0 = l;
    if (l0 > 0.0 && l > 1e-12) {
      fi = mul(d, k * (l - l0) / l);
      r = mul(d, 1.0 / l);
      quer = std::max(1.0 - l0 / l, 0.0);
    } else {
      fi = mul(d, k);
      r = {0, 0, 0};
      quer = 1.0;
    }
  }
  V3 du = sub(ui, uj);
  V3 bd = mul(add(mul(r, dot(r, du) * (1.0 - quer)), mul(du, quer)), k);
  V3 dm = sub(mui, muj);
  return h * dot(dm, fi) - h * h * dot(dm, bd);
}

void dreh(V2 w, double a, V2& out) {
  double c = std::cos(a), s = std::sin(a);
  out = {c * w[0] - s * w[1], s * w[0] + c * w[1]};
}
Membran gedreht(const Membran& m, double a) {
  Membran o = m;
  dreh(m.kette, a, o.kette);
  dreh(m.schuss, a, o.schuss);
  return o;
}

// Contact normal and depth of the last body in contact at x (the build's
// rule, implizit.rs:873-883), with their x-derivatives by central differences
// of Koerper::kontakt. Returns false if no body is in contact.
struct KontaktAbl {
  V3 n{};
  double tiefe = 0;
  M3 dn{};    // dn[a][c] = d n_a / d x_c
  V3 dtiefe{};
};
bool kontakt_abl(const Koerper& kb, V3 x, double abstand, KontaktAbl& o) {
  auto k0 = kb.kontakt(x, abstand);
  if (!k0) return false;
  o.n = k0->normale;
  o.tiefe = k0->tiefe;
  const double eps = 1e-7;
  for (int c = 0; c < 3; ++c) {
    V3 xp = x, xm = x;
    xp[c] += eps;
    xm[c] -= eps;
    auto kp = kb.kontakt(xp, abstand), km = kb.kontakt(xm, abstand);
    // one-sided at the rim of the contact band
    V3 np = kp ? kp->normale : k0->normale, nm = km ? km->normale : k0->normale;
    double tp = kp ? kp->tiefe : k0->tiefe, tm = km ? km->tiefe : k0->tiefe;
    double sp = kp ? eps : 0.0, sm = km ? eps : 0.0;
    double span = sp + sm;
    if (span == 0.0) continue;
    for (int a = 0; a < 3; ++a) o.dn[a][c] = (np[a] - nm[a]) / span;
    o.dtiefe[c] = (tp - tm) / span;
  }
  return true;
}
V3 mtv(const M3& m, V3 v) {  // m^T v
  return {m[0][0] * v[0] + m[1][0] * v[1] + m[2][0] * v[2], m[0][1] * v[0] + m[1][1] * v[1] + m[2][1] * v[2],
          m[0][2] * v[0] + m[1][2] * v[1] + m[2][2] * v[2]};
}

}  // namespace

void ImplizitCg::adjoint_schritt(Szene& s, const Aufnahme& a, std::vector<V3>& xq, std::vector<V3>& vq,
                                 AdjGrad& g, std::vector<V3>& lam, AdjStat& st, double adj_toleranz) {
  const size_t n = a.x.size();
  const double h = a.h;
  s.x = a.x;
  s.v = a.v;
  s.koerper = a.koerper;
  std::vector<std::optional<Fest>> fest0;
  System sys = system_bauen(s, h, fest0);
  const auto& fest = a.fest;
  const auto& loes = a.fest_loes;
  // rho = A dv - b
  std::vector<V3> adv(n), rho(n);
  sys.mal_a(a.dv, adv);
  for (size_t i = 0; i < n; ++i) rho[i] = sub(adv[i], sys.rhs[i]);

  // ---- friction, integration and push-outs, backwards per point
  std::vector<V3> gq(n), rq(n), nq(n), xa(n), va(n);
  for (size_t i = 0; i < n; ++i) {
    if (s.w[i] <= 0.0) {
      xa[i] = xq[i];
      va[i] = vq[i];
      continue;
    }
    // replay of the forward
    const V3 v1 = add(a.v[i], a.dv[i]);
    V3 v2 = v1, nn{}, vk{}, rel{}, t{};
    double lt = 0.0, grenze = 0.0;
    const bool held = fest[i].has_value();
    if (held) {
      nn = fest[i]->normale;
      vk = fest[i]->v_koerper;
      rel = sub(v1, vk);
      t = sub(rel, mul(nn, dot(rel, nn)));
      lt = norm(t);
      grenze = s.reibung[i] * a.fn[i] * h * s.w[i];
      if (a.reib[i] == 1)
        v2 = sub(v1, t);
      else if (a.reib[i] == 2)
        v2 = sub(v1, mul(t, grenze / lt));
    }
    const size_t nk = a.koerper.size();
    std::vector<V3> xs(nk), vs(nk);
    V3 x = add(a.x[i], mul(v2, h)), v = v2;
    for (size_t kb = 0; kb < nk; ++kb) {
      xs[kb] = x;
      vs[kb] = v;
      if (!(a.stoss[i] & (1u << (2 * kb)))) continue;
      auto kt = a.koerper[kb].kontakt(x, s.kollisionsabstand[i]);
      x = add(x, mul(kt->normale, kt->tiefe));
      if (a.stoss[i] & (1u << (2 * kb + 1))) v = sub(v, mul(kt->normale, dot(sub(v, kt->geschwindigkeit), kt->normale)));
    }
    // backwards through the push-outs
    V3 xb = xq[i], vb = vq[i];
    for (size_t kb = nk; kb-- > 0;) {
      if (!(a.stoss[i] & (1u << (2 * kb)))) continue;
      KontaktAbl ka;
      kontakt_abl(a.koerper[kb], xs[kb], s.kollisionsabstand[i], ka);
      V3 nbar = mul(xb, ka.tiefe);
      const double tbar = dot(xb, ka.n);
      if (a.stoss[i] & (1u << (2 * kb + 1))) {
        const V3 vr = sub(vs[kb], a.koerper[kb].geschwindigkeit);
        nbar = sub(nbar, add(mul(vb, dot(ka.n, vr)), mul(vr, dot(ka.n, vb))));
        vb = sub(vb, mul(ka.n, dot(ka.n, vb)));
      }
      xb = add(add(xb, mtv(ka.dn, nbar)), mul(ka.dtiefe, tbar));
    }
    // x1 = x + h v2
    xa[i] = xb;
    const V3 v2b = add(vb, mul(xb, h));
    V3 v1b = v2b;
    if (held && a.reib[i] == 1) {
      v1b = mul(nn, dot(nn, v2b));
      nq[i] = add(nq[i], add(mul(v2b, dot(nn, rel)), mul(rel, dot(nn, v2b))));
    } else if (held && a.reib[i] == 2) {
      const double sk = grenze / lt;
      const V3 th = mul(t, 1.0 / lt);
      const V3 q = mul(sub(v2b, mul(th, dot(th, v2b))), sk);
      v1b = sub(v2b, sub(q, mul(nn, dot(nn, q))));
      nq[i] = add(nq[i], add(mul(q, dot(nn, rel)), mul(rel, dot(nn, q))));
      const double gb = -dot(v2b, th) * s.reibung[i] * s.w[i];
      rq[i] = mul(nn, gb);
      nq[i] = add(nq[i], mul(rho[i], gb));
    }
    va[i] = v1b;
    gq[i] = v1b;
  }

  // ---- adjoint solve on the filtered system
  std::vector<V3> arq(n), gg(n);
  sys.mal_a(rq, arq);
  for (size_t i = 0; i < n; ++i) gg[i] = add(gq[i], arq[i]);
  System adj = sys;
  adj.rhs = gg;
  adj.cg_toleranz = adj_toleranz;
  adj.cg_max = 100000;
  std::vector<std::optional<Fest>> fa = loes;
  for (size_t i = 0; i < n; ++i)
    if (fa[i]) fa[i]->vn_soll = dot(a.v[i], fa[i]->normale);  // zero target
  if (lam.size() != n) lam.assign(n, V3{0, 0, 0});
  CgLauf lauf = cpu_loese(adj, fa, lam);
  st.cg_iterationen += lauf.iterationen;
  st.loesungen += 1;
  if (lauf.nicht_konvergiert) st.nicht_konvergiert += 1;
  std::vector<V3> alam(n), mu(n), amu(n);
  sys.mal_a(lam, alam);
  for (size_t i = 0; i < n; ++i) {
    mu[i] = sub(lam[i], rq[i]);
    amu[i] = sub(alam[i], arq[i]);
  }

  // ---- point terms: damping and the H v part of b, constraint, normals
  std::vector<V3> xo(n), vo(n);
  for (size_t i = 0; i < n; ++i) {
    xo[i] = xa[i];
    vo[i] = add(va[i], sub(mul(mu[i], s.masse[i]), amu[i]));
    if (!loes[i] || s.w[i] <= 0.0) continue;
    const V3 nn = loes[i]->normale;
    const double zeta = dot(nn, sub(gg[i], alam[i]));
    vo[i] = sub(vo[i], mul(nn, zeta));
    V3 nbar = nq[i];
    nbar = add(nbar, mul(lam[i], dot(nn, rho[i])));
    nbar = sub(nbar, mul(a.dv[i], zeta));
    nbar = add(nbar, mul(sub(loes[i]->v_koerper, a.v[i]), zeta));
    // the build's contact: the last body in contact at x
    KontaktAbl ka, kl;
    bool hat = false;
    for (const auto& kb : a.koerper)
      if (kontakt_abl(kb, a.x[i], s.kollisionsabstand[i] + param.kontakt_rand, ka)) {
        kl = ka;
        hat = true;
      }
    if (!hat) continue;
    xo[i] = add(xo[i], add(mul(kl.dtiefe, zeta / h), mtv(kl.dn, nbar)));
  }

  // ---- element terms: grad of mu.Phi, Phi = h f - h^2 H(x)(v + dv)
  std::vector<V3> u(n);
  for (size_t i = 0; i < n; ++i) u[i] = add(a.v[i], a.dv[i]);
  for (size_t t = 0; t < s.membran_elemente.size(); ++t) {
    const auto& me = s.membran_elemente[t];
    std::array<V3, 3> p, m3, u3;
    double lmax = 0.0;
    for (int k = 0; k < 3; ++k) {
      p[k] = a.x[me.punkte[k]];
      m3[k] = mu[me.punkte[k]];
      u3[k] = u[me.punkte[k]];
    }
    for (int k = 1; k < 3; ++k) lmax = std::max(lmax, norm(sub(p[k], p[0])));
    const double ex = 1e-7 * lmax;
    for (int k = 0; k < 3; ++k)
      for (int c = 0; c < 3; ++c) {
        auto pp = p, pm = p;
        pp[k][c] += ex;
        pm[k][c] -= ex;
        const double d = (phi_membran(me.element, pp, m3, u3, h) - phi_membran(me.element, pm, m3, u3, h)) / (2 * ex);
        xo[me.punkte[k]][c] += d;
      }
    const double ep = 1e-6;
    for (int q = 0; q < 3; ++q) {
      Membran mp = me.element, mm = me.element;
      double* fp = q == 0 ? &mp.kette_n_m : q == 1 ? &mp.dehnung_n_m : &mp.schub_n_m;
      double* fm = q == 0 ? &mm.kette_n_m : q == 1 ? &mm.dehnung_n_m : &mm.schub_n_m;
      const double e0 = *fp, de = ep * std::max(std::abs(e0), 1e-30);
      *fp = e0 + de;
      *fm = e0 - de;
      g.membran[t][q] += (phi_membran(mp, p, m3, u3, h) - phi_membran(mm, p, m3, u3, h)) / (2 * de);
    }
    g.membran[t][3] +=
        (phi_membran(gedreht(me.element, ep), p, m3, u3, h) - phi_membran(gedreht(me.element, -ep), p, m3, u3, h)) /
        (2 * ep);
  }
  for (size_t b = 0; b < s.biegung.size(); ++b) {
    const auto& idx = s.biegung.punkte[b];
    const double k = 1.0 / s.biegung.nachgiebigkeit[b], ruhe = s.biegung.ruhe[b];
    std::array<V3, 4> p, m4, u4;
    for (int q = 0; q < 4; ++q) {
      p[q] = a.x[idx[q]];
      m4[q] = mu[idx[q]];
      u4[q] = u[idx[q]];
    }
    const double ex = 1e-7 * norm(sub(p[1], p[0]));
    for (int q = 0; q < 4; ++q)
      for (int c = 0; c < 3; ++c) {
        auto pp = p, pm = p;
        pp[q][c] += ex;
        pm[q][c] -= ex;
        xo[idx[q]][c] += (phi_biegung(pp, k, ruhe, m4, u4, h) - phi_biegung(pm, k, ruhe, m4, u4, h)) / (2 * ex);
      }
    // Phi is linear in k
    g.biegung[b] += phi_biegung(p, 1.0, ruhe, m4, u4, h);
  }
  auto federn = [&](int art, size_t e, uint32_t i, uint32_t j, double k, double l0) {
    const double ex = 1e-7 * std::max(norm(sub(a.x[j], a.x[i])), 1e-6);
    for (int side = 0; side < 2; ++side)
      for (int c = 0; c < 3; ++c) {
        V3 xi = a.x[i], xj = a.x[j], xi2 = a.x[i], xj2 = a.x[j];
        if (side == 0) {
          xi[c] += ex;
          xi2[c] -= ex;
        } else {
          xj[c] += ex;
          xj2[c] -= ex;
        }
        const double d = (phi_feder(art, xi, xj, k, l0, mu[i], mu[j], u[i], u[j], h) -
                          phi_feder(art, xi2, xj2, k, l0, mu[i], mu[j], u[i], u[j], h)) /
                         (2 * ex);
        xo[side == 0 ? i : j][c] += d;
      }
    (void)e;
  };
  for (size_t e = 0; e < s.abstand.size(); ++e) {
    if (e < s.membran_kante.size() && s.membran_kante[e]) continue;
    federn(0, e, s.abstand.punkte[e][0], s.abstand.punkte[e][1], 1.0 / s.abstand.nachgiebigkeit[e],
           s.abstand.ruhe[e]);
  }
  for (size_t e = 0; e < s.naht.size(); ++e)
    federn(1, e, s.naht.punkte[e][0], s.naht.punkte[e][1], param.naht_k, s.naht.ruhe[e]);
  xq = std::move(xo);
  vq = std::move(vo);
}

}  // namespace orc
