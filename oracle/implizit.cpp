// ORACLE (test infrastructure). Restatement of the implicit CG step
// (sim/src/implizit.rs) in FP64, same loops and summation order: System::mal_h,
// mal_a, diag, CpuLoeser::loese, ImplizitCg::system_bauen / schritt / bild.
// Glue zones, and the penetration and impact stages of self-collision, are
// not part of this restatement; its proximity springs are (selbst.cpp).
#include <algorithm>
#include <cfloat>
#include <limits>

#include "oracle.hpp"

namespace orc {
namespace {
// implizit.rs:429-443
void m3_add_skal(M3& m, double s) {
  for (int k = 0; k < 3; ++k) m[k][k] += s;
}
void m3_add_aus(M3& m, V3 a, V3 b, double s) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) m[i][j] += s * a[i] * b[j];
}
// implizit.rs:283-288
V3 filtern(const std::optional<Fest>& f, V3 v) { return f ? sub(v, mul(f->normale, dot(v, f->normale))) : v; }
}  // namespace

V3 m3_mal(const M3& m, V3 v) { return {dot(m[0], v), dot(m[1], v), dot(m[2], v)}; }
// implizit.rs:444-453
M3 m3_inv(const M3& m) {
  double a = m[0][0], b = m[0][1], c = m[0][2], d = m[1][0], e = m[1][1], f = m[1][2], g = m[2][0], h = m[2][1],
         i = m[2][2];
  double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
  double s = 1.0 / det;
  return {V3{(e * i - f * h) * s, (c * h - b * i) * s, (b * f - c * e) * s},
          V3{(f * g - d * i) * s, (a * i - c * g) * s, (c * d - a * f) * s},
          V3{(d * h - e * g) * s, (b * g - a * h) * s, (a * e - b * d) * s}};
}

// implizit.rs:63-70: the (first side, second side, |g_q g_r|) pairs of a spring
template <typename F>
static void feder_paare(const Feder& fe, F&& f) {
  for (int q = 0; q < 5; ++q)
    for (int r = 0; r < 5; ++r) {
      double gq = fe.gewichte[q], gr = fe.gewichte[r];
      if (gq > 0.0 && gr < 0.0) f(size_t(fe.punkte[q]), size_t(fe.punkte[r]), -gq * gr);
    }
}

// implizit.rs:185-221
void System::mal_h(const std::vector<V3>& p, std::vector<V3>& out) const {
  for (auto& o : out) o = {0, 0, 0};
  auto federn = [&](const std::vector<Kante>& ks) {
    for (const auto& k : ks) {
      if (k.k == 0.0) continue;
      V3 d = sub(p[k.i], p[k.j]);
      V3 bd = mul(add(mul(k.richtung, dot(k.richtung, d) * (1.0 - k.quer)), mul(d, k.quer)), k.k);
      out[k.i] = add(out[k.i], bd);
      out[k.j] = sub(out[k.j], bd);
    }
  };
  federn(kanten);
  federn(naehte);
  for (const auto& b : biegungen) {
    double gp = 0.0;
    for (int m = 0; m < 4; ++m) gp += dot(b.grad[m], p[b.punkte[m]]);
    for (int m = 0; m < 4; ++m) out[b.punkte[m]] = add(out[b.punkte[m]], mul(b.grad[m], b.k * gp));
  }
  for (size_t t = 0; t < membran->size(); ++t) {
    const auto& m = (*membran)[t];
    std::array<V3, 3> d3 = {p[m.punkte[0]], p[m.punkte[1]], p[m.punkte[2]]};
    auto hu = membran_mal_h_aus(m.element, membran_h[t], d3);
    for (int k = 0; k < 3; ++k) out[m.punkte[k]] = add(out[m.punkte[k]], hu[k]);
  }
  for (const auto& fe : this->federn)
    feder_paare(fe, [&](size_t q, size_t r, double om) {
      V3 t = mul(m3_mal(fe.block, sub(p[q], p[r])), om);
      out[q] = add(out[q], t);
      out[r] = sub(out[r], t);
    });
}
// implizit.rs:224-229
void System::mal_a(const std::vector<V3>& p, std::vector<V3>& out) const {
  mal_h(p, out);
  for (size_t i = 0; i < p.size(); ++i)
    out[i] = add(mul(out[i], h * h), mul(p[i], (*masse)[i] * (1.0 + h * c)));
}
// implizit.rs:232-279
std::vector<M3> System::diag() const {
  double h2 = h * h;
  std::vector<M3> dg(masse->size());
  for (size_t i = 0; i < dg.size(); ++i) {
    dg[i] = {};
    m3_add_skal(dg[i], (*masse)[i] * (1.0 + h * c));
  }
  auto federn = [&](const std::vector<Kante>& ks) {
    for (const auto& k : ks) {
      if (k.k == 0.0) continue;
      for (uint32_t q : {k.i, k.j}) {
        m3_add_skal(dg[q], k.k * h2 * k.quer);
        m3_add_aus(dg[q], k.richtung, k.richtung, k.k * h2 * (1.0 - k.quer));
      }
    }
  };
  federn(kanten);
  federn(naehte);
  for (const auto& b : biegungen)
    for (int m = 0; m < 4; ++m) m3_add_aus(dg[b.punkte[m]], b.grad[m], b.grad[m], b.k * h2);
  for (size_t t = 0; t < membran->size(); ++t) {
    const auto& m = (*membran)[t];
    auto bl = membran_diag_bloecke_aus(m.element, membran_h[t]);
    for (int k = 0; k < 3; ++k)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) dg[m.punkte[k]][a][b] += h2 * bl[k][a][b];
  }
  for (const auto& fe : this->federn)
    feder_paare(fe, [&](size_t q, size_t r, double om) {
      for (size_t pt : {q, r})
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) dg[pt][a][b] += h2 * om * fe.block[a][b];
    });
  return dg;
}

// implizit.rs:370-426 (CpuLoeser::loese, modified PCG of Baraff & Witkin)
CgLauf cpu_loese(const System& sys, const std::vector<std::optional<Fest>>& fest, std::vector<V3>& dv) {
  const size_t n = sys.masse->size();
  const auto& w = *sys.w;
  const auto& b = sys.rhs;
  const auto& pinv = sys.pinv;
  for (size_t i = 0; i < n; ++i) {
    if (w[i] <= 0.0) {
      dv[i] = {0, 0, 0};
      continue;
    }
    if (fest[i]) {
      double soll = fest[i]->vn_soll - dot((*sys.v)[i], fest[i]->normale);
      dv[i] = add(filtern(fest[i], dv[i]), mul(fest[i]->normale, soll));
    }
  }
  std::vector<V3> ap(n), r(n), z(n), cdir(n);
  sys.mal_a(dv, ap);
  for (size_t i = 0; i < n; ++i) r[i] = w[i] > 0.0 ? filtern(fest[i], sub(b[i], ap[i])) : V3{0, 0, 0};
  double bb = 0.0;
  for (size_t i = 0; i < n; ++i)
    if (w[i] > 0.0) {
      V3 fb = filtern(fest[i], b[i]);
      bb += dot(fb, m3_mal(pinv[i], fb));
    }
  for (size_t i = 0; i < n; ++i) z[i] = m3_mal(pinv[i], r[i]);
  for (size_t i = 0; i < n; ++i) cdir[i] = filtern(fest[i], z[i]);
  double delta = 0.0;
  for (size_t i = 0; i < n; ++i) delta += dot(r[i], cdir[i]);
  double boden = 0.0;
  for (double m : *sys.masse) boden += m;
  boden *= 1e-18;
  double ziel = std::max(sys.cg_toleranz * sys.cg_toleranz * std::max(bb, delta), boden);
  size_t it = 0;
  while (delta > ziel && it < sys.cg_max) {
    sys.mal_a(cdir, ap);
    for (size_t i = 0; i < n; ++i) ap[i] = w[i] > 0.0 ? filtern(fest[i], ap[i]) : V3{0, 0, 0};
    double ca = 0.0;
    for (size_t i = 0; i < n; ++i) ca += dot(cdir[i], ap[i]);
    if (ca <= DBL_MIN || !std::isfinite(ca)) break;
    double alpha = delta / ca;
    for (size_t i = 0; i < n; ++i) {
      dv[i] = add(dv[i], mul(cdir[i], alpha));
      r[i] = sub(r[i], mul(ap[i], alpha));
    }
    for (size_t i = 0; i < n; ++i) z[i] = m3_mal(pinv[i], r[i]);
    double neu = 0.0;
    for (size_t i = 0; i < n; ++i) neu += dot(r[i], z[i]);
    double beta = neu / delta;
    delta = neu;
    for (size_t i = 0; i < n; ++i) cdir[i] = w[i] > 0.0 ? filtern(fest[i], add(z[i], mul(cdir[i], beta))) : V3{0, 0, 0};
    ++it;
  }
  return {it, delta > ziel, std::sqrt(delta / std::max(bb, boden))};
}

// implizit.rs:663-896 (without glue zones and self-collision springs)
System ImplizitCg::system_bauen(Szene& s, double h, std::vector<std::optional<Fest>>& fest) {
  const size_t n = s.x.size();
  const V3 g = s.param.schwerkraft;
  const double c = s.param.daempfung;
  // implizit.rs:668-691: proximity pairs and springs; their approach damping
  // acts on v before every other force
  std::vector<Feder> fed;
  if (param.selbstkollision) {
    if (!selbst || selbst->first.r_punkt.size() != n) selbst = aus_szene(s, param.selbst_zusatzdicke);
    const auto& netz = selbst->first;
    const auto& werte = selbst->second;
    std::vector<Naehe> naehe = finde(netz, s.x, s.w, true, true);
    for (const auto& p : naehe) {
      if (p.art == Art::PunktDreieck)
        statistik.naehe_punkt_dreieck += 1;
      else
        statistik.naehe_kante_kante += 1;
    }
    fed = federn(netz, werte, naehe, param.selbst_steifigkeit, s.masse, s.w, s.naht.ruhe, s.v);
    // implizit.rs:692-707: edges through triangles, their regions, push
    // springs; a region is switched off where the body holds the edge side and
    // the triangle side from opposite directions
    std::vector<Schnitt> schn = finde_schnitte(netz, s.x, param.selbst_schnitte_an_naehten);
    std::vector<size_t> wurzeln = gebiete(netz, schn);
    statistik.durchdringungen += schn.size();
    for (size_t i = 0; i < wurzeln.size(); ++i)
      if (wurzeln[i] == i) statistik.durchdringungsgebiete += 1;
    const double rand = param.kontakt_rand;
    auto normale = [&](uint32_t i) -> std::optional<V3> {
      for (const auto& kb : s.koerper) {
        auto kt = kb.kontakt(s.x[i], s.kollisionsabstand[i] + rand);
        if (kt) return kt->normale;
      }
      return std::nullopt;
    };
    auto eingeklemmt = [&](std::array<uint32_t, 2> kp, std::array<uint32_t, 3> dp) {
      V3 summe{0, 0, 0};
      for (uint32_t i : dp)
        if (auto nk = normale(i)) summe = add(summe, *nk);
      if (!(norm(summe) > 0.0)) return false;
      for (uint32_t i : kp)
        if (auto nk = normale(i))
          if (dot(*nk, summe) < 0.0) return true;
      return false;
    };
    std::vector<Feder> schub = schubfedern(netz, werte, schn, wurzeln, param.selbst_steifigkeit, folge, eingeklemmt);
    fed.insert(fed.end(), schub.begin(), schub.end());
    schnitte = std::move(schn);
  }
  std::vector<V3> f(n), last(n);
  for (size_t i = 0; i < n; ++i) {
    f[i] = sub(mul(g, s.masse[i]), mul(s.v[i], c * s.masse[i]));
    last[i] = mul(g, s.masse[i]);
  }
  System sys;
  sys.kanten.reserve(s.abstand.size());
  for (size_t e = 0; e < s.abstand.size(); ++e) {
    uint32_t i = s.abstand.punkte[e][0], j = s.abstand.punkte[e][1];
    double k = (e < s.membran_kante.size() && s.membran_kante[e]) ? 0.0 : 1.0 / s.abstand.nachgiebigkeit[e];
    double l0 = s.abstand.ruhe[e];
    V3 d = sub(s.x[j], s.x[i]);
    double l = std::max(norm(d), 1e-12);
    V3 nr = mul(d, 1.0 / l);
    V3 fi = mul(nr, k * (l - l0));
    f[i] = add(f[i], fi);
    f[j] = sub(f[j], fi);
    if (l > l0) {
      last[i] = add(last[i], fi);
      last[j] = sub(last[j], fi);
    }
    sys.kanten.push_back({i, j, k, nr, std::max(1.0 - l0 / l, 0.0), l0});
  }
  sys.naehte.reserve(s.naht.size());
  for (size_t e = 0; e < s.naht.size(); ++e) {
    uint32_t i = s.naht.punkte[e][0], j = s.naht.punkte[e][1];
    double l0 = s.naht.ruhe[e];
    V3 d = sub(s.x[j], s.x[i]);
    double l = norm(d);
    if (!std::isfinite(l0)) l0 = l;
    V3 fi = (l0 > 0.0 && l > 1e-12) ? mul(d, param.naht_k * (l - l0) / l) : mul(d, param.naht_k);
    f[i] = add(f[i], fi);
    f[j] = sub(f[j], fi);
    V3 richtung{0, 0, 0};
    double quer = 1.0;
    if (l0 > 0.0 && l > 1e-12) {
      richtung = mul(d, 1.0 / l);
      quer = std::max(1.0 - l0 / l, 0.0);
    }
    sys.naehte.push_back({i, j, param.naht_k, richtung, quer, l0});
  }
  sys.biegungen.reserve(s.biegung.size());
  for (size_t b = 0; b < s.biegung.size(); ++b) {
    const auto& idx = s.biegung.punkte[b];
    double k = 1.0 / s.biegung.nachgiebigkeit[b];
    double ruhe = s.biegung.ruhe[b];
    double theta = 0.0;
    std::array<V3, 4> gr{};
    if (!dieder({s.x[idx[0]], s.x[idx[1]], s.x[idx[2]], s.x[idx[3]]}, theta, gr)) {
      theta = 0.0;
      gr = {};
    }
    double fehler = winkel_fehler(theta, ruhe);
    for (int m = 0; m < 4; ++m) f[idx[m]] = sub(f[idx[m]], mul(gr[m], k * fehler));
    sys.biegungen.push_back({idx, gr, k, ruhe});
  }
  // implizit.rs:798-805
  for (const auto& fe : fed)
    for (int q = 0; q < 5; ++q) f[fe.punkte[q]] = add(f[fe.punkte[q]], mul(fe.kraft, fe.gewichte[q]));
  sys.federn = std::move(fed);
  for (const auto& m : s.membran_elemente) {
    std::array<V3, 3> p3 = {s.x[m.punkte[0]], s.x[m.punkte[1]], s.x[m.punkte[2]]};
    auto fe = membran_krafte(m.element, p3);
    for (int k = 0; k < 3; ++k) f[m.punkte[k]] = add(f[m.punkte[k]], fe[k]);
    auto fz = membran_krafte_zug(m.element, p3);
    for (int k = 0; k < 3; ++k) last[m.punkte[k]] = add(last[m.punkte[k]], fz[k]);
  }
  sys.membran_h.reserve(s.membran_elemente.size());
  for (const auto& m : s.membran_elemente)
    sys.membran_h.push_back(membran_hessen(m.element, {s.x[m.punkte[0]], s.x[m.punkte[1]], s.x[m.punkte[2]]}));
  sys.h = h;
  sys.c = c;
  sys.cg_max = param.cg_max;
  sys.cg_toleranz = param.cg_toleranz;
  sys.masse = &s.masse;
  sys.w = &s.w;
  sys.v = &s.v;
  sys.membran = &s.membran_elemente;
  // implizit.rs:872-883 contact set
  fest.assign(n, std::nullopt);
  for (size_t i = 0; i < n; ++i) {
    if (s.w[i] <= 0.0) continue;
    for (const auto& kb : s.koerper) {
      auto kt = kb.kontakt(s.x[i], s.kollisionsabstand[i] + param.kontakt_rand);
      if (kt) {
        double tiefe = kt->tiefe - param.kontakt_rand;
        fest[i] = Fest{kt->normale, tiefe / h + dot(kt->geschwindigkeit, kt->normale), kt->geschwindigkeit};
      }
    }
  }
  // implizit.rs:887-894
  std::vector<V3> hv(n);
  sys.mal_h(s.v, hv);
  sys.rhs.resize(n);
  for (size_t i = 0; i < n; ++i) sys.rhs[i] = mul(sub(f[i], mul(hv[i], h)), h);
  sys.f = std::move(f);
  sys.last = std::move(last);
  auto dg = sys.diag();
  sys.pinv.resize(n);
  for (size_t i = 0; i < n; ++i) sys.pinv[i] = m3_inv(dg[i]);
  return sys;
}

// implizit.rs:899-1038
void ImplizitCg::schritt(Szene& s, double h, Aufnahme* auf) {
  const size_t n = s.x.size();
  const V3 g = s.param.schwerkraft;
  const std::vector<V3> x_anfang = param.selbstkollision ? s.x : std::vector<V3>();
  if (auf) {
    auf->h = h;
    auf->x = s.x;
    auf->v = s.v;
    auf->koerper = s.koerper;
    auf->reib.assign(n, 0);
    auf->stoss.assign(n, 0);
  }
  std::vector<std::optional<Fest>> fest;
  System sys = system_bauen(s, h, fest);
  std::vector<V3> dv = dv_vorher.size() == n ? dv_vorher : std::vector<V3>(n, mul(g, h));
  std::vector<double> fn_kraft(n, 0.0);
  for (int durchgang = 0; durchgang < 2; ++durchgang) {
    CgLauf lauf = cpu_loese(sys, fest, dv);
    if (auf) auf->fest_loes = fest;
    statistik.loesungen += 1;
    statistik.cg_iterationen += lauf.iterationen;
    statistik.rest_max = std::max(statistik.rest_max, lauf.rest);
    if (lauf.nicht_konvergiert) statistik.nicht_konvergiert += 1;
    bool irgendein = false;
    for (const auto& fe : fest) irgendein = irgendein || fe.has_value();
    if (!irgendein) break;
    std::vector<V3> rest(n);
    sys.mal_a(dv, rest);
    for (size_t i = 0; i < n; ++i) rest[i] = sub(rest[i], sys.rhs[i]);
    bool frei = false;
    for (size_t i = 0; i < n; ++i) {
      if (!fest[i]) continue;
      double fn_i = dot(rest[i], fest[i]->normale) / h;
      if (fn_i < 0.0) {
        fest[i] = std::nullopt;
        frei = true;
        statistik.freigegeben += 1;
      } else {
        fn_kraft[i] = fn_i;
      }
    }
    if (!frei) break;
  }
  dv_vorher = dv;
  if (auf) {
    auf->dv = dv;
    auf->fest = fest;
    auf->fn = fn_kraft;
  }
  const std::vector<V3>& last = sys.last;
  for (size_t i = 0; i < n; ++i) {
    if (s.w[i] <= 0.0) continue;
    V3 v = add(s.v[i], dv[i]);
    if (fest[i]) {
      const Fest& fe = *fest[i];
      statistik.kontakte += 1;
      V3 rel = sub(v, fe.v_koerper);
      V3 t = sub(rel, mul(fe.normale, dot(rel, fe.normale)));
      double lt = norm(t);
      double normal = param.normalkraft_aus_last ? std::max(-dot(last[i], fe.normale), 0.0) : fn_kraft[i];
      double grenze = s.reibung[i] * normal * h * s.w[i];
      if (lt <= grenze) {
        statistik.haftend += 1;
        v = sub(v, t);
        if (auf) auf->reib[i] = 1;
      } else if (lt > 0.0) {
        v = sub(v, mul(t, grenze / lt));
        if (auf) auf->reib[i] = 2;
      }
    }
    s.v[i] = v;
    const V3 alt = s.x[i];
    s.x[i] = add(alt, mul(v, h));
    // implizit.rs:988-1002: a path through a mesh body's skin sets down at
    // the entry; the impact removes the normal velocity relative to the body
    // and Coulomb on the impact takes up to mu |vn| of the tangential
    if (param.durchstoss_pruefen)
      for (const Koerper& kb : s.koerper) {
        auto d = kb.durchstoss(alt, s.x[i]);
        if (!d) continue;
        const V3 p = (*d)[0], nk = (*d)[1], vk = (*d)[2];
        statistik.durchstoesse += 1;
        s.x[i] = add(p, mul(nk, s.kollisionsabstand[i]));
        const V3 rel = sub(s.v[i], vk);
        const double vn = dot(rel, nk);
        if (vn < 0.0) {
          V3 t = sub(rel, mul(nk, vn));
          const double lt = norm(t);
          const double grenze = s.reibung[i] * -vn;
          t = lt <= grenze ? V3{0.0, 0.0, 0.0} : mul(t, 1.0 - grenze / lt);
          s.v[i] = add(vk, t);
        }
      }
    for (size_t kb = 0; kb < s.koerper.size(); ++kb) {
      auto kt = s.koerper[kb].kontakt(s.x[i], s.kollisionsabstand[i]);
      if (kt) {
        s.x[i] = add(s.x[i], mul(kt->normale, kt->tiefe));
        double vn = dot(sub(s.v[i], kt->geschwindigkeit), kt->normale);
        if (vn < 0.0) s.v[i] = sub(s.v[i], mul(kt->normale, vn));
        if (auf) auf->stoss[i] |= (1u << (2 * kb)) | (vn < 0.0 ? 1u << (2 * kb + 1) : 0u);
      }
    }
  }
  // implizit.rs:1015-1025: body points against cloth triangles
  for (size_t pass = 0; pass < param.koerperpunkt_durchgaenge; ++pass) {
    size_t k = 0;
    for (const Koerper& kb : s.koerper) k += kb.punkte_gegen_dreiecke(param.koerperpunkt_tiefe, s.dreiecke, s.w, s.x, s.v);
    statistik.koerperpunkte += k;
    if (k == 0) break;
  }
  // implizit.rs:1027-1037: the way x_anfang -> x, impacts between parts that
  // do not already interpenetrate, position response; held points count as
  // heavy (x 1e9)
  if (param.selbstkollision && selbst) {
    const Stoffnetz& netz = selbst->first;
    std::vector<Stoss> st = finde_stoesse(netz, x_anfang, s.x, s.w, true, true);
    st = ohne_durchdrungene(netz, std::move(st), schnitte);
    if (!st.empty()) {
      std::vector<double> m_eff(n);
      for (size_t i = 0; i < n; ++i) m_eff[i] = fest[i] ? s.masse[i] * 1e9 : s.masse[i];
      statistik.selbst_stoesse += stossantwort(st, s.x, m_eff, s.w, param.selbst_stoss_iterationen);
    }
  }
}

// implizit.rs:1042-1057
void ImplizitCg::bild(Szene& s, std::vector<Aufnahme>* auf) {
  size_t n = std::max<size_t>(param.schritte_je_bild, 1);
  double h = s.param.bild_dt / double(n);
  statistik = ImplizitStatistik{};
  std::vector<Koerper> anfang = s.koerper;
  for (size_t k = 0; k < n; ++k) {
    double weg = double(k + 1) * h;
    for (size_t b = 0; b < s.koerper.size(); ++b) s.koerper[b] = anfang[b].verschoben(weg);
    if (auf) {
      auf->emplace_back();
      schritt(s, h, &auf->back());
    } else {
      schritt(s, h);
    }
  }
  s.zeit += s.param.bild_dt;
}

// implizit.rs:637-643 (operator probe)
std::vector<V3> ImplizitCg::op(Szene& s, const std::vector<V3>& p) {
  double h = s.param.bild_dt / double(std::max<size_t>(param.schritte_je_bild, 1));
  std::vector<std::optional<Fest>> fest;
  System sys = system_bauen(s, h, fest);
  std::vector<V3> out(p.size());
  sys.mal_a(p, out);
  return out;
}

}  // namespace orc
