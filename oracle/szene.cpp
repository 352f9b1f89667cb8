// ORACLE (test infrastructure). Restatement of Szene::bauen
// (sim/src/szene.rs:320-715) for a pattern given as pieces + seam point pairs,
// without the folded allowance band (saumfalte, out of scope).
#include <algorithm>
#include <limits>

#include "oracle.hpp"

namespace orc {
namespace {
// szene.rs:272-279
double l2(V2 a, V2 b) { return std::sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1])); }
double flaeche(V2 a, V2 b, V2 c) { return 0.5 * ((b[0] - a[0]) * (c[1] - a[1]) - (c[0] - a[0]) * (b[1] - a[1])); }

// szene.rs:141-170 (Gruppe::geordnet_mit_extra)
template <int N>
Gruppe<N> geordnet(const std::vector<std::array<uint32_t, N>>& punkte, const std::vector<double>& ruhe,
                   const std::vector<double>& alpha, size_t npunkte, const std::vector<uint8_t>* extra,
                   std::vector<uint8_t>* extra_out) {
  std::vector<std::vector<uint32_t>> pv(punkte.size());
  for (size_t c = 0; c < punkte.size(); ++c) pv[c].assign(punkte[c].begin(), punkte[c].end());
  auto [farbe, zahl] = faerbe(punkte.size(), npunkte, pv);
  auto [idx, farben] = ordnung(farbe, zahl);
  Gruppe<N> g;
  for (size_t c : idx) {
    g.punkte.push_back(punkte[c]);
    g.ruhe.push_back(ruhe[c]);
    g.nachgiebigkeit.push_back(alpha[c]);
  }
  g.farben = farben;
  if (extra && extra_out) {
    extra_out->clear();
    for (size_t c : idx) extra_out->push_back((*extra)[c]);
  }
  return g;
}
}  // namespace

Szene szene_bauen(const Muster& netz, const std::vector<Koerper>& koerper, Simparameter param) {
  Szene s;
  std::vector<std::array<uint32_t, 2>> a_p;
  std::vector<double> a_r, a_a;
  std::vector<std::array<uint32_t, 4>> b_p;
  std::vector<double> b_r, b_a;
  std::vector<uint32_t> versatz;
  using Key = std::pair<uint32_t, uint32_t>;
  std::vector<std::map<Key, std::pair<uint32_t, double>>> randkanten;
  std::vector<std::map<Key, size_t>> randkanten_index;
  std::vector<std::vector<V2>> punkte_m;
  std::vector<double> biegesteif, skala_je_teil;
  std::vector<V2> dir2_je_teil;
  std::vector<std::map<Key, size_t>> kanten_index_je_teil;
  struct DT {
    size_t ti;
    std::array<uint32_t, 3> d, global;
  };
  std::vector<DT> dreieck_teil;

  // szene.rs:360-490
  for (size_t ti = 0; ti < netz.teile.size(); ++ti) {
    const Teil& t = netz.teile[ti];
    const Material& mat = t.material;
    double skala = 1.0 - t.reduktion;
    uint32_t off = uint32_t(s.x.size());
    versatz.push_back(off);
    const size_t d_anfang = s.dreiecke.size();
    std::vector<V2> p_m;
    for (const auto& p : t.punkte_mm) p_m.push_back({p[0] * 1e-3, p[1] * 1e-3});
    V2 dir2 = t.fadenlauf;
    for (size_t k = 0; k < t.punkte_mm.size(); ++k) {
      s.x.push_back(t.lage[k]);
      s.masse.push_back(0.0);
      s.kollisionsabstand.push_back(mat.dicke_m / 2.0);
      s.reibung.push_back(mat.reibung);
    }
    std::map<Key, std::pair<double, std::vector<uint32_t>>> kanten;
    std::map<Key, size_t> rand_index, kanten_e;
    for (const auto& d : t.dreiecke) {
      V2 pa = p_m[d[0]], pb = p_m[d[1]], pc = p_m[d[2]];
      double a = std::fabs(flaeche(pa, pb, pc));
      for (uint32_t i : d) s.masse[off + i] += a * skala * skala * mat.flaechengewicht_kg_m2 / 3.0;
      for (int k = 0; k < 3; ++k) {
        uint32_t i = d[k], j = d[(k + 1) % 3], o = d[(k + 2) % 3];
        auto& e = kanten[{std::min(i, j), std::max(i, j)}];
        e.first += a;
        e.second.push_back(o);
      }
      auto sc = [&](V2 q) -> V2 { return {q[0] * skala, q[1] * skala}; };
      V2 qa = sc(pa), qb = sc(pb), qc = sc(pc);
      double m00 = qb[0] - qa[0], m10 = qb[1] - qa[1], m01 = qc[0] - qa[0], m11 = qc[1] - qa[1];
      double det = m00 * m11 - m01 * m10;
      s.ruhe_inv.push_back({m11 / det, -m01 / det, -m10 / det, m00 / det});
      std::array<uint32_t, 3> g = {d[0] + off, d[1] + off, d[2] + off};
      s.dreiecke.push_back(g);
      dreieck_teil.push_back({ti, d, g});
    }
    for (const auto& [key, val] : kanten) {
      uint32_t i = key.first, j = key.second;
      double asum = val.first;
      const auto& gegen = val.second;
      double l = l2(p_m[i], p_m[j]);
      if (l <= 0.0) continue;
      double k = mat.dehnung_n_m * asum / (l * l);
      a_p.push_back({i + off, j + off});
      a_r.push_back(l * skala);
      a_a.push_back(1.0 / k);
      kanten_e[key] = a_r.size() - 1;
      if (gegen.size() == 1) rand_index[key] = a_r.size() - 1;
      if (gegen.size() == 2) {
        uint32_t o1 = gegen[0], o2 = gegen[1];
        V2 pi = p_m[i], pj = p_m[j];
        uint32_t o_a = o1, o_b = o2;
        if (!(flaeche(pi, pj, p_m[o1]) > 0.0)) std::swap(o_a, o_b);
        double a12 = std::fabs(flaeche(pi, pj, p_m[o_a])) + std::fabs(flaeche(pj, pi, p_m[o_b]));
        double c2, s2, d;
        if (cos2_sin2({pj[0] - pi[0], pj[1] - pi[1]}, dir2, c2, s2))
          d = steifigkeit_aus(c2, s2, mat.biegung_nm, mat.biegung_kette_nm, mat.biegung_schraege_nm);
        else
          d = mat.biegung_nm;
        double kb = d * l * l / a12;
        b_p.push_back({i + off, j + off, o_a + off, o_b + off});
        b_r.push_back(0.0);
        b_a.push_back(1.0 / kb);
      }
    }
    std::map<Key, std::pair<uint32_t, double>> rand;
    for (const auto& [key, val] : kanten)
      if (val.second.size() == 1) rand[key] = {val.second[0], val.first};
    randkanten.push_back(rand);
    randkanten_index.push_back(rand_index);
    punkte_m.push_back(p_m);
    dir2_je_teil.push_back(dir2);
    skala_je_teil.push_back(skala);
    kanten_index_je_teil.push_back(kanten_e);
    biegesteif.push_back(mat.biegung_nm);
    // szene.rs:483-489
    s.teile.push_back({off, s.x.size(), d_anfang, s.dreiecke.size(), mat.dehnung_n_m, -1});
  }

  // szene.rs:492-529 bending across seams
  std::set<Key> naht_kanten;
  for (const auto& n : netz.naehte)
    for (const auto& tn : n.teilnaehte) {
      size_t ta = tn.teil_a, tb = tn.teil_b;
      for (size_t w = 0; w + 1 < tn.paare.size(); ++w) {
        uint32_t a0 = tn.paare[w].first, a1 = tn.paare[w + 1].first;
        uint32_t b0 = tn.paare[w].second, b1 = tn.paare[w + 1].second;
        auto ia = randkanten[ta].find({std::min(a0, a1), std::max(a0, a1)});
        auto ib = randkanten[tb].find({std::min(b0, b1), std::max(b0, b1)});
        if (ia == randkanten[ta].end() || ib == randkanten[tb].end()) continue;
        uint32_t oa = ia->second.first, ob = ib->second.first;
        double fa = ia->second.second, fb = ib->second.second;
        if (!naht_kanten.insert({versatz[ta] + std::min(a0, a1), versatz[ta] + std::max(a0, a1)}).second) continue;
        const auto &pa = punkte_m[ta], &pb = punkte_m[tb];
        uint32_t x0a, x1a, x0b, x1b;
        if (flaeche(pa[a0], pa[a1], pa[oa]) > 0.0) {
          x0a = a0; x1a = a1; x0b = b0; x1b = b1;
        } else {
          x0a = a1; x1a = a0; x0b = b1; x1b = b0;
        }
        (void)x0b;
        if (flaeche(pb[x1b], pb[x0b], pb[ob]) <= 0.0) {
          s.naht_biegung_ohne += 1;
          continue;
        }
        double l = l2(pa[a0], pa[a1]);
        double kb = 0.5 * (biegesteif[ta] + biegesteif[tb]) * l * l / (fa + fb);
        b_p.push_back({x0a + versatz[ta], x1a + versatz[ta], oa + versatz[ta], ob + versatz[tb]});
        b_r.push_back(0.0);
        b_a.push_back(1.0 / kb);
      }
    }

  // szene.rs:531-544 seam pairs
  std::set<Key> paare;
  for (const auto& n : netz.naehte)
    for (const auto& tn : n.teilnaehte)
      for (const auto& pp : tn.paare) {
        uint32_t a = versatz[tn.teil_a] + pp.first, b = versatz[tn.teil_b] + pp.second;
        if (a != b) paare.insert({std::min(a, b), std::max(a, b)});
      }
  std::vector<std::array<uint32_t, 2>> n_p;
  for (const auto& pr : paare) n_p.push_back({pr.first, pr.second});
  std::vector<double> n_r(n_p.size(), 0.0), n_a(n_p.size(), param.naht_nachgiebigkeit);

  // szene.rs:556-592 ease
  if (param.einhalteweite) {
    std::set<size_t> gesetzt;
    for (const auto& n : netz.naehte) {
      double la = n.laenge_a_mm, lb = n.laenge_b_mm;
      if (!(la > 0.0 && lb > 0.0)) continue;
      double faktor = std::min(la, lb) / std::max(la, lb);
      if (faktor >= 1.0 - 1e-9) continue;
      int lang = la > lb ? 0 : 1;
      for (const auto& tn : n.teilnaehte) {
        const auto& index = lang == 0 ? randkanten_index[tn.teil_a] : randkanten_index[tn.teil_b];
        for (size_t w = 0; w + 1 < tn.paare.size(); ++w) {
          uint32_t p0 = lang == 0 ? tn.paare[w].first : tn.paare[w].second;
          uint32_t p1 = lang == 0 ? tn.paare[w + 1].first : tn.paare[w + 1].second;
          if (p0 == p1) continue;
          auto it = index.find({std::min(p0, p1), std::max(p0, p1)});
          if (it == index.end()) continue;
          if (gesetzt.insert(it->second).second) {
            a_r[it->second] *= faktor;
            s.einhalte_kanten += 1;
          }
        }
      }
    }
  }

  // szene.rs:602-647 membranes
  std::vector<uint8_t> membran_kante(a_r.size(), 0);
  for (const auto& dt : dreieck_teil) {
    const Teil& t = netz.teile[dt.ti];
    const auto& index = kanten_index_je_teil[dt.ti];
    const auto& p = punkte_m[dt.ti];
    const auto& d = dt.d;
    V3 kl{};
    bool vollstaendig = true;
    const Key ks[3] = {{std::min(d[0], d[1]), std::max(d[0], d[1])},
                       {std::min(d[1], d[2]), std::max(d[1], d[2])},
                       {std::min(d[2], d[0]), std::max(d[2], d[0])}};
    for (int k = 0; k < 3; ++k) {
      auto it = index.find(ks[k]);
      if (it != index.end())
        kl[k] = a_r[it->second];
      else
        vollstaendig = false;
    }
    std::optional<Membran> gebaut;
    if (vollstaendig)
      gebaut = membran_bauen({p[d[0]], p[d[1]], p[d[2]]}, kl, dir2_je_teil[dt.ti],
                             {t.material.kette_n_m, t.material.dehnung_n_m, t.material.schub_n_m});
    if (gebaut) {
      for (int k = 0; k < 3; ++k) {
        auto it = index.find(ks[k]);
        if (it != index.end()) membran_kante[it->second] = 1;
      }
      s.membran_elemente.push_back({dt.global, *gebaut});
    } else {
      s.membran_entartet += 1;
    }
  }

  // szene.rs:681-713
  size_t np = s.x.size();
  for (double m : s.masse) s.w.push_back(m > 0.0 ? 1.0 / m : 0.0);
  s.abstand = geordnet<2>(a_p, a_r, a_a, np, &membran_kante, &s.membran_kante);
  s.biegung = geordnet<4>(b_p, b_r, b_a, np, nullptr, nullptr);
  s.naht = geordnet<2>(n_p, n_r, n_a, np, nullptr, nullptr);
  s.v.assign(np, V3{0, 0, 0});
  s.koerper = koerper;
  s.param = param;
  return s;
}

// szene.rs:768-774
void naht_kuerzen(Szene& s, double schritt) {
  for (size_t c = 0; c < s.naht.size(); ++c) {
    auto [i, j] = s.naht.punkte[c];
    double l = norm(sub(s.x[i], s.x[j]));
    s.naht.ruhe[c] = std::max(std::min(s.naht.ruhe[c], l) - schritt, 0.0);
  }
}
// szene.rs:778-782
void naht_offen(Szene& s) {
  for (double& r : s.naht.ruhe) r = std::numeric_limits<double>::infinity();
}

}  // namespace orc
