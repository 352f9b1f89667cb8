// ORACLE (test infrastructure): the proximity stage of cloth self-collision,
// sim/src/selbstkollision.rs:41-801 — mesh adjacency, normals, the spatial
// hash, the point-triangle and edge-edge searches and the proximity springs
// with their approach damping. Same loop order and the same floating-point
// expressions as the reference, so pair lists come out in the reference's
// order with the reference's bits. The penetration regions and the impact
// stage (selbstkollision.rs:813-1343) are not restated.
#include <algorithm>
#include <cfloat>
#include <limits>

#include "oracle.hpp"

namespace orc {

// selbstkollision.rs:129-140
bool Stoffnetz::band_und_traeger(uint32_t a, uint32_t b) const {
  auto traeger = [&](uint32_t p) -> std::optional<uint32_t> {
    if (p >= band_von.size()) return std::nullopt;
    uint32_t v = band_von[p];
    if (v == KEIN) return std::nullopt;
    return v;
  };
  auto teil = [&](uint32_t p) -> std::optional<uint32_t> {
    if (p >= teil_von.size()) return std::nullopt;
    return teil_von[p];
  };
  auto ta = traeger(a), tb = traeger(b);
  if (ta && teil(b) == ta) return true;
  if (tb && teil(a) == tb) return true;
  return false;
}

// selbstkollision.rs:147-155
std::optional<double> Stoffnetz::band_abstand(uint32_t a, const uint32_t* andere, int n) const {
  bool any = false;
  for (int k = 0; k < n; ++k) any = any || band_und_traeger(a, andere[k]);
  if (!any) return std::nullopt;
  auto dick = [&](uint32_t p) { return p < dicke.size() ? dicke[p] : 0.0; };
  double m = 0.0;
  for (int k = 0; k < n; ++k) m = std::fmax(m, dick(andere[k]));
  return dick(a) + m;
}

// selbstkollision.rs:190-192
bool Stoffnetz::gleich_oder_partner(uint32_t a, uint32_t b) const {
  if (a == b) return true;
  if (a >= naht_partner.size()) return false;
  const auto& l = naht_partner[a];
  return std::find(l.begin(), l.end(), b) != l.end();
}

// selbstkollision.rs:159-187
Stoffnetz stoffnetz_neu(const std::vector<std::array<uint32_t, 3>>& dreiecke, std::vector<double> r_punkt) {
  Stoffnetz n;
  n.dreiecke = dreiecke;
  for (size_t t = 0; t < dreiecke.size(); ++t) {
    const auto& d = dreiecke[t];
    std::array<uint32_t, 3> dk{};
    for (int k = 0; k < 3; ++k) {
      uint32_t a = d[k], b = d[(k + 1) % 3];
      std::pair<uint32_t, uint32_t> key{std::min(a, b), std::max(a, b)};
      auto it = n.kanten_index.find(key);
      uint32_t e;
      if (it == n.kanten_index.end()) {
        n.kanten.push_back({key.first, key.second});
        n.kanten_dreiecke.push_back({KEIN, KEIN});
        e = uint32_t(n.kanten.size() - 1);
        n.kanten_index.emplace(key, e);
      } else {
        e = it->second;
      }
      auto& kd = n.kanten_dreiecke[e];
      if (kd[0] == KEIN)
        kd[0] = uint32_t(t);
      else if (kd[1] == KEIN)
        kd[1] = uint32_t(t);
      dk[k] = e;
    }
    n.dreieck_kanten.push_back(dk);
  }
  for (const auto& k : n.kanten) n.r_kante.push_back(std::fmax(r_punkt[k[0]], r_punkt[k[1]]));
  for (const auto& d : dreiecke) {
    double r = 0.0;
    for (uint32_t i : d) r = std::fmax(r, r_punkt[i]);
    n.r_dreieck.push_back(r);
  }
  n.r_punkt = std::move(r_punkt);
  return n;
}

namespace {
// selbstkollision.rs:196-203
V3 einheit(V3 a) {
  double l = norm(a);
  if (l > 1e-12) return mul(a, 1.0 / l);
  return {1.0, 0.0, 0.0};
}
}  // namespace

// selbstkollision.rs:216-251
Normalen normalen_neu(const Stoffnetz& netz, const std::vector<V3>& x) {
  Normalen o;
  o.dreieck.reserve(netz.dreiecke.size());
  for (const auto& d : netz.dreiecke) {
    V3 a = x[d[0]], b = x[d[1]], c = x[d[2]];
    o.dreieck.push_back(einheit(cross(sub(b, a), sub(c, a))));
  }
  o.punkt.assign(x.size(), V3{0, 0, 0});
  for (size_t t = 0; t < netz.dreiecke.size(); ++t)
    for (uint32_t i : netz.dreiecke[t]) o.punkt[i] = add(o.punkt[i], o.dreieck[t]);
  for (auto& p : o.punkt) p = einheit(p);
  o.kantenebene.reserve(netz.kanten.size());
  for (size_t e = 0; e < netz.kanten.size(); ++e) {
    const auto& k = netz.kanten[e];
    const auto& kd = netz.kanten_dreiecke[e];
    V3 m;
    if (kd[0] == KEIN) {
      m = {1.0, 0.0, 0.0};
    } else if (kd[1] == KEIN) {
      m = o.dreieck[kd[0]];
    } else {
      V3 a = o.dreieck[kd[0]], b = o.dreieck[kd[1]];
      m = dot(a, b) < 0.0 ? sub(a, b) : add(a, b);
    }
    o.kantenebene.push_back(einheit(cross(m, sub(x[k[0]], x[k[1]]))));
  }
  return o;
}

// selbstkollision.rs:263-265: floor(x / zelle) as i64, saturating like
// Rust's float-to-int `as` (NaN -> 0)
int64_t zellindex(double x, double zelle) {
  double f = std::floor(x / zelle);
  if (std::isnan(f)) return 0;
  if (f >= 9223372036854775808.0) return std::numeric_limits<int64_t>::max();
  if (f < -9223372036854775808.0) return std::numeric_limits<int64_t>::min();
  return int64_t(f);
}

namespace {
// selbstkollision.rs:270-272
bool zellbereich_ok(const Quader& q, double zelle) {
  for (int a = 0; a < 3; ++a)
    if (!(std::isfinite(q.first[a]) && std::isfinite(q.second[a]) && (q.second[a] - q.first[a]) <= 64.0 * zelle))
      return false;
  return true;
}
// inclusive i64 range loop that cannot overflow at the type's maximum
template <typename F>
void bereich(int64_t lo, int64_t hi, F&& f) {
  if (lo > hi) return;
  for (int64_t i = lo;; ++i) {
    f(i);
    if (i == hi) break;
  }
}
template <typename F>
void je_zelle(const Quader& q, double zelle, F&& f) {
  int64_t lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = zellindex(q.first[a], zelle);
    hi[a] = zellindex(q.second[a], zelle);
  }
  bereich(lo[0], hi[0], [&](int64_t i) {
    bereich(lo[1], hi[1], [&](int64_t j) { bereich(lo[2], hi[2], [&](int64_t k) { f(i, j, k); }); });
  });
}
}  // namespace

// selbstkollision.rs:274-278
size_t streue(int64_t i, int64_t j, int64_t k, size_t n) {
  uint32_t h = (uint32_t(i) * 0x8DA6B343u) ^ (uint32_t(j) * 0xD8163841u) ^ (uint32_t(k) * 0xCB1AB31Fu);
  return size_t(h) % n;
}

// selbstkollision.rs:281-324
Hashgitter hashgitter_neu(const std::vector<Quader>& quader, double zelle) {
  Hashgitter g;
  g.zelle = zelle;
  g.eimer = std::max<size_t>(2 * quader.size(), 64);
  std::vector<uint32_t> zahl(g.eimer + 1, 0);
  std::vector<size_t> hs;
  auto eimer_von = [&](const Quader& q) {
    hs.clear();
    if (!zellbereich_ok(q, zelle)) return;
    je_zelle(q, zelle, [&](int64_t i, int64_t j, int64_t k) { hs.push_back(streue(i, j, k, g.eimer)); });
    std::sort(hs.begin(), hs.end());
    hs.erase(std::unique(hs.begin(), hs.end()), hs.end());
  };
  for (const auto& q : quader) {
    eimer_von(q);
    for (size_t h : hs) zahl[h + 1] += 1;
  }
  for (size_t h = 0; h < g.eimer; ++h) zahl[h + 1] += zahl[h];
  g.anfang = zahl;
  std::vector<uint32_t> fuell = zahl;
  g.eintraege.assign(g.anfang[g.eimer], 0);
  for (size_t e = 0; e < quader.size(); ++e) {
    eimer_von(quader[e]);
    for (size_t h : hs) g.eintraege[fuell[h]++] = uint32_t(e);
  }
  return g;
}

namespace {
// selbstkollision.rs:328-344
template <typename F>
void je_eintrag(const Hashgitter& g, const Quader& q, F&& f) {
  if (!zellbereich_ok(q, g.zelle)) return;
  je_zelle(q, g.zelle, [&](int64_t i, int64_t j, int64_t k) {
    size_t h = streue(i, j, k, g.eimer);
    for (uint32_t s = g.anfang[h]; s < g.anfang[h + 1]; ++s) f(g.eintraege[s], std::array<int64_t, 3>{i, j, k});
  });
}
// selbstkollision.rs:359-361
bool ueberlappt(const Quader& a, const Quader& b) {
  for (int k = 0; k < 3; ++k)
    if (!(a.first[k] <= b.second[k] && b.first[k] <= a.second[k])) return false;
  return true;
}
// selbstkollision.rs:365-367
bool erste_zelle(const Quader& a, const Quader& b, double zelle, std::array<int64_t, 3> c) {
  for (int k = 0; k < 3; ++k)
    if (zellindex(std::fmax(a.first[k], b.first[k]), zelle) != c[k]) return false;
  return true;
}
}  // namespace

// selbstkollision.rs:347-357
Quader quader_punkte(const V3* p, int n, double m) {
  V3 lo{INFINITY, INFINITY, INFINITY}, hi{-INFINITY, -INFINITY, -INFINITY};
  for (int q = 0; q < n; ++q)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::fmin(lo[a], p[q][a] - m);
      hi[a] = std::fmax(hi[a], p[q][a] + m);
    }
  return {lo, hi};
}

// selbstkollision.rs:370-384
std::array<double, 3> naechster_dreieck(V3 p0, V3 p1, V3 p2, V3 x) {
  V3 a = naechster_auf_dreieck(x, p0, p1, p2).first;
  V3 e1 = sub(p1, p0), e2 = sub(p2, p0), r = sub(a, p0);
  double d11 = dot(e1, e1), d12 = dot(e1, e2), d22 = dot(e2, e2);
  double det = d11 * d22 - d12 * d12;
  if (det <= 1e-30) return {1.0, 0.0, 0.0};
  double r1 = dot(r, e1), r2 = dot(r, e2);
  double w1 = (d22 * r1 - d12 * r2) / det;
  double w2 = (d11 * r2 - d12 * r1) / det;
  return {1.0 - w1 - w2, w1, w2};
}

// selbstkollision.rs:469-484
Quader kanten_quader(V3 a, V3 b, double m) {
  V3 t = einheit(sub(b, a));
  V3 h = std::fabs(t[1] - 1.0) < 1e-5 ? V3{1.0, 0.0, 0.0} : V3{0.0, 1.0, 0.0};
  V3 u = einheit(cross(t, h));
  V3 v = einheit(cross(t, u));
  V3 ecken[8];
  int n = 0;
  for (V3 p : {a, b})
    for (double su : {-m, m})
      for (double sv : {-m, m}) ecken[n++] = add(add(p, mul(u, su)), mul(v, sv));
  return quader_punkte(ecken, 8, 0.0);
}

double hash_zelle(const Stoffnetz& netz) {
  double r_max = 0.0;
  for (double r : netz.r_punkt) r_max = std::fmax(r_max, r);
  return std::fmax(2.0 * r_max + ZUSCHLAG_PAAR, 1e-4) * 2.0;
}

namespace {
// selbstkollision.rs:400-466
void finde_punkt_dreieck(const Stoffnetz& netz, const std::vector<V3>& x, const std::vector<double>& w,
                         const Normalen& nrm, std::vector<Naehe>& aus) {
  std::vector<Quader> qp(x.size());
  for (size_t v = 0; v < x.size(); ++v) qp[v] = quader_punkte(&x[v], 1, netz.r_punkt[v] + ZUSCHLAG_QUADER);
  const double zelle = hash_zelle(netz);
  Hashgitter gitter = hashgitter_neu(qp, zelle);
  for (size_t t = 0; t < netz.dreiecke.size(); ++t) {
    const auto d = netz.dreiecke[t];
    const uint32_t i0 = d[0], i1 = d[1], i2 = d[2];
    if (i0 == i1 || i1 == i2 || i0 == i2) continue;
    const V3 p[3] = {x[i0], x[i1], x[i2]};
    const double rt = netz.r_dreieck[t];
    const Quader qt = quader_punkte(p, 3, rt + ZUSCHLAG_QUADER);
    const V3 nt = nrm.dreieck[t];
    V3 en[3];
    for (int k = 0; k < 3; ++k) en[k] = nrm.kantenebene[netz.dreieck_kanten[t][k]];
    const double s[3] = {dot(sub(p[2], p[0]), en[0]), dot(sub(p[0], p[1]), en[1]), dot(sub(p[1], p[2]), en[2])};
    je_eintrag(gitter, qt, [&](uint32_t v, std::array<int64_t, 3> c) {
      for (uint32_t i : d)
        if (netz.gleich_oder_partner(v, i)) return;
      if (w[v] <= 0.0 && w[i0] <= 0.0 && w[i1] <= 0.0 && w[i2] <= 0.0) return;
      if (!ueberlappt(qp[v], qt) || !erste_zelle(qt, qp[v], gitter.zelle, c)) return;
      const V3 xv = x[v];
      double ruhe = rt + netz.r_punkt[v];
      if (auto eine = netz.band_abstand(v, d.data(), 3)) ruhe = *eine;
      const double soll = ruhe + ZUSCHLAG_PAAR;
      const double sd = dot(nt, sub(xv, p[0]));
      if (std::fabs(sd) > soll) return;
      for (int k = 0; k < 3; ++k)
        if (dot(sub(xv, p[k]), en[k]) * s[k] < 0.0) return;
      auto g = naechster_dreieck(p[0], p[1], p[2], xv);
      V3 cp = add(add(mul(p[0], g[0]), mul(p[1], g[1])), mul(p[2], g[2]));
      V3 r = sub(xv, cp);
      double abstand = norm(r);
      if (abstand > soll) return;
      Naehe nh;
      nh.art = Art::PunktDreieck;
      nh.punkte = {v, i0, i1, i2};
      nh.gewichte = {1.0, -g[0], -g[1], -g[2]};
      nh.normale = abstand > 1e-12 ? mul(r, 1.0 / abstand) : nt;
      nh.abstand = abstand;
      nh.ruhe = ruhe;
      aus.push_back(nh);
    });
  }
}

// selbstkollision.rs:489-503
bool ist_kuerzeste(const Stoffnetz& netz, const Normalen& nrm, const std::vector<V3>& x, size_t e, V3 u, V3 m) {
  const uint32_t k0 = netz.kanten[e][0], k1 = netz.kanten[e][1];
  for (uint32_t t : netz.kanten_dreiecke[e]) {
    if (t == KEIN) continue;
    const auto& d = netz.dreiecke[t];
    uint32_t o = KEIN;
    for (uint32_t i : d)
      if (i != k0 && i != k1) {
        o = i;
        break;
      }
    if (o == KEIN) continue;
    V3 r = sub(x[o], x[k0]);
    V3 wr = einheit(sub(r, mul(u, dot(r, u))));
    if (dot(m, wr) > 0.0 && std::fabs(dot(m, nrm.dreieck[t])) < 0.5) return false;
  }
  return true;
}

// selbstkollision.rs:506-598
void finde_kante_kante(const Stoffnetz& netz, const std::vector<V3>& x, const std::vector<double>& w,
                       const Normalen& nrm, std::vector<Naehe>& aus) {
  std::vector<Quader> qk(netz.kanten.size());
  for (size_t e = 0; e < netz.kanten.size(); ++e)
    qk[e] = kanten_quader(x[netz.kanten[e][0]], x[netz.kanten[e][1]], netz.r_kante[e] + ZUSCHLAG_QUADER);
  const double zelle = hash_zelle(netz);
  Hashgitter gitter = hashgitter_neu(qk, zelle);
  for (size_t e = 0; e < netz.kanten.size(); ++e) {
    const uint32_t a0 = netz.kanten[e][0], a1 = netz.kanten[e][1];
    if (a0 == a1) continue;
    const V3 pa0 = x[a0], pa1 = x[a1];
    je_eintrag(gitter, qk[e], [&](uint32_t fu, std::array<int64_t, 3> c) {
      const size_t f = fu;
      if (f <= e || !ueberlappt(qk[e], qk[f]) || !erste_zelle(qk[e], qk[f], gitter.zelle, c)) return;
      const uint32_t b0 = netz.kanten[f][0], b1 = netz.kanten[f][1];
      for (uint32_t b : {b0, b1})
        if (netz.gleich_oder_partner(a0, b) || netz.gleich_oder_partner(a1, b)) return;
      const uint32_t bb[2] = {b0, b1}, aa[2] = {a0, a1};
      std::optional<double> band_dick = netz.band_abstand(a0, bb, 2);
      if (!band_dick) band_dick = netz.band_abstand(a1, bb, 2);
      if (!band_dick) band_dick = netz.band_abstand(b0, aa, 2);
      if (!band_dick) band_dick = netz.band_abstand(b1, aa, 2);
      if (w[a0] <= 0.0 && w[a1] <= 0.0 && w[b0] <= 0.0 && w[b1] <= 0.0) return;
      const V3 pb0 = x[b0], pb1 = x[b1];
      const V3 da = sub(pa1, pa0), db = sub(pb1, pb0);
      const double la = norm(da), lb = norm(db);
      if (la < KANTE_MIN || lb < KANTE_MIN) return;
      const V3 ua = mul(da, 1.0 / la), ub = mul(db, 1.0 / lb);
      const double cw = dot(ua, ub);
      if (std::fabs(cw) > 0.99999) return;
      const V3 r = sub(pb0, pa0);
      const double p = dot(r, ua), q = -dot(r, ub);
      const double nen = 1.0 - cw * cw;
      const double sa = (p + cw * q) / nen;
      const double sb = (q + cw * p) / nen;
      if (!(0.0 <= sa && sa <= la) || !(0.0 <= sb && sb <= lb)) return;
      const V3 pa = add(pa0, mul(ua, sa));
      const V3 pb = add(pb0, mul(ub, sb));
      const V3 dv = sub(pa, pb);
      const double abstand = norm(dv);
      const double ruhe = band_dick ? *band_dick : netz.r_kante[e] + netz.r_kante[f];
      if (abstand > ruhe + ZUSCHLAG_PAAR) return;
      const V3 n = einheit(dv);
      if (!ist_kuerzeste(netz, nrm, x, f, ub, n) || !ist_kuerzeste(netz, nrm, x, e, ua, mul(n, -1.0))) return;
      const double s = sa / la, t = sb / lb;
      Naehe nh;
      nh.art = Art::KanteKante;
      nh.punkte = {a0, a1, b0, b1};
      nh.gewichte = {1.0 - s, s, -(1.0 - t), -t};
      nh.normale = n;
      nh.abstand = abstand;
      nh.ruhe = ruhe;
      aus.push_back(nh);
    });
  }
}

// selbstkollision.rs:796-799
size_t kante_von(const Stoffnetz& netz, uint32_t a, uint32_t b) {
  auto it = netz.kanten_index.find({std::min(a, b), std::max(a, b)});
  return it == netz.kanten_index.end() ? 0 : it->second;
}
// selbstkollision.rs:790-794
size_t dreieck_von(const Stoffnetz& netz, const uint32_t* p) {
  size_t e = kante_von(netz, p[0], p[1]);
  for (uint32_t t : netz.kanten_dreiecke[e]) {
    if (t == KEIN) continue;
    const auto& d = netz.dreiecke[t];
    if (d[0] == p[2] || d[1] == p[2] || d[2] == p[2]) return t;
  }
  return 0;
}
}  // namespace

// selbstkollision.rs:387-398
std::vector<Naehe> finde(const Stoffnetz& netz, const std::vector<V3>& x, const std::vector<double>& w, bool pd,
                         bool kk) {
  Normalen nrm = normalen_neu(netz, x);
  std::vector<Naehe> aus;
  if (pd) finde_punkt_dreieck(netz, x, w, nrm, aus);
  if (kk) finde_kante_kante(netz, x, w, nrm, aus);
  return aus;
}

// selbstkollision.rs:623-688
std::pair<Stoffnetz, Stoffwerte> aus_szene(const Szene& s, double zusatzdicke) {
  const size_t n = s.x.size();
  std::vector<double> r(n);
  for (size_t i = 0; i < n; ++i) r[i] = s.kollisionsabstand[i] + zusatzdicke / 2.0;
  Stoffnetz netz = stoffnetz_neu(s.dreiecke, r);
  netz.naht_partner.assign(n, {});
  for (const auto& p : s.naht.punkte) {
    netz.naht_partner[p[0]].push_back(p[1]);
    netz.naht_partner[p[1]].push_back(p[0]);
  }
  for (size_t e = 0; e < s.abstand.size(); ++e) {
    uint32_t i = s.abstand.punkte[e][0], j = s.abstand.punkte[e][1];
    if (s.abstand.ruhe[e] != 0.0 || i == j) continue;
    auto& li = netz.naht_partner[i];
    if (std::find(li.begin(), li.end(), j) == li.end()) li.push_back(j);
    auto& lj = netz.naht_partner[j];
    if (std::find(lj.begin(), lj.end(), i) == lj.end()) lj.push_back(i);
  }
  netz.teil_von.assign(n, KEIN);
  netz.band_von.assign(n, KEIN);
  netz.dicke = s.kollisionsabstand;
  for (size_t ti = 0; ti < s.teile.size(); ++ti) {
    const auto& t = s.teile[ti];
    for (size_t i = t.p0; i < t.p1; ++i) netz.teil_von[i] = uint32_t(ti);
    if (t.band_von >= 0)
      for (size_t i = t.p0; i < t.p1; ++i) netz.band_von[i] = uint32_t(t.band_von);
  }
  Stoffwerte wv;
  wv.e_punkt.assign(n, 0.0);
  wv.e_dreieck.assign(s.dreiecke.size(), 0.0);
  for (const auto& t : s.teile) {
    for (size_t i = t.p0; i < t.p1; ++i) wv.e_punkt[i] = t.dehnung_n_m;
    for (size_t d = t.d0; d < t.d1; ++d) wv.e_dreieck[d] = t.dehnung_n_m;
  }
  for (const auto& m : s.ruhe_inv) wv.a_dreieck.push_back(0.5 / std::fmax(std::fabs(m[0] * m[3] - m[1] * m[2]), 1e-30));
  wv.a_punkt.assign(n, 0.0);
  for (size_t t = 0; t < s.dreiecke.size(); ++t)
    for (uint32_t i : s.dreiecke[t]) wv.a_punkt[i] += wv.a_dreieck[t] / 3.0;
  for (const auto& kd : netz.kanten_dreiecke) {
    double sa = 0.0, se = 0.0;
    int cnt = 0;
    for (uint32_t t : kd)
      if (t != KEIN) {
        sa += wv.a_dreieck[t];
        se += wv.e_dreieck[t];
        ++cnt;
      }
    double k = double(std::max(cnt, 1));
    wv.a_kante.push_back(sa / k);
    wv.e_kante.push_back(se / k);
  }
  wv.naht_partner.assign(n, {});
  for (size_t c = 0; c < s.naht.size(); ++c) {
    uint32_t i = s.naht.punkte[c][0], j = s.naht.punkte[c][1];
    wv.naht_partner[i].push_back({j, uint32_t(c)});
    wv.naht_partner[j].push_back({i, uint32_t(c)});
  }
  wv.mu_punkt = s.reibung;
  return {std::move(netz), std::move(wv)};
}

// selbstkollision.rs:713-787
std::vector<Feder> federn(const Stoffnetz& netz, const Stoffwerte& werte, const std::vector<Naehe>& naehe,
                          double steifigkeit, const std::vector<double>& masse, const std::vector<double>& w,
                          const std::vector<double>& naht_ruhe, std::vector<V3>& v) {
  std::vector<Feder> aus;
  aus.reserve(naehe.size());
  for (const auto& p : naehe) {
    const auto idx = p.punkte;
    double e, a, mu;
    if (p.art == Art::PunktDreieck) {
      size_t t = dreieck_von(netz, &p.punkte[1]);
      e = werte.e_punkt[idx[0]] + werte.e_dreieck[t];
      a = werte.a_punkt[idx[0]] + werte.a_dreieck[t];
      mu = 0.5 * (werte.mu_punkt[idx[0]] + (werte.mu_punkt[idx[1]] + werte.mu_punkt[idx[2]] + werte.mu_punkt[idx[3]]) / 3.0);
    } else {
      size_t k1 = kante_von(netz, idx[0], idx[1]), k2 = kante_von(netz, idx[2], idx[3]);
      e = werte.e_kante[k1] + werte.e_kante[k2];
      a = werte.a_kante[k1] + werte.a_kante[k2];
      mu = 0.25 * (werte.mu_punkt[idx[0]] + werte.mu_punkt[idx[1]] + werte.mu_punkt[idx[2]] + werte.mu_punkt[idx[3]]);
    }
    const double k = steifigkeit * e * a / 1e-6;
    double ruhe = p.ruhe;
    bool fertig = false;
    for (int q = 0; q < 4 && !fertig; ++q) {
      if (p.gewichte[q] <= 0.0) continue;
      for (const auto& pc : werte.naht_partner[idx[q]]) {
        bool auf_zweiter = false;
        for (int r = 0; r < 4; ++r) auf_zweiter = auf_zweiter || (p.gewichte[r] < 0.0 && p.punkte[r] == pc.first);
        double l0 = naht_ruhe[pc.second];
        if (auf_zweiter && std::isfinite(l0) && l0 < ruhe) {
          ruhe = l0;
          fertig = true;
          break;
        }
      }
    }
    const double c = std::fmin(ruhe - p.abstand, AUSLENKUNG_MAX);
    const V3 n = p.normale;
    const V3 kraft = mul(n, k * c);
    M3 block{};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) block[i][j] = k * ((1.0 - mu) * n[i] * n[j] + (i == j ? mu : 0.0));
    double m1 = 0.0, m2 = 0.0;
    V3 dv{0, 0, 0};
    for (int q = 0; q < 4; ++q) {
      double g = p.gewichte[q];
      dv = add(dv, mul(v[idx[q]], g));
      if (g > 0.0)
        m1 += g * masse[idx[q]];
      else
        m2 -= g * masse[idx[q]];
    }
    const double an = dot(dv, n) * ANNAEHERUNG_ANTEIL;
    if (an < 0.0 && m1 + m2 > 0.0) {
      V3 u = add(mul(n, an), mul(sub(dv, mul(n, an)), mu));
      for (int q = 0; q < 4; ++q) {
        double g = p.gewichte[q];
        if (w[idx[q]] <= 0.0) continue;
        double anteil = g > 0.0 ? m2 / (m1 + m2) : m1 / (m1 + m2);
        v[idx[q]] = sub(v[idx[q]], mul(u, g * anteil));
      }
    }
    Feder fe;
    fe.punkte = {p.punkte[0], p.punkte[1], p.punkte[2], p.punkte[3], p.punkte[0]};
    fe.gewichte = {p.gewichte[0], p.gewichte[1], p.gewichte[2], p.gewichte[3], 0.0};
    fe.kraft = kraft;
    fe.block = block;
    aus.push_back(fe);
  }
  return aus;
}

// ============================================================ response stages
// selbstkollision.rs:810-1350: edges through triangles, their regions and
// push springs; impacts on the way x0 -> x1 and their position response.
namespace {
// selbstkollision.rs:1116-1122
double ebenenabstand(V3 a, V3 b, V3 c, V3 p) { return dot(sub(p, a), einheit(cross(sub(b, a), sub(c, a)))); }
V3 lerp(V3 a, V3 b, double t) { return add(mul(a, 1.0 - t), mul(b, t)); }
// selbstkollision.rs:1156-1171
std::optional<std::array<double, 2>> im_dreieck(V3 a, V3 b, V3 c, V3 p) {
  V3 e1 = sub(b, a), e2 = sub(c, a), r = sub(p, a);
  double d11 = dot(e1, e1), d12 = dot(e1, e2), d22 = dot(e2, e2);
  double det = d11 * d22 - d12 * d12;
  if (det <= 1e-4 * d11 * d22) return std::nullopt;
  double r1 = dot(r, e1), r2 = dot(r, e2);
  double u = (d22 * r1 - d12 * r2) / det;
  double v = (d11 * r2 - d12 * r1) / det;
  if (u < 0.0 || v < 0.0 || u + v > 1.0) return std::nullopt;
  return std::array<double, 2>{u, v};
}
// selbstkollision.rs:830-846
std::optional<std::pair<double, std::array<double, 3>>> kante_durch_dreieck(V3 a, V3 b, const std::array<V3, 3>& v,
                                                                             V3 n) {
  double d0 = dot(n, sub(a, v[0])), d1 = dot(n, sub(b, v[0]));
  if ((d0 > 0.0 && d1 > 0.0) || (d0 < 0.0 && d1 < 0.0) || std::abs(d1 - d0) < 1e-12) return std::nullopt;
  double t = -d0 / (d1 - d0);
  if (std::abs(t) < 1e-5 || std::abs(t - 1.0) < 1e-5) return std::nullopt;
  V3 p = lerp(a, b, t);
  V3 e1 = sub(v[1], v[0]), e2 = sub(v[2], v[0]);
  if (norm(e1) < STOSS_KANTE_MIN || norm(e2) < STOSS_KANTE_MIN) return std::nullopt;
  auto uv = im_dreieck(v[0], v[1], v[2], p);
  if (!uv) return std::nullopt;
  return std::make_pair(t, std::array<double, 3>{1.0 - (*uv)[0] - (*uv)[1], (*uv)[0], (*uv)[1]});
}
// selbstkollision.rs:1128-1153 (regula falsi on the plane distance)
std::optional<double> koplanar_zeit(const std::array<V3, 4>& x0, const std::array<V3, 4>& x1, double tol) {
  auto f = [&](double t) {
    std::array<V3, 4> q;
    for (int k = 0; k < 4; ++k) q[k] = lerp(x0[k], x1[k], t);
    return ebenenabstand(q[0], q[1], q[2], q[3]);
  };
  double t0 = 0.0, t1 = 1.0, d0 = f(0.0), d1 = f(1.0);
  for (int it = 0; it < 16; ++it) {
    if (d0 * d1 > 0.0) return std::nullopt;
    double tau = t0 + (t1 - t0) * std::abs(d0) / std::max(std::abs(d0) + std::abs(d1), DBL_MIN);
    double d = f(tau);
    if (std::abs(d) < tol || t1 - t0 < 1e-4) return tau;
    if (d0 * d > 0.0) {
      t0 = tau;
      d0 = d;
    } else {
      t1 = tau;
      d1 = d;
    }
  }
  return std::nullopt;
}
// selbstkollision.rs:1173-1193
std::optional<std::array<double, 2>> kanten_kreuzen(V3 a, V3 b, V3 c, V3 d) {
  V3 e1 = sub(b, a), e2 = sub(d, c);
  double l1 = norm(e1), l2 = norm(e2);
  if (l1 < STOSS_KANTE_MIN || l2 < STOSS_KANTE_MIN) return std::nullopt;
  V3 u1 = mul(e1, 1.0 / l1), u2 = mul(e2, 1.0 / l2);
  double g = dot(u1, u2);
  if (std::abs(g) > 0.99999) return std::nullopt;
  V3 q = sub(c, a);
  double nen = 1.0 - g * g;
  double s = (dot(q, u1) - g * dot(q, u2)) / nen;
  double w = (g * dot(q, u1) - dot(q, u2)) / nen;
  if (s <= 0.0 || s >= l1 || w <= 0.0 || w >= l2) return std::nullopt;
  return std::array<double, 2>{s / l1, w / l2};
}
// selbstkollision.rs:910-925 (union-find with path halving; root = the smallest index)
size_t wurzel(std::vector<size_t>& eltern, size_t i) {
  while (eltern[i] != i) {
    eltern[i] = eltern[eltern[i]];
    i = eltern[i];
  }
  return i;
}
void vereinige(std::vector<size_t>& eltern, size_t a, size_t b) {
  size_t ra = wurzel(eltern, a), rb = wurzel(eltern, b);
  if (ra != rb) eltern[std::max(ra, rb)] = std::min(ra, rb);
}
}  // namespace

// selbstkollision.rs:858-907
std::vector<Schnitt> finde_schnitte(const Stoffnetz& netz, const std::vector<V3>& x, bool an_naehten) {
  Normalen nrm = normalen_neu(netz, x);
  std::vector<Quader> qt(netz.dreiecke.size());
  for (size_t t = 0; t < qt.size(); ++t) {
    V3 p[3] = {x[netz.dreiecke[t][0]], x[netz.dreiecke[t][1]], x[netz.dreiecke[t][2]]};
    qt[t] = quader_punkte(p, 3, ZUSCHLAG_QUADER);
  }
  double laenge = 0.0;
  for (const auto& k : netz.kanten) laenge = std::fmax(laenge, norm(sub(x[k[0]], x[k[1]])));
  Hashgitter gitter = hashgitter_neu(qt, std::fmax(laenge, 1e-3));
  std::vector<Schnitt> aus;
  for (size_t e = 0; e < netz.kanten.size(); ++e) {
    uint32_t a0 = netz.kanten[e][0], a1 = netz.kanten[e][1];
    const auto& kd = netz.kanten_dreiecke[e];
    if (a0 == a1 || kd[0] == KEIN) continue;
    V3 pa = x[a0], pb = x[a1];
    V3 pe[2] = {pa, pb};
    Quader qe = quader_punkte(pe, 2, ZUSCHLAG_QUADER);
    V3 ehat = einheit(sub(pb, pa));
    je_eintrag(gitter, qe, [&](uint32_t t, std::array<int64_t, 3> c) {
      const auto& d = netz.dreiecke[t];
      bool nachbar = false;
      for (uint32_t i : d)
        nachbar = nachbar || (an_naehten ? (i == a0 || i == a1)
                                         : (netz.gleich_oder_partner(a0, i) || netz.gleich_oder_partner(a1, i)));
      if (nachbar || !ueberlappt(qt[t], qe) || !erste_zelle(qe, qt[t], gitter.zelle, c)) return;
      V3 n = nrm.dreieck[t];
      auto kd_t = kante_durch_dreieck(pa, pb, {x[d[0]], x[d[1]], x[d[2]]}, n);
      if (!kd_t) return;
      double cn = dot(n, ehat);
      if (std::abs(cn) < 1e-6) return;
      V3 p = lerp(pa, pb, kd_t->first);
      V3 g{0, 0, 0};
      for (uint32_t k : kd) {
        if (k == KEIN) continue;
        const auto& dk = netz.dreiecke[k];
        uint32_t o = KEIN;
        for (uint32_t i : dk)
          if (i != a0 && i != a1) {
            o = i;
            break;
          }
        if (o == KEIN) continue;
        V3 m = einheit(cross(n, nrm.dreieck[k]));
        V3 r = sub(x[o], p);
        V3 r_quer = sub(r, mul(ehat, dot(ehat, r)));
        if (dot(m, r_quer) < 0.0) m = mul(m, -1.0);
        g = add(g, sub(m, mul(n, dot(ehat, m) / cn)));
      }
      double lg = norm(g);
      aus.push_back(Schnitt{uint32_t(e), t, kd_t->first, kd_t->second, einheit(g), lg / std::sqrt(lg * lg + 2.25)});
    });
  }
  return aus;
}

// selbstkollision.rs:931-1009
std::vector<size_t> gebiete(const Stoffnetz& netz, std::vector<Schnitt>& schnitte) {
  const size_t n = schnitte.size();
  std::map<std::pair<uint32_t, uint32_t>, size_t> index;
  for (size_t i = 0; i < n; ++i) index.emplace(std::make_pair(schnitte[i].kante, schnitte[i].dreieck), i);
  auto finde = [&](uint32_t e, uint32_t t, std::vector<size_t>& out) {
    auto it = index.find({e, t});
    if (it != index.end()) out.push_back(it->second);
  };
  auto nachbardreiecke = [&](uint32_t t) {
    std::vector<uint32_t> v;
    for (uint32_t k : netz.dreieck_kanten[t])
      for (uint32_t u : netz.kanten_dreiecke[k])
        if (u != KEIN && u != t) v.push_back(u);
    return v;
  };
  std::vector<size_t> eltern(n);
  for (size_t i = 0; i < n; ++i) eltern[i] = i;
  std::vector<std::pair<size_t, size_t>> tausch;
  for (size_t i = 0; i < n; ++i) {
    uint32_t e = schnitte[i].kante, t = schnitte[i].dreieck;
    std::vector<uint32_t> kde;
    for (uint32_t k : netz.kanten_dreiecke[e])
      if (k != KEIN) kde.push_back(k);
    std::vector<uint32_t> andere;
    for (uint32_t k : kde)
      for (uint32_t f : netz.dreieck_kanten[k])
        if (f != e) andere.push_back(f);
    std::vector<uint32_t> tn = nachbardreiecke(t);
    std::vector<size_t> gleich;
    for (uint32_t f : andere) finde(f, t, gleich);
    for (uint32_t u : tn) {
      finde(e, u, gleich);
      for (uint32_t f : andere) finde(f, u, gleich);
    }
    for (size_t j : gleich) vereinige(eltern, i, j);
    for (uint32_t f : netz.dreieck_kanten[t])
      for (uint32_t k : kde) {
        std::vector<size_t> j;
        finde(f, k, j);
        if (!j.empty()) tausch.push_back({i, j[0]});
      }
  }
  for (int runde = 0; runde < 2; ++runde) {
    std::vector<size_t> partner(n, SIZE_MAX);
    for (auto [i, j] : tausch) {
      size_t ri = wurzel(eltern, i), rj = wurzel(eltern, j);
      partner[ri] = std::min(partner[ri], rj);
      partner[rj] = std::min(partner[rj], ri);
    }
    for (auto [i, j] : tausch) {
      size_t rj = wurzel(eltern, j);
      if (partner[rj] != SIZE_MAX) vereinige(eltern, i, partner[rj]);
    }
  }
  std::vector<size_t> wurzeln(n);
  for (size_t i = 0; i < n; ++i) wurzeln[i] = wurzel(eltern, i);
  std::vector<V3> summe(n, V3{0, 0, 0});
  for (size_t i = 0; i < n; ++i) summe[wurzeln[i]] = add(summe[wurzeln[i]], mul(schnitte[i].richtung, schnitte[i].gewicht));
  for (size_t i = 0; i < n; ++i) schnitte[i].richtung = einheit(summe[wurzeln[i]]);
  return wurzeln;
}

// selbstkollision.rs:1014-1058
std::vector<Feder> schubfedern(const Stoffnetz& netz, const Stoffwerte& werte, const std::vector<Schnitt>& schnitte,
                               const std::vector<size_t>& wurzeln, double steifigkeit, std::vector<uint32_t>& folge,
                               const std::function<bool(std::array<uint32_t, 2>, std::array<uint32_t, 3>)>& eingeklemmt) {
  if (folge.size() != netz.dreiecke.size()) folge.assign(netz.dreiecke.size(), 1u);
  std::vector<uint8_t> hat(netz.dreiecke.size(), 0), klemm(schnitte.size(), 0);
  for (size_t i = 0; i < schnitte.size(); ++i) {
    hat[schnitte[i].dreieck] = 1;
    if (eingeklemmt(netz.kanten[schnitte[i].kante], netz.dreiecke[schnitte[i].dreieck])) klemm[wurzeln[i]] = 1;
  }
  for (size_t t = 0; t < folge.size(); ++t) folge[t] = hat[t] ? folge[t] + 1 : 1u;
  std::vector<Feder> aus;
  for (size_t i = 0; i < schnitte.size(); ++i) {
    if (klemm[wurzeln[i]]) continue;
    const Schnitt& s = schnitte[i];
    size_t e = s.kante, t = s.dreieck;
    double k = 2.0 * steifigkeit * (werte.e_kante[e] + werte.e_dreieck[t]) * (werte.a_kante[e] + werte.a_dreieck[t]) / 1e-6;
    V3 g = s.richtung;
    Feder f;
    f.kraft = mul(g, k * double(std::min(folge[t], FOLGE_MAX)) * SCHUB_HEBEL);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) f.block[a][b] = k * g[a] * g[b];
    f.punkte = {netz.kanten[e][0], netz.kanten[e][1], netz.dreiecke[t][0], netz.dreiecke[t][1], netz.dreiecke[t][2]};
    f.gewichte = {1.0 - s.t, s.t, -s.w[0], -s.w[1], -s.w[2]};
    aus.push_back(f);
  }
  return aus;
}

// selbstkollision.rs:1063-1084
std::vector<Stoss> ohne_durchdrungene(const Stoffnetz& netz, std::vector<Stoss> stoesse,
                                      const std::vector<Schnitt>& schnitte) {
  if (schnitte.empty()) return stoesse;
  std::set<std::pair<uint32_t, uint32_t>> paare;
  for (const auto& s : schnitte) paare.insert({s.kante, s.dreieck});
  std::vector<Stoss> aus;
  for (const auto& st : stoesse) {
    bool weg = false;
    if (st.art == Art::PunktDreieck) {
      uint32_t t = uint32_t(dreieck_von(netz, &st.punkte[1]));
      for (const auto& s : schnitte)
        if (s.dreieck == t && (netz.kanten[s.kante][0] == st.punkte[0] || netz.kanten[s.kante][1] == st.punkte[0]))
          weg = true;
    } else {
      size_t i = kante_von(netz, st.punkte[0], st.punkte[1]), j = kante_von(netz, st.punkte[2], st.punkte[3]);
      auto trifft = [&](size_t a, size_t b) {
        for (uint32_t t : netz.kanten_dreiecke[b]) {
          if (t == KEIN) continue;
          const auto& dk = netz.dreieck_kanten[t];
          if (paare.count({uint32_t(a), t}) && (dk[0] == b || dk[1] == b || dk[2] == b)) return true;
        }
        return false;
      };
      weg = trifft(i, j) || trifft(j, i);
    }
    if (!weg) aus.push_back(st);
  }
  return aus;
}

// selbstkollision.rs:1196-1285
std::vector<Stoss> finde_stoesse(const Stoffnetz& netz, const std::vector<V3>& x0, const std::vector<V3>& x1,
                                 const std::vector<double>& w, bool pd, bool kk) {
  std::vector<Stoss> aus;
  auto weg = [&](const uint32_t* idx, int m) {
    V3 p[8];
    for (int k = 0; k < m; ++k) {
      p[k] = x0[idx[k]];
      p[m + k] = x1[idx[k]];
    }
    return quader_punkte(p, 2 * m, 1e-8);
  };
  double laenge = 0.0;
  for (const auto& k : netz.kanten) laenge = std::fmax(laenge, norm(sub(x1[k[0]], x1[k[1]])));
  const double zelle = std::fmax(laenge, 1e-3);
  auto bew = [](const std::array<V3, 4>& a0, const std::array<V3, 4>& a1, int k) { return sub(a1[k], a0[k]); };
  if (pd) {
    std::vector<Quader> qp(x0.size());
    for (uint32_t v = 0; v < qp.size(); ++v) qp[v] = weg(&v, 1);
    Hashgitter gitter = hashgitter_neu(qp, zelle);
    for (const auto& d : netz.dreiecke) {
      if (d[0] == d[1] || d[1] == d[2] || d[0] == d[2]) continue;
      Quader qt = weg(d.data(), 3);
      std::optional<Stoss> best;
      je_eintrag(gitter, qt, [&](uint32_t v, std::array<int64_t, 3> c) {
        bool nb = false;
        for (uint32_t i : d) nb = nb || netz.gleich_oder_partner(v, i);
        if (nb || !ueberlappt(qp[v], qt) || !erste_zelle(qt, qp[v], zelle, c)) return;
        std::array<uint32_t, 4> idx = {d[0], d[1], d[2], v};
        bool alle_fest = true;
        for (uint32_t i : idx) alle_fest = alle_fest && w[i] <= 0.0;
        if (alle_fest) return;
        std::array<V3, 4> a0, a1;
        for (int k = 0; k < 4; ++k) {
          a0[k] = x0[idx[k]];
          a1[k] = x1[idx[k]];
        }
        auto zeit = koplanar_zeit(a0, a1, STOSS_ABSTAND * 0.1);
        if (!zeit) return;
        if (best && best->zeit <= *zeit) return;
        std::array<V3, 4> q;
        for (int k = 0; k < 4; ++k) q[k] = lerp(a0[k], a1[k], *zeit);
        auto uv = im_dreieck(q[0], q[1], q[2], q[3]);
        if (!uv) return;
        V3 n = einheit(cross(sub(q[1], q[0]), sub(q[2], q[0])));
        double g[3] = {1.0 - (*uv)[0] - (*uv)[1], (*uv)[0], (*uv)[1]};
        V3 rel = sub(bew(a0, a1, 3), add(add(mul(bew(a0, a1, 0), g[0]), mul(bew(a0, a1, 1), g[1])), mul(bew(a0, a1, 2), g[2])));
        double seite = dot(rel, n) <= 0.0 ? 1.0 : -1.0;
        best = Stoss{Art::PunktDreieck, {v, d[0], d[1], d[2]}, *uv, *zeit, seite, mul(n, seite)};
      });
      if (best) aus.push_back(*best);
    }
  }
  if (kk) {
    std::vector<Quader> qk(netz.kanten.size());
    for (size_t e = 0; e < qk.size(); ++e) qk[e] = weg(netz.kanten[e].data(), 2);
    Hashgitter gitter = hashgitter_neu(qk, zelle);
    for (size_t i = 0; i < netz.kanten.size(); ++i) {
      uint32_t i0 = netz.kanten[i][0], i1 = netz.kanten[i][1];
      if (i0 == i1) continue;
      std::optional<Stoss> best;
      je_eintrag(gitter, qk[i], [&](uint32_t jj, std::array<int64_t, 3> c) {
        size_t j = jj;
        if (j <= i || !ueberlappt(qk[i], qk[j]) || !erste_zelle(qk[i], qk[j], zelle, c)) return;
        uint32_t j0 = netz.kanten[j][0], j1 = netz.kanten[j][1];
        for (uint32_t q : {j0, j1})
          if (netz.gleich_oder_partner(q, i0) || netz.gleich_oder_partner(q, i1)) return;
        std::array<uint32_t, 4> idx = {i1, j0, j1, i0};
        bool alle_fest = true;
        for (uint32_t k : idx) alle_fest = alle_fest && w[k] <= 0.0;
        if (alle_fest) return;
        std::array<V3, 4> a0, a1;
        for (int k = 0; k < 4; ++k) {
          a0[k] = x0[idx[k]];
          a1[k] = x1[idx[k]];
        }
        auto zeit = koplanar_zeit(a0, a1, STOSS_ABSTAND * 0.1);
        if (!zeit) return;
        if (best && best->zeit <= *zeit) return;
        std::array<V3, 4> q;
        for (int k = 0; k < 4; ++k) q[k] = lerp(a0[k], a1[k], *zeit);
        auto sw = kanten_kreuzen(q[3], q[0], q[1], q[2]);
        if (!sw) return;
        V3 n = einheit(cross(sub(q[0], q[3]), sub(q[2], q[1])));
        V3 auf_i = add(mul(bew(a0, a1, 3), 1.0 - (*sw)[0]), mul(bew(a0, a1, 0), (*sw)[0]));
        V3 auf_j = add(mul(bew(a0, a1, 1), 1.0 - (*sw)[1]), mul(bew(a0, a1, 2), (*sw)[1]));
        double seite = dot(sub(auf_i, auf_j), n) <= 0.0 ? 1.0 : -1.0;
        best = Stoss{Art::KanteKante, {i0, i1, j0, j1}, *sw, *zeit, seite, mul(n, seite)};
      });
      if (best) aus.push_back(*best);
    }
  }
  return aus;
}

// selbstkollision.rs:1288-1343
size_t stossantwort(const std::vector<Stoss>& stoesse, std::vector<V3>& x, const std::vector<double>& masse,
                    const std::vector<double>& w, size_t iterationen) {
  size_t zahl = 0;
  for (size_t it = 0; it < iterationen; ++it) {
    std::vector<V3> dx(x.size(), V3{0, 0, 0});
    std::vector<uint32_t> cnt(x.size(), 0);
    for (const auto& s : stoesse) {
      size_t p0 = s.punkte[0], p1 = s.punkte[1], p2 = s.punkte[2], p3 = s.punkte[3];
      std::vector<std::pair<size_t, double>> erste, zweite;
      V3 n;
      double d;
      if (s.art == Art::PunktDreieck) {
        n = mul(einheit(cross(sub(x[p2], x[p1]), sub(x[p3], x[p1]))), s.seite);
        double g0 = 1.0 - s.lage[0] - s.lage[1];
        erste = {{p0, 1.0}};
        zweite = {{p1, g0}, {p2, s.lage[0]}, {p3, s.lage[1]}};
        d = dot(n, sub(x[p0], x[p1]));
      } else {
        n = s.normale;
        V3 a = lerp(x[p0], x[p1], s.lage[0]), b = lerp(x[p2], x[p3], s.lage[1]);
        erste = {{p0, 1.0 - s.lage[0]}, {p1, s.lage[0]}};
        zweite = {{p2, 1.0 - s.lage[1]}, {p3, s.lage[1]}};
        d = dot(n, sub(a, b));
      }
      double tief = STOSS_ABSTAND - d;
      if (tief <= 0.0) continue;
      double m1 = 0.0, m2 = 0.0;
      bool fest1 = true, fest2 = true;
      for (auto [i, g] : erste) {
        m1 += g * masse[i];
        fest1 = fest1 && w[i] <= 0.0;
      }
      for (auto [i, g] : zweite) {
        m2 += g * masse[i];
        fest2 = fest2 && w[i] <= 0.0;
      }
      double alpha = fest2 ? 1.0 : (fest1 ? 0.0 : m2 / (m1 + m2));
      for (auto [i, g] : erste)
        if (w[i] > 0.0) {
          dx[i] = add(dx[i], mul(n, tief * alpha));
          cnt[i] += 1;
        }
      for (auto [i, g] : zweite)
        if (w[i] > 0.0) {
          dx[i] = sub(dx[i], mul(n, tief * (1.0 - alpha)));
          cnt[i] += 1;
        }
      zahl += 1;
    }
    bool bewegt = false;
    for (size_t i = 0; i < x.size(); ++i)
      if (cnt[i] > 0) {
        x[i] = add(x[i], mul(dx[i], 1.0 / double(cnt[i])));
        bewegt = true;
      }
    if (!bewegt) break;
  }
  return zahl;
}

}  // namespace orc
