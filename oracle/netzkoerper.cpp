// ORACLE (test infrastructure): a CPU FP64 restatement of the body mesh as a
// signed-distance collider, sim/src/netzkoerper.rs (Koerpernetz). Only the
// tests, smoke() and the bench's CPU legs load it, as the checker.
//
// Restated: the exact nearest point on a triangle (Ericson 2005, 5.1.5), the
// point-dependent tables (face normals, angle-weighted point normals, bounding
// spheres, volume), the topology checks and edge neighbours of Koerpernetz::neu,
// the triangle grid (cells of 2 x the search depth over the point hull grown
// by the search depth, grow-only on nachfuehren), the nearest query within a
// radius, the nearest over all triangles, and the segment penetration test
// (Moeller-Trumbore from outside). The sampled grid (netz_sdf) has no
// counterpart in the reference: it is the definition the device voxeliser is
// checked against, naechster_alle at every node, clamped to +-band.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <string>

#include "oracle.hpp"

namespace orc {

namespace {

// `f64 as i64` of Rust: saturating, NaN to 0.
int64_t als_i64(double v) {
  if (std::isnan(v)) return 0;
  if (v >= 9.2233720368547758e18) return std::numeric_limits<int64_t>::max();
  if (v <= -9.2233720368547758e18) return std::numeric_limits<int64_t>::min();
  return int64_t(v);
}

// netzkoerper.rs:220-227
V3 normiert(V3 a) {
  double l = norm(a);
  if (l > 0.0) return mul(a, 1.0 / l);
  return {0.0, 0.0, 0.0};
}

// netzkoerper.rs:246-248
double winkel(V3 u, V3 v) { return std::atan2(norm(cross(u, v)), dot(u, v)); }

// netzkoerper.rs:257-290: face normals, angle-weighted point normals (summed
// in triangle order), bounding spheres, volume.
double punktabhaengig(const std::vector<V3>& p, const std::vector<std::array<uint32_t, 3>>& d, std::vector<V3>& fn,
                      std::vector<V3>& pn, std::vector<std::pair<V3, double>>& kugel) {
  fn.clear();
  for (const auto& t : d) fn.push_back(normiert(cross(sub(p[t[1]], p[t[0]]), sub(p[t[2]], p[t[0]]))));
  pn.assign(p.size(), V3{0.0, 0.0, 0.0});
  kugel.clear();
  double volumen = 0.0;
  for (size_t t = 0; t < d.size(); ++t) {
    const V3 q[3] = {p[d[t][0]], p[d[t][1]], p[d[t][2]]};
    for (int k = 0; k < 3; ++k) {
      const double w = winkel(sub(q[(k + 1) % 3], q[k]), sub(q[(k + 2) % 3], q[k]));
      V3& s = pn[d[t][k]];
      s = add(s, mul(fn[t], w));
    }
    volumen += dot(q[0], cross(q[1], q[2])) / 6.0;
    const V3 m = mul(add(add(q[0], q[1]), q[2]), 1.0 / 3.0);
    double r = 0.0;
    for (int k = 0; k < 3; ++k) r = std::max(r, norm(sub(q[k], m)));
    kugel.push_back({m, r});
  }
  for (V3& s : pn) s = normiert(s);
  return volumen;
}

// netzkoerper.rs:232-243: barycentric weights of p's projection
std::array<double, 3> schwerpunktgewichte(V3 p, V3 a, V3 b, V3 c) {
  const V3 e1 = sub(b, a), e2 = sub(c, a), e3 = sub(p, a);
  const double d00 = dot(e1, e1), d01 = dot(e1, e2), d11 = dot(e2, e2);
  const double d20 = dot(e3, e1), d21 = dot(e3, e2);
  const double nenner = d00 * d11 - d01 * d01;
  if (nenner == 0.0) return {1.0, 0.0, 0.0};
  const double u = (d11 * d20 - d01 * d21) / nenner;
  const double w = (d00 * d21 - d01 * d20) / nenner;
  return {1.0 - u - w, u, w};
}

// netzkoerper.rs:785-797
void huelle(const std::vector<V3>& p, V3& lo, V3& hi) {
  lo = {INFINITY, INFINITY, INFINITY};
  hi = {-INFINITY, -INFINITY, -INFINITY};
  for (const V3& q : p)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], q[a]);
      hi[a] = std::max(hi[a], q[a]);
    }
}

}  // namespace

// netzkoerper.rs:87-92
std::array<int64_t, 3> NetzGitter::index(V3 x) const {
  std::array<int64_t, 3> k{};
  for (int a = 0; a < 3; ++a) k[a] = als_i64(std::floor((x[a] - ursprung[a]) / zelle));
  return k;
}
// netzkoerper.rs:95-97
size_t NetzGitter::zellnummer(size_t kx, size_t ky, size_t kz) const { return (kz * zahl[1] + ky) * zahl[0] + kx; }
// netzkoerper.rs:117-128
bool NetzGitter::bereich(V3 lo, V3 hi, std::array<std::pair<size_t, size_t>, 3>& r) const {
  const auto a = index(lo), b = index(hi);
  for (int d = 0; d < 3; ++d) {
    const int64_t n = int64_t(zahl[d]);
    if (b[d] < 0 || a[d] >= n) return false;
    r[d] = {size_t(std::max<int64_t>(a[d], 0)), size_t(std::min<int64_t>(b[d], n - 1))};
  }
  return true;
}

// netzkoerper.rs:185-216 (Ericson 2005, 5.1.5). Regions: 0-2 corner k, 3-5
// edge k (edge k runs from corner k to k+1), 6 face.
std::pair<V3, int> naechster_auf_dreieck(V3 p, V3 a, V3 b, V3 c) {
  auto quot = [](double z, double n) { return n > 0.0 ? z / n : 0.0; };
  const V3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
  const double d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) return {a, 0};
  const V3 bp = sub(p, b);
  const double d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0.0 && d4 <= d3) return {b, 1};
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) return {add(a, mul(ab, quot(d1, d1 - d3))), 3};
  const V3 cp = sub(p, c);
  const double d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) return {c, 2};
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return {add(a, mul(ac, quot(d2, d2 - d6))), 5};
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0.0 && d4 - d3 >= 0.0 && d5 - d6 >= 0.0) {
    const double w = quot(d4 - d3, (d4 - d3) + (d5 - d6));
    return {add(b, mul(sub(c, b), w)), 4};
  }
  const double s = va + vb + vc;
  const double v = quot(vb, s), w = quot(vc, s);
  return {add(a, add(mul(ab, v), mul(ac, w))), 6};
}

// netzkoerper.rs:820-858 (the triangle grid only; the point grid serves the
// body-point pass, which is not restated) and :881-910.
void Koerpernetz::gitter_bauen() {
  V3 lo, hi;
  huelle(punkte, lo, hi);
  const double z = 2.0 * suchtiefe;
  V3 u = sub(lo, V3{suchtiefe, suchtiefe, suchtiefe});
  V3 e = hi;
  for (int a = 0; a < 3; ++a) e[a] += suchtiefe;
  if (!(gitter.zahl[0] == 0 && gitter.zahl[1] == 0 && gitter.zahl[2] == 0)) {
    for (int a = 0; a < 3; ++a) {
      u[a] = std::min(u[a], gitter.ursprung[a]);
      e[a] = std::max(e[a], gitter.ursprung[a] + gitter.zelle * double(gitter.zahl[a]));
    }
  }
  std::array<size_t, 3> zahl{};
  for (int a = 0; a < 3; ++a) {
    const double c = std::ceil((e[a] - u[a]) / z);
    zahl[a] = std::max<size_t>(c > 0.0 ? size_t(c) : 0, 1);
  }
  gitter.ursprung = u;
  gitter.zelle = z;
  gitter.zahl = zahl;
  std::vector<std::array<int64_t, 3>> zellen(punkte.size());
  for (size_t i = 0; i < punkte.size(); ++i) zellen[i] = gitter.index(punkte[i]);
  const size_t nz = zahl[0] * zahl[1] * zahl[2];
  gitter.anfang.assign(nz + 1, 0);
  auto spanne = [&](const std::array<uint32_t, 3>& d, std::array<std::pair<size_t, size_t>, 3>& r) {
    std::array<int64_t, 3> a = zellen[d[0]], b = zellen[d[0]];
    for (int j = 1; j < 3; ++j)
      for (int q = 0; q < 3; ++q) {
        a[q] = std::min(a[q], zellen[d[j]][q]);
        b[q] = std::max(b[q], zellen[d[j]][q]);
      }
    for (int q = 0; q < 3; ++q) {
      const int64_t n = int64_t(zahl[q]);
      r[q] = {size_t(std::max<int64_t>(a[q], 0)), size_t(std::min<int64_t>(b[q], n - 1))};
    }
  };
  // the point grid on the same cells (gitter_punkte, :863-879): each point in
  // its own cell, in point order
  punktgitter.ursprung = u;
  punktgitter.zelle = z;
  punktgitter.zahl = zahl;
  punktgitter.anfang.assign(nz + 1, 0);
  auto zelle_von = [&](size_t i) {
    std::array<size_t, 3> k{};
    for (int q = 0; q < 3; ++q)
      k[q] = size_t(std::min<int64_t>(std::max<int64_t>(zellen[i][q], 0), int64_t(zahl[q]) - 1));
    return gitter.zellnummer(k[0], k[1], k[2]);
  };
  for (size_t i = 0; i < punkte.size(); ++i) punktgitter.anfang[zelle_von(i) + 1] += 1;
  for (size_t q = 0; q < nz; ++q) punktgitter.anfang[q + 1] += punktgitter.anfang[q];
  punktgitter.eintraege.assign(punktgitter.anfang[nz], 0);
  {
    std::vector<uint32_t> frei(punktgitter.anfang.begin(), punktgitter.anfang.end());
    for (size_t i = 0; i < punkte.size(); ++i) punktgitter.eintraege[frei[zelle_von(i)]++] = uint32_t(i);
  }
  std::array<std::pair<size_t, size_t>, 3> r{};
  for (const auto& d : dreiecke) {
    spanne(d, r);
    for (size_t kz = r[2].first; kz <= r[2].second; ++kz)
      for (size_t ky = r[1].first; ky <= r[1].second; ++ky)
        for (size_t kx = r[0].first; kx <= r[0].second; ++kx) gitter.anfang[gitter.zellnummer(kx, ky, kz) + 1] += 1;
  }
  for (size_t q = 0; q < nz; ++q) gitter.anfang[q + 1] += gitter.anfang[q];
  gitter.eintraege.assign(gitter.anfang[nz], 0);
  std::vector<uint32_t> frei(gitter.anfang.begin(), gitter.anfang.end());
  for (size_t t = 0; t < dreiecke.size(); ++t) {
    spanne(dreiecke[t], r);
    for (size_t kz = r[2].first; kz <= r[2].second; ++kz)
      for (size_t ky = r[1].first; ky <= r[1].second; ++ky)
        for (size_t kx = r[0].first; kx <= r[0].second; ++kx)
          gitter.eintraege[frei[gitter.zellnummer(kx, ky, kz)]++] = uint32_t(t);
  }
}

// netzkoerper.rs:297-367
std::optional<std::string> Koerpernetz::neu(std::vector<V3> p, std::vector<std::array<uint32_t, 3>> d,
                                            double suchtiefe_, Koerpernetz& out) {
  if (d.empty()) return std::string("body mesh without triangles");
  if (!(suchtiefe_ > 0.0)) return std::string("search depth must be positive");
  const size_t n = p.size();
  for (const auto& t : d)
    for (uint32_t i : t)
      if (size_t(i) >= n) return std::string("a triangle names a point out of range");
  // per undirected edge: (triangle, edge number, direction)
  std::map<std::pair<uint32_t, uint32_t>, std::vector<std::array<uint32_t, 3>>> kanten;
  for (size_t t = 0; t < d.size(); ++t)
    for (uint32_t k = 0; k < 3; ++k) {
      const uint32_t i = d[t][k], j = d[t][(k + 1) % 3];
      kanten[{std::min(i, j), std::max(i, j)}].push_back({uint32_t(t), k, uint32_t(i < j)});
    }
  std::vector<std::array<uint32_t, 3>> nachbar(d.size(), {0, 0, 0});
  size_t rand = 0;
  for (const auto& [ij, l] : kanten) {
    if (l.size() == 1) {
      ++rand;
      nachbar[l[0][0]][l[0][1]] = l[0][0];
    } else if (l.size() == 2) {
      if (l[0][2] == l[1][2]) return std::string("mesh orientation is inconsistent at an edge");
      nachbar[l[0][0]][l[0][1]] = l[1][0];
      nachbar[l[1][0]][l[1][1]] = l[0][0];
    } else {
      return std::string("an edge has more than two triangles");
    }
  }
  Koerpernetz k;
  k.volumen = punktabhaengig(p, d, k.flaechennormale, k.punktnormale, k.kugel);
  if (k.volumen <= 0.0) return std::string("volume <= 0: the normals point inwards");
  k.punkte = std::move(p);
  k.dreiecke = std::move(d);
  k.nachbar = std::move(nachbar);
  k.randkanten = rand;
  k.suchtiefe = suchtiefe_;
  k.gitter_bauen();
  out = std::move(k);
  return std::nullopt;
}

// netzkoerper.rs:390-411
std::optional<std::string> Koerpernetz::nachfuehren(const std::vector<V3>& p) {
  if (p.size() != punkte.size()) return std::string("nachfuehren: point count differs");
  const double v = punktabhaengig(p, dreiecke, flaechennormale, punktnormale, kugel);
  if (v <= 0.0) return std::string("volume <= 0 after deforming: the mesh turned inside out");
  punkte = p;
  volumen = v;
  punktgeschwindigkeit.clear();  // the field belonged to the old positions
  gitter_bauen();
  return std::nullopt;
}

// netzkoerper.rs:454-463
std::optional<std::string> Koerpernetz::setze_punktgeschwindigkeit(const std::vector<V3>& v) {
  if (!v.empty() && v.size() != punkte.size()) return std::string("velocity field size differs from the points");
  punktgeschwindigkeit = v;
  return std::nullopt;
}
// netzkoerper.rs:474-489
V3 Koerpernetz::geschwindigkeit_an(size_t t, V3 p, V3 starr) const {
  if (punktgeschwindigkeit.empty()) return starr;
  const auto& d = dreiecke[t];
  const auto g = schwerpunktgewichte(p, punkte[d[0]], punkte[d[1]], punkte[d[2]]);
  V3 q{0.0, 0.0, 0.0};
  for (int j = 0; j < 3; ++j) {
    const V3 v = punktgeschwindigkeit[d[j]];
    for (int k = 0; k < 3; ++k) q[k] += g[j] * v[k];
  }
  return q;
}

// netzkoerper.rs:431-438
V3 Koerpernetz::kantennormale(size_t t, int k) const {
  const size_t o = nachbar[t][size_t(k)];
  if (o == t) return flaechennormale[t];
  return normiert(add(flaechennormale[t], flaechennormale[o]));
}
// netzkoerper.rs:441-447
V3 Koerpernetz::pseudonormale(size_t t, int r) const {
  if (r == 6) return flaechennormale[t];
  if (r >= 3) return kantennormale(t, r - 3);
  return punktnormale[dreiecke[t][size_t(r)]];
}
// netzkoerper.rs:492-499
Naechster Koerpernetz::ergebnis(V3 x, size_t t, V3 c, int r) const {
  const V3 pn = pseudonormale(t, r);
  const V3 d = sub(x, c);
  const double l = norm(d);
  const bool aussen = dot(d, pn) >= 0.0;
  const V3 nrm = l > 1e-12 ? mul(d, aussen ? 1.0 / l : -1.0 / l) : pn;
  return Naechster{aussen ? l : -l, c, nrm, uint32_t(t), r};
}

// netzkoerper.rs:503-539
std::optional<Naechster> Koerpernetz::naechster(V3 x, double radius) const {
  std::array<std::pair<size_t, size_t>, 3> r{};
  if (!gitter.bereich(sub(x, V3{radius, radius, radius}), add(x, V3{radius, radius, radius}), r)) return std::nullopt;
  double best = radius;
  bool hit = false;
  size_t bt = 0;
  V3 bq{};
  int br = 0;
  for (size_t kz = r[2].first; kz <= r[2].second; ++kz)
    for (size_t ky = r[1].first; ky <= r[1].second; ++ky)
      for (size_t kx = r[0].first; kx <= r[0].second; ++kx) {
        const size_t z = gitter.zellnummer(kx, ky, kz);
        for (uint32_t e = gitter.anfang[z]; e < gitter.anfang[z + 1]; ++e) {
          const size_t t = gitter.eintraege[e];
          if (norm(sub(x, kugel[t].first)) - kugel[t].second >= best) continue;
          const auto [q, reg] =
              naechster_auf_dreieck(x, punkte[dreiecke[t][0]], punkte[dreiecke[t][1]], punkte[dreiecke[t][2]]);
          const double l = norm(sub(x, q));
          if (l < best) {
            best = l;
            hit = true;
            bt = t;
            bq = q;
            br = reg;
          }
        }
      }
  if (!hit) return std::nullopt;
  return ergebnis(x, bt, bq, br);
}

// netzkoerper.rs:770-782
Naechster Koerpernetz::naechster_alle(V3 x) const {
  double best = INFINITY;
  size_t bt = 0;
  V3 bq{};
  int br = 6;
  for (size_t t = 0; t < dreiecke.size(); ++t) {
    const auto [q, reg] =
        naechster_auf_dreieck(x, punkte[dreiecke[t][0]], punkte[dreiecke[t][1]], punkte[dreiecke[t][2]]);
    const double l = norm(sub(x, q));
    if (l < best) {
      best = l;
      bt = t;
      bq = q;
      br = reg;
    }
  }
  return ergebnis(x, bt, bq, br);
}

// netzkoerper.rs:541-593 (the body velocity at the hit is not restated: a
// rigid body's is its own velocity)
std::optional<Durchstoss> Koerpernetz::durchstoss(V3 a, V3 b) const {
  const V3 d = sub(b, a);
  if (dot(d, d) < 1e-24) return std::nullopt;
  V3 lo = a, hi = a;
  for (int k = 0; k < 3; ++k) {
    lo[k] = std::min(lo[k], b[k]);
    hi[k] = std::max(hi[k], b[k]);
  }
  std::array<std::pair<size_t, size_t>, 3> r{};
  if (!gitter.bereich(lo, hi, r)) return std::nullopt;
  const double eps = 1e-12;
  bool hit = false;
  double sb = 0.0;
  size_t tb = 0;
  for (size_t kz = r[2].first; kz <= r[2].second; ++kz)
    for (size_t ky = r[1].first; ky <= r[1].second; ++ky)
      for (size_t kx = r[0].first; kx <= r[0].second; ++kx) {
        const size_t z = gitter.zellnummer(kx, ky, kz);
        for (uint32_t e = gitter.anfang[z]; e < gitter.anfang[z + 1]; ++e) {
          const size_t t = gitter.eintraege[e];
          if (dot(d, flaechennormale[t]) >= 0.0) continue;
          const V3 p0 = punkte[dreiecke[t][0]], p1 = punkte[dreiecke[t][1]], p2 = punkte[dreiecke[t][2]];
          const V3 e1 = sub(p1, p0), e2 = sub(p2, p0);
          const V3 pv = cross(d, e2);
          const double det = dot(e1, pv);
          if (std::fabs(det) < 1e-30) continue;
          const V3 tv = sub(a, p0);
          const double u = dot(tv, pv) / det;
          if (u < -eps || u > 1.0 + eps) continue;
          const V3 qv = cross(tv, e1);
          const double v = dot(d, qv) / det;
          if (v < -eps || u + v > 1.0 + eps) continue;
          const double s = dot(e2, qv) / det;
          if (s >= -eps && s <= 1.0 + eps && (!hit || s < sb)) {
            hit = true;
            sb = s;
            tb = t;
          }
        }
      }
  if (!hit) return std::nullopt;
  const V3 p = add(a, mul(d, std::min(std::max(sb, 0.0), 1.0)));
  return Durchstoss{p, flaechennormale[tb], uint32_t(tb)};
}

// netzkoerper.rs:612-665 (punkte_gegen_dreiecke) with stiche (:677-735):
// every body point whose line p + t n (n its point normal) meets a cloth
// triangle at -tief < t < -1e-9 stabs it; per triangle the deepest stab (the
// first of equal depth in the point grid's order) lifts the triangle, in
// triangle order, by barycentric weight and inverse mass, and takes the
// triangle's velocity into the body point's away.
size_t Koerpernetz::punkte_gegen_dreiecke(double tief, V3 versatz, V3 geschwindigkeit,
                                          const std::vector<std::array<uint32_t, 3>>& dreiecke,
                                          const std::vector<double>& w, std::vector<V3>& x,
                                          std::vector<V3>& v) const {
  struct Stich {
    bool hat = false;
    double d = 0;
    V3 n{}, bary{};
    uint32_t kir = 0;
  };
  std::vector<Stich> tiefster(dreiecke.size());
  const double band = -1e-9, rand = std::max(tief, band);
  for (size_t di = 0; di < dreiecke.size(); ++di) {
    const V3 a = x[dreiecke[di][0]], b = x[dreiecke[di][1]], c = x[dreiecke[di][2]];
    V3 lo = a, hi = a;
    for (const V3& q : {b, c})
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], q[k]);
        hi[k] = std::max(hi[k], q[k]);
      }
    lo = sub(sub(lo, versatz), V3{rand, rand, rand});
    hi = add(sub(hi, versatz), V3{rand, rand, rand});
    const V3 e1 = sub(b, a), e2 = sub(c, a);
    std::array<std::pair<size_t, size_t>, 3> r{};
    if (!punktgitter.bereich(lo, hi, r)) continue;
    for (size_t kz = r[2].first; kz <= r[2].second; ++kz)
      for (size_t ky = r[1].first; ky <= r[1].second; ++ky)
        for (size_t kx = r[0].first; kx <= r[0].second; ++kx) {
          const size_t z = punktgitter.zellnummer(kx, ky, kz);
          for (uint32_t e = punktgitter.anfang[z]; e < punktgitter.anfang[z + 1]; ++e) {
            const uint32_t k = punktgitter.eintraege[e];
            const V3 p = add(punkte[k], versatz);
            const V3 n = punktnormale[k];
            const V3 pv = cross(n, e2);
            const double det = dot(e1, pv);
            if (std::fabs(det) < 1e-18) continue;
            const V3 tv = sub(p, a);
            const double bu = dot(tv, pv) / det;
            if (!(bu >= 0.0 && bu <= 1.0)) continue;
            const V3 qv = cross(tv, e1);
            const double bv = dot(n, qv) / det;
            if (bv < 0.0 || bu + bv > 1.0) continue;
            const double t = dot(e2, qv) / det;
            if (t > -tief && t < band) {
              Stich& s = tiefster[di];
              if (!s.hat || -t > s.d) s = Stich{true, -t, n, V3{1.0 - bu - bv, bu, bv}, k};
            }
          }
        }
  }
  size_t zahl = 0;
  for (size_t di = 0; di < dreiecke.size(); ++di) {
    const Stich& s = tiefster[di];
    if (!s.hat) continue;
    const auto& idx = dreiecke[di];
    const double gew[3] = {w[idx[0]], w[idx[1]], w[idx[2]]};
    double nenner = -0.0;
    for (int j = 0; j < 3; ++j) nenner += s.bary[j] * s.bary[j] * gew[j];
    if (nenner <= 0.0) continue;
    const V3 vk = punktgeschwindigkeit.empty() ? geschwindigkeit : punktgeschwindigkeit[s.kir];
    V3 vq{0.0, 0.0, 0.0};
    for (int j = 0; j < 3; ++j) vq = add(vq, mul(v[idx[j]], s.bary[j]));
    vq = sub(vq, vk);
    const double vn = std::min(dot(vq, s.n), 0.0);
    for (int j = 0; j < 3; ++j) {
      const double f = s.bary[j] * gew[j] / nenner;
      x[idx[j]] = add(x[idx[j]], mul(s.n, f * s.d));
      v[idx[j]] = sub(v[idx[j]], mul(s.n, f * vn));
    }
    ++zahl;
  }
  return zahl;
}

// The sampled grid: node (i, j, k) at ursprung + spacing * (i, j, k); its
// value is the signed distance of naechster_alle, clamped to [-band, band]
// when band > 0.
void Koerpernetz::sdf(const int32_t dims[3], V3 ursprung, double spacing, double band, float* out) const {
  for (int64_t k = 0; k < dims[2]; ++k)
    for (int64_t j = 0; j < dims[1]; ++j)
      for (int64_t i = 0; i < dims[0]; ++i) {
        const V3 x = {ursprung[0] + spacing * double(i), ursprung[1] + spacing * double(j),
                      ursprung[2] + spacing * double(k)};
        double d = naechster_alle(x).abstand;
        if (band > 0.0) d = std::min(std::max(d, -band), band);
        out[(k * dims[1] + j) * int64_t(dims[0]) + i] = float(d);
      }
}

}  // namespace orc

// ------------------------------------------------------------ C entry points
using namespace orc;

namespace {
std::vector<V3> punkte_aus(const double* p, int64_t n) {
  std::vector<V3> o(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) o[size_t(i)] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
  return o;
}
void fehler_setzen(const std::string& s, char* err, int64_t cap) {
  if (!err || cap <= 0) return;
  const size_t m = std::min<size_t>(s.size(), size_t(cap - 1));
  std::memcpy(err, s.data(), m);
  err[m] = 0;
}
void schreibe(const Naechster& r, int64_t q, double* abstand, double* punkt, double* normale, int32_t* dreieck,
              int32_t* region) {
  if (abstand) abstand[q] = r.abstand;
  for (int a = 0; a < 3; ++a) {
    if (punkt) punkt[3 * q + a] = r.punkt[a];
    if (normale) normale[3 * q + a] = r.normale[a];
  }
  if (dreieck) dreieck[q] = int32_t(r.dreieck);
  if (region) region[q] = r.region;
}
}  // namespace

extern "C" {

void* orc_netz_neu(const double* punkte, int64_t n, const uint32_t* dreiecke, int64_t nd, double suchtiefe, char* err,
                   int64_t err_cap) {
  std::vector<std::array<uint32_t, 3>> d(static_cast<size_t>(nd));
  for (int64_t t = 0; t < nd; ++t) d[size_t(t)] = {dreiecke[3 * t], dreiecke[3 * t + 1], dreiecke[3 * t + 2]};
  auto k = std::make_unique<Koerpernetz>();
  if (auto e = Koerpernetz::neu(punkte_aus(punkte, n), std::move(d), suchtiefe, *k)) {
    fehler_setzen(*e, err, err_cap);
    return nullptr;
  }
  return k.release();
}
void orc_netz_free(void* h) { delete static_cast<Koerpernetz*>(h); }
int32_t orc_netz_nachfuehren(void* h, const double* punkte, char* err, int64_t err_cap) {
  auto* k = static_cast<Koerpernetz*>(h);
  if (auto e = k->nachfuehren(punkte_aus(punkte, int64_t(k->punkte.size())))) {
    fehler_setzen(*e, err, err_cap);
    return 1;
  }
  return 0;
}
// randkanten, volumen, gitter: ursprung (3), zelle, zahl (3), entries
void orc_netz_info(void* h, int64_t* randkanten, double* volumen, double* ursprung3, double* zelle, int64_t* zahl3,
                   int64_t* eintraege) {
  const auto* k = static_cast<const Koerpernetz*>(h);
  *randkanten = int64_t(k->randkanten);
  *volumen = k->volumen;
  for (int a = 0; a < 3; ++a) {
    ursprung3[a] = k->gitter.ursprung[a];
    zahl3[a] = int64_t(k->gitter.zahl[a]);
  }
  *zelle = k->gitter.zelle;
  *eintraege = int64_t(k->gitter.eintraege.size());
}
// face normals (3 nd), point normals (3 n), neighbours (3 nd), spheres (4 nd)
void orc_netz_tabellen(void* h, double* fn, double* pn, uint32_t* nachbar, double* kugel) {
  const auto* k = static_cast<const Koerpernetz*>(h);
  for (size_t t = 0; t < k->dreiecke.size(); ++t)
    for (int a = 0; a < 3; ++a) {
      if (fn) fn[3 * t + a] = k->flaechennormale[t][a];
      if (nachbar) nachbar[3 * t + a] = k->nachbar[t][a];
      if (kugel) kugel[4 * t + a] = k->kugel[t].first[a];
    }
  if (kugel)
    for (size_t t = 0; t < k->dreiecke.size(); ++t) kugel[4 * t + 3] = k->kugel[t].second;
  if (pn)
    for (size_t i = 0; i < k->punkte.size(); ++i)
      for (int a = 0; a < 3; ++a) pn[3 * i + a] = k->punktnormale[i][a];
}
// radius > 0: naechster (dreieck -1 where nothing is closer); otherwise naechster_alle
void orc_netz_naechster(void* h, const double* x, int64_t n, double radius, double* abstand, double* punkt,
                        double* normale, int32_t* dreieck, int32_t* region) {
  const auto* k = static_cast<const Koerpernetz*>(h);
  for (int64_t q = 0; q < n; ++q) {
    const V3 p = {x[3 * q], x[3 * q + 1], x[3 * q + 2]};
    if (radius > 0.0) {
      auto r = k->naechster(p, radius);
      if (r) {
        schreibe(*r, q, abstand, punkt, normale, dreieck, region);
      } else {
        if (dreieck) dreieck[q] = -1;
        if (region) region[q] = -1;
      }
    } else {
      schreibe(k->naechster_alle(p), q, abstand, punkt, normale, dreieck, region);
    }
  }
}
void orc_netz_durchstoss(void* h, const double* a, const double* b, int64_t n, int32_t* dreieck, double* punkt,
                         double* normale) {
  const auto* k = static_cast<const Koerpernetz*>(h);
  for (int64_t q = 0; q < n; ++q) {
    auto r = k->durchstoss({a[3 * q], a[3 * q + 1], a[3 * q + 2]}, {b[3 * q], b[3 * q + 1], b[3 * q + 2]});
    dreieck[q] = r ? int32_t(r->dreieck) : -1;
    for (int c = 0; c < 3; ++c) {
      if (punkt) punkt[3 * q + c] = r ? r->punkt[c] : 0.0;
      if (normale) normale[3 * q + c] = r ? r->normale[c] : 0.0;
    }
  }
}
// punkte_gegen_dreiecke on raw cloth arrays (x, v changed in place)
int64_t orc_netz_punkte_gegen_dreiecke(void* h, double tief, const double* versatz3, const double* geschw3,
                                       const uint32_t* dreiecke, int64_t nd, const double* w, double* x, double* v,
                                       int64_t n) {
  const auto* k = static_cast<const Koerpernetz*>(h);
  std::vector<std::array<uint32_t, 3>> d(static_cast<size_t>(nd));
  for (int64_t t = 0; t < nd; ++t) d[size_t(t)] = {dreiecke[3 * t], dreiecke[3 * t + 1], dreiecke[3 * t + 2]};
  std::vector<V3> xs = punkte_aus(x, n), vs = punkte_aus(v, n);
  const std::vector<double> ws(w, w + n);
  const size_t z = k->punkte_gegen_dreiecke(tief, {versatz3[0], versatz3[1], versatz3[2]},
                                            {geschw3[0], geschw3[1], geschw3[2]}, d, ws, xs, vs);
  for (int64_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) x[3 * i + a] = xs[size_t(i)][a], v[3 * i + a] = vs[size_t(i)][a];
  return int64_t(z);
}
// setze_punktgeschwindigkeit: v 3 per point, or null to clear
int32_t orc_netz_setze_geschwindigkeit(void* h, const double* v, int64_t n, char* err, int64_t err_cap) {
  auto* k = static_cast<Koerpernetz*>(h);
  std::vector<V3> f;
  if (v) f = punkte_aus(v, n);
  if (auto e = k->setze_punktgeschwindigkeit(f)) {
    fehler_setzen(*e, err, err_cap);
    return 1;
  }
  return 0;
}
void orc_netz_geschwindigkeit_an(void* h, const int32_t* dreieck, const double* punkt, int64_t n,
                                 const double* starr3, double* out) {
  const auto* k = static_cast<const Koerpernetz*>(h);
  const V3 starr = {starr3[0], starr3[1], starr3[2]};
  for (int64_t q = 0; q < n; ++q) {
    const V3 v = k->geschwindigkeit_an(size_t(dreieck[q]), {punkt[3 * q], punkt[3 * q + 1], punkt[3 * q + 2]}, starr);
    for (int a = 0; a < 3; ++a) out[3 * q + a] = v[a];
  }
}
void orc_netz_sdf(void* h, const int32_t* dims3, const double* ursprung3, double spacing, double band, float* out) {
  static_cast<const Koerpernetz*>(h)->sdf(dims3, {ursprung3[0], ursprung3[1], ursprung3[2]}, spacing, band, out);
}

}  // extern "C"
