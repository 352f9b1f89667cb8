// ORACLE (test infrastructure). Bending stiffness, dihedral angle, colouring,
// collision bodies and scene measurements, restated from the reference in FP64.
#include <algorithm>
#include <limits>

#include "oracle.hpp"

namespace orc {

// ------------------------------------------------------------ sim/src/biegung.rs
// biegung.rs:136-142
static double positiv(double d, double weft, double warp, double bias) {
  if (d > 0.0) return d;
  double kleinste = std::fabs(std::min(std::min(weft, warp), bias));
  return 1.0e-3 * kleinste;
}
// biegung.rs:92-104
double steifigkeit(double weft, double warp, double bias, double theta) {
  if (weft == warp && warp == bias) return weft;
  double s = std::sin(theta), c = std::cos(theta);
  double s2 = s * s, c2 = c * c;
  return positiv(warp * (c2 * c2) + weft * (s2 * s2) + (4.0 * bias - warp - weft) * (c2 * s2), weft, warp,
                 bias);
}
// biegung.rs:111-121
double steifigkeit_aus(double c2, double s2, double weft, double warp, double bias) {
  if (weft == warp && warp == bias) return weft;
  return positiv(warp * (c2 * c2) + weft * (s2 * s2) + (4.0 * bias - warp - weft) * (c2 * s2), weft, warp,
                 bias);
}
// biegung.rs:156-173
bool cos2_sin2(V2 e, V2 warp, double& c2, double& s2) {
  double le = std::sqrt(e[0] * e[0] + e[1] * e[1]);
  double lw = std::sqrt(warp[0] * warp[0] + warp[1] * warp[1]);
  if (!(le > 1e-12) || !(lw > 1e-12)) return false;
  double ex = e[0] / le, ey = e[1] / le;
  double wx = warp[0] / lw, wy = warp[1] / lw;
  double c_edge = ex * wx + ey * wy;
  double s_edge = ex * wy - ey * wx;
  double c = -s_edge, s = c_edge;
  c2 = c * c;
  s2 = s * s;
  return true;
}

// ------------------------------------------------------------ sim/src/cpu.rs
// cpu.rs:279-282: difference wrapped to (-pi, pi]; Rust's f64::round rounds
// half away from zero, which std::round also does.
double winkel_fehler(double theta, double ruhe) {
  const double tau = 6.283185307179586476925286766559;
  double d = theta - ruhe;
  return d - tau * std::round(d / tau);
}
// cpu.rs:288-307 (Bridson et al. 2003 dihedral angle and gradients)
bool dieder(const std::array<V3, 4>& q, double& theta, std::array<V3, 4>& g) {
  const V3 &x0 = q[0], &x1 = q[1], &x2 = q[2], &x3 = q[3];
  V3 e = sub(x1, x0);
  double le = norm(e);
  V3 n1 = cross(sub(x2, x0), sub(x2, x1));
  V3 n2 = cross(sub(x3, x1), sub(x3, x0));
  double q1 = dot(n1, n1), q2 = dot(n2, n2);
  if (le < 1e-12 || q1 < 1e-30 || q2 < 1e-30) return false;
  V3 m1 = mul(n1, 1.0 / std::sqrt(q1)), m2 = mul(n2, 1.0 / std::sqrt(q2));
  theta = std::atan2(dot(cross(m1, m2), mul(e, 1.0 / le)), dot(m1, m2));
  g[2] = mul(n1, -le / q1);
  g[3] = mul(n2, -le / q2);
  g[0] = mul(add(mul(n1, dot(sub(x2, x1), e) / le / q1), mul(n2, dot(sub(x3, x1), e) / le / q2)), -1.0);
  g[1] = add(mul(n1, dot(sub(x2, x0), e) / le / q1), mul(n2, dot(sub(x3, x0), e) / le / q2));
  return true;
}

// ------------------------------------------------------------ sim/src/faerbung.rs
// faerbung.rs:11-43: greedy colouring in input order, 64-bit mask fast path.
std::pair<std::vector<uint32_t>, size_t> faerbe(size_t anzahl, size_t npunkte,
                                                 const std::vector<std::vector<uint32_t>>& punkte) {
  std::vector<uint64_t> maske(npunkte, 0);
  std::vector<std::vector<uint32_t>> mehr(npunkte);
  std::vector<uint32_t> farbe(anzahl, 0);
  size_t zahl = 0;
  for (size_t c = 0; c < anzahl; ++c) {
    const auto& p = punkte[c];
    uint64_t belegt = 0;
    for (uint32_t i : p) belegt |= maske[i];
    uint32_t f;
    if (belegt != ~uint64_t(0)) {
      f = static_cast<uint32_t>(__builtin_ctzll(~belegt));
    } else {
      f = 64;
      for (;; ++f) {
        bool frei = true;
        for (uint32_t i : p)
          if (std::find(mehr[i].begin(), mehr[i].end(), f) != mehr[i].end()) frei = false;
        if (frei) break;
      }
    }
    for (uint32_t i : p) {
      if (f < 64)
        maske[i] |= uint64_t(1) << f;
      else
        mehr[i].push_back(f);
    }
    farbe[c] = f;
    zahl = std::max(zahl, size_t(f) + 1);
  }
  return {farbe, zahl};
}
// faerbung.rs:46-57: stable order by colour
std::pair<std::vector<size_t>, std::vector<std::pair<size_t, size_t>>> ordnung(const std::vector<uint32_t>& farbe,
                                                                                size_t zahl) {
  std::vector<size_t> idx(farbe.size());
  for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return farbe[a] < farbe[b]; });
  std::vector<std::pair<size_t, size_t>> bereiche;
  size_t start = 0;
  for (uint32_t f = 0; f < zahl; ++f) {
    size_t ende = start;
    while (ende < idx.size() && farbe[idx[ende]] == f) ++ende;
    bereiche.push_back({start, ende});
    start = ende;
  }
  return {idx, bereiche};
}

// ------------------------------------------------------------ bodies
// koerper.rs:69-91 (Zylinder, Netz); art 1 is the sampled signed-distance grid.
std::optional<Kontakt> Koerper::kontakt(V3 x, double abstand) const {
  if (art == 2) {
    auto n = netz->naechster(sub(x, punkt), std::max(netz->suchtiefe, abstand));
    if (!n) return std::nullopt;
    const double tiefe = abstand - n->abstand;
    if (!(tiefe > 0.0)) return std::nullopt;
    return Kontakt{n->normale, tiefe, netz->geschwindigkeit_an(n->dreieck, n->punkt, geschwindigkeit)};
  }
  if (art == 0) {
    V3 a = mul(achse, 1.0 / norm(achse));
    V3 d = sub(x, punkt);
    V3 quer = sub(d, mul(a, dot(d, a)));
    double r = norm(quer);
    double tiefe = radius + abstand - r;
    if (tiefe <= 0.0 || r < 1e-12) return std::nullopt;
    return Kontakt{mul(quer, 1.0 / r), tiefe, geschwindigkeit};
  }
  // Trilinear value and gradient of the node values; outside the grid there
  // is no contact.
  double u[3];
  int64_t ii[3];
  double t[3];
  for (int a = 0; a < 3; ++a) {
    u[a] = (x[a] - punkt[a] - ursprung[a]) / spacing;
    double fl = std::floor(u[a]);
    if (!(fl >= 0.0) || !(fl < double(dims[a] - 1))) return std::nullopt;
    ii[a] = int64_t(fl);
    t[a] = u[a] - fl;
  }
  auto phi = [&](int64_t i, int64_t j, int64_t k) -> double {
    return double(sdf[(k * dims[1] + j) * int64_t(dims[0]) + i]);
  };
  const int64_t i = ii[0], j = ii[1], k = ii[2];
  double c000 = phi(i, j, k), c100 = phi(i + 1, j, k), c010 = phi(i, j + 1, k), c110 = phi(i + 1, j + 1, k);
  double c001 = phi(i, j, k + 1), c101 = phi(i + 1, j, k + 1), c011 = phi(i, j + 1, k + 1),
         c111 = phi(i + 1, j + 1, k + 1);
  double tx = t[0], ty = t[1], tz = t[2];
  double c00 = c000 + (c100 - c000) * tx, c10 = c010 + (c110 - c010) * tx;
  double c01 = c001 + (c101 - c001) * tx, c11 = c011 + (c111 - c011) * tx;
  double c0 = c00 + (c10 - c00) * ty, c1 = c01 + (c11 - c01) * ty;
  double wert = c0 + (c1 - c0) * tz;
  double d00 = c100 - c000, d10 = c110 - c010, d01 = c101 - c001, d11 = c111 - c011;
  double d0 = d00 + (d10 - d00) * ty, d1 = d01 + (d11 - d01) * ty;
  double gx = (d0 + (d1 - d0) * tz) / spacing;
  double e0 = c10 - c00, e1 = c11 - c01;
  double gy = (e0 + (e1 - e0) * tz) / spacing;
  double gz = (c1 - c0) / spacing;
  double tiefe = abstand - wert;
  if (tiefe <= 0.0) return std::nullopt;
  V3 g = {gx, gy, gz};
  double gl = norm(g);
  if (gl < 1e-12) return std::nullopt;
  return Kontakt{mul(g, 1.0 / gl), tiefe, geschwindigkeit};
}
// koerper.rs:122-133
// koerper.rs:99-107 (only the mesh has a skin to pass through)
std::optional<std::array<V3, 3>> Koerper::durchstoss(V3 von, V3 nach) const {
  if (art != 2) return std::nullopt;
  auto r = netz->durchstoss(sub(von, punkt), sub(nach, punkt));
  if (!r) return std::nullopt;
  return std::array<V3, 3>{add(r->punkt, punkt), r->normale, netz->geschwindigkeit_an(r->dreieck, r->punkt, geschwindigkeit)};
}

size_t Koerper::punkte_gegen_dreiecke(double tief, const std::vector<std::array<uint32_t, 3>>& dreiecke,
                                      const std::vector<double>& w, std::vector<V3>& x, std::vector<V3>& v) const {
  if (art != 2) return 0;
  return netz->punkte_gegen_dreiecke(tief, punkt, geschwindigkeit, dreiecke, w, x, v);
}

Koerper Koerper::verschoben(double t) const {
  Koerper k = *this;
  k.punkt = add(punkt, mul(geschwindigkeit, t));
  return k;
}

// ------------------------------------------------------------ sim/src/messung.rs
// messung.rs:10-30
double umfang_in_ebene(const Szene& s, V3 punkt, V3 normale) {
  V3 n = mul(normale, 1.0 / norm(normale));
  double summe = 0.0;
  for (const auto& d : s.dreiecke) {
    V3 p[3] = {s.x[d[0]], s.x[d[1]], s.x[d[2]]};
    double h[3];
    for (int k = 0; k < 3; ++k) h[k] = dot(sub(p[k], punkt), n);
    std::vector<V3> schnitt;
    for (int k = 0; k < 3; ++k) {
      int a = k, b = (k + 1) % 3;
      if ((h[a] < 0.0) != (h[b] < 0.0)) {
        double tt = h[a] / (h[a] - h[b]);
        schnitt.push_back(add(p[a], mul(sub(p[b], p[a]), tt)));
      }
    }
    if (schnitt.size() == 2) summe += norm(sub(schnitt[1], schnitt[0]));
  }
  return summe;
}
// messung.rs:35-51
std::vector<std::pair<double, double>> dehnung_je_dreieck(const Szene& s) {
  std::vector<std::pair<double, double>> out;
  for (size_t t = 0; t < s.dreiecke.size(); ++t) {
    const auto& d = s.dreiecke[t];
    const auto& r = s.ruhe_inv[t];
    V3 e1 = sub(s.x[d[1]], s.x[d[0]]), e2 = sub(s.x[d[2]], s.x[d[0]]);
    V3 f1 = add(mul(e1, r[0]), mul(e2, r[2]));
    V3 f2 = add(mul(e1, r[1]), mul(e2, r[3]));
    double a = dot(f1, f1), b = dot(f1, f2), c = dot(f2, f2);
    double mitte = 0.5 * (a + c);
    double rad = std::sqrt(0.25 * (a - c) * (a - c) + b * b);
    out.push_back({std::sqrt(mitte + rad) - 1.0, std::sqrt(std::max(mitte - rad, 0.0)) - 1.0});
  }
  return out;
}
// messung.rs:54-60
double nahtspalt(const Szene& s) {
  double m = 0.0;
  for (const auto& p : s.naht.punkte) m = std::max(m, norm(sub(s.x[p[0]], s.x[p[1]])));
  return m;
}
// messung.rs:82-116
double mittlere_geschwindigkeit(const Szene& s) {
  double e = 0.0, m = 0.0;
  for (size_t i = 0; i < s.v.size(); ++i) e += 0.5 * s.masse[i] * dot(s.v[i], s.v[i]);
  for (double mi : s.masse) m += mi;
  return std::sqrt(2.0 * e / m);
}
V3 schwerpunkt(const Szene& s) {
  double m = 0.0;
  for (double mi : s.masse) m += mi;
  V3 q{};
  for (size_t i = 0; i < s.x.size(); ++i) q = add(q, mul(s.x[i], s.masse[i]));
  return mul(q, 1.0 / m);
}

}  // namespace orc
