// Test infrastructure (oracle): the reference's XPBD cross-check solver,
// CpuReferenz (crates/klon3d-sim/src/cpu.rs:76-245), restated in FP64 in the
// same loop order, with the membrane's three strain constraints
// (kontinuum.rs:526-551). The device step does not run XPBD; it stays a
// host-side cross-check of the implicit step, as in the reference.
#include <cmath>
#include <limits>

#include "oracle.hpp"

namespace orc {

// cpu.rs:251-270: C = |p_i - p_j| - ruhe with p = x + delta + korr; corrects korr.
void xpbd_abstand(const std::vector<V3>& x, const std::vector<V3>& delta, std::vector<V3>& korr,
                  const std::vector<double>& w, std::array<uint32_t, 2> p, double ruhe, double alpha_h2) {
  const size_t i = p[0], j = p[1];
  const V3 d = add(add(sub(x[i], x[j]), sub(delta[i], delta[j])), sub(korr[i], korr[j]));
  const double l = norm(d);
  const double wsum = w[i] + w[j] + alpha_h2;
  if (l < 1e-12 || wsum <= 0.0) return;
  const double dl = -(l - ruhe) / wsum;
  const V3 nrm = mul(d, 1.0 / l);
  korr[i] = add(korr[i], mul(nrm, w[i] * dl));
  korr[j] = sub(korr[j], mul(nrm, w[j] * dl));
}

// cpu.rs:312-335: C = theta - ruhe (wrapped), positions relative to the first
// point; corrects korr.
void xpbd_biegung(const std::vector<V3>& x, const std::vector<V3>& delta, std::vector<V3>& korr,
                  const std::vector<double>& w, std::array<uint32_t, 4> p, double ruhe, double alpha_h2) {
  const size_t p0 = p[0];
  std::array<V3, 4> q{};
  for (int k = 0; k < 4; ++k) {
    const size_t i = p[k];
    q[k] = add(add(sub(x[i], x[p0]), sub(delta[i], delta[p0])), sub(korr[i], korr[p0]));
  }
  double theta = 0.0;
  std::array<V3, 4> g{};
  if (!dieder(q, theta, g)) return;
  double nenner = alpha_h2;
  for (int k = 0; k < 4; ++k) nenner += w[p[k]] * dot(g[k], g[k]);
  if (nenner <= 0.0) return;
  const double dl = -winkel_fehler(theta, ruhe) / nenner;
  for (int k = 0; k < 4; ++k) korr[p[k]] = add(korr[p[k]], mul(g[k], w[p[k]] * dl));
}

namespace {
// The colour ranges of a constraint group; a scene handed over through the C
// ABI carries its constraints already in colour order (Szene::bauen sorts
// them, faerbung.rs:46-57) without the ranges, and one range over all of them
// visits them in the same order.
template <int N>
std::vector<std::pair<size_t, size_t>> bereiche(const Gruppe<N>& g) {
  if (!g.farben.empty()) return g.farben;
  return {{size_t(0), g.size()}};
}
}  // namespace

// cpu.rs:92-219: one substep of length h; s.x is the frame-start position.
void CpuReferenz::unterschritt(Szene& s, double h) {
  const size_t n = s.x.size();
  const V3 g = s.param.schwerkraft;
  const double daempf = std::max(1.0 - s.param.daempfung * h, 0.0);
  auto kante_membran = [&](size_t c) { return c < s.membran_kante.size() && s.membran_kante[c] != 0; };
  // load per point at the substep's start: edge tension and weight
  for (size_t i = 0; i < n; ++i) last[i] = mul(g, s.masse[i]);
  for (const auto& [f0, f1] : bereiche(s.abstand))
    for (size_t c = f0; c < f1; ++c) {
      if (kante_membran(c)) continue;
      const size_t i = s.abstand.punkte[c][0], j = s.abstand.punkte[c][1];
      const V3 d = add(sub(s.x[j], s.x[i]), sub(delta[j], delta[i]));
      const double l = norm(d);
      const double zug = std::max(l - s.abstand.ruhe[c], 0.0) / s.abstand.nachgiebigkeit[c];
      if (l > 1e-12 && zug > 0.0) {
        const V3 fij = mul(d, zug / l);
        last[i] = add(last[i], fij);
        last[j] = sub(last[j], fij);
      }
    }
  for (const MembranElement& m : s.membran_elemente) {
    std::array<V3, 3> p{};
    for (int k = 0; k < 3; ++k) {
      const size_t i = m.punkte[k];
      p[k] = add(add(s.x[i], delta[i]), korr[i]);
    }
    const auto fz = membran_krafte_zug(m.element, p);
    for (int k = 0; k < 3; ++k) last[m.punkte[k]] = add(last[m.punkte[k]], fz[k]);
  }
  // prediction
  for (size_t i = 0; i < n; ++i) {
    korr[i] = {0.0, 0.0, 0.0};
    if (s.w[i] > 0.0) {
      s.v[i] = mul(add(s.v[i], mul(g, h)), daempf);
      delta[i] = add(delta[i], mul(s.v[i], h));
    }
  }
  const double h2 = h * h;
  for (const auto& [f0, f1] : bereiche(s.abstand))
    for (size_t c = f0; c < f1; ++c) {
      if (kante_membran(c)) continue;
      xpbd_abstand(s.x, delta, korr, s.w, s.abstand.punkte[c], s.abstand.ruhe[c], s.abstand.nachgiebigkeit[c] / h2);
    }
  // membranes: three scalar constraints each, one triangle after the other
  for (const MembranElement& m : s.membran_elemente) {
    std::array<V3, 3> p{};
    for (int k = 0; k < 3; ++k) {
      const size_t i = m.punkte[k];
      p[k] = add(add(s.x[i], delta[i]), korr[i]);
    }
    for (const Zug& z : membran_zuege(m.element, p)) {
      if (!std::isfinite(z.alpha)) continue;
      double wsum = z.alpha / h2;
      for (int k = 0; k < 3; ++k) wsum += s.w[m.punkte[k]] * dot(z.grad[k], z.grad[k]);
      if (!(wsum > 0.0)) continue;
      const double dl = -z.c / wsum;
      for (int k = 0; k < 3; ++k) {
        const size_t i = m.punkte[k];
        korr[i] = add(korr[i], mul(z.grad[k], s.w[i] * dl));
      }
    }
  }
  for (const auto& [f0, f1] : bereiche(s.naht))
    for (size_t c = f0; c < f1; ++c)
      xpbd_abstand(s.x, delta, korr, s.w, s.naht.punkte[c], s.naht.ruhe[c], s.naht.nachgiebigkeit[c] / h2);
  for (const auto& [f0, f1] : bereiche(s.biegung))
    for (size_t c = f0; c < f1; ++c)
      xpbd_biegung(s.x, delta, korr, s.w, s.biegung.punkte[c], s.biegung.ruhe[c], s.biegung.nachgiebigkeit[c] / h2);
  // bodies with Coulomb friction as a position correction
  for (size_t i = 0; i < n; ++i) {
    if (s.w[i] <= 0.0) continue;
    for (const Koerper& k : s.koerper) {
      const V3 p = add(add(s.x[i], delta[i]), korr[i]);
      const auto kt = k.kontakt(p, s.kollisionsabstand[i]);
      if (!kt) continue;
      korr[i] = add(korr[i], mul(kt->normale, kt->tiefe));
      const V3 dx = sub(add(mul(s.v[i], h), korr[i]), mul(kt->geschwindigkeit, h));
      const V3 t = sub(dx, mul(kt->normale, dot(dx, kt->normale)));
      const double lt = norm(t);
      const double normallast = std::max(-dot(last[i], kt->normale), 0.0);
      const double grenze = s.reibung[i] * std::max(kt->tiefe, normallast * h2 * s.w[i]);
      statistik.kontakte += 1;
      statistik.tiefe += kt->tiefe;
      statistik.tangential += lt;
      if (lt <= grenze) {
        statistik.haftend += 1;
        korr[i] = sub(korr[i], t);
      } else if (lt > 0.0) {
        korr[i] = sub(korr[i], mul(t, grenze / lt));
      }
    }
  }
  for (size_t i = 0; i < n; ++i)
    if (s.w[i] > 0.0) {
      delta[i] = add(delta[i], korr[i]);
      s.v[i] = add(s.v[i], mul(korr[i], 1.0 / h));
    }
}

// cpu.rs:222-245: a frame of `unterschritte` substeps; the bodies are set
// from their frame-start positions at every substep.
void CpuReferenz::bild(Szene& s, size_t unterschritte) {
  const size_t n = std::max<size_t>(unterschritte, 1);
  const double h = s.param.bild_dt / double(n);
  const size_t np = s.x.size();
  statistik = Kontaktstatistik{};
  delta.assign(np, V3{0.0, 0.0, 0.0});
  korr.assign(np, V3{0.0, 0.0, 0.0});
  last.assign(np, V3{0.0, 0.0, 0.0});
  const std::vector<Koerper> anfang = s.koerper;
  for (size_t k = 0; k < n; ++k) {
    const double weg = double(k + 1) * h;
    for (size_t b = 0; b < s.koerper.size(); ++b) s.koerper[b] = anfang[b].verschoben(weg);
    unterschritt(s, h);
  }
  for (size_t i = 0; i < np; ++i) s.x[i] = add(s.x[i], delta[i]);
  s.zeit += s.param.bild_dt;
}

}  // namespace orc
