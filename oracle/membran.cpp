// ORACLE (test infrastructure). Restatement of the orthotropic StVK membrane
// of sim/src/kontinuum.rs in FP64, same operation order as the reference.
#include <limits>
#include "oracle.hpp"

namespace orc {
namespace {

// kontinuum.rs:143-150  a(w), c(w, v) Voigt rows
V3 a3(V2 w) { return {w[0] * w[0], w[1] * w[1], w[0] * w[1]}; }
V3 c3(V2 w, V2 v) { return {w[0] * v[0], w[1] * v[1], 0.5 * (w[0] * v[1] + w[1] * v[0])}; }

struct Basis {
  V3 a, b, c;
};
// kontinuum.rs:292-298
Basis basis(const Membran& m) { return {a3(m.kette), a3(m.schuss), c3(m.kette, m.schuss)}; }
// kontinuum.rs:302-312
V3 c1(const Membran& m) {
  const auto& r = m.ruhe_inv;
  return {-(r[0] + r[2]), r[0], r[2]};
}
V3 c2(const Membran& m) {
  const auto& r = m.ruhe_inv;
  return {-(r[1] + r[3]), r[1], r[3]};
}
// kontinuum.rs:326-328
V3 g_aus(V3 f1, V3 f2) { return {dot(f1, f1), dot(f2, f2), 2.0 * dot(f1, f2)}; }
// kontinuum.rs:338-346
V3 dehnung_aus(const Membran& m, V3 f1, V3 f2) {
  Basis B = basis(m);
  V3 g = g_aus(f1, f2);
  return {0.5 * (dot(B.a, g) - 1.0), 0.5 * (dot(B.b, g) - 1.0), 0.5 * dot(B.c, g)};
}
// kontinuum.rs:376-386
V3 dU_dg_aus(const Membran& m, V3 e) {
  Basis B = basis(m);
  V3 out{};
  for (int i = 0; i < 3; ++i)
    out[i] = m.flaeche * (0.5 * m.kette_n_m * e[0] * B.a[i] + 0.5 * m.dehnung_n_m * e[1] * B.b[i] +
                          2.0 * m.schub_n_m * e[2] * B.c[i]);
  return out;
}
// kontinuum.rs:391-406
M3 kg_aus_basis(const Membran& m) {
  Basis B = basis(m);
  M3 out{};
  const std::array<std::pair<double, V3>, 3> terms = {
      std::make_pair(0.25 * m.kette_n_m, B.a), std::make_pair(0.25 * m.dehnung_n_m, B.b),
      std::make_pair(m.schub_n_m, B.c)};
  for (const auto& [wt, v] : terms)
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 3; ++k) out[i][k] += m.flaeche * wt * v[i] * v[k];
  return out;
}
// kontinuum.rs:421-435
V3 kg_mal(const Membran& m, V3 q) {
  Basis B = basis(m);
  V3 w{};
  const std::array<std::pair<double, V3>, 3> terms = {
      std::make_pair(0.25 * m.kette_n_m, B.a), std::make_pair(0.25 * m.dehnung_n_m, B.b),
      std::make_pair(m.schub_n_m, B.c)};
  for (const auto& [s, v] : terms) {
    double t = m.flaeche * s * dot(v, q);
    for (int i = 0; i < 3; ++i) w[i] += t * v[i];
  }
  return w;
}
using J3 = std::array<M3, 3>;  // J[k][row][col]
// kontinuum.rs:446-472
J3 jacobi_aus(const Membran& m, V3 f1, V3 f2) {
  const auto& r = m.ruhe_inv;
  auto zeile = [&](double a, double b) -> V3 {
    return {a * f1[0] + b * f2[0], a * f1[1] + b * f2[1], a * f1[2] + b * f2[2]};
  };
  M3 j1 = {zeile(2.0 * r[0], 0.0), zeile(0.0, 2.0 * r[1]), zeile(2.0 * r[1], 2.0 * r[0])};
  M3 j2 = {zeile(2.0 * r[2], 0.0), zeile(0.0, 2.0 * r[3]), zeile(2.0 * r[3], 2.0 * r[2])};
  M3 j0{};
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) j0[i][k] = -(j1[i][k] + j2[i][k]);
  return {j0, j1, j2};
}
// kontinuum.rs:504-520
std::array<V3, 3> kraefte_aus(const Membran& m, const std::array<V3, 3>& p, V3 d) {
  V3 f1, f2;
  membran_f(m, p, f1, f2);
  V3 k1 = c1(m), k2 = c2(m);
  std::array<V3, 3> out{};
  for (int k = 0; k < 3; ++k) {
    double s1 = 2.0 * (d[0] * k1[k] + d[2] * k2[k]);
    double s2 = 2.0 * (d[1] * k2[k] + d[2] * k1[k]);
    out[k] = {-(s1 * f1[0] + s2 * f2[0]), -(s1 * f1[1] + s2 * f2[1]), -(s1 * f1[2] + s2 * f2[2])};
  }
  return out;
}
// kontinuum.rs:584-591
V3 geo_w_aus(const Membran& m, V3 f1, V3 f2) {
  V3 e = dehnung_aus(m, f1, f2);
  V3 d = dU_dg_aus(m, {std::max(e[0], 0.0), std::max(e[1], 0.0), e[2]});
  return psd2(d[0], d[1], d[2]);
}
// kontinuum.rs:193-216
bool rest_aus_kanten(V3 kanten, std::array<double, 4>& inv, double& flaeche) {
  double l01 = kanten[0], l12 = kanten[1], l20 = kanten[2];
  if (!(l01 > 0.0 && l12 > 0.0 && l20 > 0.0)) return false;
  double x = (l01 * l01 + l20 * l20 - l12 * l12) / (2.0 * l01);
  double y2 = l20 * l20 - x * x;
  if (!(y2 > 0.0)) return false;
  double y = std::sqrt(y2);
  double det = l01 * y;
  if (!(det > 0.0)) return false;
  inv = {1.0 / l01, -x / det, 0.0, 1.0 / y};
  flaeche = 0.5 * det;
  return true;
}

}  // namespace

// kontinuum.rs:158-177
V3 psd2(double a, double b, double c) {
  double m = 0.5 * (a + b);
  double d = 0.5 * (a - b);
  double r = std::sqrt(d * d + c * c);
  if (m - r >= 0.0) return {a, b, c};
  double l_max = m + r;
  if (!(l_max > 0.0)) return {0.0, 0.0, 0.0};
  double u0 = l_max - b, u1 = c;
  double n2 = u0 * u0 + u1 * u1;
  if (!(n2 > 0.0)) return {0.0, 0.0, 0.0};
  double f = l_max / n2;
  return {f * u0 * u0, f * u1 * u1, f * u0 * u1};
}

// kontinuum.rs:229-286
std::optional<Membran> membran_bauen(std::array<V2, 3> ruhe, V3 kanten, V2 dir2, V3 material) {
  Membran m;
  if (!rest_aus_kanten(kanten, m.ruhe_inv, m.flaeche)) return std::nullopt;
  V3 d01 = sub({ruhe[1][0], ruhe[1][1], 0.0}, {ruhe[0][0], ruhe[0][1], 0.0});
  double l01 = norm(d01);
  if (!(l01 > 0.0)) return std::nullopt;
  double c = d01[0] / l01, s = d01[1] / l01;
  auto dreh = [&](V2 v) -> V2 { return {c * v[0] + s * v[1], -s * v[0] + c * v[1]}; };
  auto nach_ruhe = [&](V2 v, V2& out) -> bool {
    double l = norm({v[0], v[1], 0.0});
    if (l > 0.0) {
      out = dreh({v[0] / l, v[1] / l});
      return true;
    }
    return false;
  };
  V2 kette, q;
  if (!nach_ruhe(dir2, kette)) return std::nullopt;
  if (!nach_ruhe({-dir2[1], dir2[0]}, q)) return std::nullopt;
  double along = q[0] * kette[0] + q[1] * kette[1];
  V2 w = {q[0] - along * kette[0], q[1] - along * kette[1]};
  double lw = norm({w[0], w[1], 0.0});
  if (!(lw > 1e-12)) return std::nullopt;
  m.kette = kette;
  m.schuss = {w[0] / lw, w[1] / lw};
  m.kette_n_m = material[0];
  m.dehnung_n_m = material[1];
  m.schub_n_m = material[2];
  return m;
}

// kontinuum.rs:315-322
void membran_f(const Membran& m, const std::array<V3, 3>& p, V3& f1, V3& f2) {
  V3 e1 = sub(p[1], p[0]), e2 = sub(p[2], p[0]);
  const auto& r = m.ruhe_inv;
  f1 = add(mul(e1, r[0]), mul(e2, r[2]));
  f2 = add(mul(e1, r[1]), mul(e2, r[3]));
}
// kontinuum.rs:331-334
V3 membran_dehnung(const Membran& m, const std::array<V3, 3>& p) {
  V3 f1, f2;
  membran_f(m, p, f1, f2);
  return dehnung_aus(m, f1, f2);
}
// kontinuum.rs:351-358
V3 membran_spannung(const Membran& m, const std::array<V3, 3>& p) {
  V3 e = membran_dehnung(m, p);
  return {m.kette_n_m * e[0], m.dehnung_n_m * e[1], 2.0 * m.schub_n_m * e[2]};
}
// kontinuum.rs:361-367
double membran_energie(const Membran& m, const std::array<V3, 3>& p) {
  V3 e = membran_dehnung(m, p);
  return m.flaeche * (0.5 * m.kette_n_m * e[0] * e[0] + 0.5 * m.dehnung_n_m * e[1] * e[1] +
                      2.0 * m.schub_n_m * e[2] * e[2]);
}
// kontinuum.rs:475-478
std::array<V3, 3> membran_krafte(const Membran& m, const std::array<V3, 3>& p) {
  V3 d = dU_dg_aus(m, membran_dehnung(m, p));
  return kraefte_aus(m, p, d);
}
// kontinuum.rs:484-495
std::array<V3, 3> membran_krafte_zug(const Membran& m, const std::array<V3, 3>& p) {
  V3 e = membran_dehnung(m, p);
  Basis B = basis(m);
  V3 d{};
  for (int i = 0; i < 3; ++i)
    d[i] = m.flaeche * (0.5 * m.kette_n_m * std::max(e[0], 0.0) * B.a[i] +
                        0.5 * m.dehnung_n_m * std::max(e[1], 0.0) * B.b[i] +
                        2.0 * m.schub_n_m * e[2] * B.c[i]);
  return kraefte_aus(m, p, d);
}
// kontinuum.rs:608-612
Hessen membran_hessen(const Membran& m, const std::array<V3, 3>& p) {
  Hessen h;
  membran_f(m, p, h.f1, h.f2);
  h.w = geo_w_aus(m, h.f1, h.f2);
  return h;
}
// kontinuum.rs:616-664
std::array<V3, 3> membran_mal_h_aus(const Membran& m, const Hessen& h, const std::array<V3, 3>& delta) {
  const V3& f1 = h.f1;
  const V3& f2 = h.f2;
  V3 k1 = c1(m), k2 = c2(m);
  V3 q{};
  for (int l = 0; l < 3; ++l) {
    double d1 = dot(f1, delta[l]), d2 = dot(f2, delta[l]);
    q[0] += 2.0 * k1[l] * d1;
    q[1] += 2.0 * k2[l] * d2;
    q[2] += 2.0 * (k2[l] * d1 + k1[l] * d2);
  }
  V3 w = kg_mal(m, q);
  std::array<V3, 3> out{};
  for (int k = 0; k < 3; ++k) {
    double s1 = 2.0 * (k1[k] * w[0] + k2[k] * w[2]);
    double s2 = 2.0 * (k2[k] * w[1] + k1[k] * w[2]);
    out[k] = {s1 * f1[0] + s2 * f2[0], s1 * f1[1] + s2 * f2[1], s1 * f1[2] + s2 * f2[2]};
  }
  double w11 = h.w[0], w22 = h.w[1], w12 = h.w[2];
  V3 t1{}, t2{};
  for (int b = 0; b < 3; ++b)
    for (int c = 0; c < 3; ++c) {
      t1[c] += k1[b] * delta[b][c];
      t2[c] += k2[b] * delta[b][c];
    }
  for (int a = 0; a < 3; ++a) {
    double pa = 2.0 * (w11 * k1[a] + w12 * k2[a]);
    double qa = 2.0 * (w12 * k1[a] + w22 * k2[a]);
    for (int c = 0; c < 3; ++c) out[a][c] += pa * t1[c] + qa * t2[c];
  }
  return out;
}
// kontinuum.rs:675-708
std::array<M3, 3> membran_diag_bloecke_aus(const Membran& m, const Hessen& h) {
  J3 j = jacobi_aus(m, h.f1, h.f2);
  M3 kg = kg_aus_basis(m);
  std::array<M3, 3> out{};
  for (int k = 0; k < 3; ++k) {
    M3 tmp{};
    for (int i = 0; i < 3; ++i)
      for (int c = 0; c < 3; ++c)
        for (int mm = 0; mm < 3; ++mm) tmp[i][c] += kg[i][mm] * j[k][mm][c];
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c)
        for (int i = 0; i < 3; ++i) out[k][a][c] += j[k][i][a] * tmp[i][c];
  }
  double w11 = h.w[0], w22 = h.w[1], w12 = h.w[2];
  V3 k1 = c1(m), k2 = c2(m);
  for (int k = 0; k < 3; ++k) {
    double s = 2.0 * (w11 * k1[k] * k1[k] + w22 * k2[k] * k2[k] + 2.0 * w12 * k1[k] * k2[k]);
    for (int c = 0; c < 3; ++c) out[k][c][c] += s;
  }
  return out;
}

// kontinuum.rs:526-551: warp strain, weft strain and the engineering shear
// angle 2*e_ks, each with its gradient per point and its compliance
// 1 / (k * area) (infinite when the stiffness or the area is not positive).
std::array<Zug, 3> membran_zuege(const Membran& m, const std::array<V3, 3>& p) {
  V3 f1, f2;
  membran_f(m, p, f1, f2);
  const V3 e = membran_dehnung(m, p);
  const J3 j = jacobi_aus(m, f1, f2);
  const Basis B = basis(m);
  auto grad = [&](const V3& v, bool halb) {
    std::array<V3, 3> g{};
    for (int k = 0; k < 3; ++k)
      for (int col = 0; col < 3; ++col) {
        double s = 0.0;
        for (int i = 0; i < 3; ++i) s += j[k][i][col] * v[i];
        g[k][col] = halb ? 0.5 * s : s;
      }
    return g;
  };
  const double fl = m.flaeche;
  auto alpha = [&](double k) {
    return (k > 0.0 && fl > 0.0) ? 1.0 / (k * fl) : std::numeric_limits<double>::infinity();
  };
  return {Zug{e[0], grad(B.a, true), alpha(m.kette_n_m)}, Zug{e[1], grad(B.b, true), alpha(m.dehnung_n_m)},
          Zug{2.0 * e[2], grad(B.c, false), alpha(m.schub_n_m)}};
}

}  // namespace orc
