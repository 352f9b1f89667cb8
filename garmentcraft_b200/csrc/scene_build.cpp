// Scene builder: Szene::aus_netz (sim/src/szene.rs:284-292, 320-715) for a
// pattern given as pieces plus seam point pairs, without the folded allowance
// band. Edges are grouped by sorting (key, triangle order) instead of a
// search tree; the floating-point operations and their order are those of
// the reference, so masses, rest lengths, stiffnesses and membranes come out
// identical, and the greedy colouring (sim/src/faerbung.rs:11-57) gives the
// same constraint order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <unordered_map>
#include <vector>

#include "../../include/klon3d_step.h"
#include "scene_build.h"

namespace k3d {
namespace {

inline uint64_t key2(uint32_t a, uint32_t b) { return (uint64_t(std::min(a, b)) << 32) | std::max(a, b); }
inline double l2(const double* a, const double* b) {
  return std::sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]));
}
inline double area2(const double* a, const double* b, const double* c) {
  return 0.5 * ((b[0] - a[0]) * (c[1] - a[1]) - (c[0] - a[0]) * (b[1] - a[1]));
}

// biegung.rs:111-142
double bend_stiffness(double c2, double s2, double weft, double warp, double bias) {
  if (weft == warp && warp == bias) return weft;
  double d = warp * (c2 * c2) + weft * (s2 * s2) + (4.0 * bias - warp - weft) * (c2 * s2);
  if (d > 0.0) return d;
  return 1.0e-3 * std::fabs(std::min(std::min(weft, warp), bias));
}
// biegung.rs:156-173
bool grain_cos2_sin2(double ex0, double ey0, const double* warp, double& c2, double& s2) {
  double le = std::sqrt(ex0 * ex0 + ey0 * ey0);
  double lw = std::sqrt(warp[0] * warp[0] + warp[1] * warp[1]);
  if (!(le > 1e-12) || !(lw > 1e-12)) return false;
  double ex = ex0 / le, ey = ey0 / le, wx = warp[0] / lw, wy = warp[1] / lw;
  double ce = ex * wx + ey * wy, se = ex * wy - ey * wx;
  c2 = se * se;
  s2 = ce * ce;
  return true;
}

struct Membrane {
  double fl, ri[4], kette[2], schuss[2];
};
// kontinuum.rs:193-286 (rest triangle from eased edge lengths + material basis)
bool membrane_build(const double* p0, const double* p1, const double* kanten, const double* dir2, Membrane& m) {
  double l01 = kanten[0], l12 = kanten[1], l20 = kanten[2];
  if (!(l01 > 0.0 && l12 > 0.0 && l20 > 0.0)) return false;
  double x = (l01 * l01 + l20 * l20 - l12 * l12) / (2.0 * l01);
  double y2 = l20 * l20 - x * x;
  if (!(y2 > 0.0)) return false;
  double y = std::sqrt(y2);
  double det = l01 * y;
  if (!(det > 0.0)) return false;
  m.ri[0] = 1.0 / l01;
  m.ri[1] = -x / det;
  m.ri[2] = 0.0;
  m.ri[3] = 1.0 / y;
  m.fl = 0.5 * det;
  double dx = p1[0] - p0[0], dy = p1[1] - p0[1];
  double ld = std::sqrt(dx * dx + dy * dy + 0.0 * 0.0);
  if (!(ld > 0.0)) return false;
  double c = dx / ld, s = dy / ld;
  auto to_rest = [&](double vx, double vy, double* out) -> bool {
    double l = std::sqrt(vx * vx + vy * vy + 0.0 * 0.0);
    if (!(l > 0.0)) return false;
    double ux = vx / l, uy = vy / l;
    out[0] = c * ux + s * uy;
    out[1] = -s * ux + c * uy;
    return true;
  };
  double q[2];
  if (!to_rest(dir2[0], dir2[1], m.kette)) return false;
  if (!to_rest(-dir2[1], dir2[0], q)) return false;
  double along = q[0] * m.kette[0] + q[1] * m.kette[1];
  double wx = q[0] - along * m.kette[0], wy = q[1] - along * m.kette[1];
  double lw = std::sqrt(wx * wx + wy * wy + 0.0 * 0.0);
  if (!(lw > 1e-12)) return false;
  m.schuss[0] = wx / lw;
  m.schuss[1] = wy / lw;
  return true;
}

// faerbung.rs:11-57: greedy colouring in input order, then stable order by colour.
std::vector<uint32_t> colour_order(const uint32_t* pts, int width, size_t count, size_t npoints, size_t& ncolours) {
  std::vector<uint64_t> mask(npoints, 0);
  std::vector<std::vector<uint32_t>> more;
  std::vector<uint32_t> colour(count);
  ncolours = 0;
  for (size_t c = 0; c < count; ++c) {
    const uint32_t* p = pts + c * width;
    uint64_t used = 0;
    for (int k = 0; k < width; ++k) used |= mask[p[k]];
    uint32_t f;
    if (used != ~uint64_t(0)) {
      f = uint32_t(__builtin_ctzll(~used));
    } else {
      if (more.empty()) more.resize(npoints);
      for (f = 64;; ++f) {
        bool ok = true;
        for (int k = 0; k < width && ok; ++k)
          ok = std::find(more[p[k]].begin(), more[p[k]].end(), f) == more[p[k]].end();
        if (ok) break;
      }
    }
    for (int k = 0; k < width; ++k) {
      if (f < 64)
        mask[p[k]] |= uint64_t(1) << f;
      else
        more[p[k]].push_back(f);
    }
    colour[c] = f;
    ncolours = std::max(ncolours, size_t(f) + 1);
  }
  // counting sort by colour (stable)
  std::vector<size_t> start(ncolours + 1, 0);
  for (uint32_t f : colour) start[f + 1]++;
  for (size_t f = 0; f < ncolours; ++f) start[f + 1] += start[f];
  std::vector<uint32_t> order(count);
  for (size_t c = 0; c < count; ++c) order[start[colour[c]]++] = uint32_t(c);
  return order;
}

template <int W>
void apply_order(const std::vector<uint32_t>& order, std::vector<uint32_t>& pts, std::vector<double>& a,
                 std::vector<double>& b) {
  std::vector<uint32_t> p2(pts.size());
  std::vector<double> a2(a.size()), b2(b.size());
  for (size_t i = 0; i < order.size(); ++i) {
    for (int k = 0; k < W; ++k) p2[W * i + k] = pts[W * order[i] + k];
    a2[i] = a[order[i]];
    b2[i] = b[order[i]];
  }
  pts.swap(p2);
  a.swap(a2);
  b.swap(b2);
}

struct EdgeRec {
  uint64_t key;
  uint32_t tri;  // triangle order within the piece
  uint32_t opp;
  double area;
};

}  // namespace

k3d_status build_scene_impl(const k3d_pattern* pat, BuiltScene& S) {
  if (!pat || pat->n_teile < 0 || pat->n_naehte < 0) return K3D_BAD_ARGUMENT;
  const int np = pat->n_teile;
  std::vector<uint32_t> a_p, b_p;
  std::vector<double> a_r, a_a, b_r, b_a;
  std::vector<uint32_t> versatz(np);
  // per piece: boundary edge key -> (opposite point, area, index in a_r); every edge key -> index in a_r
  std::vector<std::unordered_map<uint64_t, std::pair<uint32_t, double>>> rand(np);
  std::vector<std::unordered_map<uint64_t, size_t>> rand_index(np), edge_index(np);
  std::vector<std::vector<double>> pts_m(np);
  struct TriRef {
    int piece;
    uint32_t d[3];
  };
  std::vector<TriRef> tris;

  for (int ti = 0; ti < np; ++ti) {
    const k3d_piece& t = pat->teile[ti];
    if (t.n_punkte < 0 || t.n_dreiecke < 0 || (t.n_punkte > 0 && (!t.punkte_mm || !t.lage)) ||
        (t.n_dreiecke > 0 && !t.dreiecke))
      return K3D_BAD_ARGUMENT;
    const k3d_material& mat = t.material;
    const double skala = 1.0 - t.reduktion;
    const uint32_t off = uint32_t(S.masse.size());
    versatz[ti] = off;
    // Teilinfo (szene.rs:483-489): point and triangle ranges, stretch stiffness
    S.teil_bereiche.insert(S.teil_bereiche.end(), {int64_t(off), int64_t(off) + t.n_punkte,
                                                   int64_t(S.dreiecke.size() / 3),
                                                   int64_t(S.dreiecke.size() / 3) + t.n_dreiecke});
    S.teil_dehnung.push_back(t.material.dehnung_n_m);
    S.teil_band_von.push_back(-1);
    std::vector<double>& pm = pts_m[ti];
    pm.resize(2 * size_t(t.n_punkte));
    for (int64_t i = 0; i < t.n_punkte; ++i) {
      pm[2 * i] = t.punkte_mm[2 * i] * 1e-3;
      pm[2 * i + 1] = t.punkte_mm[2 * i + 1] * 1e-3;
      for (int a = 0; a < 3; ++a) S.x.push_back(t.lage[3 * i + a]);
      S.masse.push_back(0.0);
      S.kabst.push_back(mat.dicke_m / 2.0);
      S.reib.push_back(mat.reibung);
    }
    std::vector<EdgeRec> edges;
    edges.reserve(3 * size_t(t.n_dreiecke));
    for (int64_t q = 0; q < t.n_dreiecke; ++q) {
      const uint32_t* d = t.dreiecke + 3 * q;
      for (int k = 0; k < 3; ++k)
        if (int64_t(d[k]) >= t.n_punkte) return K3D_BAD_ARGUMENT;
      const double *pa = &pm[2 * d[0]], *pb = &pm[2 * d[1]], *pc = &pm[2 * d[2]];
      double a = std::fabs(area2(pa, pb, pc));
      for (int k = 0; k < 3; ++k) S.masse[off + d[k]] += a * skala * skala * mat.flaechengewicht_kg_m2 / 3.0;
      for (int k = 0; k < 3; ++k) edges.push_back({key2(d[k], d[(k + 1) % 3]), uint32_t(q), d[(k + 2) % 3], a});
      // reduced rest matrix inverse (szene.rs:398-402)
      double qa[2] = {pa[0] * skala, pa[1] * skala}, qb[2] = {pb[0] * skala, pb[1] * skala},
             qc[2] = {pc[0] * skala, pc[1] * skala};
      double m00 = qb[0] - qa[0], m10 = qb[1] - qa[1], m01 = qc[0] - qa[0], m11 = qc[1] - qa[1];
      double det = m00 * m11 - m01 * m10;
      S.ruhe_inv.insert(S.ruhe_inv.end(), {m11 / det, -m01 / det, -m10 / det, m00 / det});
      for (int k = 0; k < 3; ++k) S.dreiecke.push_back(d[k] + off);
      tris.push_back({ti, {d[0], d[1], d[2]}});
    }
    std::stable_sort(edges.begin(), edges.end(), [](const EdgeRec& x, const EdgeRec& y) { return x.key < y.key; });
    for (size_t e0 = 0; e0 < edges.size();) {
      size_t e1 = e0;
      double asum = 0.0;
      while (e1 < edges.size() && edges[e1].key == edges[e0].key) asum += edges[e1++].area;
      const size_t cnt = e1 - e0;
      const uint32_t i = uint32_t(edges[e0].key >> 32), j = uint32_t(edges[e0].key & 0xffffffffu);
      if (cnt == 1) rand[ti][edges[e0].key] = {edges[e0].opp, asum};
      double l = l2(&pm[2 * i], &pm[2 * j]);
      if (l > 0.0) {
        double k = mat.dehnung_n_m * asum / (l * l);
        a_p.push_back(i + off);
        a_p.push_back(j + off);
        a_r.push_back(l * skala);
        a_a.push_back(1.0 / k);
        edge_index[ti][edges[e0].key] = a_r.size() - 1;
        if (cnt == 1) rand_index[ti][edges[e0].key] = a_r.size() - 1;
        if (cnt == 2) {
          uint32_t o1 = edges[e0].opp, o2 = edges[e0 + 1].opp;
          const double *pi = &pm[2 * i], *pj = &pm[2 * j];
          uint32_t oa = o1, ob = o2;
          if (!(area2(pi, pj, &pm[2 * o1]) > 0.0)) std::swap(oa, ob);
          double a12 = std::fabs(area2(pi, pj, &pm[2 * oa])) + std::fabs(area2(pj, pi, &pm[2 * ob]));
          double c2, s2, dd;
          if (grain_cos2_sin2(pj[0] - pi[0], pj[1] - pi[1], t.fadenlauf, c2, s2))
            dd = bend_stiffness(c2, s2, mat.biegung_nm, mat.biegung_kette_nm, mat.biegung_schraege_nm);
          else
            dd = mat.biegung_nm;
          double kb = dd * l * l / a12;
          b_p.insert(b_p.end(), {i + off, j + off, oa + off, ob + off});
          b_r.push_back(0.0);
          b_a.push_back(1.0 / kb);
        }
      }
      e0 = e1;
    }
  }

  // bending across seams (szene.rs:492-529)
  std::unordered_map<uint64_t, char> seam_edges;
  for (int n = 0; n < pat->n_naehte; ++n) {
    const k3d_seam& sm = pat->naehte[n];
    for (int q = 0; q < sm.n_teilnaehte; ++q) {
      const k3d_seam_part& tn = sm.teilnaehte[q];
      if (tn.teil_a < 0 || tn.teil_a >= np || tn.teil_b < 0 || tn.teil_b >= np) return K3D_BAD_ARGUMENT;
      const int ta = tn.teil_a, tb = tn.teil_b;
      for (int64_t w = 0; w + 1 < tn.n_paare; ++w) {
        uint32_t a0 = tn.paare[2 * w], a1 = tn.paare[2 * w + 2], b0 = tn.paare[2 * w + 1], b1 = tn.paare[2 * w + 3];
        auto ia = rand[ta].find(key2(a0, a1));
        auto ib = rand[tb].find(key2(b0, b1));
        if (ia == rand[ta].end() || ib == rand[tb].end()) continue;
        if (!seam_edges.emplace(key2(versatz[ta] + std::min(a0, a1), versatz[ta] + std::max(a0, a1)), 1).second)
          continue;
        const uint32_t oa = ia->second.first, ob = ib->second.first;
        const double fa = ia->second.second, fb = ib->second.second;
        const std::vector<double>&pa = pts_m[ta], &pb = pts_m[tb];
        uint32_t x0a = a0, x1a = a1, x0b = b0, x1b = b1;
        if (!(area2(&pa[2 * a0], &pa[2 * a1], &pa[2 * oa]) > 0.0)) {
          x0a = a1;
          x1a = a0;
          x0b = b1;
          x1b = b0;
        }
        if (area2(&pb[2 * x1b], &pb[2 * x0b], &pb[2 * ob]) <= 0.0) {
          S.naht_biegung_ohne++;
          continue;
        }
        double l = l2(&pa[2 * a0], &pa[2 * a1]);
        const double ba = pat->teile[ta].material.biegung_nm, bbv = pat->teile[tb].material.biegung_nm;
        double kb = 0.5 * (ba + bbv) * l * l / (fa + fb);
        b_p.insert(b_p.end(), {x0a + versatz[ta], x1a + versatz[ta], oa + versatz[ta], ob + versatz[tb]});
        b_r.push_back(0.0);
        b_a.push_back(1.0 / kb);
      }
    }
  }

  // seam pairs, sorted and unique (szene.rs:531-544)
  std::vector<uint64_t> pairs;
  for (int n = 0; n < pat->n_naehte; ++n) {
    const k3d_seam& sm = pat->naehte[n];
    for (int q = 0; q < sm.n_teilnaehte; ++q) {
      const k3d_seam_part& tn = sm.teilnaehte[q];
      for (int64_t w = 0; w < tn.n_paare; ++w) {
        uint32_t a = versatz[tn.teil_a] + tn.paare[2 * w], b = versatz[tn.teil_b] + tn.paare[2 * w + 1];
        if (a != b) pairs.push_back(key2(a, b));
      }
    }
  }
  std::sort(pairs.begin(), pairs.end());
  pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
  std::vector<uint32_t> n_p;
  for (uint64_t k : pairs) {
    n_p.push_back(uint32_t(k >> 32));
    n_p.push_back(uint32_t(k & 0xffffffffu));
  }
  std::vector<double> n_r(pairs.size(), 0.0), n_a(pairs.size(), pat->naht_nachgiebigkeit);

  // ease (szene.rs:556-592)
  if (pat->einhalteweite) {
    std::unordered_map<size_t, char> set;
    for (int n = 0; n < pat->n_naehte; ++n) {
      const k3d_seam& sm = pat->naehte[n];
      double la = sm.laenge_a_mm, lb = sm.laenge_b_mm;
      if (!(la > 0.0 && lb > 0.0)) continue;
      double f = std::min(la, lb) / std::max(la, lb);
      if (f >= 1.0 - 1e-9) continue;
      const int lang = la > lb ? 0 : 1;
      for (int q = 0; q < sm.n_teilnaehte; ++q) {
        const k3d_seam_part& tn = sm.teilnaehte[q];
        const auto& index = rand_index[lang == 0 ? tn.teil_a : tn.teil_b];
        for (int64_t w = 0; w + 1 < tn.n_paare; ++w) {
          uint32_t p0 = tn.paare[2 * w + lang], p1 = tn.paare[2 * w + 2 + lang];
          if (p0 == p1) continue;
          auto it = index.find(key2(p0, p1));
          if (it == index.end()) continue;
          if (set.emplace(it->second, 1).second) {
            a_r[it->second] *= f;
            S.einhalte_kanten++;
          }
        }
      }
    }
  }

  // membranes (szene.rs:602-647)
  std::vector<uint8_t> mkante(a_r.size(), 0);
  for (size_t q = 0; q < tris.size(); ++q) {
    const TriRef& tr = tris[q];
    const k3d_piece& t = pat->teile[tr.piece];
    const auto& index = edge_index[tr.piece];
    const uint64_t ks[3] = {key2(tr.d[0], tr.d[1]), key2(tr.d[1], tr.d[2]), key2(tr.d[2], tr.d[0])};
    double kl[3] = {0, 0, 0};
    bool full = true;
    for (int k = 0; k < 3; ++k) {
      auto it = index.find(ks[k]);
      if (it != index.end())
        kl[k] = a_r[it->second];
      else
        full = false;
    }
    Membrane m;
    const std::vector<double>& pm = pts_m[tr.piece];
    if (full && membrane_build(&pm[2 * tr.d[0]], &pm[2 * tr.d[1]], kl, t.fadenlauf, m)) {
      for (int k = 0; k < 3; ++k) {
        auto it = index.find(ks[k]);
        if (it != index.end()) mkante[it->second] = 1;
      }
      const uint32_t off = versatz[tr.piece];
      for (int k = 0; k < 3; ++k) S.m_punkte.push_back(tr.d[k] + off);
      S.m_flaeche.push_back(m.fl);
      S.m_ruhe_inv.insert(S.m_ruhe_inv.end(), {m.ri[0], m.ri[1], m.ri[2], m.ri[3]});
      S.m_kette.insert(S.m_kette.end(), {m.kette[0], m.kette[1]});
      S.m_schuss.insert(S.m_schuss.end(), {m.schuss[0], m.schuss[1]});
      S.m_steif.insert(S.m_steif.end(), {t.material.kette_n_m, t.material.dehnung_n_m, t.material.schub_n_m});
    } else {
      S.membran_entartet++;
    }
  }

  // colour order (szene.rs:681-694)
  const size_t npts = S.masse.size();
  S.w.resize(npts);
  for (size_t i = 0; i < npts; ++i) S.w[i] = S.masse[i] > 0.0 ? 1.0 / S.masse[i] : 0.0;
  size_t nc = 0;
  {
    auto ord = colour_order(a_p.data(), 2, a_r.size(), npts, nc);
    std::vector<uint8_t> mk2(mkante.size());
    for (size_t i = 0; i < ord.size(); ++i) mk2[i] = mkante[ord[i]];
    mkante.swap(mk2);
    apply_order<2>(ord, a_p, a_r, a_a);
    S.farben[0] = nc;
  }
  {
    auto ord = colour_order(b_p.data(), 4, b_r.size(), npts, nc);
    apply_order<4>(ord, b_p, b_r, b_a);
    S.farben[1] = nc;
  }
  {
    auto ord = colour_order(n_p.data(), 2, n_r.size(), npts, nc);
    apply_order<2>(ord, n_p, n_r, n_a);
    S.farben[2] = nc;
  }
  S.a_p.swap(a_p);
  S.a_r.swap(a_r);
  S.a_a.swap(a_a);
  S.mkante.swap(mkante);
  S.b_p.swap(b_p);
  S.b_r.swap(b_r);
  S.b_a.swap(b_a);
  S.n_p.swap(n_p);
  S.n_r.swap(n_r);
  S.v.assign(3 * npts, 0.0);
  S.param = pat->param;
  return K3D_OK;
}

void built_scene_view(BuiltScene& S, k3d_scene* o) {
  std::memset(o, 0, sizeof(*o));
  o->n_punkte = int64_t(S.masse.size());
  o->x = S.x.data();
  o->v = S.v.data();
  o->masse = S.masse.data();
  o->w = S.w.data();
  o->kollisionsabstand = S.kabst.data();
  o->reibung = S.reib.data();
  o->n_abstand = int64_t(S.a_r.size());
  o->abstand_punkte = S.a_p.data();
  o->abstand_ruhe = S.a_r.data();
  o->abstand_nachgiebigkeit = S.a_a.data();
  o->membran_kante = S.mkante.data();
  o->n_naht = int64_t(S.n_r.size());
  o->naht_punkte = S.n_p.data();
  o->naht_ruhe = S.n_r.data();
  o->n_biegung = int64_t(S.b_r.size());
  o->biegung_punkte = S.b_p.data();
  o->biegung_ruhe = S.b_r.data();
  o->biegung_nachgiebigkeit = S.b_a.data();
  o->n_membran = int64_t(S.m_flaeche.size());
  o->membran_punkte = S.m_punkte.data();
  o->membran_flaeche = S.m_flaeche.data();
  o->membran_ruhe_inv = S.m_ruhe_inv.data();
  o->membran_kette = S.m_kette.data();
  o->membran_schuss = S.m_schuss.data();
  o->membran_steif = S.m_steif.data();
  o->n_dreiecke = int64_t(S.dreiecke.size() / 3);
  o->dreiecke = S.dreiecke.data();
  o->ruhe_inv = S.ruhe_inv.data();
  o->param = S.param;
  o->n_teile = int64_t(S.teil_dehnung.size());
  o->teil_bereiche = S.teil_bereiche.data();
  o->teil_dehnung = S.teil_dehnung.data();
  o->teil_band_von = S.teil_band_von.data();
}

}  // namespace k3d
