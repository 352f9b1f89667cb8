// ORACLE (test infrastructure). Flat C entry points over the FP64
// restatement, for tests/ and the CPU-baseline leg of bench.py (ctypes). The
// scene and parameter structs reuse the public ABI layouts of
// include/klon3d_step.h so both sides read the same inputs.
#include <algorithm>
#include <cstring>
#include <memory>
#include <string>

#include "../include/klon3d_step.h"
#include "oracle.hpp"

using namespace orc;

namespace {

Material mat_aus(const k3d_material& m) {
  Material o;
  o.dehnung_n_m = m.dehnung_n_m;
  o.kette_n_m = m.kette_n_m;
  o.schub_n_m = m.schub_n_m;
  o.biegung_nm = m.biegung_nm;
  o.biegung_kette_nm = m.biegung_kette_nm;
  o.biegung_schraege_nm = m.biegung_schraege_nm;
  o.flaechengewicht_kg_m2 = m.flaechengewicht_kg_m2;
  o.dicke_m = m.dicke_m;
  o.reibung = m.reibung;
  return o;
}

struct Koerperdaten {
  std::vector<Koerper> koerper;
  std::vector<std::vector<float>> gitter;
};

Koerperdaten koerper_aus(const k3d_body* kb, int32_t n) {
  Koerperdaten out;
  out.gitter.resize(n);
  for (int32_t b = 0; b < n; ++b) {
    const k3d_body& s = kb[b];
    Koerper k;
    k.art = s.art;
    for (int a = 0; a < 3; ++a) {
      k.punkt[a] = s.punkt[a];
      k.achse[a] = s.achse[a];
      k.geschwindigkeit[a] = s.geschwindigkeit[a];
      k.ursprung[a] = s.ursprung[a];
      k.dims[a] = s.dims[a];
    }
    k.radius = s.radius;
    k.spacing = s.spacing;
    // the oracle's mesh bodies carry an oracle Koerpernetz (orc_netz_neu) in `netz`
    if (s.art == K3D_BODY_MESH) k.netz = reinterpret_cast<const Koerpernetz*>(s.netz);
    if (s.art == K3D_BODY_SDF_GRID && s.sdf) {
      size_t nn = size_t(s.dims[0]) * size_t(s.dims[1]) * size_t(s.dims[2]);
      out.gitter[b].assign(s.sdf, s.sdf + nn);
    }
    out.koerper.push_back(k);
  }
  for (int32_t b = 0; b < n; ++b)
    if (!out.gitter[b].empty()) out.koerper[b].sdf = out.gitter[b].data();
  return out;
}

Simparameter sim_aus(const k3d_simparams& p) {
  Simparameter o;
  o.bild_dt = p.bild_dt;
  for (int a = 0; a < 3; ++a) o.schwerkraft[a] = p.schwerkraft[a];
  o.daempfung = p.daempfung;
  return o;
}

struct Gebaut {
  Szene s;
  // flat copies for the k3d_scene view
  std::vector<double> x, v, ruhe_a, alpha_a, ruhe_n, ruhe_b, alpha_b, m_fl, m_ri, m_k, m_s, m_st, ri;
  std::vector<uint32_t> p_a, p_n, p_b, p_m, dr;
  std::vector<uint8_t> mk;
  void flach() {
    auto v3 = [](const std::vector<V3>& a) {
      std::vector<double> o;
      for (auto& q : a) o.insert(o.end(), q.begin(), q.end());
      return o;
    };
    x = v3(s.x);
    v = v3(s.v);
    for (auto& p : s.abstand.punkte) p_a.insert(p_a.end(), p.begin(), p.end());
    ruhe_a = s.abstand.ruhe;
    alpha_a = s.abstand.nachgiebigkeit;
    mk = s.membran_kante;
    for (auto& p : s.naht.punkte) p_n.insert(p_n.end(), p.begin(), p.end());
    ruhe_n = s.naht.ruhe;
    for (auto& p : s.biegung.punkte) p_b.insert(p_b.end(), p.begin(), p.end());
    ruhe_b = s.biegung.ruhe;
    alpha_b = s.biegung.nachgiebigkeit;
    for (auto& m : s.membran_elemente) {
      p_m.insert(p_m.end(), m.punkte.begin(), m.punkte.end());
      m_fl.push_back(m.element.flaeche);
      m_ri.insert(m_ri.end(), m.element.ruhe_inv.begin(), m.element.ruhe_inv.end());
      m_k.insert(m_k.end(), m.element.kette.begin(), m.element.kette.end());
      m_s.insert(m_s.end(), m.element.schuss.begin(), m.element.schuss.end());
      m_st.push_back(m.element.kette_n_m);
      m_st.push_back(m.element.dehnung_n_m);
      m_st.push_back(m.element.schub_n_m);
    }
    for (auto& d : s.dreiecke) dr.insert(dr.end(), d.begin(), d.end());
    for (auto& r : s.ruhe_inv) ri.insert(ri.end(), r.begin(), r.end());
    for (auto& t : s.teile) {
      tb.insert(tb.end(), {int64_t(t.p0), int64_t(t.p1), int64_t(t.d0), int64_t(t.d1)});
      te.push_back(t.dehnung_n_m);
      tv.push_back(int32_t(t.band_von));
    }
  }
  std::vector<int64_t> tb;
  std::vector<double> te;
  std::vector<int32_t> tv;
};

Szene szene_aus(const k3d_scene* k, Koerperdaten& kd) {
  Szene s;
  size_t n = size_t(k->n_punkte);
  s.x.resize(n);
  s.v.resize(n);
  for (size_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      s.x[i][a] = k->x[3 * i + a];
      s.v[i][a] = k->v[3 * i + a];
    }
  s.masse.assign(k->masse, k->masse + n);
  s.w.assign(k->w, k->w + n);
  s.kollisionsabstand.assign(k->kollisionsabstand, k->kollisionsabstand + n);
  s.reibung.assign(k->reibung, k->reibung + n);
  for (int64_t e = 0; e < k->n_abstand; ++e) {
    s.abstand.punkte.push_back({k->abstand_punkte[2 * e], k->abstand_punkte[2 * e + 1]});
    s.abstand.ruhe.push_back(k->abstand_ruhe[e]);
    s.abstand.nachgiebigkeit.push_back(k->abstand_nachgiebigkeit[e]);
    s.membran_kante.push_back(k->membran_kante ? k->membran_kante[e] : 0);
  }
  for (int64_t e = 0; e < k->n_naht; ++e) {
    s.naht.punkte.push_back({k->naht_punkte[2 * e], k->naht_punkte[2 * e + 1]});
    s.naht.ruhe.push_back(k->naht_ruhe[e]);
    s.naht.nachgiebigkeit.push_back(0.0);
  }
  for (int64_t e = 0; e < k->n_biegung; ++e) {
    s.biegung.punkte.push_back({k->biegung_punkte[4 * e], k->biegung_punkte[4 * e + 1], k->biegung_punkte[4 * e + 2],
                                k->biegung_punkte[4 * e + 3]});
    s.biegung.ruhe.push_back(k->biegung_ruhe[e]);
    s.biegung.nachgiebigkeit.push_back(k->biegung_nachgiebigkeit[e]);
  }
  for (int64_t t = 0; t < k->n_membran; ++t) {
    MembranElement m;
    for (int a = 0; a < 3; ++a) m.punkte[a] = k->membran_punkte[3 * t + a];
    m.element.flaeche = k->membran_flaeche[t];
    for (int a = 0; a < 4; ++a) m.element.ruhe_inv[a] = k->membran_ruhe_inv[4 * t + a];
    for (int a = 0; a < 2; ++a) {
      m.element.kette[a] = k->membran_kette[2 * t + a];
      m.element.schuss[a] = k->membran_schuss[2 * t + a];
    }
    m.element.kette_n_m = k->membran_steif[3 * t];
    m.element.dehnung_n_m = k->membran_steif[3 * t + 1];
    m.element.schub_n_m = k->membran_steif[3 * t + 2];
    s.membran_elemente.push_back(m);
  }
  for (int64_t t = 0; t < k->n_dreiecke; ++t) {
    s.dreiecke.push_back({k->dreiecke[3 * t], k->dreiecke[3 * t + 1], k->dreiecke[3 * t + 2]});
    s.ruhe_inv.push_back({k->ruhe_inv[4 * t], k->ruhe_inv[4 * t + 1], k->ruhe_inv[4 * t + 2], k->ruhe_inv[4 * t + 3]});
  }
  for (int64_t t = 0; t < k->n_teile; ++t) {
    Teilinfo ti;
    ti.p0 = size_t(k->teil_bereiche[4 * t]);
    ti.p1 = size_t(k->teil_bereiche[4 * t + 1]);
    ti.d0 = size_t(k->teil_bereiche[4 * t + 2]);
    ti.d1 = size_t(k->teil_bereiche[4 * t + 3]);
    ti.dehnung_n_m = k->teil_dehnung[t];
    ti.band_von = k->teil_band_von ? k->teil_band_von[t] : -1;
    s.teile.push_back(ti);
  }
  kd = koerper_aus(k->koerper, k->n_koerper);
  s.koerper = kd.koerper;
  s.param = sim_aus(k->param);
  s.zeit = k->zeit;
  return s;
}

ImplizitParameter param_aus(const k3d_params* p) {
  ImplizitParameter o;
  o.schritte_je_bild = size_t(p->schritte_je_bild);
  o.cg_max = size_t(p->cg_max);
  o.cg_toleranz = p->cg_toleranz;
  o.naht_k = p->naht_k;
  o.kontakt_rand = p->kontakt_rand;
  o.normalkraft_aus_last = p->normalkraft_aus_last != 0;
  o.durchstoss_pruefen = p->durchstoss_pruefen != 0;
  o.selbstkollision = p->selbstkollision != 0;
  o.selbst_zusatzdicke = p->selbst_zusatzdicke;
  o.selbst_steifigkeit = p->selbst_steifigkeit;
  o.selbst_stoss_iterationen = size_t(std::max(p->selbst_stoss_iterationen, 0));
  o.selbst_schnitte_an_naehten = p->selbst_schnitte_an_naehten != 0;
  o.koerperpunkt_durchgaenge = size_t(std::max(p->koerperpunkt_durchgaenge, 0));
  o.koerperpunkt_tiefe = p->koerperpunkt_tiefe;
  return o;
}

struct Sim {
  Szene s;
  Koerperdaten kd;
  ImplizitCg cg;
  CpuReferenz xpbd;  // the XPBD cross-check on the same scene (cpu.rs)
};

void stats_aus(const ImplizitStatistik& st, k3d_stats* out) {
  if (!out) return;
  std::memset(out, 0, sizeof(*out));
  out->cg_iterationen = int64_t(st.cg_iterationen);
  out->loesungen = int64_t(st.loesungen);
  out->nicht_konvergiert = int64_t(st.nicht_konvergiert);
  out->kontakte = int64_t(st.kontakte);
  out->haftend = int64_t(st.haftend);
  out->freigegeben = int64_t(st.freigegeben);
  out->durchstoesse = int64_t(st.durchstoesse);
  out->koerperpunkte = int64_t(st.koerperpunkte);
  out->rest_max = st.rest_max;
  out->naehe_punkt_dreieck = int64_t(st.naehe_punkt_dreieck);
  out->naehe_kante_kante = int64_t(st.naehe_kante_kante);
  out->selbst_stoesse = int64_t(st.selbst_stoesse);
  out->durchdringungen = int64_t(st.durchdringungen);
  out->durchdringungsgebiete = int64_t(st.durchdringungsgebiete);
}

}  // namespace

extern "C" {

// ------------------------------------------------------------ scene builder
void* orc_build_scene(const k3d_pattern* p) {
  Muster m;
  for (int32_t t = 0; t < p->n_teile; ++t) {
    const k3d_piece& kp = p->teile[t];
    Teil tl;
    for (int64_t i = 0; i < kp.n_punkte; ++i) {
      tl.punkte_mm.push_back({kp.punkte_mm[2 * i], kp.punkte_mm[2 * i + 1]});
      tl.lage.push_back({kp.lage[3 * i], kp.lage[3 * i + 1], kp.lage[3 * i + 2]});
    }
    for (int64_t d = 0; d < kp.n_dreiecke; ++d)
      tl.dreiecke.push_back({kp.dreiecke[3 * d], kp.dreiecke[3 * d + 1], kp.dreiecke[3 * d + 2]});
    tl.fadenlauf = {kp.fadenlauf[0], kp.fadenlauf[1]};
    tl.material = mat_aus(kp.material);
    tl.reduktion = kp.reduktion;
    m.teile.push_back(std::move(tl));
  }
  for (int32_t n = 0; n < p->n_naehte; ++n) {
    const k3d_seam& ks = p->naehte[n];
    Naht nh;
    nh.laenge_a_mm = ks.laenge_a_mm;
    nh.laenge_b_mm = ks.laenge_b_mm;
    for (int32_t q = 0; q < ks.n_teilnaehte; ++q) {
      const k3d_seam_part& kt = ks.teilnaehte[q];
      Teilnaht tn;
      tn.teil_a = size_t(kt.teil_a);
      tn.teil_b = size_t(kt.teil_b);
      for (int64_t i = 0; i < kt.n_paare; ++i) tn.paare.push_back({kt.paare[2 * i], kt.paare[2 * i + 1]});
      nh.teilnaehte.push_back(std::move(tn));
    }
    m.naehte.push_back(std::move(nh));
  }
  Simparameter sp = sim_aus(p->param);
  sp.naht_nachgiebigkeit = p->naht_nachgiebigkeit;
  sp.einhalteweite = p->einhalteweite != 0;
  auto* g = new Gebaut;
  g->s = szene_bauen(m, {}, sp);
  g->flach();
  return g;
}

void orc_built_scene_view(void* h, k3d_scene* out) {
  auto* g = static_cast<Gebaut*>(h);
  std::memset(out, 0, sizeof(*out));
  out->n_punkte = int64_t(g->s.x.size());
  out->x = g->x.data();
  out->v = g->v.data();
  out->masse = g->s.masse.data();
  out->w = g->s.w.data();
  out->kollisionsabstand = g->s.kollisionsabstand.data();
  out->reibung = g->s.reibung.data();
  out->n_abstand = int64_t(g->s.abstand.size());
  out->abstand_punkte = g->p_a.data();
  out->abstand_ruhe = g->ruhe_a.data();
  out->abstand_nachgiebigkeit = g->alpha_a.data();
  out->membran_kante = g->mk.data();
  out->n_naht = int64_t(g->s.naht.size());
  out->naht_punkte = g->p_n.data();
  out->naht_ruhe = g->ruhe_n.data();
  out->n_biegung = int64_t(g->s.biegung.size());
  out->biegung_punkte = g->p_b.data();
  out->biegung_ruhe = g->ruhe_b.data();
  out->biegung_nachgiebigkeit = g->alpha_b.data();
  out->n_membran = int64_t(g->s.membran_elemente.size());
  out->membran_punkte = g->p_m.data();
  out->membran_flaeche = g->m_fl.data();
  out->membran_ruhe_inv = g->m_ri.data();
  out->membran_kette = g->m_k.data();
  out->membran_schuss = g->m_s.data();
  out->membran_steif = g->m_st.data();
  out->n_dreiecke = int64_t(g->s.dreiecke.size());
  out->dreiecke = g->dr.data();
  out->ruhe_inv = g->ri.data();
  out->param.bild_dt = g->s.param.bild_dt;
  for (int a = 0; a < 3; ++a) out->param.schwerkraft[a] = g->s.param.schwerkraft[a];
  out->param.daempfung = g->s.param.daempfung;
  out->n_teile = int64_t(g->s.teile.size());
  out->teil_bereiche = g->tb.data();
  out->teil_dehnung = g->te.data();
  out->teil_band_von = g->tv.data();
}

int64_t orc_built_scene_counts(void* h, int64_t* out6) {
  auto* g = static_cast<Gebaut*>(h);
  out6[0] = int64_t(g->s.membran_entartet);
  out6[1] = int64_t(g->s.naht_biegung_ohne);
  out6[2] = int64_t(g->s.einhalte_kanten);
  out6[3] = int64_t(g->s.abstand.farben.size());
  out6[4] = int64_t(g->s.biegung.farben.size());
  out6[5] = int64_t(g->s.naht.farben.size());
  return 0;
}

void orc_built_scene_free(void* h) { delete static_cast<Gebaut*>(h); }

// ------------------------------------------------------------ simulation
void* orc_sim_create(const k3d_scene* s, const k3d_params* p) {
  auto* sim = new Sim;
  sim->s = szene_aus(s, sim->kd);
  sim->cg.param = param_aus(p);
  return sim;
}
void orc_sim_free(void* h) { delete static_cast<Sim*>(h); }

// Impacts on the way x0 -> x1 of a small mesh (triangles, or with nt == 0
// the edges alone) and their response (selbstkollision.rs:1196-1343); x1 is
// updated. Writes per impact (art, zeit, seite) up to cap; returns the number
// of impacts, *antworten the response's count.
int64_t orc_stoesse(int64_t np, const double* x0, double* x1, const double* w, const double* masse, int64_t nt,
                    const uint32_t* tris, int64_t ne, const uint32_t* kanten, int32_t pd, int32_t kk,
                    int32_t iterationen, double* out3, int64_t cap, int64_t* antworten) {
  std::vector<std::array<uint32_t, 3>> d(static_cast<size_t>(nt));
  for (int64_t t = 0; t < nt; ++t) d[size_t(t)] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
  Stoffnetz netz = stoffnetz_neu(d, std::vector<double>(static_cast<size_t>(np), 1e-3));
  if (nt == 0)
    for (int64_t e = 0; e < ne; ++e) netz.kanten.push_back({kanten[2 * e], kanten[2 * e + 1]});
  std::vector<V3> a(static_cast<size_t>(np)), b(static_cast<size_t>(np));
  std::vector<double> wv(w, w + np), mv(masse, masse + np);
  for (int64_t i = 0; i < np; ++i)
    for (int k = 0; k < 3; ++k) {
      a[size_t(i)][k] = x0[3 * i + k];
      b[size_t(i)][k] = x1[3 * i + k];
    }
  std::vector<Stoss> st = finde_stoesse(netz, a, b, wv, pd != 0, kk != 0);
  for (size_t q = 0; q < st.size() && int64_t(q) < cap; ++q) {
    out3[3 * q] = st[q].art == Art::PunktDreieck ? 0.0 : 1.0;
    out3[3 * q + 1] = st[q].zeit;
    out3[3 * q + 2] = st[q].seite;
  }
  size_t z = stossantwort(st, b, mv, wv, size_t(std::max(iterationen, 0)));
  for (int64_t i = 0; i < np; ++i)
    for (int k = 0; k < 3; ++k) x1[3 * i + k] = b[size_t(i)][k];
  if (antworten) *antworten = int64_t(z);
  return int64_t(st.size());
}

// finde_schnitte (selbstkollision.rs:858) at the simulation's current state,
// with the scene's cloth tables (aus_szene, zusatzdicke 2.5 mm); writes the
// region roots (gebiete) up to cap; returns the number of intersections.
int64_t orc_sim_schnitte(void* h, int32_t an_naehten, int64_t cap, int64_t* wurzeln) {
  auto* sim = static_cast<Sim*>(h);
  auto nw = aus_szene(sim->s, 2.5e-3);
  std::vector<Schnitt> schn = finde_schnitte(nw.first, sim->s.x, an_naehten != 0);
  std::vector<size_t> r = gebiete(nw.first, schn);
  for (size_t q = 0; q < r.size() && int64_t(q) < cap; ++q) wurzeln[q] = int64_t(r[q]);
  return int64_t(schn.size());
}

// Adjoint of n frames (adjoint.cpp): runs the frames from the current state,
// recording every substep, then goes back through them. gx, gv: cotangents of
// the final x, v (3 per point); out: those of the initial x, v, and per
// membrane (E_warp, E_weft, G, grain rotation) and per hinge (k) the
// parameter cotangents. iters: adjoint CG iterations (may be null).
void orc_sim_adjoint(void* h, int32_t n, const double* gx, const double* gv, double* gx0, double* gv0,
                     double* g_membran, double* g_biegung, double toleranz, int64_t* iters) {
  auto* sim = static_cast<Sim*>(h);
  std::vector<Aufnahme> auf;
  for (int32_t f = 0; f < n; ++f) sim->cg.bild(sim->s, &auf);
  const size_t np = sim->s.x.size();
  std::vector<V3> xq(np), vq(np), lam;
  for (size_t i = 0; i < np; ++i)
    for (int a = 0; a < 3; ++a) {
      xq[i][a] = gx[3 * i + a];
      vq[i][a] = gv[3 * i + a];
    }
  AdjGrad g;
  g.membran.assign(sim->s.membran_elemente.size(), {0, 0, 0, 0});
  g.biegung.assign(sim->s.biegung.size(), 0.0);
  AdjStat st;
  Szene s = sim->s;
  ImplizitCg cg = sim->cg;
  for (size_t k = auf.size(); k-- > 0;) cg.adjoint_schritt(s, auf[k], xq, vq, g, lam, st, toleranz);
  for (size_t i = 0; i < np; ++i)
    for (int a = 0; a < 3; ++a) {
      gx0[3 * i + a] = xq[i][a];
      gv0[3 * i + a] = vq[i][a];
    }
  for (size_t t = 0; t < g.membran.size(); ++t)
    for (int q = 0; q < 4; ++q) g_membran[4 * t + q] = g.membran[t][q];
  for (size_t b = 0; b < g.biegung.size(); ++b) g_biegung[b] = g.biegung[b];
  if (iters) *iters = int64_t(st.cg_iterationen);
}

void orc_sim_frames(void* h, int32_t n, k3d_stats* st) {
  auto* sim = static_cast<Sim*>(h);
  ImplizitStatistik summe;
  for (int32_t f = 0; f < n; ++f) {
    sim->cg.bild(sim->s);
    const auto& b = sim->cg.statistik;
    summe.cg_iterationen += b.cg_iterationen;
    summe.loesungen += b.loesungen;
    summe.nicht_konvergiert += b.nicht_konvergiert;
    summe.kontakte += b.kontakte;
    summe.haftend += b.haftend;
    summe.freigegeben += b.freigegeben;
    summe.durchstoesse += b.durchstoesse;
    summe.koerperpunkte += b.koerperpunkte;
    summe.rest_max = std::max(summe.rest_max, b.rest_max);
    summe.naehe_punkt_dreieck += b.naehe_punkt_dreieck;
    summe.naehe_kante_kante += b.naehe_kante_kante;
    summe.selbst_stoesse += b.selbst_stoesse;
    summe.durchdringungen += b.durchdringungen;
    summe.durchdringungsgebiete += b.durchdringungsgebiete;
  }
  stats_aus(summe, st);
}

// n frames of the XPBD cross-check (CpuReferenz::bild, cpu.rs:222-245) with
// `unterschritte` substeps each; out4 = contacts, sticking, depth sum and
// tangential sum of the last frame (Kontaktstatistik).
void orc_sim_xpbd_frames(void* h, int32_t n, int32_t unterschritte, double* out4) {
  auto* sim = static_cast<Sim*>(h);
  for (int32_t f = 0; f < n; ++f) sim->xpbd.bild(sim->s, size_t(std::max(unterschritte, 1)));
  if (out4) {
    out4[0] = double(sim->xpbd.statistik.kontakte);
    out4[1] = double(sim->xpbd.statistik.haftend);
    out4[2] = sim->xpbd.statistik.tiefe;
    out4[3] = sim->xpbd.statistik.tangential;
  }
}

// One distance constraint on two points (cpu.rs:251-270): korr6 is updated.
void orc_xpbd_abstand(const double* x6, const double* delta6, double* korr6, const double* w2, double ruhe,
                      double alpha_h2) {
  std::vector<V3> x = {{x6[0], x6[1], x6[2]}, {x6[3], x6[4], x6[5]}};
  std::vector<V3> d = {{delta6[0], delta6[1], delta6[2]}, {delta6[3], delta6[4], delta6[5]}};
  std::vector<V3> k = {{korr6[0], korr6[1], korr6[2]}, {korr6[3], korr6[4], korr6[5]}};
  std::vector<double> w = {w2[0], w2[1]};
  xpbd_abstand(x, d, k, w, {0u, 1u}, ruhe, alpha_h2);
  for (int i = 0; i < 2; ++i)
    for (int c = 0; c < 3; ++c) korr6[3 * i + c] = k[size_t(i)][size_t(c)];
}

// The membrane's three XPBD constraints (kontinuum.rs:526-551) for the
// element m12 (orc_membran_eval's layout) at p9: c3, grad27 (constraint,
// point, axis), alpha3.
void orc_membran_zuege(const double* m12, const double* p9, double* c3, double* grad27, double* alpha3);

void orc_sim_get_state(void* h, double* x, double* v) {
  auto* sim = static_cast<Sim*>(h);
  for (size_t i = 0; i < sim->s.x.size(); ++i)
    for (int a = 0; a < 3; ++a) {
      if (x) x[3 * i + a] = sim->s.x[i][a];
      if (v) v[3 * i + a] = sim->s.v[i][a];
    }
}
void orc_sim_set_state(void* h, const double* x, const double* v) {
  auto* sim = static_cast<Sim*>(h);
  for (size_t i = 0; i < sim->s.x.size(); ++i)
    for (int a = 0; a < 3; ++a) {
      if (x) sim->s.x[i][a] = x[3 * i + a];
      if (v) sim->s.v[i][a] = v[3 * i + a];
    }
}
void orc_sim_set_naht_ruhe(void* h, const double* r) {
  auto* sim = static_cast<Sim*>(h);
  for (size_t c = 0; c < sim->s.naht.ruhe.size(); ++c) sim->s.naht.ruhe[c] = r[c];
}
void orc_sim_get_naht_ruhe(void* h, double* r) {
  auto* sim = static_cast<Sim*>(h);
  for (size_t c = 0; c < sim->s.naht.ruhe.size(); ++c) r[c] = sim->s.naht.ruhe[c];
}
void orc_sim_naht_kuerzen(void* h, double schritt) { naht_kuerzen(static_cast<Sim*>(h)->s, schritt); }
void orc_sim_naht_offen(void* h) { naht_offen(static_cast<Sim*>(h)->s); }
void orc_sim_set_reibung(void* h, double mu) {
  for (double& r : static_cast<Sim*>(h)->s.reibung) r = mu;
}
void orc_sim_set_dv_warm(void* h, const double* dv) {
  auto* sim = static_cast<Sim*>(h);
  sim->cg.dv_vorher.resize(sim->s.x.size());
  for (size_t i = 0; i < sim->cg.dv_vorher.size(); ++i)
    for (int a = 0; a < 3; ++a) sim->cg.dv_vorher[i][a] = dv[3 * i + a];
}
void orc_sim_get_dv_warm(void* h, double* dv) {
  auto* sim = static_cast<Sim*>(h);
  for (size_t i = 0; i < sim->cg.dv_vorher.size(); ++i)
    for (int a = 0; a < 3; ++a) dv[3 * i + a] = sim->cg.dv_vorher[i][a];
}

void orc_sim_operator(void* h, const double* p, double* out) {
  auto* sim = static_cast<Sim*>(h);
  size_t n = sim->s.x.size();
  std::vector<V3> pv(n);
  for (size_t i = 0; i < n; ++i) pv[i] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
  auto r = sim->cg.op(sim->s, pv);
  for (size_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) out[3 * i + a] = r[i][a];
}

static double substep_h(Sim* sim) {
  return sim->s.param.bild_dt / double(std::max<size_t>(sim->cg.param.schritte_je_bild, 1));
}

void orc_sim_system(void* h, k3d_system_readback* rb) {
  auto* sim = static_cast<Sim*>(h);
  std::vector<std::optional<Fest>> fest;
  System sys = sim->cg.system_bauen(sim->s, substep_h(sim), fest);
  size_t n = sim->s.x.size();
  for (size_t i = 0; i < n; ++i) {
    for (int a = 0; a < 3; ++a) {
      if (rb->rhs) rb->rhs[3 * i + a] = sys.rhs[i][a];
      if (rb->f) rb->f[3 * i + a] = sys.f[i][a];
      if (rb->last) rb->last[3 * i + a] = sys.last[i][a];
      if (rb->normale) rb->normale[3 * i + a] = fest[i] ? fest[i]->normale[a] : 0.0;
    }
    if (rb->pinv)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) rb->pinv[9 * i + 3 * a + b] = sys.pinv[i][a][b];
    if (rb->vn_soll) rb->vn_soll[i] = fest[i] ? fest[i]->vn_soll : 0.0;
    if (rb->fest) rb->fest[i] = fest[i] ? 1 : 0;
  }
}

void orc_sim_solve(void* h, double* dv, k3d_cg_result* out) {
  auto* sim = static_cast<Sim*>(h);
  std::vector<std::optional<Fest>> fest;
  System sys = sim->cg.system_bauen(sim->s, substep_h(sim), fest);
  size_t n = sim->s.x.size();
  std::vector<V3> d(n);
  for (size_t i = 0; i < n; ++i) d[i] = {dv[3 * i], dv[3 * i + 1], dv[3 * i + 2]};
  CgLauf l = cpu_loese(sys, fest, d);
  for (size_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) dv[3 * i + a] = d[i][a];
  out->iterationen = int64_t(l.iterationen);
  out->nicht_konvergiert = l.nicht_konvergiert ? 1 : 0;
  out->breakdown = 0;
  out->rest = l.rest;
}

// Loeser::loese with a given contact set (implizit.rs:308): the system of the
// current state, the caller's Fest in place of the one system_bauen found.
void orc_sim_solve_contacts(void* h, const uint8_t* on, const double* nrm, const double* soll, double* dv,
                            k3d_cg_result* out) {
  auto* sim = static_cast<Sim*>(h);
  std::vector<std::optional<Fest>> fest;
  System sys = sim->cg.system_bauen(sim->s, substep_h(sim), fest);
  size_t n = sim->s.x.size();
  for (size_t i = 0; i < n; ++i) {
    if (!on[i]) {
      fest[i].reset();
      continue;
    }
    Fest f;
    f.normale = {nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]};
    f.vn_soll = soll[i];
    fest[i] = f;
  }
  std::vector<V3> d(n);
  for (size_t i = 0; i < n; ++i) d[i] = {dv[3 * i], dv[3 * i + 1], dv[3 * i + 2]};
  CgLauf l = cpu_loese(sys, fest, d);
  for (size_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) dv[3 * i + a] = d[i][a];
  out->iterationen = int64_t(l.iterationen);
  out->nicht_konvergiert = l.nicht_konvergiert ? 1 : 0;
  out->breakdown = 0;
  out->rest = l.rest;
}

// ------------------------------------------------------------ measurement
double orc_sim_umfang(void* h, const double* punkt, const double* normale) {
  auto* sim = static_cast<Sim*>(h);
  return umfang_in_ebene(sim->s, {punkt[0], punkt[1], punkt[2]}, {normale[0], normale[1], normale[2]});
}
double orc_sim_nahtspalt(void* h) { return nahtspalt(static_cast<Sim*>(h)->s); }
double orc_sim_mittlere_geschwindigkeit(void* h) { return mittlere_geschwindigkeit(static_cast<Sim*>(h)->s); }
void orc_sim_dehnung(void* h, double* out2) {
  auto d = dehnung_je_dreieck(static_cast<Sim*>(h)->s);
  for (size_t t = 0; t < d.size(); ++t) {
    out2[2 * t] = d[t].first;
    out2[2 * t + 1] = d[t].second;
  }
}
void orc_sim_schwerpunkt(void* h, double* out3) {
  V3 q = schwerpunkt(static_cast<Sim*>(h)->s);
  for (int a = 0; a < 3; ++a) out3[a] = q[a];
}

// ------------------------------------------------------------ element-level probes
// m12 = flaeche, ruhe_inv[4], kette[2], schuss[2], steif[3]
static Membran membran_aus(const double* m) {
  Membran e;
  e.flaeche = m[0];
  for (int a = 0; a < 4; ++a) e.ruhe_inv[a] = m[1 + a];
  e.kette = {m[5], m[6]};
  e.schuss = {m[7], m[8]};
  e.kette_n_m = m[9];
  e.dehnung_n_m = m[10];
  e.schub_n_m = m[11];
  return e;
}
static std::array<V3, 3> p3_aus(const double* p) {
  return {V3{p[0], p[1], p[2]}, V3{p[3], p[4], p[5]}, V3{p[6], p[7], p[8]}};
}
int32_t orc_membran_bauen(const double* ruhe6, const double* kanten3, const double* dir2, const double* mat3,
                          double* out12) {
  auto m = membran_bauen({V2{ruhe6[0], ruhe6[1]}, V2{ruhe6[2], ruhe6[3]}, V2{ruhe6[4], ruhe6[5]}},
                         {kanten3[0], kanten3[1], kanten3[2]}, {dir2[0], dir2[1]}, {mat3[0], mat3[1], mat3[2]});
  if (!m) return 0;
  out12[0] = m->flaeche;
  for (int a = 0; a < 4; ++a) out12[1 + a] = m->ruhe_inv[a];
  out12[5] = m->kette[0];
  out12[6] = m->kette[1];
  out12[7] = m->schuss[0];
  out12[8] = m->schuss[1];
  out12[9] = m->kette_n_m;
  out12[10] = m->dehnung_n_m;
  out12[11] = m->schub_n_m;
  return 1;
}
void orc_membran_eval(const double* m12, const double* p9, double* dehnung3, double* spannung3, double* energie,
                      double* krafte9, double* zug9, double* hessen9) {
  Membran m = membran_aus(m12);
  auto p = p3_aus(p9);
  V3 d = membran_dehnung(m, p), s = membran_spannung(m, p);
  for (int a = 0; a < 3; ++a) {
    dehnung3[a] = d[a];
    spannung3[a] = s[a];
  }
  *energie = membran_energie(m, p);
  auto f = membran_krafte(m, p), z = membran_krafte_zug(m, p);
  Hessen hs = membran_hessen(m, p);
  for (int k = 0; k < 3; ++k)
    for (int a = 0; a < 3; ++a) {
      krafte9[3 * k + a] = f[k][a];
      zug9[3 * k + a] = z[k][a];
    }
  for (int a = 0; a < 3; ++a) {
    hessen9[a] = hs.f1[a];
    hessen9[3 + a] = hs.f2[a];
    hessen9[6 + a] = hs.w[a];
  }
}
void orc_membran_zuege(const double* m12, const double* p9, double* c3, double* grad27, double* alpha3) {
  const auto z = membran_zuege(membran_aus(m12), p3_aus(p9));
  for (int q = 0; q < 3; ++q) {
    c3[q] = z[size_t(q)].c;
    alpha3[q] = z[size_t(q)].alpha;
    for (int k = 0; k < 3; ++k)
      for (int a = 0; a < 3; ++a) grad27[9 * q + 3 * k + a] = z[size_t(q)].grad[size_t(k)][size_t(a)];
  }
}
void orc_membran_mal_h(const double* m12, const double* p9, const double* d9, double* out9) {
  Membran m = membran_aus(m12);
  auto r = membran_mal_h_aus(m, membran_hessen(m, p3_aus(p9)), p3_aus(d9));
  for (int k = 0; k < 3; ++k)
    for (int a = 0; a < 3; ++a) out9[3 * k + a] = r[k][a];
}
void orc_membran_diag(const double* m12, const double* p9, double* out27) {
  Membran m = membran_aus(m12);
  auto r = membran_diag_bloecke_aus(m, membran_hessen(m, p3_aus(p9)));
  for (int k = 0; k < 3; ++k)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) out27[9 * k + 3 * a + b] = r[k][a][b];
}
void orc_psd2(double a, double b, double c, double* out3) {
  V3 r = psd2(a, b, c);
  for (int i = 0; i < 3; ++i) out3[i] = r[i];
}
double orc_steifigkeit(double weft, double warp, double bias, double theta) {
  return steifigkeit(weft, warp, bias, theta);
}
int32_t orc_cos2_sin2(const double* e, const double* warp, double* out2) {
  double c2 = 0, s2 = 0;
  bool ok = cos2_sin2({e[0], e[1]}, {warp[0], warp[1]}, c2, s2);
  out2[0] = c2;
  out2[1] = s2;
  return ok ? 1 : 0;
}
int32_t orc_dieder(const double* q12, double* theta, double* grad12) {
  std::array<V3, 4> q = {V3{q12[0], q12[1], q12[2]}, V3{q12[3], q12[4], q12[5]}, V3{q12[6], q12[7], q12[8]},
                         V3{q12[9], q12[10], q12[11]}};
  std::array<V3, 4> g{};
  bool ok = dieder(q, *theta, g);
  for (int k = 0; k < 4; ++k)
    for (int a = 0; a < 3; ++a) grad12[3 * k + a] = g[k][a];
  return ok ? 1 : 0;
}
double orc_winkel_fehler(double theta, double ruhe) { return winkel_fehler(theta, ruhe); }
void orc_m3_inv(const double* m9, double* out9) {
  M3 m = {V3{m9[0], m9[1], m9[2]}, V3{m9[3], m9[4], m9[5]}, V3{m9[6], m9[7], m9[8]}};
  M3 r = m3_inv(m);
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) out9[3 * a + b] = r[a][b];
}
// colours of `anzahl` constraints with `breite` points each; returns the number of colours
int64_t orc_faerbe(int64_t anzahl, int32_t breite, int64_t npunkte, const uint32_t* punkte, uint32_t* farbe_out,
                   int64_t* ordnung_out) {
  std::vector<std::vector<uint32_t>> pv(static_cast<size_t>(anzahl));
  for (int64_t c = 0; c < anzahl; ++c) pv[c].assign(punkte + c * breite, punkte + (c + 1) * breite);
  auto [farbe, zahl] = faerbe(size_t(anzahl), size_t(npunkte), pv);
  auto [idx, ber] = ordnung(farbe, zahl);
  for (int64_t c = 0; c < anzahl; ++c) {
    farbe_out[c] = farbe[c];
    ordnung_out[c] = int64_t(idx[c]);
  }
  return int64_t(zahl);
}
int32_t orc_kontakt(const k3d_body* kb, const double* x, double abstand, double* normale3, double* tiefe) {
  Koerperdaten kd = koerper_aus(kb, 1);
  auto k = kd.koerper[0].kontakt({x[0], x[1], x[2]}, abstand);
  if (!k) return 0;
  for (int a = 0; a < 3; ++a) normale3[a] = k->normale[a];
  *tiefe = k->tiefe;
  return 1;
}

}  // extern "C"

// ------------------------------------------------------------ self-collision probes
namespace {
std::vector<V3> v3_aus(const double* p, size_t n) {
  std::vector<V3> o(n);
  for (size_t i = 0; i < n; ++i) o[i] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
  return o;
}
int64_t naehe_aus(const std::vector<Naehe>& nh, int64_t cap, int32_t* art, uint32_t* punkte4, double* gewichte4,
                  double* normale3, double* abstand, double* ruhe) {
  const int64_t n = int64_t(nh.size());
  for (int64_t q = 0; q < std::min(n, cap); ++q) {
    const Naehe& p = nh[size_t(q)];
    if (art) art[q] = int32_t(p.art);
    for (int k = 0; k < 4; ++k) {
      if (punkte4) punkte4[4 * q + k] = p.punkte[k];
      if (gewichte4) gewichte4[4 * q + k] = p.gewichte[k];
    }
    for (int k = 0; k < 3; ++k)
      if (normale3) normale3[3 * q + k] = p.normale[k];
    if (abstand) abstand[q] = p.abstand;
    if (ruhe) ruhe[q] = p.ruhe;
  }
  return n;
}
std::pair<Stoffnetz, Stoffwerte> netz_von(Sim* sim) {
  return aus_szene(sim->s, sim->cg.param.selbst_zusatzdicke);
}
}  // namespace

extern "C" {

int64_t orc_zellindex(double x, double zelle) { return zellindex(x, zelle); }
uint64_t orc_streue(int64_t i, int64_t j, int64_t k, uint64_t n) { return uint64_t(streue(i, j, k, size_t(n))); }

// Stoffnetz::neu on raw triangles and radii, then finde (the reference's
// own unit tests build the mesh this way, selbstkollision.rs:1352-1396)
int64_t orc_finde_roh(int64_t n, const double* x, const double* w, int64_t nt, const uint32_t* dreiecke,
                      const double* r_punkt, int32_t pd, int32_t kk, int64_t cap, int32_t* art, uint32_t* punkte4,
                      double* gewichte4, double* normale3, double* abstand, double* ruhe) {
  std::vector<std::array<uint32_t, 3>> d(static_cast<size_t>(nt));
  for (int64_t t = 0; t < nt; ++t) d[size_t(t)] = {dreiecke[3 * t], dreiecke[3 * t + 1], dreiecke[3 * t + 2]};
  Stoffnetz netz = stoffnetz_neu(d, std::vector<double>(r_punkt, r_punkt + n));
  std::vector<double> wv(w, w + n);
  return naehe_aus(finde(netz, v3_aus(x, size_t(n)), wv, pd != 0, kk != 0), cap, art, punkte4, gewichte4, normale3,
                   abstand, ruhe);
}

// Proximity pairs of the simulation's scene at positions x (its own w).
int64_t orc_selbst_finde(void* h, const double* x, int32_t pd, int32_t kk, int64_t cap, int32_t* art,
                         uint32_t* punkte4, double* gewichte4, double* normale3, double* abstand, double* ruhe) {
  auto* sim = static_cast<Sim*>(h);
  auto nw = netz_von(sim);
  return naehe_aus(finde(nw.first, v3_aus(x, sim->s.x.size()), sim->s.w, pd != 0, kk != 0), cap, art, punkte4,
                   gewichte4, normale3, abstand, ruhe);
}

// Edge list of the scene's self-collision mesh (Stoffnetz::neu order),
// 2 per edge, and the hash cell size; returns the edge count.
int64_t orc_selbst_kanten(void* h, int64_t cap, uint32_t* kanten2, double* zelle) {
  auto* sim = static_cast<Sim*>(h);
  auto nw = netz_von(sim);
  const auto& k = nw.first.kanten;
  for (size_t e = 0; e < std::min(k.size(), size_t(cap)); ++e) {
    kanten2[2 * e] = k[e][0];
    kanten2[2 * e + 1] = k[e][1];
  }
  if (zelle) *zelle = hash_zelle(nw.first);
  return int64_t(k.size());
}

// Hashgitter::neu of the point boxes (kanten = 0) or the edge boxes
// (kanten = 1) at positions x: bucket starts (eimer + 1) and entries.
// Returns the bucket count; *n_eintraege = entry count.
int64_t orc_selbst_hash(void* h, const double* x, int32_t kanten, int64_t cap_anfang, uint32_t* anfang,
                        int64_t cap_eintraege, uint32_t* eintraege, int64_t* n_eintraege) {
  auto* sim = static_cast<Sim*>(h);
  auto nw = netz_von(sim);
  const Stoffnetz& netz = nw.first;
  std::vector<V3> xv = v3_aus(x, sim->s.x.size());
  std::vector<Quader> q;
  if (kanten) {
    for (size_t e = 0; e < netz.kanten.size(); ++e)
      q.push_back(kanten_quader(xv[netz.kanten[e][0]], xv[netz.kanten[e][1]], netz.r_kante[e] + ZUSCHLAG_QUADER));
  } else {
    for (size_t v = 0; v < xv.size(); ++v) q.push_back(quader_punkte(&xv[v], 1, netz.r_punkt[v] + ZUSCHLAG_QUADER));
  }
  Hashgitter g = hashgitter_neu(q, hash_zelle(netz));
  for (size_t b = 0; b < std::min(g.anfang.size(), size_t(cap_anfang)); ++b) anfang[b] = g.anfang[b];
  for (size_t e = 0; e < std::min(g.eintraege.size(), size_t(cap_eintraege)); ++e) eintraege[e] = g.eintraege[e];
  if (n_eintraege) *n_eintraege = int64_t(g.eintraege.size());
  return int64_t(g.eimer);
}

// finde + federn on the simulation's scene at (x, v): springs (5 points and
// weights, force, 3x3 block) and the damped velocities in v_inout.
int64_t orc_selbst_federn(void* h, const double* x, double* v_inout, int64_t cap, uint32_t* punkte5,
                          double* gewichte5, double* kraft3, double* block9) {
  auto* sim = static_cast<Sim*>(h);
  auto nw = netz_von(sim);
  const size_t n = sim->s.x.size();
  std::vector<V3> xv = v3_aus(x, n), vv = v3_aus(v_inout, n);
  auto nh = finde(nw.first, xv, sim->s.w, true, true);
  auto fe = federn(nw.first, nw.second, nh, sim->cg.param.selbst_steifigkeit, sim->s.masse, sim->s.w,
                   sim->s.naht.ruhe, vv);
  for (size_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) v_inout[3 * i + a] = vv[i][a];
  for (size_t q = 0; q < std::min(fe.size(), size_t(cap)); ++q) {
    for (int k = 0; k < 5; ++k) {
      punkte5[5 * q + k] = fe[q].punkte[k];
      gewichte5[5 * q + k] = fe[q].gewichte[k];
    }
    for (int a = 0; a < 3; ++a) {
      kraft3[3 * q + a] = fe[q].kraft[a];
      for (int b = 0; b < 3; ++b) block9[9 * q + 3 * a + b] = fe[q].block[a][b];
    }
  }
  return int64_t(fe.size());
}

}  // extern "C"
