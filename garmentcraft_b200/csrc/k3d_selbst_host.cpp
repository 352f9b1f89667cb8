// Host side of the self-collision proximity stage: the mesh tables of
// Stoffnetz::neu / aus_szene (sim/src/selbstkollision.rs:159-187, 623-688),
// built once per upload, the device buffers (grown when a run needs more),
// and one run per substep.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <utility>
#include <vector>

#include "k3d_selbst_host.h"

namespace k3d {
namespace {

template <typename T>
cudaError_t up(T*& dst, const std::vector<T>& src, std::vector<void*>& owned, cudaStream_t st) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, std::max<size_t>(src.size(), 1) * sizeof(T));
  if (e != cudaSuccess) return e;
  owned.push_back(p);
  dst = static_cast<T*>(p);
  if (!src.empty()) return cudaMemcpyAsync(p, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, st);
  return cudaSuccess;
}
template <typename T>
cudaError_t alloc(T*& dst, size_t count, std::vector<void*>& owned) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) return e;
  owned.push_back(p);
  dst = static_cast<T*>(p);
  return cudaSuccess;
}
void free_all(std::vector<void*>& v) {
  for (void* p : v) cudaFree(p);
  v.clear();
}

}  // namespace

void selbst_free(SelbstHost& H) {
  free_all(H.fest);
  free_all(H.pairs);
  free_all(H.hashk);
  free_all(H.schn);
  free_all(H.wege);
  H.on = false;
  H.ran = false;
}

cudaError_t selbst_upload(SelbstHost& H, const k3d_scene* sc, double zusatzdicke, double steifigkeit, int rsize,
                          const double* x, double* v, const double* masse, const double* w, const double* reib,
                          cudaStream_t st) {
  selbst_free(H);
  SelbstArgs& s = H.s;
  std::memset(&s, 0, sizeof(s));
  const int64_t n = sc->n_punkte, nd = sc->n_dreiecke;
  s.n = n;
  s.nd = nd;
  s.rsize = rsize;
  s.steifigkeit = steifigkeit;
  s.x = x;
  s.v = v;
  s.masse = masse;
  s.w = w;
  s.mu = reib;

  // Stoffnetz::neu: edges in order of first appearance, their triangles, the
  // triangles' edges, radii (selbstkollision.rs:159-187)
  std::vector<double> r(n);
  for (int64_t i = 0; i < n; ++i) r[i] = sc->kollisionsabstand[i] + zusatzdicke / 2.0;
  std::vector<uint4> d_idx(nd), d_kan(nd);
  std::vector<uint2> k_idx, k_dr;
  std::map<std::pair<uint32_t, uint32_t>, uint32_t> karte;
  for (int64_t t = 0; t < nd; ++t) {
    const uint32_t* d = sc->dreiecke + 3 * t;
    uint32_t dk[3];
    for (int k = 0; k < 3; ++k) {
      const uint32_t a = d[k], b = d[(k + 1) % 3];
      const std::pair<uint32_t, uint32_t> key{std::min(a, b), std::max(a, b)};
      auto it = karte.find(key);
      uint32_t e;
      if (it == karte.end()) {
        e = uint32_t(k_idx.size());
        k_idx.push_back(make_uint2(key.first, key.second));
        k_dr.push_back(make_uint2(kKein, kKein));
        karte.emplace(key, e);
      } else {
        e = it->second;
      }
      uint2& kd = k_dr[e];
      if (kd.x == kKein)
        kd.x = uint32_t(t);
      else if (kd.y == kKein)
        kd.y = uint32_t(t);
      dk[k] = e;
    }
    d_idx[t] = make_uint4(d[0], d[1], d[2], 0u);
    d_kan[t] = make_uint4(dk[0], dk[1], dk[2], 0u);
  }
  const int64_t ne = int64_t(k_idx.size());
  s.ne = ne;
  std::vector<double> r_kante(ne), r_dreieck(nd);
  for (int64_t e = 0; e < ne; ++e) r_kante[e] = std::fmax(r[k_idx[e].x], r[k_idx[e].y]);
  for (int64_t t = 0; t < nd; ++t) {
    double m = 0.0;
    const uint32_t* d = sc->dreiecke + 3 * t;
    for (int k = 0; k < 3; ++k) m = std::fmax(m, r[d[k]]);
    r_dreieck[t] = m;
  }
  double r_max = 0.0;
  for (double q : r) r_max = std::fmax(r_max, q);
  s.zelle = std::fmax(2.0 * r_max + 4e-5, 1e-4) * 2.0;
  s.eimer_p = uint32_t(std::max<int64_t>(2 * n, 64));
  s.eimer_k = uint32_t(std::max<int64_t>(2 * ne, 64));

  // seam and weld partners (selbstkollision.rs:628-647)
  std::vector<std::vector<uint32_t>> partner(n);
  for (int64_t c = 0; c < sc->n_naht; ++c) {
    const uint32_t i = sc->naht_punkte[2 * c], j = sc->naht_punkte[2 * c + 1];
    partner[i].push_back(j);
    partner[j].push_back(i);
  }
  for (int64_t e = 0; e < sc->n_abstand; ++e) {
    const uint32_t i = sc->abstand_punkte[2 * e], j = sc->abstand_punkte[2 * e + 1];
    if (sc->abstand_ruhe[e] != 0.0 || i == j) continue;
    if (std::find(partner[i].begin(), partner[i].end(), j) == partner[i].end()) partner[i].push_back(j);
    if (std::find(partner[j].begin(), partner[j].end(), i) == partner[j].end()) partner[j].push_back(i);
  }
  std::vector<uint32_t> np_off(n + 1, 0), np_ent;
  for (int64_t i = 0; i < n; ++i) {
    np_off[i + 1] = np_off[i] + uint32_t(partner[i].size());
    np_ent.insert(np_ent.end(), partner[i].begin(), partner[i].end());
  }
  // parts, bands, stretch stiffness and areas (selbstkollision.rs:648-680)
  std::vector<uint32_t> teil_von(n, kKein), band_von(n, kKein);
  std::vector<double> e_punkt(n, 0.0), e_dreieck(nd, 0.0), a_dreieck(nd), a_punkt(n, 0.0);
  s.has_band = 0;
  for (int64_t ti = 0; ti < sc->n_teile; ++ti) {
    const int64_t* b = sc->teil_bereiche + 4 * ti;
    const int32_t bv = sc->teil_band_von ? sc->teil_band_von[ti] : -1;
    for (int64_t i = std::max<int64_t>(b[0], 0); i < std::min(b[1], n); ++i) {
      teil_von[i] = uint32_t(ti);
      e_punkt[i] = sc->teil_dehnung[ti];
      if (bv >= 0) {
        band_von[i] = uint32_t(bv);
        s.has_band = 1;
      }
    }
    for (int64_t d = std::max<int64_t>(b[2], 0); d < std::min(b[3], nd); ++d) e_dreieck[d] = sc->teil_dehnung[ti];
  }
  for (int64_t t = 0; t < nd; ++t) {
    const double* m = sc->ruhe_inv + 4 * t;
    a_dreieck[t] = 0.5 / std::fmax(std::fabs(m[0] * m[3] - m[1] * m[2]), 1e-30);
  }
  for (int64_t t = 0; t < nd; ++t)
    for (int k = 0; k < 3; ++k) a_punkt[sc->dreiecke[3 * t + k]] += a_dreieck[t] / 3.0;
  std::vector<double> a_kante(ne), e_kante(ne);
  for (int64_t e = 0; e < ne; ++e) {
    double sa = 0.0, se = 0.0;
    int cnt = 0;
    for (uint32_t t : {k_dr[e].x, k_dr[e].y})
      if (t != kKein) {
        sa += a_dreieck[t];
        se += e_dreieck[t];
        ++cnt;
      }
    const double k = double(std::max(cnt, 1));
    a_kante[e] = sa / k;
    e_kante[e] = se / k;
  }
  std::vector<std::vector<uint2>> wp(n);
  for (int64_t c = 0; c < sc->n_naht; ++c) {
    const uint32_t i = sc->naht_punkte[2 * c], j = sc->naht_punkte[2 * c + 1];
    wp[i].push_back(make_uint2(j, uint32_t(c)));
    wp[j].push_back(make_uint2(i, uint32_t(c)));
  }
  std::vector<uint32_t> wp_off(n + 1, 0);
  std::vector<uint2> wp_ent;
  for (int64_t i = 0; i < n; ++i) {
    wp_off[i + 1] = wp_off[i] + uint32_t(wp[i].size());
    wp_ent.insert(wp_ent.end(), wp[i].begin(), wp[i].end());
  }
  H.naht_ruhe.assign(sc->naht_ruhe, sc->naht_ruhe + sc->n_naht);
  std::vector<double> dicke(sc->kollisionsabstand, sc->kollisionsabstand + n);

  cudaError_t e;
#define SC_UP(field, vec)                                          \
  do {                                                             \
    if ((e = up(field, vec, H.fest, st)) != cudaSuccess) return e; \
  } while (0)
  uint4 *di, *dk;
  uint2 *ki, *kd, *we;
  double *rp, *rk, *rd, *ep, *ap, *ek, *ak, *ed, *ad, *dc, *nr;
  uint32_t *npo, *npe, *tv, *bv, *wo;
  SC_UP(di, d_idx);
  SC_UP(dk, d_kan);
  SC_UP(ki, k_idx);
  SC_UP(kd, k_dr);
  SC_UP(rp, r);
  SC_UP(rk, r_kante);
  SC_UP(rd, r_dreieck);
  SC_UP(npo, np_off);
  SC_UP(npe, np_ent);
  SC_UP(tv, teil_von);
  SC_UP(bv, band_von);
  SC_UP(dc, dicke);
  SC_UP(ep, e_punkt);
  SC_UP(ap, a_punkt);
  SC_UP(ek, e_kante);
  SC_UP(ak, a_kante);
  SC_UP(ed, e_dreieck);
  SC_UP(ad, a_dreieck);
  SC_UP(wo, wp_off);
  SC_UP(we, wp_ent);
  SC_UP(nr, H.naht_ruhe);
#undef SC_UP
  s.d_idx = di;
  s.d_kan = dk;
  s.k_idx = ki;
  s.k_dr = kd;
  s.r_punkt = rp;
  s.r_kante = rk;
  s.r_dreieck = rd;
  s.np_off = npo;
  s.np_ent = npe;
  s.teil_von = tv;
  s.band_von = bv;
  s.dicke = dc;
  s.e_punkt = ep;
  s.a_punkt = ap;
  s.e_kante = ek;
  s.a_kante = ak;
  s.e_dreieck = ed;
  s.a_dreieck = ad;
  s.wp_off = wo;
  s.wp_ent = we;
  s.naht_ruhe = nr;
  H.naht_ruhe_dev = nr;

  // per-run arrays of fixed size
  if ((e = alloc(s.nrm_t, size_t(nd), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.keb, size_t(ne), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.qp_lo, size_t(n), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.qp_hi, size_t(n), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.qk_lo, size_t(ne), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.qk_hi, size_t(ne), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.anf_p, size_t(s.eimer_p) + 1, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.cur_p, size_t(s.eimer_p), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.anf_k, size_t(s.eimer_k) + 1, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.cur_k, size_t(s.eimer_k), H.fest)) != cudaSuccess) return e;
  // a point box spans at most two cells per axis (its extent is at most half
  // a cell), so 8 buckets per point bound the point hash
  s.cap_ep = uint32_t(std::min<int64_t>(8 * std::max<int64_t>(n, 1), int64_t(0xffffffffu)));
  if ((e = alloc(s.ein_p, size_t(s.cap_ep), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.ebp_lo, size_t(s.cap_ep), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.ebp_hi, size_t(s.cap_ep), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.off_t, size_t(nd) + 1, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.off_e, size_t(ne) + 1, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.aktiv_p, size_t(nd) + size_t(ne) + 1, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.inc_off, size_t(n) + 1, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.inc_cur, size_t(n), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.zahl, size_t(SZ_COUNT), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.slot_of, size_t(n), H.fest)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(s.slot_of, 0xff, sizeof(int32_t) * std::max<size_t>(size_t(n), 1), st)) != cudaSuccess)
    return e;
  // penetration regions: the triangle hash (a triangle box spans at most
  // three cells per axis: its extent is at most the cell, the longest edge,
  // plus the margin), per edge and per triangle lists, the fold counts
  s.hs.m = nd;
  s.hs.eimer = uint32_t(std::max<int64_t>(2 * nd, 64));
  s.hs.cap = uint32_t(std::min<int64_t>(27 * std::max<int64_t>(nd, 1), int64_t(0xffffffffu)));
  if ((e = alloc(s.hs.lo, size_t(nd), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.hs.hi, size_t(nd), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.hs.anf, size_t(s.hs.eimer) + 1, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.hs.cur, size_t(s.hs.eimer), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.hs.ein, size_t(s.hs.cap), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.hs.elo, size_t(s.hs.cap), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.hs.ehi, size_t(s.hs.cap), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.lmax, 2, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.off_s, size_t(ne) + 1, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.aktiv_s, size_t(ne) + 1, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.t_off, size_t(nd) + 1, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.t_cur, size_t(nd), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.hat, size_t(nd), H.fest)) != cudaSuccess) return e;
  {
    std::vector<uint32_t> eins(size_t(std::max<int64_t>(nd, 1)), 1u);
    if ((e = up(s.folge, eins, H.fest, st)) != cudaSuccess) return e;
  }
  // impacts: path hashes (entries sized per run), per triangle and edge slots
  s.hp2.m = n;
  s.hp2.eimer = uint32_t(std::max<int64_t>(2 * n, 64));
  s.hk2.m = ne;
  s.hk2.eimer = uint32_t(std::max<int64_t>(2 * ne, 64));
  if ((e = alloc(s.hp2.lo, size_t(n), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.hp2.hi, size_t(n), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.hp2.anf, size_t(s.hp2.eimer) + 1, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.hp2.cur, size_t(s.hp2.eimer), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.hk2.lo, size_t(ne), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.hk2.hi, size_t(ne), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.hk2.anf, size_t(s.hk2.eimer) + 1, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.hk2.cur, size_t(s.hk2.eimer), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.qt2_lo, size_t(nd), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.qt2_hi, size_t(nd), H.fest)) != cudaSuccess) return e;
  const size_t slots = size_t(nd + ne);
  if ((e = alloc(s.st_art, slots, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.st_idx, slots, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.st_lzs, slots, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.st_n, slots, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.st_off, slots + 1, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.schwer_pd, size_t(std::max<int64_t>(nd, 1)), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.schwer_kk, size_t(std::max<int64_t>(ne, 1)), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.im, slots, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.im_off, size_t(n) + 1, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.im_cur, size_t(n), H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.im_ent, 4 * slots, H.fest)) != cudaSuccess) return e;
  if ((e = alloc(s.im_c, 4 * slots, H.fest)) != cudaSuccess) return e;
  double* x0 = nullptr;
  if ((e = alloc(x0, 3 * size_t(n), H.fest)) != cudaSuccess) return e;
  s.x0 = x0;
  H.x0 = x0;
  Body* bd = nullptr;
  if ((e = alloc(bd, size_t(kMaxBodies), H.fest)) != cudaSuccess) return e;
  s.bodies = bd;
  H.bodies_dev = bd;
  if ((e = alloc(H.acc, 3, H.fest)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(H.acc, 0, 3 * sizeof(unsigned long long), st)) != cudaSuccess) return e;
  const int64_t longest = std::max({int64_t(s.eimer_p) + 1, int64_t(s.eimer_k) + 1, nd + 1, ne + 1, n + 1,
                                    int64_t(s.hs.eimer) + 1, int64_t(s.hp2.eimer) + 1, int64_t(s.hk2.eimer) + 1,
                                    nd + ne + 1});
  if ((e = alloc(s.scan_tmp, selbst_scan_tmp_words(longest), H.fest)) != cudaSuccess) return e;
  if ((e = selbst_grow_schnitte(H, 1024)) != cudaSuccess) return e;
  if ((e = selbst_grow_wege(H, uint32_t(std::min<int64_t>(8 * std::max<int64_t>(n, 1), 0x7fffffff)),
                            uint32_t(std::min<int64_t>(8 * std::max<int64_t>(ne, 1), 0x7fffffff)))) != cudaSuccess)
    return e;
  if ((e = selbst_grow_edge_hash(H, uint32_t(std::min<int64_t>(27 * std::max<int64_t>(ne, 1), 0x7fffffff)))) !=
      cudaSuccess)
    return e;
  if ((e = selbst_grow_pairs(H, uint32_t(std::min<int64_t>(std::max<int64_t>(n, 1024), 0x3fffffff)))) !=
      cudaSuccess)
    return e;
  H.on = true;
  return cudaStreamSynchronize(st);
}

cudaError_t selbst_grow_schnitte(SelbstHost& H, uint32_t cap) {
  free_all(H.schn);
  SelbstArgs& s = H.s;
  s.cap_s = cap;
  cudaError_t e;
  if ((e = alloc(s.sn_ke, cap, H.schn)) != cudaSuccess) return e;
  if ((e = alloc(s.sn_t, cap, H.schn)) != cudaSuccess) return e;
  if ((e = alloc(s.sn_w, cap, H.schn)) != cudaSuccess) return e;
  if ((e = alloc(s.sn_g, cap, H.schn)) != cudaSuccess) return e;
  if ((e = alloc(s.sn_wurzel, cap, H.schn)) != cudaSuccess) return e;
  if ((e = alloc(s.sn_eltern, cap, H.schn)) != cudaSuccess) return e;
  if ((e = alloc(s.sn_partner, cap, H.schn)) != cudaSuccess) return e;
  if ((e = alloc(s.sn_sp, size_t(cap) + 1, H.schn)) != cudaSuccess) return e;
  if ((e = alloc(s.sn_tausch, 6 * size_t(cap), H.schn)) != cudaSuccess) return e;
  if ((e = alloc(s.sn_toff, size_t(cap) + 1, H.schn)) != cudaSuccess) return e;
  if ((e = alloc(s.sn_scan_tmp, selbst_scan_tmp_words(int64_t(cap) + 1), H.schn)) != cudaSuccess) return e;
  if ((e = alloc(s.sn_summe, cap, H.schn)) != cudaSuccess) return e;
  if ((e = alloc(s.klemm, cap, H.schn)) != cudaSuccess) return e;
  return alloc(s.t_ent, cap, H.schn);
}

cudaError_t selbst_grow_wege(SelbstHost& H, uint32_t cap_p, uint32_t cap_k) {
  free_all(H.wege);
  cudaError_t e;
  H.s.hp2.cap = cap_p;
  H.s.hk2.cap = cap_k;
  if ((e = alloc(H.s.hp2.ein, size_t(cap_p), H.wege)) != cudaSuccess) return e;
  if ((e = alloc(H.s.hp2.elo, size_t(cap_p), H.wege)) != cudaSuccess) return e;
  if ((e = alloc(H.s.hp2.ehi, size_t(cap_p), H.wege)) != cudaSuccess) return e;
  if ((e = alloc(H.s.hk2.elo, size_t(cap_k), H.wege)) != cudaSuccess) return e;
  if ((e = alloc(H.s.hk2.ehi, size_t(cap_k), H.wege)) != cudaSuccess) return e;
  return alloc(H.s.hk2.ein, size_t(cap_k), H.wege);
}

cudaError_t selbst_grow_edge_hash(SelbstHost& H, uint32_t cap) {
  free_all(H.hashk);
  H.s.cap_ek = cap;
  cudaError_t e;
  if ((e = alloc(H.s.ebk_lo, size_t(cap), H.hashk)) != cudaSuccess) return e;
  if ((e = alloc(H.s.ebk_hi, size_t(cap), H.hashk)) != cudaSuccess) return e;
  return alloc(H.s.ein_k, size_t(cap), H.hashk);
}

cudaError_t selbst_grow_pairs(SelbstHost& H, uint32_t cap) {
  free_all(H.pairs);
  SelbstArgs& s = H.s;
  s.cap_pairs = cap;
  s.cap_inc = 5u * cap;
  cudaError_t e;
  if ((e = alloc(s.pr_idx, cap, H.pairs)) != cudaSuccess) return e;
  if ((e = alloc(s.pr_src, cap, H.pairs)) != cudaSuccess) return e;
  if ((e = alloc(s.pr_w, cap, H.pairs)) != cudaSuccess) return e;
  if ((e = alloc(s.pr_nab, cap, H.pairs)) != cudaSuccess) return e;
  if ((e = alloc(s.pr_ruhe, cap, H.pairs)) != cudaSuccess) return e;
  if ((e = alloc(s.pr_kf, cap, H.pairs)) != cudaSuccess) return e;
  if ((e = alloc(s.pr_b0, cap, H.pairs)) != cudaSuccess) return e;
  if ((e = alloc(s.pr_b1, cap, H.pairs)) != cudaSuccess) return e;
  if ((e = alloc(s.pr_ga, cap, H.pairs)) != cudaSuccess) return e;
  char* bR = nullptr;
  if ((e = alloc(bR, size_t(cap) * 8 * size_t(s.rsize), H.pairs)) != cudaSuccess) return e;
  s.pr_bR = bR;
  char* wR = nullptr;
  if ((e = alloc(wR, size_t(cap) * 4 * size_t(s.rsize), H.pairs)) != cudaSuccess) return e;
  s.pr_wR = wR;
  if ((e = alloc(s.pr_x5, cap, H.pairs)) != cudaSuccess) return e;
  if ((e = alloc(s.pr_g5, cap, H.pairs)) != cudaSuccess) return e;
  char* g5R = nullptr;
  if ((e = alloc(g5R, size_t(cap) * size_t(s.rsize), H.pairs)) != cudaSuccess) return e;
  s.pr_g5R = g5R;
  if ((e = alloc(s.inc_pos, size_t(8) * cap, H.pairs)) != cudaSuccess) return e;
  // the per-entry products are in the PCG's vector precision, which is FP64
  // also where the operator copies are FP32 (K3D_MIXED_STORAGE)
  char* out = nullptr;
  if ((e = alloc(out, size_t(s.cap_inc) * 4 * sizeof(double), H.pairs)) != cudaSuccess) return e;
  s.inc_out = out;
  return alloc(s.inc_ent, size_t(s.cap_inc), H.pairs);
}

cudaError_t selbst_set_naht_ruhe(SelbstHost& H, const double* ruhe, int64_t n_naht, cudaStream_t st) {
  if (!H.on || n_naht != int64_t(H.naht_ruhe.size()) || n_naht == 0 || !ruhe) return cudaSuccess;
  if (std::memcmp(H.naht_ruhe.data(), ruhe, sizeof(double) * size_t(n_naht)) == 0) return cudaSuccess;
  H.naht_ruhe.assign(ruhe, ruhe + n_naht);
  return cudaMemcpyAsync(H.naht_ruhe_dev, H.naht_ruhe.data(), sizeof(double) * size_t(n_naht),
                         cudaMemcpyHostToDevice, st);
}

cudaError_t selbst_run(SelbstHost& H, double h, cudaStream_t st, int& launches) {
  SelbstArgs& s = H.s;
  s.h = h;
  cudaError_t e;
  uint32_t z[SZ_COUNT];
  if ((e = cudaMemsetAsync(s.anf_p, 0, sizeof(uint32_t) * (size_t(s.eimer_p) + 1), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(s.anf_k, 0, sizeof(uint32_t) * (size_t(s.eimer_k) + 1), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(s.cur_p, 0, sizeof(uint32_t) * size_t(s.eimer_p), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(s.cur_k, 0, sizeof(uint32_t) * size_t(s.eimer_k), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(s.zahl, 0, sizeof(uint32_t) * SZ_COUNT, st)) != cudaSuccess) return e;
  if ((e = selbst_hash_zaehlen(s, st)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(z, s.zahl, sizeof(z), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  if (z[SZ_HASH_P] > s.cap_ep) return cudaErrorInvalidValue;  // cannot happen: 8 buckets per point box
  if (z[SZ_HASH_K] > s.cap_ek) {
    const uint64_t want = uint64_t(z[SZ_HASH_K]) + z[SZ_HASH_K] / 2 + 1024;
    if ((e = selbst_grow_edge_hash(H, uint32_t(std::min<uint64_t>(want, 0xffffffffu)))) != cudaSuccess) return e;
  }
  if ((e = cudaMemsetAsync(s.lmax, 0, 2 * sizeof(unsigned long long), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(s.hs.anf, 0, sizeof(uint32_t) * (size_t(s.hs.eimer) + 1), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(s.hs.cur, 0, sizeof(uint32_t) * size_t(s.hs.eimer), st)) != cudaSuccess) return e;
  if ((e = selbst_hash_fuellen_und_paare_zaehlen(s, st)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(z, s.zahl, sizeof(z), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  if (z[SZ_HASH_S] > s.hs.cap) return cudaErrorInvalidValue;  // cannot happen: 27 buckets per triangle box
  const uint32_t n_s = z[SZ_SCHNITTE];
  if (n_s > s.cap_s) {
    const uint64_t want = uint64_t(n_s) + n_s / 2 + 1024;
    if (want > 0x0fffffffu) return cudaErrorMemoryAllocation;
    if ((e = selbst_grow_schnitte(H, uint32_t(want))) != cudaSuccess) return e;
  }
  // the proximity pairs, then one push spring per intersection
  const uint64_t paare = uint64_t(z[SZ_PAARE_PT]) + z[SZ_PAARE_KK], federn = paare + n_s;
  if (federn > s.cap_pairs) {
    const uint64_t want = federn + federn / 2 + 1024;
    if (want > 0x1fffffffu) return cudaErrorMemoryAllocation;
    if ((e = selbst_grow_pairs(H, uint32_t(want))) != cudaSuccess) return e;
  }
  if ((e = cudaMemsetAsync(s.inc_off, 0, sizeof(uint32_t) * (size_t(s.n) + 1), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(s.inc_cur, 0, sizeof(uint32_t) * size_t(s.n), st)) != cudaSuccess) return e;
  if (federn > 0 && (e = cudaMemsetAsync(s.inc_pos, 0xff, sizeof(uint32_t) * 8 * size_t(federn), st)) != cudaSuccess)
    return e;
  if ((e = cudaMemsetAsync(s.hat, 0, size_t(std::max<int64_t>(s.nd, 1)), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(s.klemm, 0, size_t(s.cap_s), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(s.t_off, 0, sizeof(uint32_t) * (size_t(s.nd) + 1), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(s.t_cur, 0, sizeof(uint32_t) * size_t(std::max<int64_t>(s.nd, 1)), st)) != cudaSuccess)
    return e;
  if ((e = selbst_paare_und_federn(s, z[SZ_AKTIV_P], z[SZ_AKTIV_S], n_s, st)) != cudaSuccess) return e;
  H.n_pt = z[SZ_PAARE_PT];
  H.n_kk = z[SZ_PAARE_KK];
  H.n_s = n_s;
  H.naehe_pt += z[SZ_PAARE_PT];
  H.naehe_kk += z[SZ_PAARE_KK];
  H.ran = true;
  launches += selbst_launches_per_run();
  return cudaSuccess;
}

cudaError_t selbst_stoss_run(SelbstHost& H, double* x, const double* nrm_fest, int iterationen, cudaStream_t st,
                            int& launches) {
  if (!H.on) return cudaSuccess;
  SelbstArgs& s = H.s;
  s.xs = x;
  s.nrm_fest = nrm_fest;
  cudaError_t e;
  if ((e = cudaMemsetAsync(&s.lmax[1], 0, sizeof(unsigned long long), st)) != cudaSuccess) return e;
  for (HashG* g : {&s.hp2, &s.hk2}) {
    if ((e = cudaMemsetAsync(g->anf, 0, sizeof(uint32_t) * (size_t(g->eimer) + 1), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(g->cur, 0, sizeof(uint32_t) * size_t(g->eimer), st)) != cudaSuccess) return e;
  }
  if ((e = selbst_stoss_zaehlen(s, st)) != cudaSuccess) return e;
  uint32_t z[SZ_COUNT];
  if ((e = cudaMemcpyAsync(z, s.zahl, sizeof(z), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  if (z[SZ_HASH_P2] > s.hp2.cap || z[SZ_HASH_K2] > s.hk2.cap) {
    const uint64_t wp = std::max<uint64_t>(s.hp2.cap, uint64_t(z[SZ_HASH_P2]) + z[SZ_HASH_P2] / 2 + 1024);
    const uint64_t wk = std::max<uint64_t>(s.hk2.cap, uint64_t(z[SZ_HASH_K2]) + z[SZ_HASH_K2] / 2 + 1024);
    if (wp > 0x7fffffffu || wk > 0x7fffffffu) return cudaErrorMemoryAllocation;
    if ((e = selbst_grow_wege(H, uint32_t(wp), uint32_t(wk))) != cudaSuccess) return e;
  }
  if ((e = cudaMemsetAsync(s.im_off, 0, sizeof(uint32_t) * (size_t(s.n) + 1), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(s.im_cur, 0, sizeof(uint32_t) * size_t(s.n), st)) != cudaSuccess) return e;
  if ((e = selbst_stoss_antwort(s, iterationen, H.acc, st)) != cudaSuccess) return e;
  launches += selbst_stoss_launches(iterationen);
  return cudaSuccess;
}

void selbst_step_args(const SelbstHost& H, StepArgs& a) {
  if (!H.on) {
    a.sc_off = a.sc_ent = a.sc_pos = nullptr;
    a.sc_idx = nullptr;
    a.sc_w = a.sc_kf = a.sc_b0 = a.sc_b1 = nullptr;
    a.sc_bR = a.sc_wR = nullptr;
    a.sc_out = nullptr;
    a.sc_np = 0;
    a.sc_x5 = nullptr;
    a.sc_g5 = nullptr;
    a.sc_g5R = nullptr;
    return;
  }
  const SelbstArgs& s = H.s;
  a.sc_off = s.inc_off;
  a.sc_ent = s.inc_ent;
  a.sc_idx = s.pr_idx;
  a.sc_w = s.pr_w;
  a.sc_kf = s.pr_kf;
  a.sc_b0 = s.pr_b0;
  a.sc_b1 = s.pr_b1;
  a.sc_bR = s.pr_bR;
  a.sc_wR = s.pr_wR;
  a.sc_pos = s.inc_pos;
  a.sc_out = s.inc_out;
  a.sc_x5 = s.pr_x5;
  a.sc_g5 = s.pr_g5;
  a.sc_g5R = s.pr_g5R;
  a.sc_np = std::min<uint32_t>(H.n_pt + H.n_kk + H.n_s, s.cap_pairs);
}

}  // namespace k3d
