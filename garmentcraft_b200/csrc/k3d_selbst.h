// Cloth self-collision, proximity stage (sim/src/selbstkollision.rs:41-801),
// on the device: normals, the two spatial hashes, the point-triangle and
// edge-edge searches, the proximity springs and their approach damping, and
// the per-point incidence lists through which the springs enter the system
// (internal to the library).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "k3d_device.cuh"

namespace k3d {

constexpr uint32_t kKein = 0xffffffffu;  // no triangle / no part

// device counters of one stage run
enum SelbstZahl : int {
  SZ_HASH_P = 0,    // entries of the point hash
  SZ_HASH_K = 1,    // entries of the edge hash
  SZ_PAARE_PT = 2,  // point-triangle pairs
  SZ_PAARE_KK = 3,  // edge-edge pairs
  SZ_INZIDENZ = 4,  // incidence entries
  SZ_SCHUB = 5,     // push springs of the penetration regions, after the pairs
  SZ_SCHNITTE = 6,  // edges through triangles
  SZ_GEBIETE = 7,   // their regions
  SZ_HASH_S = 8,    // entries of the triangle hash of the intersection search
  SZ_HASH_P2 = 9,   // entries of the point-path hash of the impact search
  SZ_HASH_K2 = 10,  // entries of the edge-path hash
  SZ_STOSS = 11,    // impacts kept for the response
  SZ_ANTWORT = 12,  // impact corrections applied (ImplizitStatistik::selbst_stoesse)
  SZ_BEWEGT = 13,   // points moved by the last response pass
  SZ_HALT = 14,     // set when a response pass moved no point (the passes stop)
  SZ_AKTIV_P = 15,  // triangles and edges with proximity pairs (the fill pass's list)
  SZ_AKTIV_S = 16,  // edges through a triangle (the intersection fill pass's list)
  SZ_SCHWER_PD = 17,  // triangles whose impact search runs one warp each (many candidates)
  SZ_SCHWER_KK = 18,  // edges likewise
  SZ_ARBEIT_P = 19,   // the proximity count pass's next item (triangles, then nd + edges)
  SZ_ARBEIT_S = 20,   // the intersection count pass's next edge
  SZ_ARBEIT_PD = 21,  // the heavy point-triangle impact search's next list entry
  SZ_ARBEIT_KK = 22,  // the heavy edge-edge impact search's next list entry
  SZ_COUNT = 24
};

// A spatial hash over boxes (Hashgitter, selbstkollision.rs:281-345): the
// boxes, bucket starts (eimer + 1), entries (cap), fill cursors.
struct HashG {
  double4 *lo, *hi;
  int64_t m;
  uint32_t eimer, cap;
  uint32_t *anf, *ein, *cur;
  float4 *elo, *ehi;  // per entry its box in FP32, rounded outward (a search's pre-test; null: none)
};

struct SelbstArgs {
  int64_t n, nd, ne;   // points, triangles, edges
  double zelle;        // hash cell edge (selbstkollision.rs:402)
  uint32_t eimer_p, eimer_k;
  int has_band;        // any folded allowance band in the scene
  int rsize;           // operator precision (4 or 8)
  double h;            // substep
  double steifigkeit;  // ImplizitParameter::selbst_steifigkeit
  // mesh (Stoffnetz::neu, selbstkollision.rs:159-187)
  const uint4* d_idx;  // triangle points
  const uint4* d_kan;  // triangle edges (edge k runs from point k to k+1)
  const uint2* k_idx;  // edge points (smaller, larger)
  const uint2* k_dr;   // up to two triangles per edge, kKein = none
  const double *r_punkt, *r_kante, *r_dreieck;
  const uint32_t *np_off, *np_ent;  // seam and weld partners per point
  const uint32_t *teil_von, *band_von;
  const double* dicke;
  // spring values (Stoffwerte, selbstkollision.rs:623-688)
  const double *e_punkt, *a_punkt, *e_kante, *a_kante, *e_dreieck, *a_dreieck, *mu;
  const uint32_t* wp_off;
  const uint2* wp_ent;      // (partner, seam)
  const double* naht_ruhe;  // per seam
  // state
  const double* x;
  double* v;
  const double *masse, *w;
  // per run
  double4 *nrm_t, *keb;                    // triangle normals, edge planes
  double4 *qp_lo, *qp_hi, *qk_lo, *qk_hi;  // point and edge boxes
  uint32_t *anf_p, *ein_p, *cur_p;         // point hash: starts (eimer+1), entries, fill cursors
  uint32_t *anf_k, *ein_k, *cur_k;         // edge hash
  float4 *ebp_lo, *ebp_hi, *ebk_lo, *ebk_hi;  // per entry of the point / edge hash its box in FP32, rounded outward
  uint32_t cap_ep, cap_ek;
  uint32_t *off_t, *off_e;  // pair counts -> starts per triangle / edge (n + 1)
  uint32_t* aktiv_p;        // triangles (t) and edges (nd + e) with pairs, in no order (nd + ne)
  uint32_t cap_pairs;
  uint4* pr_idx;           // 4 points
  uint2* pr_src;           // triangle (point-triangle) or the two edges (edge-edge)
  double4* pr_w;           // weights
  double4* pr_nab;         // normal, distance
  double* pr_ruhe;         // rest distance as found
  double4* pr_kf;          // force on the first side, k
  double4 *pr_b0, *pr_b1;  // block k[(1-mu) n n^T + mu I]: (xx, yy, zz, xy), (xz, yz, mu, m1 + m2 > 0)
  double4* pr_ga;          // per slot g * (mass share of the other side), the damping's update factor
  void* pr_bR;             // h^2 * block in operator precision, 2 R4 per pair
  void* pr_wR;             // weights in operator precision, R4 per pair
  // a fifth point per spring (the push springs of penetration regions join
  // an edge to a triangle; kKein and weight 0 for the proximity pairs)
  uint32_t* pr_x5;
  double* pr_g5;
  void* pr_g5R;                           // in operator precision
  uint32_t *inc_off, *inc_cur, *inc_ent;  // per point: (spring << 3 | slot)
  uint32_t cap_inc;
  uint32_t* inc_pos;  // per (spring << 3 | slot): its entry index, all ones for a zero weight
  void* inc_out;      // per entry: the PCG's spring product of that slot, R4
  int32_t* slot_of;  // damping scratch per point: its shared-memory slot, -1 between batches
  uint32_t* zahl;    // SZ_COUNT counters
  uint32_t* scan_tmp;

  // ---- penetration regions (selbstkollision.rs:810-1058)
  int an_naehten;                 // ImplizitParameter::selbst_schnitte_an_naehten
  unsigned long long* lmax;       // 2: the longest edge (as bits) at x and at the impact stage's x1
  HashG hs;                       // triangle boxes
  uint32_t* off_s;                // per edge: its intersections' count, then start (ne + 1)
  uint32_t* aktiv_s;              // edges with intersections, in no order (ne)
  uint32_t cap_s;
  uint2* sn_ke;                   // per intersection: edge, triangle
  double* sn_t;                   // position on the edge
  double4* sn_w;                  // triangle weights
  double4* sn_g;                  // direction (xyz) and weight
  uint32_t *sn_wurzel, *sn_eltern, *sn_partner, *sn_sp;  // regions; push-spring slots (cap_s + 1)
  uint2* sn_tausch;               // role swaps (6 per intersection at most)
  uint32_t* sn_toff;              // role swaps per intersection, then their starts (cap_s + 1)
  uint32_t* sn_scan_tmp;          // scan scratch for sn_toff
  double4* sn_summe;
  uint32_t *t_off, *t_cur, *t_ent;  // per triangle: its intersections (nd + 1)
  uint8_t *hat, *klemm;           // per triangle; per region root
  uint32_t* folge;                // per triangle: steps in a row with an edge through it (kept)
  const Body* bodies;             // for the pinch test (first body in contact)
  int n_bodies;
  const double* kabst;
  double rand;
  // ---- impacts (selbstkollision.rs:1063-1343)
  const double* x0;               // the positions at the start of the substep
  double* xs;                     // the positions the response moves (the step's x)
  const double* nrm_fest;         // held points (nonzero normal) weigh 1e9 times their mass
  int iterationen;
  HashG hp2, hk2;                 // point paths, edge paths
  double4 *qt2_lo, *qt2_hi;       // triangle paths
  // the earliest impact per triangle (slots 0..nd) and per edge (nd..nd+ne)
  uint32_t* st_art;               // 0 none, 1 point-triangle, 2 edge-edge
  uint4* st_idx;
  double4* st_lzs;                // lage (2), zeit, seite
  double4* st_n;                  // normal (edge-edge)
  uint32_t* st_off;               // kept impacts: count, then start (nd + ne + 1)
  uint32_t *schwer_pd, *schwer_kk;  // triangles / edges with many candidates, in no order (nd / ne)
  uint32_t* im;                   // the kept impacts' slots in order
  uint32_t *im_off, *im_cur, *im_ent;  // per point: (impact << 2 | slot) (n + 1)
  double4* im_c;                  // per (impact, slot): the correction, w = 1 if it applies
};

// The stage in three parts with host reads of the counters between them
// (the host sizes the hash and pair buffers from the counts).
cudaError_t selbst_hash_zaehlen(const SelbstArgs& s, cudaStream_t st);
cudaError_t selbst_hash_fuellen_und_paare_zaehlen(const SelbstArgs& s, cudaStream_t st);
// n_aktiv_p, n_aktiv_s: the fill lists' lengths (counters SZ_AKTIV_P, SZ_AKTIV_S)
// n_s: the intersections (counter SZ_SCHNITTE, at most cap_s)
cudaError_t selbst_paare_und_federn(const SelbstArgs& s, uint32_t n_aktiv_p, uint32_t n_aktiv_s, uint32_t n_s,
                                    cudaStream_t st);
int selbst_launches_per_run();
// Impacts after the step's integration, in two parts with a host read of the
// path hashes' entry counts between them.
cudaError_t selbst_stoss_zaehlen(const SelbstArgs& s, cudaStream_t st);
cudaError_t selbst_stoss_antwort(const SelbstArgs& s, int iterationen, unsigned long long* acc, cudaStream_t st);
int selbst_stoss_launches(int iterationen);
size_t selbst_scan_tmp_words(int64_t n);
// Exclusive prefix sum of n uint32 in place (3 launches); tmp holds
// selbst_scan_tmp_words(n) words; `total` (device, may be null) gets the sum.
cudaError_t exclusive_scan_u32(uint32_t* data, int64_t n, uint32_t* tmp, uint32_t* total, cudaStream_t st);

}  // namespace k3d
