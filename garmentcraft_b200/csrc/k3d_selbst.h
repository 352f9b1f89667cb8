// Cloth self-collision, proximity stage (sim/src/selbstkollision.rs:41-801),
// on the device: normals, the two spatial hashes, the point-triangle and
// edge-edge searches, the proximity springs and their approach damping, and
// the per-point incidence lists through which the springs enter the system
// (internal to the library).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace k3d {

constexpr uint32_t kKein = 0xffffffffu;  // no triangle / no part

// device counters of one stage run
enum SelbstZahl : int {
  SZ_HASH_P = 0,    // entries of the point hash
  SZ_HASH_K = 1,    // entries of the edge hash
  SZ_PAARE_PT = 2,  // point-triangle pairs
  SZ_PAARE_KK = 3,  // edge-edge pairs
  SZ_INZIDENZ = 4,  // incidence entries
  SZ_COUNT = 8
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
  uint32_t cap_ep, cap_ek;
  uint32_t *off_t, *off_e;  // pair counts -> starts per triangle / edge (n + 1)
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
  uint32_t *inc_off, *inc_cur, *inc_ent;  // per point: (pair << 2 | slot)
  uint32_t cap_inc;
  uint32_t* inc_pos;  // per (pair << 2 | slot): its entry index, all ones for a zero weight
  void* inc_out;      // per entry: the PCG's spring product of that slot, R4
  int32_t* slot_of;  // damping scratch per point: its shared-memory slot, -1 between batches
  uint32_t* zahl;    // SZ_COUNT counters
  uint32_t* scan_tmp;
};

// The stage in three parts with host reads of the counters between them
// (the host sizes the hash and pair buffers from the counts).
cudaError_t selbst_hash_zaehlen(const SelbstArgs& s, cudaStream_t st);
cudaError_t selbst_hash_fuellen_und_paare_zaehlen(const SelbstArgs& s, cudaStream_t st);
cudaError_t selbst_paare_und_federn(const SelbstArgs& s, cudaStream_t st);
int selbst_launches_per_run();
size_t selbst_scan_tmp_words(int64_t n);

}  // namespace k3d
