// Cloth self-collision, proximity stage, on the device
// (sim/src/selbstkollision.rs:41-801; the stage is called from
// ImplizitCg::system_bauen, implizit.rs:668-691).
//
// This file is compiled with -fmad=false: every product and sum rounds on its
// own, as in the reference, so cell indices, bucket contents, the candidate
// pairs and their distances come out with the reference's bits.
//
// One run:
//   triangle normals; edge planes; point and edge boxes with their distinct
//   hash buckets counted                                  -> host reads sizes
//   bucket starts (scan), fill, entries sorted per bucket; pair counts per
//   triangle (point-triangle) and per edge (edge-edge)    -> host reads sizes
//   pairs written in the reference's order; springs per pair; the approach
//   damping in pair order; per-point incidence lists (pair, slot)
#include <cfloat>
#include <cstdint>

#include "k3d_device.cuh"
#include "k3d_selbst.h"

namespace k3d {
namespace {

constexpr int kT = 256;
constexpr double kZuschlagQuader = 2e-5;     // selbstkollision.rs:44
constexpr double kZuschlagPaar = 4e-5;       // :46
constexpr double kKanteMin = 1e-4;           // :48
constexpr double kAuslenkungMax = 2.5e-3;    // :606
constexpr double kAnnaeherung = 1.0 / 32.0;  // :608
constexpr int kCellCache = 64;

#define SC_FOR(i, n) \
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < int64_t(n); i += int64_t(gridDim.x) * blockDim.x)

// selbstkollision.rs:196-203
__device__ __forceinline__ D3 einheit(D3 a) {
  const double l = norm(a);
  if (l > 1e-12) return a * (1.0 / l);
  return d3(1.0, 0.0, 0.0);
}

// selbstkollision.rs:263-265: floor(x / zelle) as i64, saturating, NaN -> 0
__device__ __forceinline__ int64_t zellindex(double x, double zelle) {
  const double f = floor(x / zelle);
  if (isnan(f)) return 0;
  if (f >= 9223372036854775808.0) return INT64_MAX;
  if (f < -9223372036854775808.0) return INT64_MIN;
  return int64_t(f);
}

// selbstkollision.rs:274-278
__device__ __forceinline__ uint32_t streue(int64_t i, int64_t j, int64_t k, uint32_t n) {
  const uint32_t h = (uint32_t(i) * 0x8DA6B343u) ^ (uint32_t(j) * 0xD8163841u) ^ (uint32_t(k) * 0xCB1AB31Fu);
  return h % n;
}

struct Box {
  D3 lo, hi;
};
__device__ __forceinline__ Box box_of(const double4* lo, const double4* hi, int64_t i) {
  const double4 a = lo[i], b = hi[i];
  return {d3(a.x, a.y, a.z), d3(b.x, b.y, b.z)};
}
__device__ __forceinline__ double ax(D3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// selbstkollision.rs:270-272
__device__ __forceinline__ bool zellbereich_ok(const Box& q, double zelle) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double l = ax(q.lo, a), h = ax(q.hi, a);
    if (!(isfinite(l) && isfinite(h) && (h - l) <= 64.0 * zelle)) return false;
  }
  return true;
}

// The cell range of a box (both ends inclusive) and its cell count (each
// axis spans at most 66 cells once zellbereich_ok holds).
struct Cells {
  int64_t lo[3], hi[3];
  uint32_t n[3];
  uint32_t total;
};
__device__ __forceinline__ Cells cells_of(const Box& q, double zelle) {
  Cells c;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    c.lo[a] = zellindex(ax(q.lo, a), zelle);
    c.hi[a] = zellindex(ax(q.hi, a), zelle);
    c.n[a] = c.hi[a] >= c.lo[a] ? uint32_t(uint64_t(c.hi[a]) - uint64_t(c.lo[a]) + 1u) : 0u;
  }
  c.total = c.n[0] * c.n[1] * c.n[2];
  return c;
}
// cell number q in the reference's loop order (i outer, k inner)
__device__ __forceinline__ void cell_at(const Cells& c, uint32_t q, int64_t& i, int64_t& j, int64_t& k) {
  const uint32_t kk = q % c.n[2], r = q / c.n[2];
  const uint32_t jj = r % c.n[1], ii = r / c.n[1];
  i = int64_t(uint64_t(c.lo[0]) + ii);
  j = int64_t(uint64_t(c.lo[1]) + jj);
  k = int64_t(uint64_t(c.lo[2]) + kk);
}

// Calls f(bucket) once for every distinct bucket of the box's cells
// (selbstkollision.rs:284-303).
template <typename F>
__device__ void je_eimer(const Box& q, double zelle, uint32_t eimer, F&& f) {
  if (!zellbereich_ok(q, zelle)) return;
  const Cells c = cells_of(q, zelle);
  uint32_t cache[kCellCache];
  for (uint32_t a = 0; a < c.total; ++a) {
    int64_t i, j, k;
    cell_at(c, a, i, j, k);
    const uint32_t h = streue(i, j, k, eimer);
    bool first = true;
    if (c.total <= kCellCache) {
      for (uint32_t b = 0; b < a && first; ++b) first = cache[b] != h;
      cache[a] = h;
    } else {
      for (uint32_t b = 0; b < a && first; ++b) {
        int64_t i2, j2, k2;
        cell_at(c, b, i2, j2, k2);
        first = streue(i2, j2, k2, eimer) != h;
      }
    }
    if (first) f(h);
  }
}

// A box in FP32 rounded outward (lo down, hi up). Every search below tests
// ueberlappt(query, entry) in FP64 among its conditions; if the outward FP32
// boxes do not overlap, the FP64 ones do not either (lo32 <= lo and hi <= hi32),
// so a candidate that fails the FP32 test is skipped without loading its FP64
// box, and no result changes.
struct Box32 {
  float lx, ly, lz, hx, hy, hz;
};
__device__ __forceinline__ Box32 box32(const Box& b) {
  return {__double2float_rd(b.lo.x), __double2float_rd(b.lo.y), __double2float_rd(b.lo.z),
          __double2float_ru(b.hi.x), __double2float_ru(b.hi.y), __double2float_ru(b.hi.z)};
}
__device__ __forceinline__ bool ueberlappt32(const Box32& q, const float4& l, const float4& h) {
  return q.lx <= h.x && l.x <= q.hx && q.ly <= h.y && l.y <= q.hy && q.lz <= h.z && l.z <= q.hz;
}

// The entries s = a, a + st, ... < b of a bucket, in that order: f(ein[s], s)
// for those whose index passes `vor` and whose FP32 box overlaps q32. The
// indices of D entries are loaded, then the boxes of those that pass `vor`,
// before any of them is tested: the searches are bound by load latency, and
// several loads in flight per lane hide more of it than one.
template <int D, typename V, typename F>
__device__ __forceinline__ void je_ueberlappend(uint32_t a, uint32_t b, uint32_t st, const Box32& q32,
                                                const float4* elo, const float4* ehi, const uint32_t* ein, V&& vor,
                                                F&& f) {
  for (uint32_t s = a; s < b; s += uint32_t(D) * st) {
    uint32_t n[D];
    bool ok[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
      const uint32_t t = s + uint32_t(k) * st;
      n[k] = t < b ? __ldg(&ein[t]) : 0u;
      ok[k] = t < b && vor(n[k]);
    }
    unsigned m = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
      const uint32_t t = s + uint32_t(k) * st;
      if (ok[k] && ueberlappt32(q32, __ldg(&elo[t]), __ldg(&ehi[t]))) m |= 1u << k;
    }
    // the overlapping ones in order, through one call of f
    while (m != 0u) {
      const int k = __ffs(m) - 1;
      m &= m - 1u;
      uint32_t en = n[0];
#pragma unroll
      for (int q = 1; q < D; ++q)
        if (q == k) en = n[q];
      f(en, s + uint32_t(k) * st);
    }
  }
}

// selbstkollision.rs:328-344: f(entry, i, j, k, position) over the entries of
// the box's cells. With entry boxes (elo, ehi: FP32, entry order) an entry
// whose box misses q is skipped; without (null), every entry goes to f. The
// pre-test pays where the box test is the search's first condition; where a
// cheaper test on the entry's index comes first (edge against later edge), f
// makes the pre-test itself after that test, from the entry's position.
template <typename F>
__device__ void je_eintrag(const Box& q, double zelle, uint32_t eimer, const uint32_t* anf, const uint32_t* ein,
                           const float4* elo, const float4* ehi, F&& f) {
  if (!zellbereich_ok(q, zelle)) return;
  const Cells c = cells_of(q, zelle);
  const Box32 q32 = box32(q);
  for (uint32_t a = 0; a < c.total; ++a) {
    int64_t i, j, k;
    cell_at(c, a, i, j, k);
    const uint32_t h = streue(i, j, k, eimer);
    const uint32_t e1 = anf[h + 1];
    for (uint32_t s = anf[h]; s < e1; ++s)
      if (!elo || ueberlappt32(q32, elo[s], ehi[s])) f(ein[s], i, j, k, s);
  }
}

// je_eintrag for a group of kG lanes working on one item: the lanes take
// consecutive entries of each cell's bucket, in the reference's order; `pruefe`
// tests one entry (filling the payload), `schreibe` writes a hit at its
// position. The hits keep the order of the one-thread loop: within a chunk of
// kG entries a hit's rank is the number of hits on lower lanes. Returns the
// number of hits (the same on every lane of the group).
constexpr int kG = 8;
struct Gruppe {
  unsigned maske;  // the group's lanes within the warp
  int lane;        // this lane's index in the group
};
__device__ __forceinline__ Gruppe gruppe() {
  const int l = threadIdx.x & 31;
  return Gruppe{((1u << kG) - 1u) << (l & ~(kG - 1)), l & (kG - 1)};
}
template <bool FILL, typename Payload, typename T, typename W>
__device__ uint32_t je_eintrag_gruppe(const Gruppe& gr, const Box& q, double zelle, uint32_t eimer,
                                      const uint32_t* anf, const uint32_t* ein, const float4* elo, const float4* ehi,
                                      uint32_t pos, T&& pruefe, W&& schreibe) {
  if (!zellbereich_ok(q, zelle)) return 0;
  const Cells c = cells_of(q, zelle);
  const Box32 q32 = box32(q);
  const unsigned unter = gr.maske & ((1u << (threadIdx.x & 31)) - 1u);
  uint32_t cnt = 0;
  for (uint32_t a = 0; a < c.total; ++a) {
    int64_t i, j, k;
    cell_at(c, a, i, j, k);
    const uint32_t h = streue(i, j, k, eimer);
    const uint32_t lo = anf[h], hi = anf[h + 1];
    for (uint32_t b0 = lo; b0 < hi; b0 += kG) {
      const uint32_t e = b0 + uint32_t(gr.lane);
      Payload pl;
      const bool hit = e < hi && (!elo || ueberlappt32(q32, elo[e], ehi[e])) && pruefe(ein[e], i, j, k, e, pl);
      const unsigned b = __ballot_sync(gr.maske, hit);
      if (FILL && hit) schreibe(pl, pos + cnt + uint32_t(__popc(b & unter)));
      cnt += uint32_t(__popc(b));
    }
  }
  return cnt;
}

// The count of a query's hits for a count pass, the group's lanes over the
// query's cells: lane l takes cells l, l + kG, ... and walks each one's
// bucket itself, so a query whose box spans many cells is not walked cell by
// cell; a bucket of more than kGross entries is walked by the whole group
// (lanes over its entries) after its round. The same candidates as
// je_eintrag_gruppe, tested by the same predicate: a count needs no order.
// With VOR, the walks test an entry's index with `vor` before its FP32 box
// (elo, ehi) and keep several entries' loads in flight (je_ueberlappend).
constexpr uint32_t kGross = 32;
template <typename Payload, bool VOR = false, typename T, typename V = int>
__device__ uint32_t zaehle_gruppe(const Gruppe& gr, const Box& q, double zelle, uint32_t eimer, const uint32_t* anf,
                                  const uint32_t* ein, const float4* elo, const float4* ehi, T&& pruefe,
                                  V vor = V()) {
  if (!zellbereich_ok(q, zelle)) return 0;
  const Cells c = cells_of(q, zelle);
  const Box32 q32 = box32(q);
  uint32_t cnt = 0;
  for (uint32_t a0 = 0; a0 < c.total; a0 += kG) {
    const uint32_t a = a0 + uint32_t(gr.lane);
    int64_t i = 0, j = 0, k = 0;
    uint32_t lo = 0, hi = 0;
    if (a < c.total) {
      cell_at(c, a, i, j, k);
      const uint32_t h = streue(i, j, k, eimer);
      lo = anf[h];
      hi = anf[h + 1];
    }
    const bool gross = hi - lo > kGross;
    if (!gross) {
      if constexpr (VOR) {
        je_ueberlappend<8>(lo, hi, 1u, q32, elo, ehi, ein, vor, [&](uint32_t en, uint32_t e) {
          Payload pl;
          if (pruefe(en, i, j, k, e, pl)) ++cnt;
        });
      } else {
        for (uint32_t e = lo; e < hi; ++e) {
          Payload pl;
          if ((!elo || ueberlappt32(q32, elo[e], ehi[e])) && pruefe(ein[e], i, j, k, e, pl)) ++cnt;
        }
      }
    }
    for (unsigned m = __ballot_sync(gr.maske, gross); m != 0u; m &= m - 1u) {
      const int l = __ffs(m) - 1;  // the warp lane that holds the cell
      const uint32_t glo = __shfl_sync(gr.maske, lo, l), ghi = __shfl_sync(gr.maske, hi, l);
      const int64_t gi = __shfl_sync(gr.maske, (long long)i, l), gj = __shfl_sync(gr.maske, (long long)j, l),
                    gk = __shfl_sync(gr.maske, (long long)k, l);
      if constexpr (VOR) {
        je_ueberlappend<8>(glo + uint32_t(gr.lane), ghi, uint32_t(kG), q32, elo, ehi, ein, vor,
                           [&](uint32_t en, uint32_t e) {
                             Payload pl;
                             if (pruefe(en, gi, gj, gk, e, pl)) ++cnt;
                           });
      } else {
        for (uint32_t e = glo + uint32_t(gr.lane); e < ghi; e += kG) {
          Payload pl;
          if ((!elo || ueberlappt32(q32, elo[e], ehi[e])) && pruefe(ein[e], gi, gj, gk, e, pl)) ++cnt;
        }
      }
    }
  }
#pragma unroll
  for (int o = kG / 2; o > 0; o >>= 1) cnt += __shfl_xor_sync(gr.maske, cnt, o);
  return cnt;
}

// selbstkollision.rs:347-357, on p[0..n) with margin m
__device__ __forceinline__ Box quader_punkte(const D3* p, int n, double m) {
  Box b{d3(INFINITY, INFINITY, INFINITY), d3(-INFINITY, -INFINITY, -INFINITY)};
  for (int q = 0; q < n; ++q) {
    b.lo = d3(fmin(b.lo.x, p[q].x - m), fmin(b.lo.y, p[q].y - m), fmin(b.lo.z, p[q].z - m));
    b.hi = d3(fmax(b.hi.x, p[q].x + m), fmax(b.hi.y, p[q].y + m), fmax(b.hi.z, p[q].z + m));
  }
  return b;
}

// selbstkollision.rs:469-484
__device__ __forceinline__ Box kanten_quader(D3 a, D3 b, double m) {
  const D3 t = einheit(b - a);
  const D3 h = fabs(t.y - 1.0) < 1e-5 ? d3(1.0, 0.0, 0.0) : d3(0.0, 1.0, 0.0);
  const D3 u = einheit(cross(t, h));
  const D3 v = einheit(cross(t, u));
  D3 e[8];
  int n = 0;
  const D3 ends[2] = {a, b};
  const double s[2] = {-m, m};
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) e[n++] = (ends[p] + u * s[i]) + v * s[j];
  return quader_punkte(e, 8, 0.0);
}

// selbstkollision.rs:359-367
__device__ __forceinline__ bool ueberlappt(const Box& a, const Box& b) {
  return a.lo.x <= b.hi.x && b.lo.x <= a.hi.x && a.lo.y <= b.hi.y && b.lo.y <= a.hi.y && a.lo.z <= b.hi.z &&
         b.lo.z <= a.hi.z;
}
__device__ __forceinline__ bool erste_zelle(const Box& a, const Box& b, double zelle, int64_t i, int64_t j,
                                            int64_t k) {
  return zellindex(fmax(a.lo.x, b.lo.x), zelle) == i && zellindex(fmax(a.lo.y, b.lo.y), zelle) == j &&
         zellindex(fmax(a.lo.z, b.lo.z), zelle) == k;
}

// Stoffnetz::gleich_oder_partner (selbstkollision.rs:190-192)
__device__ __forceinline__ bool gleich_oder_partner(const SelbstArgs& s, uint32_t a, uint32_t b) {
  if (a == b) return true;
  for (uint32_t q = s.np_off[a]; q < s.np_off[a + 1]; ++q)
    if (s.np_ent[q] == b) return true;
  return false;
}
// Stoffnetz::band_und_traeger / band_abstand (selbstkollision.rs:129-155)
__device__ __forceinline__ bool band_und_traeger(const SelbstArgs& s, uint32_t a, uint32_t b) {
  const uint32_t ta = s.band_von[a], tb = s.band_von[b];
  if (ta != kKein && s.teil_von[b] == ta) return true;
  if (tb != kKein && s.teil_von[a] == tb) return true;
  return false;
}
__device__ __forceinline__ bool band_abstand(const SelbstArgs& s, uint32_t a, const uint32_t* andere, int n,
                                             double& out) {
  if (!s.has_band) return false;
  bool any = false;
  for (int k = 0; k < n; ++k) any = any || band_und_traeger(s, a, andere[k]);
  if (!any) return false;
  double m = 0.0;
  for (int k = 0; k < n; ++k) m = fmax(m, s.dicke[andere[k]]);
  out = s.dicke[a] + m;
  return true;
}

// netzkoerper.rs:185-218 (Ericson's closest point on a triangle)
__device__ D3 naechster_auf_dreieck(D3 p, D3 a, D3 b, D3 c) {
  auto quot = [](double z, double n) { return n > 0.0 ? z / n : 0.0; };
  const D3 ab = b - a, ac = c - a, ap = p - a;
  const double d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) return a;
  const D3 bp = p - b;
  const double d3v = dot(ab, bp), d4 = dot(ac, bp);
  if (d3v >= 0.0 && d4 <= d3v) return b;
  const double vc = d1 * d4 - d3v * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3v <= 0.0) return a + ab * quot(d1, d1 - d3v);
  const D3 cp = p - c;
  const double d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) return c;
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return a + ac * quot(d2, d2 - d6);
  const double va = d3v * d6 - d5 * d4;
  if (va <= 0.0 && d4 - d3v >= 0.0 && d5 - d6 >= 0.0) {
    const double w = quot(d4 - d3v, (d4 - d3v) + (d5 - d6));
    return b + (c - b) * w;
  }
  const double sum = va + vb + vc;
  const double v = quot(vb, sum), w = quot(vc, sum);
  return a + (ab * v + ac * w);
}

// selbstkollision.rs:370-384
__device__ void naechster_dreieck(D3 p0, D3 p1, D3 p2, D3 x, double g[3]) {
  const D3 a = naechster_auf_dreieck(x, p0, p1, p2);
  const D3 e1 = p1 - p0, e2 = p2 - p0, r = a - p0;
  const double d11 = dot(e1, e1), d12 = dot(e1, e2), d22 = dot(e2, e2);
  const double det = d11 * d22 - d12 * d12;
  if (det <= 1e-30) {
    g[0] = 1.0;
    g[1] = 0.0;
    g[2] = 0.0;
    return;
  }
  const double r1 = dot(r, e1), r2 = dot(r, e2);
  const double w1 = (d22 * r1 - d12 * r2) / det;
  const double w2 = (d11 * r2 - d12 * r1) / det;
  g[0] = 1.0 - w1 - w2;
  g[1] = w1;
  g[2] = w2;
}

// ------------------------------------------------------------ kernels
// selbstkollision.rs:216-225 (the point normals of :226-234 feed nothing the
// proximity stage returns, so they are not formed)
__global__ void __launch_bounds__(kT) tri_normals_kernel(const __grid_constant__ SelbstArgs s) {
  SC_FOR(t, s.nd) {
    const uint4 d = s.d_idx[t];
    const D3 a = ld3(s.x, d.x), b = ld3(s.x, d.y), c = ld3(s.x, d.z);
    const D3 n = einheit(cross(b - a, c - a));
    s.nrm_t[t] = make_double4(n.x, n.y, n.z, 0.0);
  }
}

// Edge planes (selbstkollision.rs:235-249), point and edge boxes (:401, :507-512)
// and the distinct buckets per box counted into the bucket-count arrays.
__global__ void __launch_bounds__(kT) boxes_kernel(const __grid_constant__ SelbstArgs s) {
  SC_FOR(v, s.n) {
    const D3 p = ld3(s.x, uint32_t(v));
    const Box b = quader_punkte(&p, 1, s.r_punkt[v] + kZuschlagQuader);
    s.qp_lo[v] = make_double4(b.lo.x, b.lo.y, b.lo.z, 0.0);
    s.qp_hi[v] = make_double4(b.hi.x, b.hi.y, b.hi.z, 0.0);
    uint32_t c = 0;
    je_eimer(b, s.zelle, s.eimer_p, [&](uint32_t h) {
      atomicAdd(&s.anf_p[h], 1u);
      ++c;
    });
    if (c) atomicAdd(&s.zahl[SZ_HASH_P], c);
  }
  SC_FOR(e, s.ne) {
    const uint2 k = s.k_idx[e];
    const uint2 kd = s.k_dr[e];
    D3 m;
    if (kd.x == kKein) {
      m = d3(1.0, 0.0, 0.0);
    } else {
      const double4 a4 = s.nrm_t[kd.x];
      const D3 a = d3(a4.x, a4.y, a4.z);
      if (kd.y == kKein) {
        m = a;
      } else {
        const double4 b4 = s.nrm_t[kd.y];
        const D3 b = d3(b4.x, b4.y, b4.z);
        m = dot(a, b) < 0.0 ? a - b : a + b;
      }
    }
    const D3 x0 = ld3(s.x, k.x), x1 = ld3(s.x, k.y);
    const D3 pl = einheit(cross(m, x0 - x1));
    s.keb[e] = make_double4(pl.x, pl.y, pl.z, 0.0);
    const Box b = kanten_quader(x0, x1, s.r_kante[e] + kZuschlagQuader);
    s.qk_lo[e] = make_double4(b.lo.x, b.lo.y, b.lo.z, 0.0);
    s.qk_hi[e] = make_double4(b.hi.x, b.hi.y, b.hi.z, 0.0);
    uint32_t c = 0;
    je_eimer(b, s.zelle, s.eimer_k, [&](uint32_t h) {
      atomicAdd(&s.anf_k[h], 1u);
      ++c;
    });
    if (c) atomicAdd(&s.zahl[SZ_HASH_K], c);
  }
}

// Entries into their buckets (any order; sorted per bucket afterwards).
__global__ void __launch_bounds__(kT) hash_fill_kernel(const __grid_constant__ SelbstArgs s) {
  SC_FOR(v, s.n) {
    const Box b = box_of(s.qp_lo, s.qp_hi, v);
    je_eimer(b, s.zelle, s.eimer_p, [&](uint32_t h) {
      const uint32_t pos = s.anf_p[h] + atomicAdd(&s.cur_p[h], 1u);
      if (pos < s.cap_ep) s.ein_p[pos] = uint32_t(v);
    });
  }
  SC_FOR(e, s.ne) {
    const Box b = box_of(s.qk_lo, s.qk_hi, e);
    je_eimer(b, s.zelle, s.eimer_k, [&](uint32_t h) {
      const uint32_t pos = s.anf_k[h] + atomicAdd(&s.cur_k[h], 1u);
      if (pos < s.cap_ek) s.ein_k[pos] = uint32_t(e);
    });
  }
}

// Ascending entries inside each bucket: the reference fills its buckets in
// entry order (selbstkollision.rs:316-322). The keys of a range are distinct,
// so any sort gives the same result. Ranges of up to kKurzSort entries are
// sorted by one thread each (insertion sort); longer ones by a block each
// (lang_sort_kernel), so that a crowded bucket does not stall its thread.
constexpr uint32_t kKurzSort = 32, kLangSort = 16384;
constexpr size_t kLangSortSmem = sizeof(uint32_t) * kLangSort;  // dynamic shared memory of lang_sort_kernel
__device__ __forceinline__ void sort_range(uint32_t* a, uint32_t lo, uint32_t hi) {
  if (hi - lo < 2 || hi - lo > kKurzSort) return;
  for (uint32_t i = lo + 1; i < hi; ++i) {
    const uint32_t key = a[i];
    uint32_t j = i;
    while (j > lo && a[j - 1] > key) {
      a[j] = a[j - 1];
      --j;
    }
    a[j] = key;
  }
}
// ranges [off[b], off[b + 1]) longer than kWarpSort: bitonic in the block's
// dynamic shared memory up to kLangSort entries (a path hash of the garment
// has buckets of 5-6k entries), Shell sort (Ciura's gaps) on one thread beyond.
__device__ __forceinline__ void lang_sortieren(uint32_t* a, uint32_t lo, uint32_t hi, uint32_t* sh) {
  const uint32_t n = hi - lo;
  if (n > kLangSort) {
    if (threadIdx.x == 0) {
      const uint32_t gaps[8] = {701u, 301u, 132u, 57u, 23u, 10u, 4u, 1u};
      for (int g = 0; g < 8; ++g) {
        const uint32_t gap = gaps[g];
        for (uint32_t i = lo + gap; i < hi; ++i) {
          const uint32_t key = a[i];
          uint32_t j = i;
          while (j >= lo + gap && a[j - gap] > key) {
            a[j] = a[j - gap];
            j -= gap;
          }
          a[j] = key;
        }
      }
    }
    __syncthreads();
    return;
  }
  uint32_t m = 1;
  while (m < n) m <<= 1;
  for (uint32_t i = threadIdx.x; i < m; i += kT) sh[i] = i < n ? a[lo + i] : 0xffffffffu;
  __syncthreads();
  for (uint32_t k = 2; k <= m; k <<= 1)
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < m; i += kT) {
        const uint32_t p = i ^ j;
        if (p > i) {
          const bool auf = (i & k) == 0;
          const uint32_t x = sh[i], y = sh[p];
          if ((x > y) == auf) sh[i] = y, sh[p] = x;
        }
      }
      __syncthreads();
    }
  for (uint32_t i = threadIdx.x; i < n; i += kT) a[lo + i] = sh[i];
  __syncthreads();
}
// a range of up to kWarpSort entries by one warp: bitonic in the warp's part
// of shared memory
constexpr uint32_t kWarpSort = 256;
__device__ __forceinline__ void warp_sortieren(uint32_t* a, uint32_t lo, uint32_t hi, uint32_t* sh) {
  const uint32_t n = hi - lo, lane = threadIdx.x & 31;
  uint32_t m = 1;
  while (m < n) m <<= 1;
  for (uint32_t i = lane; i < m; i += 32) sh[i] = i < n ? a[lo + i] : 0xffffffffu;
  __syncwarp();
  for (uint32_t k = 2; k <= m; k <<= 1)
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = lane; i < m; i += 32) {
        const uint32_t p = i ^ j;
        if (p > i) {
          const bool auf = (i & k) == 0;
          const uint32_t x = sh[i], y = sh[p];
          if ((x > y) == auf) sh[i] = y, sh[p] = x;
        }
      }
      __syncwarp();
    }
  for (uint32_t i = lane; i < n; i += 32) a[lo + i] = sh[i];
  __syncwarp();
}
// The ranges longer than kKurzSort of kT buckets at a time: those up to
// kWarpSort entries one per warp, side by side; the longer ones by the whole
// block, one after another.
__global__ void __launch_bounds__(kT) lang_sort_kernel(const uint32_t* off, uint32_t* a, int64_t nb) {
  extern __shared__ uint32_t sh[];  // kLangSort entries
  __shared__ uint32_t lang[kT];
  __shared__ uint32_t zahl, gross;
  uint32_t* wsh = sh + (threadIdx.x >> 5) * kWarpSort;  // kT / 32 warps x kWarpSort <= kLangSort
  for (int64_t base = int64_t(blockIdx.x) * kT; base < nb; base += int64_t(gridDim.x) * kT) {
    if (threadIdx.x == 0) zahl = gross = 0;
    __syncthreads();
    const int64_t b = base + threadIdx.x;
    const uint32_t len = b < nb ? off[b + 1] - off[b] : 0u;
    if (len > kKurzSort && len <= kWarpSort) lang[atomicAdd(&zahl, 1u)] = threadIdx.x;
    __syncthreads();
    const uint32_t m = zahl;
    if (len > kWarpSort) lang[kT - 1 - atomicAdd(&gross, 1u)] = threadIdx.x;  // from the list's other end
    for (uint32_t q = threadIdx.x >> 5; q < m; q += kT / 32) {
      const int64_t bq = base + lang[q];
      warp_sortieren(a, off[bq], off[bq + 1], wsh);
    }
    __syncthreads();
    const uint32_t g = gross;
    for (uint32_t q = 0; q < g; ++q) {
      const int64_t bq = base + lang[kT - 1 - q];
      lang_sortieren(a, off[bq], off[bq + 1], sh);
    }
    __syncthreads();
  }
}
// The FP32 boxes of a hash's entries, in entry order (after the per-bucket
// sort), rounded outward: the searches' pre-test (see Box32).
__global__ void __launch_bounds__(kT) eintrag_boxen_kernel(const uint32_t* anf, uint32_t eimer, uint32_t cap,
                                                           const uint32_t* ein, const double4* lo, const double4* hi,
                                                           float4* elo, float4* ehi) {
  const uint32_t n = anf[eimer] < cap ? anf[eimer] : cap;
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const uint32_t b = ein[q];
    const double4 l = lo[b], h = hi[b];
    elo[q] = make_float4(__double2float_rd(l.x), __double2float_rd(l.y), __double2float_rd(l.z), 0.f);
    ehi[q] = make_float4(__double2float_ru(h.x), __double2float_ru(h.y), __double2float_ru(h.z), 0.f);
  }
}
constexpr unsigned kEintragGrid = 148 * 8;

unsigned grid_lang(int64_t nb);
// lang_sort_kernel over nb ranges with its shared memory (set once per process)
cudaError_t lang_sort(const uint32_t* off, uint32_t* a, int64_t nb, cudaStream_t st) {
  static bool gesetzt = false;
  if (!gesetzt) {
    const cudaError_t e =
        cudaFuncSetAttribute(lang_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kLangSortSmem));
    if (e != cudaSuccess) return e;
    gesetzt = true;
  }
  lang_sort_kernel<<<grid_lang(nb), kT, kLangSortSmem, st>>>(off, a, nb);
  return cudaSuccess;
}
unsigned grid_lang(int64_t nb) {
  const int64_t b = (nb + kT - 1) / kT;
  return unsigned(b < 1 ? 1 : (b > 148 * 4 ? 148 * 4 : b));
}
__global__ void __launch_bounds__(kT) bucket_sort_kernel(const __grid_constant__ SelbstArgs s) {
  SC_FOR(b, s.eimer_p) sort_range(s.ein_p, s.anf_p[b], s.anf_p[b + 1]);
  SC_FOR(b, s.eimer_k) sort_range(s.ein_k, s.anf_k[b], s.anf_k[b + 1]);
}

// Point-triangle search for triangle t (selbstkollision.rs:400-466) and
// edge-edge search for edge e (:506-598): see punkt_dreieck_gruppe and
// kante_kante_gruppe below (a group of lanes per triangle or edge).

// selbstkollision.rs:489-503
__device__ bool ist_kuerzeste(const SelbstArgs& s, uint32_t e, D3 u, D3 m) {
  const uint2 k = s.k_idx[e];
  const uint2 kd = s.k_dr[e];
  const uint32_t ts[2] = {kd.x, kd.y};
  for (int q = 0; q < 2; ++q) {
    const uint32_t t = ts[q];
    if (t == kKein) continue;
    const uint4 d = s.d_idx[t];
    const uint32_t dd[3] = {d.x, d.y, d.z};
    uint32_t o = kKein;
    for (int a = 0; a < 3; ++a)
      if (dd[a] != k.x && dd[a] != k.y) {
        o = dd[a];
        break;
      }
    if (o == kKein) continue;
    const D3 r = ld3(s.x, o) - ld3(s.x, k.x);
    const D3 wr = einheit(r - u * dot(r, u));
    const double4 n4 = s.nrm_t[t];
    if (dot(m, wr) > 0.0 && fabs(dot(m, d3(n4.x, n4.y, n4.z))) < 0.5) return false;
  }
  return true;
}

// The searches, one group of kG lanes per triangle or edge: the tests of
// selbstkollision.rs:400-466 (point-triangle) and :506-598 (edge-edge) per
// candidate, the hits written in the reference's order.
struct PaarPT {
  uint32_t v;
  double g0, g1, g2, ab, ruhe;
  D3 n;
};
template <bool FILL>
__device__ uint32_t punkt_dreieck_gruppe(const SelbstArgs& s, const Gruppe& gr, int64_t t, uint32_t pos) {
  const uint4 dq = s.d_idx[t];
  const uint32_t i0 = dq.x, i1 = dq.y, i2 = dq.z;
  if (i0 == i1 || i1 == i2 || i0 == i2) return 0;
  const uint32_t d[3] = {i0, i1, i2};
  const D3 p[3] = {ld3(s.x, i0), ld3(s.x, i1), ld3(s.x, i2)};
  const double rt = s.r_dreieck[t];
  const Box qt = quader_punkte(p, 3, rt + kZuschlagQuader);
  const double4 n4 = s.nrm_t[t];
  const D3 nt = d3(n4.x, n4.y, n4.z);
  const uint4 dk = s.d_kan[t];
  const uint32_t ek[3] = {dk.x, dk.y, dk.z};
  D3 en[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double4 q = s.keb[ek[k]];
    en[k] = d3(q.x, q.y, q.z);
  }
  const double sg[3] = {dot(p[2] - p[0], en[0]), dot(p[0] - p[1], en[1]), dot(p[1] - p[2], en[2])};
  const bool alle_fest = s.w[i0] <= 0.0 && s.w[i1] <= 0.0 && s.w[i2] <= 0.0;
  const auto pruefe = [&](uint32_t v, int64_t ci, int64_t cj, int64_t ck, uint32_t, PaarPT& o) -> bool {
    // the reference's conditions, the cheapest rejection first (each is
    // a plain condition on the candidate, so the order changes no result)
    const Box qv = box_of(s.qp_lo, s.qp_hi, v);
    if (!ueberlappt(qv, qt) || !erste_zelle(qt, qv, s.zelle, ci, cj, ck)) return false;
    for (int k = 0; k < 3; ++k)
      if (gleich_oder_partner(s, v, d[k])) return false;
    if (s.w[v] <= 0.0 && alle_fest) return false;
    const D3 xv = ld3(s.x, v);
    double ruhe = rt + s.r_punkt[v];
    double eine;
    if (band_abstand(s, v, d, 3, eine)) ruhe = eine;
    const double soll = ruhe + kZuschlagPaar;
    const double sd = dot(nt, xv - p[0]);
    if (fabs(sd) > soll) return false;
    for (int k = 0; k < 3; ++k)
      if (dot(xv - p[k], en[k]) * sg[k] < 0.0) return false;
    double g[3];
    naechster_dreieck(p[0], p[1], p[2], xv, g);
    const D3 cp = (p[0] * g[0] + p[1] * g[1]) + p[2] * g[2];
    const D3 r = xv - cp;
    const double abstand = norm(r);
    if (abstand > soll) return false;
    if (FILL) {
      o.v = v;
      o.g0 = g[0], o.g1 = g[1], o.g2 = g[2];
      o.ab = abstand;
      o.ruhe = ruhe;
      o.n = abstand > 1e-12 ? r * (1.0 / abstand) : nt;
    }
    return true;
  };
  const auto schreibe = [&](const PaarPT& o, uint32_t q) {
    if (q < s.cap_pairs) {
      s.pr_idx[q] = make_uint4(o.v, i0, i1, i2);
      s.pr_src[q] = make_uint2(uint32_t(t), kKein);
      s.pr_w[q] = make_double4(1.0, -o.g0, -o.g1, -o.g2);
      s.pr_nab[q] = make_double4(o.n.x, o.n.y, o.n.z, o.ab);
      s.pr_ruhe[q] = o.ruhe;
    }
  };
  if constexpr (FILL) {
    return je_eintrag_gruppe<true, PaarPT>(gr, qt, s.zelle, s.eimer_p, s.anf_p, s.ein_p, s.ebp_lo, s.ebp_hi,
                                      pos, pruefe, schreibe);
  } else {
    return zaehle_gruppe<PaarPT, true>(gr, qt, s.zelle, s.eimer_p, s.anf_p, s.ein_p, s.ebp_lo, s.ebp_hi, pruefe,
                                       [](uint32_t) { return true; });
  }
}
struct PaarKK {
  uint32_t f, b0, b1;
  double sp, tp, ab, ruhe;
  D3 n;
};
template <bool FILL>
__device__ uint32_t kante_kante_gruppe(const SelbstArgs& s, const Gruppe& gr, int64_t e, uint32_t pos) {
  const uint2 ka = s.k_idx[e];
  const uint32_t a0 = ka.x, a1 = ka.y;
  if (a0 == a1) return 0;
  const D3 pa0 = ld3(s.x, a0), pa1 = ld3(s.x, a1);
  const Box qe = box_of(s.qk_lo, s.qk_hi, e);
  const Box32 qe32 = box32(qe);
  const auto pruefe = [&](uint32_t f, int64_t ci, int64_t cj, int64_t ck, uint32_t sq, PaarKK& o) -> bool {
    if (int64_t(f) <= e) return false;
    if (!ueberlappt32(qe32, s.ebk_lo[sq], s.ebk_hi[sq])) return false;
    const Box qf = box_of(s.qk_lo, s.qk_hi, f);
    if (!ueberlappt(qe, qf) || !erste_zelle(qe, qf, s.zelle, ci, cj, ck)) return false;
    const uint2 kb = s.k_idx[f];
    const uint32_t b0 = kb.x, b1 = kb.y;
    if (gleich_oder_partner(s, a0, b0) || gleich_oder_partner(s, a1, b0) || gleich_oder_partner(s, a0, b1) ||
        gleich_oder_partner(s, a1, b1))
      return false;
    const uint32_t bb[2] = {b0, b1}, aa[2] = {a0, a1};
    double band = 0.0;
    const bool hat_band = band_abstand(s, a0, bb, 2, band) || band_abstand(s, a1, bb, 2, band) ||
                          band_abstand(s, b0, aa, 2, band) || band_abstand(s, b1, aa, 2, band);
    if (s.w[a0] <= 0.0 && s.w[a1] <= 0.0 && s.w[b0] <= 0.0 && s.w[b1] <= 0.0) return false;
    const D3 pb0 = ld3(s.x, b0), pb1 = ld3(s.x, b1);
    const D3 da = pa1 - pa0, db = pb1 - pb0;
    const double la = norm(da), lb = norm(db);
    if (la < kKanteMin || lb < kKanteMin) return false;
    const D3 ua = da * (1.0 / la), ub = db * (1.0 / lb);
    const double cw = dot(ua, ub);
    if (fabs(cw) > 0.99999) return false;
    const D3 r = pb0 - pa0;
    const double p = dot(r, ua), q = -dot(r, ub);
    const double nen = 1.0 - cw * cw;
    const double sa = (p + cw * q) / nen;
    const double sb = (q + cw * p) / nen;
    if (!(0.0 <= sa && sa <= la) || !(0.0 <= sb && sb <= lb)) return false;
    const D3 pa = pa0 + ua * sa;
    const D3 pb = pb0 + ub * sb;
    const D3 dv = pa - pb;
    const double abstand = norm(dv);
    const double ruhe = hat_band ? band : s.r_kante[e] + s.r_kante[f];
    if (abstand > ruhe + kZuschlagPaar) return false;
    const D3 n = einheit(dv);
    if (!ist_kuerzeste(s, f, ub, n) || !ist_kuerzeste(s, uint32_t(e), ua, n * -1.0)) return false;
    if (FILL) {
      o.f = f, o.b0 = b0, o.b1 = b1;
      o.sp = sa / la, o.tp = sb / lb;
      o.ab = abstand, o.ruhe = ruhe, o.n = n;
    }
    return true;
  };
  const auto schreibe = [&](const PaarKK& o, uint32_t w) {
    if (w < s.cap_pairs) {
      s.pr_idx[w] = make_uint4(a0, a1, o.b0, o.b1);
      s.pr_src[w] = make_uint2(uint32_t(e), o.f);
      s.pr_w[w] = make_double4(1.0 - o.sp, o.sp, -(1.0 - o.tp), -o.tp);
      s.pr_nab[w] = make_double4(o.n.x, o.n.y, o.n.z, o.ab);
      s.pr_ruhe[w] = o.ruhe;
    }
  };
  if constexpr (FILL) {
    return je_eintrag_gruppe<true, PaarKK>(gr, qe, s.zelle, s.eimer_k, s.anf_k, s.ein_k, nullptr, nullptr,
                                      pos, pruefe, schreibe);
  } else {
    // the index test (later edges only) before the box loads
    return zaehle_gruppe<PaarKK, true>(gr, qe, s.zelle, s.eimer_k, s.anf_k, s.ein_k, s.ebk_lo, s.ebk_hi, pruefe,
                                       [&](uint32_t f) { return int64_t(f) > e; });
  }
}
// one group of kG lanes per item: the items of a grid-stride loop
#define GR_FOR(i, n)                                                                                   \
  for (int64_t i = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / kG; i < int64_t(n);                \
       i += int64_t(gridDim.x) * blockDim.x / kG)

// Items 0 .. n-1 taken one at a time from a counter (zeroed with the stage's
// counters) by a group of lanes: its first lane (`fuehrer`, a warp lane)
// grabs, every lane of `maske` gets the item, f(item) runs on all of them.
// Crowded parts of the cloth cluster in index ranges, so a fixed stride would
// leave some groups far more work than others.
template <typename F>
__device__ __forceinline__ void je_gezogen(unsigned maske, int fuehrer, uint32_t* zaehler, uint64_t n, F&& f) {
  for (;;) {
    uint32_t q = 0;
    if (int(threadIdx.x & 31) == fuehrer) q = atomicAdd(zaehler, 1u);
    q = __shfl_sync(maske, q, fuehrer);
    if (q >= n) break;
    f(q);
  }
}

// count pass: pair count per triangle and per edge (off_t[t], off_e[e]);
// the triangles and edges that have pairs go to a list for the fill pass
__global__ void __launch_bounds__(kT, 4) pairs_count_kernel(const __grid_constant__ SelbstArgs s) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {  // the scans run over n + 1 values
    s.off_t[s.nd] = 0u;
    s.off_e[s.ne] = 0u;
  }
  // triangles (q < nd) and edges (nd + e) from one counter, one item per
  // grab: the crowded parts of the cloth cluster in index ranges, so a fixed
  // stride would leave some groups far more work than others
  const Gruppe gr = gruppe();
  const int fuehrer = int(threadIdx.x & 31) & ~(kG - 1);
  const uint64_t gesamt = uint64_t(s.nd) + uint64_t(s.ne);
  for (;;) {
    uint32_t q = 0;
    if (gr.lane == 0) q = atomicAdd(&s.zahl[SZ_ARBEIT_P], 1u);
    q = __shfl_sync(gr.maske, q, fuehrer);
    if (q >= gesamt) break;
    if (int64_t(q) < s.nd) {
      const uint32_t c = punkt_dreieck_gruppe<false>(s, gr, q, 0);
      if (gr.lane == 0) {
        s.off_t[q] = c;
        if (c) s.aktiv_p[atomicAdd(&s.zahl[SZ_AKTIV_P], 1u)] = q;
      }
    } else {
      const int64_t e = int64_t(q) - s.nd;
      const uint32_t c = kante_kante_gruppe<false>(s, gr, e, 0);
      if (gr.lane == 0) {
        s.off_e[e] = c;
        if (c) s.aktiv_p[atomicAdd(&s.zahl[SZ_AKTIV_P], 1u)] = q;
      }
    }
  }
}

// fill pass over the listed triangles and edges only: each writes its pairs
// from its scanned start, so the buffer holds the point-triangle pairs in
// triangle order, then the edge-edge pairs in edge order, whatever the list's
// order
__global__ void __launch_bounds__(kT, 4) pairs_fill_kernel(const __grid_constant__ SelbstArgs s, uint32_t n_aktiv) {
  const uint32_t npt = s.zahl[SZ_PAARE_PT];
  const Gruppe gr = gruppe();
  GR_FOR(q, n_aktiv) {
    const uint32_t c = s.aktiv_p[q];
    if (int64_t(c) < s.nd)
      punkt_dreieck_gruppe<true>(s, gr, c, s.off_t[c]);
    else
      kante_kante_gruppe<true>(s, gr, int64_t(c) - s.nd, npt + s.off_e[c - s.nd]);
  }
}

__device__ __forceinline__ uint32_t paare(const SelbstArgs& s) {
  const uint64_t p = uint64_t(s.zahl[SZ_PAARE_PT]) + s.zahl[SZ_PAARE_KK];
  return p < s.cap_pairs ? uint32_t(p) : s.cap_pairs;
}
// all springs: the proximity pairs, then the push springs
__device__ __forceinline__ uint32_t federn_alle(const SelbstArgs& s) {
  const uint32_t ns = s.zahl[SZ_SCHNITTE] < s.cap_s ? s.zahl[SZ_SCHNITTE] : s.cap_s;
  const uint64_t p = uint64_t(s.zahl[SZ_PAARE_PT]) + s.zahl[SZ_PAARE_KK] + ns;
  return p < s.cap_pairs ? uint32_t(p) : s.cap_pairs;
}

// Spring of each pair (selbstkollision.rs:715-752, 779-785) without the
// approach damping: stiffness, rest (seam override), force, block; and the
// operator copies (h^2 block, weights) in precision R.
template <typename R>
__global__ void __launch_bounds__(kT) federn_kernel(const __grid_constant__ SelbstArgs s) {
  const uint32_t P = paare(s), npt = s.zahl[SZ_PAARE_PT];
  R4<R>* bR = static_cast<R4<R>*>(s.pr_bR);
  R4<R>* wR = static_cast<R4<R>*>(s.pr_wR);
  const double h2 = s.h * s.h;
  SC_FOR(q, P) {
    const uint4 id = s.pr_idx[q];
    const uint2 src = s.pr_src[q];
    const double4 g4 = s.pr_w[q];
    const double4 nab = s.pr_nab[q];
    const uint32_t idx[4] = {id.x, id.y, id.z, id.w};
    const double gw[4] = {g4.x, g4.y, g4.z, g4.w};
    double e, a, mu;
    if (uint32_t(q) < npt) {
      // dreieck_von (selbstkollision.rs:790-794): the first triangle of the
      // pair's edge 0 -> 1 that holds its point 2
      const uint32_t ke = s.d_kan[src.x].x;
      const uint2 kd = s.k_dr[ke];
      uint32_t t = 0;
      const uint32_t cand[2] = {kd.x, kd.y};
      for (int c = 0; c < 2; ++c) {
        if (cand[c] == kKein) continue;
        const uint4 d = s.d_idx[cand[c]];
        if (d.x == id.w || d.y == id.w || d.z == id.w) {
          t = cand[c];
          break;
        }
      }
      e = s.e_punkt[id.x] + s.e_dreieck[t];
      a = s.a_punkt[id.x] + s.a_dreieck[t];
      mu = 0.5 * (s.mu[id.x] + (s.mu[id.y] + s.mu[id.z] + s.mu[id.w]) / 3.0);
    } else {
      e = s.e_kante[src.x] + s.e_kante[src.y];
      a = s.a_kante[src.x] + s.a_kante[src.y];
      mu = 0.25 * (s.mu[id.x] + s.mu[id.y] + s.mu[id.z] + s.mu[id.w]);
    }
    const double k = s.steifigkeit * e * a / 1e-6;
    // a seam spring between the two sides with a shorter rest replaces the rest distance
    double ruhe = s.pr_ruhe[q];
    bool fertig = false;
    for (int qq = 0; qq < 4 && !fertig; ++qq) {
      if (gw[qq] <= 0.0) continue;
      for (uint32_t c = s.wp_off[idx[qq]]; c < s.wp_off[idx[qq] + 1]; ++c) {
        const uint2 pc = s.wp_ent[c];
        bool auf_zweiter = false;
        for (int r = 0; r < 4; ++r) auf_zweiter = auf_zweiter || (gw[r] < 0.0 && idx[r] == pc.x);
        const double l0 = s.naht_ruhe[pc.y];
        if (auf_zweiter && isfinite(l0) && l0 < ruhe) {
          ruhe = l0;
          fertig = true;
          break;
        }
      }
    }
    const double c = fmin(ruhe - nab.w, kAuslenkungMax);
    const D3 n = d3(nab.x, nab.y, nab.z);
    const double kc = k * c;
    s.pr_kf[q] = make_double4(n.x * kc, n.y * kc, n.z * kc, k);
    const double om = 1.0 - mu;
    const double bxx = k * (om * n.x * n.x + mu), byy = k * (om * n.y * n.y + mu), bzz = k * (om * n.z * n.z + mu);
    const double bxy = k * (om * n.x * n.y + 0.0), bxz = k * (om * n.x * n.z + 0.0), byz = k * (om * n.y * n.z + 0.0);
    // the damping's mass shares (selbstkollision.rs:759-777), in the reference's order
    double m1 = 0.0, m2 = 0.0;
    for (int kq = 0; kq < 4; ++kq) {
      if (gw[kq] > 0.0)
        m1 += gw[kq] * s.masse[idx[kq]];
      else
        m2 -= gw[kq] * s.masse[idx[kq]];
    }
    double ga[4];
    for (int kq = 0; kq < 4; ++kq) ga[kq] = gw[kq] * (gw[kq] > 0.0 ? m2 / (m1 + m2) : m1 / (m1 + m2));
    s.pr_b0[q] = make_double4(bxx, byy, bzz, bxy);
    s.pr_b1[q] = make_double4(bxz, byz, mu, m1 + m2 > 0.0 ? 1.0 : 0.0);
    s.pr_ga[q] = make_double4(ga[0], ga[1], ga[2], ga[3]);
    bR[2 * q] = {R(h2 * bxx), R(h2 * byy), R(h2 * bzz), R(h2 * bxy)};
    bR[2 * q + 1] = {R(h2 * bxz), R(h2 * byz), R(0), R(0)};
    wR[q] = {R(gw[0]), R(gw[1]), R(gw[2]), R(gw[3])};
    s.pr_x5[q] = kKein;
    s.pr_g5[q] = 0.0;
    static_cast<R*>(s.pr_g5R)[q] = R(0);
  }
}

// The approach damping (selbstkollision.rs:753-778). The reference applies
// it pair by pair: each pair reads the velocities its predecessors left.
// Here one block takes the pairs in batches of kDB. The batch's free points
// get shared-memory slots; one thread gives each pair a level, one more than
// the highest level of the earlier pairs in the batch that share a free
// point with it; then the levels run one after another, all pairs of a level
// at once. Pairs of one level share no free point, and every pair runs after
// all earlier pairs it shares a free point with, so every pair reads exactly
// the velocities the sequential order gives it. Points that are held (w <= 0)
// are never written and are read from global memory.
constexpr int kDB = 512;
constexpr int kDSlots = 4 * kDB;
constexpr uint16_t kFest = 0xffffu;
constexpr size_t kDampSmem = size_t(kDSlots) * (3 * sizeof(double) + sizeof(uint32_t) + sizeof(uint16_t)) +
                             size_t(kDB) * (4 + 1) * sizeof(uint16_t) + 64;

__global__ void __launch_bounds__(kDB, 1) daempfung_kernel(const __grid_constant__ SelbstArgs s) {
  extern __shared__ __align__(16) unsigned char dsm[];
  double* vx = reinterpret_cast<double*>(dsm);
  double* vy = vx + kDSlots;
  double* vz = vy + kDSlots;
  uint32_t* slot_pt = reinterpret_cast<uint32_t*>(vz + kDSlots);
  uint16_t* last = reinterpret_cast<uint16_t*>(slot_pt + kDSlots);
  uint16_t* pslot = last + kDSlots;  // 4 per pair
  uint16_t* level = pslot + 4 * kDB;
  __shared__ uint32_t nslots, maxlevel;
  const uint32_t P = paare(s);
  const int tid = threadIdx.x;
  for (uint32_t b0 = 0; b0 < P; b0 += kDB) {
    const uint32_t nb = P - b0 < uint32_t(kDB) ? P - b0 : uint32_t(kDB);
    if (tid == 0) {
      nslots = 0;
      maxlevel = 0;
    }
    __syncthreads();
    // 1. the pair's data into registers; slots for its free points (first
    //    come, first served); held points' velocities are constant
    const bool mine = uint32_t(tid) < nb;
    double gw[4] = {0, 0, 0, 0}, ga[4] = {0, 0, 0, 0}, mu = 0.0, flag = 0.0;
    D3 n = d3(0, 0, 0), vk[4];
    uint16_t sl[4] = {kFest, kFest, kFest, kFest};
    if (mine) {
      const uint32_t q = b0 + tid;
      const uint4 id = s.pr_idx[q];
      const double4 g4 = s.pr_w[q], nab = s.pr_nab[q], b1 = s.pr_b1[q], ga4 = s.pr_ga[q];
      const uint32_t pts[4] = {id.x, id.y, id.z, id.w};
      gw[0] = g4.x, gw[1] = g4.y, gw[2] = g4.z, gw[3] = g4.w;
      ga[0] = ga4.x, ga[1] = ga4.y, ga[2] = ga4.z, ga[3] = ga4.w;
      n = d3(nab.x, nab.y, nab.z);
      mu = b1.z;
      flag = b1.w;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (s.w[pts[k]] > 0.0) {
          int32_t cur = atomicAdd(&s.slot_of[pts[k]], 0);
          if (cur < 0) {
            const uint32_t me = atomicAdd(&nslots, 1u);
            const int32_t old = atomicCAS(&s.slot_of[pts[k]], -1, int32_t(me));
            slot_pt[me] = old < 0 ? pts[k] : kKein;
            cur = old < 0 ? int32_t(me) : old;
          }
          sl[k] = uint16_t(cur);
          vk[k] = d3(0, 0, 0);
        } else {
          vk[k] = ld3(s.v, pts[k]);
        }
        pslot[4 * tid + k] = sl[k];
      }
    }
    __syncthreads();
    // 2. the slots' velocities
    for (uint32_t q = tid; q < nslots; q += kDB) {
      const uint32_t pt = slot_pt[q];
      if (pt != kKein) {
        const D3 v = ld3(s.v, pt);
        vx[q] = v.x;
        vy[q] = v.y;
        vz[q] = v.z;
      }
      last[q] = 0;
    }
    __syncthreads();
    // 3. levels, in pair order (pairs without a free point write nothing: level 0)
    if (tid == 0) {
      uint32_t mx = 0;
      for (uint32_t q = 0; q < nb; ++q) {
        const uint16_t s0 = pslot[4 * q], s1 = pslot[4 * q + 1], s2 = pslot[4 * q + 2], s3 = pslot[4 * q + 3];
        uint32_t l = 0;
        bool frei = false;
        if (s0 != kFest) { l = last[s0] > l ? last[s0] : l; frei = true; }
        if (s1 != kFest) { l = last[s1] > l ? last[s1] : l; frei = true; }
        if (s2 != kFest) { l = last[s2] > l ? last[s2] : l; frei = true; }
        if (s3 != kFest) { l = last[s3] > l ? last[s3] : l; frei = true; }
        if (!frei) {
          level[q] = 0;
          continue;
        }
        ++l;
        level[q] = uint16_t(l);
        if (s0 != kFest) last[s0] = uint16_t(l);
        if (s1 != kFest) last[s1] = uint16_t(l);
        if (s2 != kFest) last[s2] = uint16_t(l);
        if (s3 != kFest) last[s3] = uint16_t(l);
        mx = l > mx ? l : mx;
      }
      maxlevel = mx;
    }
    __syncthreads();
    // 4. the levels one after another
    const uint32_t L = maxlevel;
    const uint32_t my = mine ? level[tid] : 0u;
    for (uint32_t lv = 1; lv <= L; ++lv) {
      if (my == lv) {
        D3 cur[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) cur[k] = sl[k] != kFest ? d3(vx[sl[k]], vy[sl[k]], vz[sl[k]]) : vk[k];
        D3 dv = d3(0.0, 0.0, 0.0);
#pragma unroll
        for (int k = 0; k < 4; ++k) dv = dv + cur[k] * gw[k];
        const double an = dot(dv, n) * kAnnaeherung;
        if (an < 0.0 && flag != 0.0) {
          const D3 u = n * an + (dv - n * an) * mu;
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            if (sl[k] == kFest) continue;
            const D3 nv = cur[k] - u * ga[k];
            vx[sl[k]] = nv.x;
            vy[sl[k]] = nv.y;
            vz[sl[k]] = nv.z;
          }
        }
      }
      __syncthreads();
    }
    // 5. back to global memory; the slots are free again
    for (uint32_t q = tid; q < nslots; q += kDB) {
      const uint32_t pt = slot_pt[q];
      if (pt != kKein) {
        st3(s.v, pt, d3(vx[q], vy[q], vz[q]));
        s.slot_of[pt] = -1;
      }
    }
    __syncthreads();
  }
}

// Per-point incidence lists of the springs' nonzero slots, ascending.
__global__ void __launch_bounds__(kT) inc_count_kernel(const __grid_constant__ SelbstArgs s) {
  const uint32_t P = federn_alle(s);
  SC_FOR(q, P) {
    const uint4 id = s.pr_idx[q];
    const double4 g = s.pr_w[q];
    if (g.x != 0.0) atomicAdd(&s.inc_off[id.x], 1u);
    if (g.y != 0.0) atomicAdd(&s.inc_off[id.y], 1u);
    if (g.z != 0.0) atomicAdd(&s.inc_off[id.z], 1u);
    if (g.w != 0.0) atomicAdd(&s.inc_off[id.w], 1u);
    if (s.pr_g5[q] != 0.0) atomicAdd(&s.inc_off[s.pr_x5[q]], 1u);
  }
}
__global__ void __launch_bounds__(kT) inc_fill_kernel(const __grid_constant__ SelbstArgs s) {
  const uint32_t P = federn_alle(s);
  SC_FOR(q, P) {
    const uint4 id = s.pr_idx[q];
    const double4 g = s.pr_w[q];
    const uint32_t pts[5] = {id.x, id.y, id.z, id.w, s.pr_x5[q]};
    const double gw[5] = {g.x, g.y, g.z, g.w, s.pr_g5[q]};
    for (int k = 0; k < 5; ++k) {
      if (gw[k] == 0.0) continue;
      const uint32_t pos = s.inc_off[pts[k]] + atomicAdd(&s.inc_cur[pts[k]], 1u);
      if (pos < s.cap_inc) s.inc_ent[pos] = (uint32_t(q) << 3) | uint32_t(k);
    }
  }
}
__global__ void __launch_bounds__(kT) inc_sort_kernel(const __grid_constant__ SelbstArgs s) {
  SC_FOR(i, s.n) sort_range(s.inc_ent, s.inc_off[i], s.inc_off[i + 1]);
}
// The inverse of the lists: each nonzero slot's entry index (the PCG writes a
// spring's slot products there and sums them per point in list order).
__global__ void __launch_bounds__(kT) inc_pos_kernel(const __grid_constant__ SelbstArgs s) {
  const uint32_t E = s.inc_off[s.n] < s.cap_inc ? s.inc_off[s.n] : s.cap_inc;
  SC_FOR(e, E) s.inc_pos[s.inc_ent[e]] = uint32_t(e);
}

// ------------------------------------------------------------ exclusive scan
// Exclusive prefix sum of n uint32 in place, 1024 per block; block totals in
// tmp, scanned by one block; `total` receives the sum.
constexpr int kScanT = 256, kScanPer = 4, kScanChunk = kScanT * kScanPer;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[wid] = x;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    uint32_t w = lane < nw ? sh[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) sh[lane] = w;
  }
  __syncthreads();
  total = sh[(blockDim.x >> 5) - 1];
  const uint32_t before = wid > 0 ? sh[wid - 1] : 0u;
  __syncthreads();
  return before + x - v;
}

__global__ void __launch_bounds__(kScanT) scan_blocks_kernel(uint32_t* data, int64_t n, uint32_t* tmp) {
  __shared__ uint32_t sh[32];
  const int64_t base = int64_t(blockIdx.x) * kScanChunk + int64_t(threadIdx.x) * kScanPer;
  uint32_t v[kScanPer], s = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    v[k] = base + k < n ? data[base + k] : 0u;
    s += v[k];
  }
  uint32_t total;
  uint32_t run = block_excl_scan(s, sh, total);
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    if (base + k < n) data[base + k] = run;
    run += v[k];
  }
  if (threadIdx.x == 0) tmp[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanT) scan_tops_kernel(uint32_t* tmp, int64_t nb, uint32_t* total_out) {
  __shared__ uint32_t sh[32];
  uint32_t carry = 0;
  for (int64_t b0 = 0; b0 < nb; b0 += kScanT) {
    const int64_t b = b0 + threadIdx.x;
    const uint32_t v = b < nb ? tmp[b] : 0u;
    uint32_t total;
    const uint32_t ex = block_excl_scan(v, sh, total);
    if (b < nb) tmp[b] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0 && total_out) *total_out = carry;
}

__global__ void __launch_bounds__(kScanT) scan_add_kernel(uint32_t* data, int64_t n, const uint32_t* tmp) {
  const uint32_t add = tmp[blockIdx.x];
  const int64_t base = int64_t(blockIdx.x) * kScanChunk;
  for (int k = threadIdx.x; k < kScanChunk; k += kScanT)
    if (base + k < n) data[base + k] += add;
}

cudaError_t scan(uint32_t* data, int64_t n, uint32_t* tmp, uint32_t* total, cudaStream_t st) {
  const int64_t nb = (n + kScanChunk - 1) / kScanChunk;
  if (nb == 0) return cudaSuccess;
  scan_blocks_kernel<<<unsigned(nb), kScanT, 0, st>>>(data, n, tmp);
  scan_tops_kernel<<<1, kScanT, 0, st>>>(tmp, nb, total);
  scan_add_kernel<<<unsigned(nb), kScanT, 0, st>>>(data, n, tmp);
  return cudaGetLastError();
}

unsigned grid_for(int64_t work) {
  int64_t b = (work + kT - 1) / kT;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return unsigned(b);
}


// ============================================================ penetration regions
// selbstkollision.rs:810-1058: edges through triangles (a hash of triangle
// boxes with the longest edge as cell), their regions (the reference's
// union-find, one thread), the push springs after the proximity pairs.

// the longest edge at positions x (atomicMax on the bits of a non-negative double)
__global__ void __launch_bounds__(kT) kante_max_kernel(const __grid_constant__ SelbstArgs s, const double* x,
                                                       unsigned long long* out) {
  double m = 0.0;
  SC_FOR(e, s.ne) {
    const uint2 k = s.k_idx[e];
    m = fmax(m, norm(ld3(x, k.x) - ld3(x, k.y)));
  }
  if (m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}
__device__ __forceinline__ double zelle_aus(const unsigned long long* lm) {
  return fmax(__longlong_as_double((long long)*lm), 1e-3);
}

// Hashgitter::neu over the boxes of g with the cell in *lm (selbstkollision.rs:281-322):
// distinct buckets per box counted, then (after a scan) filled, then sorted.
__global__ void __launch_bounds__(kT) hg_count_kernel(const HashG g, const unsigned long long* lm, uint32_t* zahl) {
  const double z = zelle_aus(lm);
  SC_FOR(b, g.m) {
    const Box q = box_of(g.lo, g.hi, b);
    uint32_t c = 0;
    je_eimer(q, z, g.eimer, [&](uint32_t h) {
      atomicAdd(&g.anf[h], 1u);
      ++c;
    });
    if (c) atomicAdd(zahl, c);
  }
}
__global__ void __launch_bounds__(kT) hg_fill_kernel(const HashG g, const unsigned long long* lm) {
  const double z = zelle_aus(lm);
  SC_FOR(b, g.m) {
    const Box q = box_of(g.lo, g.hi, b);
    je_eimer(q, z, g.eimer, [&](uint32_t h) {
      const uint32_t pos = g.anf[h] + atomicAdd(&g.cur[h], 1u);
      if (pos < g.cap) g.ein[pos] = uint32_t(b);
    });
  }
}
__global__ void __launch_bounds__(kT) hg_sort_kernel(const HashG g) {
  SC_FOR(b, g.eimer) sort_range(g.ein, g.anf[b], g.anf[b + 1]);
}

// triangle boxes of the intersection search (selbstkollision.rs:860)
__global__ void __launch_bounds__(kT) schnitt_boxen_kernel(const __grid_constant__ SelbstArgs s) {
  SC_FOR(t, s.nd) {
    const uint4 d = s.d_idx[t];
    const D3 p[3] = {ld3(s.x, d.x), ld3(s.x, d.y), ld3(s.x, d.z)};
    const Box b = quader_punkte(p, 3, kZuschlagQuader);
    s.hs.lo[t] = make_double4(b.lo.x, b.lo.y, b.lo.z, 0.0);
    s.hs.hi[t] = make_double4(b.hi.x, b.hi.y, b.hi.z, 0.0);
  }
}

__device__ __forceinline__ D3 lerp3(D3 a, D3 b, double t) { return a * (1.0 - t) + b * t; }
// selbstkollision.rs:1156-1171
__device__ bool im_dreieck(D3 a, D3 b, D3 c, D3 p, double& u, double& v) {
  const D3 e1 = b - a, e2 = c - a, r = p - a;
  const double d11 = dot(e1, e1), d12 = dot(e1, e2), d22 = dot(e2, e2);
  const double det = d11 * d22 - d12 * d12;
  if (det <= 1e-4 * d11 * d22) return false;
  const double r1 = dot(r, e1), r2 = dot(r, e2);
  u = (d22 * r1 - d12 * r2) / det;
  v = (d11 * r2 - d12 * r1) / det;
  return !(u < 0.0 || v < 0.0 || u + v > 1.0);
}
// selbstkollision.rs:830-846
__device__ bool kante_durch_dreieck(D3 a, D3 b, D3 v0, D3 v1, D3 v2, D3 n, double& t, double w[3]) {
  const double d0 = dot(n, a - v0), d1 = dot(n, b - v0);
  if ((d0 > 0.0 && d1 > 0.0) || (d0 < 0.0 && d1 < 0.0) || fabs(d1 - d0) < 1e-12) return false;
  t = -d0 / (d1 - d0);
  if (fabs(t) < 1e-5 || fabs(t - 1.0) < 1e-5) return false;
  const D3 p = lerp3(a, b, t);
  if (norm(v1 - v0) < kKanteMin || norm(v2 - v0) < kKanteMin) return false;
  double u, v;
  if (!im_dreieck(v0, v1, v2, p, u, v)) return false;
  w[0] = 1.0 - u - v;
  w[1] = u;
  w[2] = v;
  return true;
}

// The intersections of edge e (selbstkollision.rs:866-903), counted or
// written from `pos` on in the reference's order.
struct SchnittT {
  uint32_t t;
  double tk, w0, w1, w2;
  D3 n;
  double cn;
};
template <bool FILL>
__device__ uint32_t kante_schnitte(const SelbstArgs& s, const Gruppe& gr, int64_t e, uint32_t pos, double zelle) {
  const uint2 ka = s.k_idx[e];
  const uint2 kd = s.k_dr[e];
  const uint32_t a0 = ka.x, a1 = ka.y;
  if (a0 == a1 || kd.x == kKein) return 0;
  const D3 pa = ld3(s.x, a0), pb = ld3(s.x, a1);
  const D3 pe[2] = {pa, pb};
  const Box qe = quader_punkte(pe, 2, kZuschlagQuader);
  const D3 ehat = einheit(pb - pa);
  const auto pruefe = [&](uint32_t t, int64_t ci, int64_t cj, int64_t ck, uint32_t, SchnittT& o) -> bool {
    // the box first: the cheapest rejection (plain conditions, any order)
    const Box qt = box_of(s.hs.lo, s.hs.hi, t);
    if (!ueberlappt(qt, qe) || !erste_zelle(qe, qt, zelle, ci, cj, ck)) return false;
    const uint4 d = s.d_idx[t];
    const uint32_t dd[3] = {d.x, d.y, d.z};
    bool nachbar = false;
    for (int k = 0; k < 3; ++k)
      nachbar = nachbar || (s.an_naehten ? (dd[k] == a0 || dd[k] == a1)
                                         : (gleich_oder_partner(s, a0, dd[k]) || gleich_oder_partner(s, a1, dd[k])));
    if (nachbar) return false;
    const double4 n4 = s.nrm_t[t];
    const D3 n = d3(n4.x, n4.y, n4.z);
    double tk, w[3];
    if (!kante_durch_dreieck(pa, pb, ld3(s.x, d.x), ld3(s.x, d.y), ld3(s.x, d.z), n, tk, w)) return false;
    const double cn = dot(n, ehat);
    if (fabs(cn) < 1e-6) return false;
    if (FILL) {
      o.t = t;
      o.tk = tk;
      o.w0 = w[0], o.w1 = w[1], o.w2 = w[2];
      o.n = n;
      o.cn = cn;
    }
    return true;
  };
  const auto schreibe = [&](const SchnittT& o, uint32_t q) {
    const D3 p = lerp3(pa, pb, o.tk);
    D3 g = d3(0, 0, 0);
    const uint32_t kk[2] = {kd.x, kd.y};
    for (int r = 0; r < 2; ++r) {
      if (kk[r] == kKein) continue;
      const uint4 dk = s.d_idx[kk[r]];
      const uint32_t dkk[3] = {dk.x, dk.y, dk.z};
      uint32_t ot = kKein;
      for (int a = 0; a < 3; ++a)
        if (dkk[a] != a0 && dkk[a] != a1) {
          ot = dkk[a];
          break;
        }
      if (ot == kKein) continue;
      const double4 m4 = s.nrm_t[kk[r]];
      D3 m = einheit(cross(o.n, d3(m4.x, m4.y, m4.z)));
      const D3 rr = ld3(s.x, ot) - p;
      const D3 r_quer = rr - ehat * dot(ehat, rr);
      if (dot(m, r_quer) < 0.0) m = m * -1.0;
      g = g + (m - o.n * (dot(ehat, m) / o.cn));
    }
    const double lg = norm(g);
    if (q < s.cap_s) {
      const D3 gh = einheit(g);
      s.sn_ke[q] = make_uint2(uint32_t(e), o.t);
      s.sn_t[q] = o.tk;
      s.sn_w[q] = make_double4(o.w0, o.w1, o.w2, 0.0);
      s.sn_g[q] = make_double4(gh.x, gh.y, gh.z, lg / sqrt(lg * lg + 2.25));
    }
  };
  if constexpr (FILL) {
    return je_eintrag_gruppe<true, SchnittT>(gr, qe, zelle, s.hs.eimer, s.hs.anf, s.hs.ein, s.hs.elo, s.hs.ehi,
                                      pos, pruefe, schreibe);
  } else {
    return zaehle_gruppe<SchnittT, true>(gr, qe, zelle, s.hs.eimer, s.hs.anf, s.hs.ein, s.hs.elo, s.hs.ehi, pruefe,
                                         [](uint32_t) { return true; });
  }
}
__global__ void __launch_bounds__(kT, 4) schnitt_count_kernel(const __grid_constant__ SelbstArgs s) {
  const double z = zelle_aus(&s.lmax[0]);
  if (blockIdx.x == 0 && threadIdx.x == 0) s.off_s[s.ne] = 0u;
  const Gruppe gr = gruppe();
  je_gezogen(gr.maske, int(threadIdx.x & 31) & ~(kG - 1), &s.zahl[SZ_ARBEIT_S], uint64_t(s.ne), [&](uint32_t e) {
    const uint32_t c = kante_schnitte<false>(s, gr, e, 0, z);
    if (gr.lane == 0) {
      s.off_s[e] = c;
      if (c) s.aktiv_s[atomicAdd(&s.zahl[SZ_AKTIV_S], 1u)] = e;
    }
  });
}
// fill pass over the listed edges (their starts come from the scan)
__global__ void __launch_bounds__(kT, 4) schnitt_fill_kernel(const __grid_constant__ SelbstArgs s, uint32_t n_aktiv) {
  const double z = zelle_aus(&s.lmax[0]);
  const Gruppe gr = gruppe();
  GR_FOR(q, n_aktiv) {
    const uint32_t e = s.aktiv_s[q];
    kante_schnitte<true>(s, gr, e, s.off_s[e], z);
  }
}

// finde(e, t): the intersection of edge e with triangle t (the list is edge by edge)
__device__ __forceinline__ uint32_t finde_schnitt(const SelbstArgs& s, uint32_t e, uint32_t t) {
  const uint32_t a = s.off_s[e], b = s.off_s[e + 1];
  for (uint32_t q = a; q < b; ++q)
    if (s.sn_ke[q].y == t) return q;
  return kKein;
}
__device__ __forceinline__ uint32_t wurzel(uint32_t* el, uint32_t i) {
  while (el[i] != i) {
    el[i] = el[el[i]];
    i = el[i];
  }
  return i;
}
__device__ __forceinline__ void vereinige(uint32_t* el, uint32_t a, uint32_t b) {
  const uint32_t ra = wurzel(el, a), rb = wurzel(el, b);
  if (ra != rb) el[ra > rb ? ra : rb] = ra < rb ? ra : rb;
}
// gebiete (selbstkollision.rs:931-1009). Linking the larger root under the
// smaller one makes every root the smallest member of its set, so the
// partition and the roots after the unions of the first loop do not depend
// on their order: those run in parallel (lock-free union-find). The role
// swaps are listed per intersection in the reference's order (counted,
// scanned, filled); the two swap rounds, whose unions do depend on the
// order, and the direction sums (in intersection order) run on one thread of
// one block, in shared memory when the intersections fit.

// the intersections of i's region (gleich) and its role swaps (tausch), in
// the reference's order (selbstkollision.rs:947-981)
template <class F, class G>
__device__ __forceinline__ void gebiet_nachbarn(const SelbstArgs& s, uint32_t i, F&& gleich, G&& tausch) {
  const uint2 et = s.sn_ke[i];
  const uint32_t e = et.x, t = et.y;
  const uint2 kd2 = s.k_dr[e];
  uint32_t kde[2], nk = 0;
  if (kd2.x != kKein) kde[nk++] = kd2.x;
  if (kd2.y != kKein) kde[nk++] = kd2.y;
  uint32_t andere[6], na = 0;
  for (uint32_t q = 0; q < nk; ++q) {
    const uint4 dk = s.d_kan[kde[q]];
    const uint32_t f3[3] = {dk.x, dk.y, dk.z};
    for (int a = 0; a < 3; ++a)
      if (f3[a] != e) andere[na++] = f3[a];
  }
  uint32_t tn[6], ntn = 0;  // nachbardreiecke(t)
  {
    const uint4 dk = s.d_kan[t];
    const uint32_t f3[3] = {dk.x, dk.y, dk.z};
    for (int a = 0; a < 3; ++a) {
      const uint2 u2 = s.k_dr[f3[a]];
      if (u2.x != kKein && u2.x != t) tn[ntn++] = u2.x;
      if (u2.y != kKein && u2.y != t) tn[ntn++] = u2.y;
    }
  }
  for (uint32_t a = 0; a < na; ++a) {
    const uint32_t j = finde_schnitt(s, andere[a], t);
    if (j != kKein) gleich(j);
  }
  for (uint32_t u = 0; u < ntn; ++u) {
    uint32_t j = finde_schnitt(s, e, tn[u]);
    if (j != kKein) gleich(j);
    for (uint32_t a = 0; a < na; ++a) {
      j = finde_schnitt(s, andere[a], tn[u]);
      if (j != kKein) gleich(j);
    }
  }
  const uint4 dt = s.d_kan[t];
  const uint32_t ft[3] = {dt.x, dt.y, dt.z};
  for (int a = 0; a < 3; ++a)
    for (uint32_t q = 0; q < nk; ++q) {
      const uint32_t j = finde_schnitt(s, ft[a], kde[q]);
      if (j != kKein) tausch(j);
    }
}
__device__ __forceinline__ uint32_t anzahl_schnitte(const SelbstArgs& s) {
  return s.zahl[SZ_SCHNITTE] < s.cap_s ? s.zahl[SZ_SCHNITTE] : s.cap_s;
}
// the root of x while other threads link roots (reads only)
__device__ __forceinline__ uint32_t wurzel_lesen(const volatile uint32_t* el, uint32_t x) {
  uint32_t p = el[x];
  while (p != x) {
    x = p;
    p = el[x];
  }
  return x;
}
__device__ __forceinline__ void vereinige_parallel(uint32_t* el, uint32_t a, uint32_t b) {
  for (;;) {
    a = wurzel_lesen(el, a);
    b = wurzel_lesen(el, b);
    if (a == b) return;
    if (a > b) {
      const uint32_t c = a;
      a = b;
      b = c;
    }
    if (atomicCAS(&el[b], b, a) == b) return;  // else b was linked meanwhile: again from the new roots
  }
}
__global__ void __launch_bounds__(kT) gebiete_init_kernel(const __grid_constant__ SelbstArgs s) {
  const uint32_t n = anzahl_schnitte(s);
  SC_FOR(i, n) s.sn_eltern[i] = uint32_t(i);
  if (blockIdx.x == 0 && threadIdx.x == 0) s.sn_toff[n] = 0u;
}
// the first loop's unions; the role swaps per intersection counted
__global__ void __launch_bounds__(kT) gebiete_vereinigen_kernel(const __grid_constant__ SelbstArgs s) {
  const uint32_t n = anzahl_schnitte(s);
  SC_FOR(i, n) {
    uint32_t nt = 0;
    gebiet_nachbarn(s, uint32_t(i), [&](uint32_t j) { vereinige_parallel(s.sn_eltern, uint32_t(i), j); },
                    [&](uint32_t) { ++nt; });
    s.sn_toff[i] = nt;
  }
}
__global__ void __launch_bounds__(kT) gebiete_tausch_kernel(const __grid_constant__ SelbstArgs s) {
  const uint32_t n = anzahl_schnitte(s);
  SC_FOR(i, n) {
    uint32_t q = s.sn_toff[i];
    gebiet_nachbarn(s, uint32_t(i), [&](uint32_t) {},
                    [&](uint32_t j) { s.sn_tausch[q++] = make_uint2(uint32_t(i), j); });
  }
}
constexpr uint32_t kGebietSmem = 2048;
constexpr size_t kGebietSmemBytes = size_t(kGebietSmem) * (2 * sizeof(uint32_t) + 3 * sizeof(double) + sizeof(double4));
// the two swap rounds, the roots, the direction sums (one block)
__global__ void __launch_bounds__(1024) gebiete_runden_kernel(const __grid_constant__ SelbstArgs s) {
  extern __shared__ double gsh[];
  __shared__ uint32_t gebiete;
  const uint32_t n = anzahl_schnitte(s), nt = s.sn_toff[n];
  const bool sm = n <= kGebietSmem;
  double4* g = reinterpret_cast<double4*>(gsh);
  double* summe = gsh + 4 * kGebietSmem;
  uint32_t* el = sm ? reinterpret_cast<uint32_t*>(summe + 3 * kGebietSmem) : s.sn_eltern;
  uint32_t* partner = sm ? el + kGebietSmem : s.sn_partner;
  if (threadIdx.x == 0) gebiete = 0;
  if (sm)
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
      el[i] = s.sn_eltern[i];
      g[i] = s.sn_g[i];
      summe[3 * i] = summe[3 * i + 1] = summe[3 * i + 2] = 0.0;
    }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int runde = 0; runde < 2; ++runde) {
      for (uint32_t i = 0; i < n; ++i) partner[i] = kKein;
      for (uint32_t q = 0; q < nt; ++q) {
        const uint2 ij = s.sn_tausch[q];
        const uint32_t ri = wurzel(el, ij.x), rj = wurzel(el, ij.y);
        if (rj < partner[ri]) partner[ri] = rj;
        if (ri < partner[rj]) partner[rj] = ri;
      }
      for (uint32_t q = 0; q < nt; ++q) {
        const uint2 ij = s.sn_tausch[q];
        const uint32_t rj = wurzel(el, ij.y);
        if (partner[rj] != kKein) vereinige(el, ij.x, partner[rj]);
      }
    }
  }
  __syncthreads();
  uint32_t eigene = 0;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const uint32_t r = wurzel_lesen(el, i);
    s.sn_wurzel[i] = r;
    if (r == i) ++eigene;
    if (!sm) s.sn_summe[i] = make_double4(0, 0, 0, 0);
  }
  if (eigene) atomicAdd(&gebiete, eigene);
  __syncthreads();
  if (threadIdx.x == 0) {  // the sums in intersection order, as the reference adds them
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t r = s.sn_wurzel[i];
      if (sm) {
        const double4 gi = g[i];
        summe[3 * r] += gi.x * gi.w;
        summe[3 * r + 1] += gi.y * gi.w;
        summe[3 * r + 2] += gi.z * gi.w;
      } else {
        const double4 gi = s.sn_g[i];
        double4& m = s.sn_summe[r];
        m.x += gi.x * gi.w;
        m.y += gi.y * gi.w;
        m.z += gi.z * gi.w;
      }
    }
    s.zahl[SZ_GEBIETE] = gebiete;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const uint32_t r = s.sn_wurzel[i];
    const D3 m = sm ? d3(summe[3 * r], summe[3 * r + 1], summe[3 * r + 2])
                    : d3(s.sn_summe[r].x, s.sn_summe[r].y, s.sn_summe[r].z);
    const D3 u = einheit(m);
    s.sn_g[i] = make_double4(u.x, u.y, u.z, s.sn_g[i].w);
  }
}

// the first body in contact at point i (implizit.rs:700)
__device__ bool erste_normale(const SelbstArgs& s, uint32_t i, D3& n) {
  const D3 x = ld3(s.x, i);
  for (int kb = 0; kb < s.n_bodies; ++kb) {
    double ti;
    if (kontakt(s.bodies[kb], x, s.kabst[i] + s.rand, n, ti)) return true;
  }
  return false;
}
// hat per triangle; pinched regions (implizit.rs:701-704)
__global__ void __launch_bounds__(kT) klemm_kernel(const __grid_constant__ SelbstArgs s) {
  const uint32_t n = s.zahl[SZ_SCHNITTE] < s.cap_s ? s.zahl[SZ_SCHNITTE] : s.cap_s;
  SC_FOR(i, n) {
    const uint2 et = s.sn_ke[i];
    s.hat[et.y] = 1;
    if (s.n_bodies == 0) continue;
    const uint2 kp = s.k_idx[et.x];
    const uint4 dp = s.d_idx[et.y];
    const uint32_t dd[3] = {dp.x, dp.y, dp.z};
    D3 summe = d3(0, 0, 0), nk;
    for (int a = 0; a < 3; ++a)
      if (erste_normale(s, dd[a], nk)) summe = summe + nk;
    if (!(norm(summe) > 0.0)) continue;
    bool k = false;
    if (erste_normale(s, kp.x, nk) && dot(nk, summe) < 0.0) k = true;
    if (!k && erste_normale(s, kp.y, nk) && dot(nk, summe) < 0.0) k = true;
    if (k) s.klemm[s.sn_wurzel[i]] = 1;
  }
}
__global__ void __launch_bounds__(kT) folge_kernel(const __grid_constant__ SelbstArgs s) {
  SC_FOR(t, s.nd) s.folge[t] = s.hat[t] ? s.folge[t] + 1u : 1u;
}
// schubfedern (selbstkollision.rs:1014-1058) after the proximity pairs
template <typename R>
__global__ void __launch_bounds__(kT) schub_kernel(const __grid_constant__ SelbstArgs s) {
  const uint32_t n = s.zahl[SZ_SCHNITTE] < s.cap_s ? s.zahl[SZ_SCHNITTE] : s.cap_s;
  const uint32_t P = paare(s);
  R4<R>* bR = static_cast<R4<R>*>(s.pr_bR);
  R4<R>* wR = static_cast<R4<R>*>(s.pr_wR);
  R* g5R = static_cast<R*>(s.pr_g5R);
  const double h2 = s.h * s.h;
  SC_FOR(i, n) {
    // spring P + i; a pinched region's springs stay in the list with zero
    // weights (no entries, no force), so the list keeps the reference's order
    const uint32_t q = P + uint32_t(i);
    if (q >= s.cap_pairs) continue;
    const bool aus = s.klemm[s.sn_wurzel[i]] != 0;
    const uint2 et = s.sn_ke[i];
    const uint32_t e = et.x, t = et.y;
    const double k = 2.0 * s.steifigkeit * (s.e_kante[e] + s.e_dreieck[t]) * (s.a_kante[e] + s.a_dreieck[t]) / 1e-6;
    const double4 g4 = s.sn_g[i];
    const D3 g = d3(g4.x, g4.y, g4.z);
    const double f = k * double(s.folge[t] < 5u ? s.folge[t] : 5u) * 1e-3;
    const double tk = s.sn_t[i];
    const double4 w = s.sn_w[i];
    const uint2 kp = s.k_idx[e];
    const uint4 dp = s.d_idx[t];
    const double on = aus ? 0.0 : 1.0;
    s.pr_idx[q] = make_uint4(kp.x, kp.y, dp.x, dp.y);
    s.pr_x5[q] = dp.z;
    s.pr_w[q] = make_double4(on * (1.0 - tk), on * tk, -on * w.x, -on * w.y);
    s.pr_g5[q] = -on * w.z;
    s.pr_kf[q] = make_double4(g.x * f, g.y * f, g.z * f, k);
    const double bxx = k * g.x * g.x, byy = k * g.y * g.y, bzz = k * g.z * g.z;
    const double bxy = k * g.x * g.y, bxz = k * g.x * g.z, byz = k * g.y * g.z;
    s.pr_b0[q] = make_double4(bxx, byy, bzz, bxy);
    s.pr_b1[q] = make_double4(bxz, byz, 0.0, 0.0);
    bR[2 * q] = {R(h2 * bxx), R(h2 * byy), R(h2 * bzz), R(h2 * bxy)};
    bR[2 * q + 1] = {R(h2 * bxz), R(h2 * byz), R(0), R(0)};
    wR[q] = {R(on * (1.0 - tk)), R(on * tk), R(-on * w.x), R(-on * w.y)};
    g5R[q] = R(-on * w.z);
  }
}
// per triangle: its intersections (for the impacts' filter)
__global__ void __launch_bounds__(kT) t_count_kernel(const __grid_constant__ SelbstArgs s) {
  const uint32_t n = s.zahl[SZ_SCHNITTE] < s.cap_s ? s.zahl[SZ_SCHNITTE] : s.cap_s;
  SC_FOR(i, n) atomicAdd(&s.t_off[s.sn_ke[i].y], 1u);
}
__global__ void __launch_bounds__(kT) t_fill_kernel(const __grid_constant__ SelbstArgs s) {
  const uint32_t n = s.zahl[SZ_SCHNITTE] < s.cap_s ? s.zahl[SZ_SCHNITTE] : s.cap_s;
  SC_FOR(i, n) {
    const uint32_t t = s.sn_ke[i].y;
    s.t_ent[s.t_off[t] + atomicAdd(&s.t_cur[t], 1u)] = uint32_t(i);
  }
}

// ============================================================ impacts
// selbstkollision.rs:1063-1343 on the way x0 -> x1 (x1 = the step's x).
constexpr double kStossAbstand = 1e-4;  // selbstkollision.rs:1090
constexpr double kStossKanteMin = 1e-4;  // :1092

// path boxes (selbstkollision.rs:1199-1203): points, edges, triangles
__global__ void __launch_bounds__(kT) weg_boxen_kernel(const __grid_constant__ SelbstArgs s) {
  SC_FOR(v, s.n) {
    const D3 p[2] = {ld3(s.x0, uint32_t(v)), ld3(s.xs, uint32_t(v))};
    const Box b = quader_punkte(p, 2, 1e-8);
    s.hp2.lo[v] = make_double4(b.lo.x, b.lo.y, b.lo.z, 0.0);
    s.hp2.hi[v] = make_double4(b.hi.x, b.hi.y, b.hi.z, 0.0);
  }
  SC_FOR(e, s.ne) {
    const uint2 k = s.k_idx[e];
    const D3 p[4] = {ld3(s.x0, k.x), ld3(s.x0, k.y), ld3(s.xs, k.x), ld3(s.xs, k.y)};
    const Box b = quader_punkte(p, 4, 1e-8);
    s.hk2.lo[e] = make_double4(b.lo.x, b.lo.y, b.lo.z, 0.0);
    s.hk2.hi[e] = make_double4(b.hi.x, b.hi.y, b.hi.z, 0.0);
  }
  SC_FOR(t, s.nd) {
    const uint4 d = s.d_idx[t];
    const D3 p[6] = {ld3(s.x0, d.x), ld3(s.x0, d.y), ld3(s.x0, d.z), ld3(s.xs, d.x), ld3(s.xs, d.y), ld3(s.xs, d.z)};
    const Box b = quader_punkte(p, 6, 1e-8);
    s.qt2_lo[t] = make_double4(b.lo.x, b.lo.y, b.lo.z, 0.0);
    s.qt2_hi[t] = make_double4(b.hi.x, b.hi.y, b.hi.z, 0.0);
  }
}

__device__ __forceinline__ double ebenenabstand(D3 a, D3 b, D3 c, D3 p) { return dot(p - a, einheit(cross(b - a, c - a))); }
// Whether the unnormalised triple product (p - a).((b - a) x (c - a)) has the
// same strict sign at the step's start and end, far enough from zero that the
// reference's ebenenabstand (the same product divided by |(b - a) x (c - a)|,
// which then exceeds its 1e-12 floor) has that sign too. The margin 1e-12 of
// the product of the operands' L1 norms is far above the rounding of either
// form. True means f(0) f(1) > 0, so koplanar_zeit returns false at once; it
// saves the two square roots and divisions of that test.
__device__ __forceinline__ double tripel(const D3 q[4], double& grenze, double& n2) {
  const D3 u = q[1] - q[0], v = q[2] - q[0], w = q[3] - q[0];
  const D3 c = cross(u, v);
  n2 = dot(c, c);
  auto l1 = [](D3 a) { return fabs(a.x) + fabs(a.y) + fabs(a.z); };
  grenze = 1e-12 * l1(w) * l1(u) * l1(v);
  return dot(w, c);
}
__device__ __forceinline__ bool gleiche_seite(const D3 x0[4], const D3 x1[4]) {
  double g0, g1, n0, n1;
  const double t0 = tripel(x0, g0, n0), t1 = tripel(x1, g1, n1);
  const double n_min = 1.0000001e-24;  // |cross| clearly above einheit's 1e-12 floor
  return n0 > n_min && n1 > n_min && fabs(t0) > g0 && fabs(t1) > g1 && ((t0 > 0.0) == (t1 > 0.0));
}

// selbstkollision.rs:1128-1153 (regula falsi, 16 steps)
__device__ bool koplanar_zeit(const D3 x0[4], const D3 x1[4], double tol, double& out) {
  if (gleiche_seite(x0, x1)) return false;
  auto f = [&](double t) {
    return ebenenabstand(lerp3(x0[0], x1[0], t), lerp3(x0[1], x1[1], t), lerp3(x0[2], x1[2], t),
                         lerp3(x0[3], x1[3], t));
  };
  double t0 = 0.0, t1 = 1.0, d0 = f(0.0), d1 = f(1.0);
  for (int it = 0; it < 16; ++it) {
    if (d0 * d1 > 0.0) return false;
    const double tau = t0 + (t1 - t0) * fabs(d0) / fmax(fabs(d0) + fabs(d1), DBL_MIN);
    const double d = f(tau);
    if (fabs(d) < tol || t1 - t0 < 1e-4) {
      out = tau;
      return true;
    }
    if (d0 * d > 0.0) {
      t0 = tau;
      d0 = d;
    } else {
      t1 = tau;
      d1 = d;
    }
  }
  return false;
}
// selbstkollision.rs:1173-1193
__device__ bool kanten_kreuzen(D3 a, D3 b, D3 c, D3 d, double& so, double& wo) {
  const D3 e1 = b - a, e2 = d - c;
  const double l1 = norm(e1), l2 = norm(e2);
  if (l1 < kStossKanteMin || l2 < kStossKanteMin) return false;
  const D3 u1 = e1 * (1.0 / l1), u2 = e2 * (1.0 / l2);
  const double g = dot(u1, u2);
  if (fabs(g) > 0.99999) return false;
  const D3 q = c - a;
  const double nen = 1.0 - g * g;
  const double sv = (dot(q, u1) - g * dot(q, u2)) / nen;
  const double wv = (g * dot(q, u1) - dot(q, u2)) / nen;
  if (sv <= 0.0 || sv >= l1 || wv <= 0.0 || wv >= l2) return false;
  so = sv / l1;
  wo = wv / l2;
  return true;
}

// One candidate of the impact searches: every condition of the reference's
// loop body, the candidate's impact time and what the search writes for it.
// `grenze`: with `hat`, a candidate at that time or later cannot win (the
// search keeps the first of equal times) and is dropped before the expensive
// part, as the reference's loop does.
struct StossPD {
  double zeit, u, v, seite;
  D3 n;
  uint32_t p;
};
__device__ __forceinline__ bool stoss_pd_kandidat(const SelbstArgs& s, const uint32_t (&d)[3], const Box& qt, double z,
                                                  uint32_t v, int64_t ci, int64_t cj, int64_t ck, bool hat,
                                                  double grenze, StossPD& o) {
  const Box qv = box_of(s.hp2.lo, s.hp2.hi, v);
  if (!ueberlappt(qv, qt) || !erste_zelle(qt, qv, z, ci, cj, ck)) return false;
  for (int k = 0; k < 3; ++k)
    if (gleich_oder_partner(s, v, d[k])) return false;
  const uint32_t idx[4] = {d[0], d[1], d[2], v};
  if (s.w[idx[0]] <= 0.0 && s.w[idx[1]] <= 0.0 && s.w[idx[2]] <= 0.0 && s.w[idx[3]] <= 0.0) return false;
  D3 a0[4], a1[4];
  for (int k = 0; k < 4; ++k) {
    a0[k] = ld3(s.x0, idx[k]);
    a1[k] = ld3(s.xs, idx[k]);
  }
  double zeit;
  if (!koplanar_zeit(a0, a1, kStossAbstand * 0.1, zeit)) return false;
  if (hat && grenze <= zeit) return false;
  D3 q[4];
  for (int k = 0; k < 4; ++k) q[k] = lerp3(a0[k], a1[k], zeit);
  double u, vv;
  if (!im_dreieck(q[0], q[1], q[2], q[3], u, vv)) return false;
  const D3 n = einheit(cross(q[1] - q[0], q[2] - q[0]));
  const double g[3] = {1.0 - u - vv, u, vv};
  const D3 rel = (a1[3] - a0[3]) - (((a1[0] - a0[0]) * g[0] + (a1[1] - a0[1]) * g[1]) + (a1[2] - a0[2]) * g[2]);
  o.zeit = zeit;
  o.u = u;
  o.v = vv;
  o.seite = dot(rel, n) <= 0.0 ? 1.0 : -1.0;
  o.n = n;
  o.p = v;
  return true;
}
__device__ __forceinline__ void stoss_pd_schreiben(const SelbstArgs& s, int64_t t, const uint32_t (&d)[3],
                                                   const StossPD& o) {
  s.st_idx[t] = make_uint4(o.p, d[0], d[1], d[2]);
  s.st_lzs[t] = make_double4(o.u, o.v, o.zeit, o.seite);
  s.st_n[t] = make_double4(o.n.x * o.seite, o.n.y * o.seite, o.n.z * o.seite, 0.0);
  s.st_art[t] = 1u;
}
struct StossKK {
  double zeit, sv, wv, seite;
  D3 n;
  uint32_t j, b0, b1;
};
__device__ __forceinline__ bool stoss_kk_kandidat(const SelbstArgs& s, int64_t i, uint32_t i0, uint32_t i1,
                                                  const Box& qi, const Box32& qi32, double z, uint32_t j, int64_t ci,
                                                  int64_t cj, int64_t ck, uint32_t sq, bool hat, double grenze,
                                                  StossKK& o) {
  if (int64_t(j) <= i) return false;
  if (!ueberlappt32(qi32, s.hk2.elo[sq], s.hk2.ehi[sq])) return false;
  const Box qj = box_of(s.hk2.lo, s.hk2.hi, j);
  if (!ueberlappt(qi, qj) || !erste_zelle(qi, qj, z, ci, cj, ck)) return false;
  const uint2 kj = s.k_idx[j];
  if (gleich_oder_partner(s, kj.x, i0) || gleich_oder_partner(s, kj.x, i1) || gleich_oder_partner(s, kj.y, i0) ||
      gleich_oder_partner(s, kj.y, i1))
    return false;
  const uint32_t idx[4] = {i1, kj.x, kj.y, i0};
  if (s.w[idx[0]] <= 0.0 && s.w[idx[1]] <= 0.0 && s.w[idx[2]] <= 0.0 && s.w[idx[3]] <= 0.0) return false;
  D3 a0[4], a1[4];
  for (int k = 0; k < 4; ++k) {
    a0[k] = ld3(s.x0, idx[k]);
    a1[k] = ld3(s.xs, idx[k]);
  }
  double zeit;
  if (!koplanar_zeit(a0, a1, kStossAbstand * 0.1, zeit)) return false;
  if (hat && grenze <= zeit) return false;
  D3 q[4];
  for (int k = 0; k < 4; ++k) q[k] = lerp3(a0[k], a1[k], zeit);
  double sv, wv;
  if (!kanten_kreuzen(q[3], q[0], q[1], q[2], sv, wv)) return false;
  const D3 n = einheit(cross(q[0] - q[3], q[2] - q[1]));
  const D3 auf_i = (a1[3] - a0[3]) * (1.0 - sv) + (a1[0] - a0[0]) * sv;
  const D3 auf_j = (a1[1] - a0[1]) * (1.0 - wv) + (a1[2] - a0[2]) * wv;
  o.zeit = zeit;
  o.sv = sv;
  o.wv = wv;
  o.seite = dot(auf_i - auf_j, n) <= 0.0 ? 1.0 : -1.0;
  o.n = n;
  o.j = j;
  o.b0 = kj.x;
  o.b1 = kj.y;
  return true;
}
__device__ __forceinline__ void stoss_kk_schreiben(const SelbstArgs& s, uint32_t slot, uint32_t i0, uint32_t i1,
                                                   const StossKK& o) {
  s.st_idx[slot] = make_uint4(i0, i1, o.b0, o.b1);
  s.st_lzs[slot] = make_double4(o.sv, o.wv, o.zeit, o.seite);
  s.st_n[slot] = make_double4(o.n.x * o.seite, o.n.y * o.seite, o.n.z * o.seite, double(o.j));  // .w: the partner edge
  s.st_art[slot] = 2u;
}

// The candidates a query visits: the entries of its cells' buckets (cells
// counted with repeats, as the search walks them), saturating.
__device__ __forceinline__ uint32_t kandidaten(const Box& q, double z, const HashG& g) {
  if (!zellbereich_ok(q, z)) return 0;
  const Cells c = cells_of(q, z);
  uint32_t n = 0;
  for (uint32_t a = 0; a < c.total && n < 0x80000000u; ++a) {
    int64_t i, j, k;
    cell_at(c, a, i, j, k);
    const uint32_t h = streue(i, j, k, g.eimer);
    n += g.anf[h + 1] - g.anf[h];
  }
  return n;
}
// A query with more candidates than this goes to the cooperative pass: one
// warp takes it, so a few queries on crowded buckets (the path boxes may span
// up to 64 cells an axis, and buckets of several thousand entries occur) do
// not hold their warps for the whole search.
constexpr uint32_t kSchwer = 256;

// The warp's first hit by (time, visit ordinal): the reference's loop keeps
// the earliest time and, among equal times, the first candidate it visits.
// Lane `beste` holds it; -1 when no lane has one.
__device__ __forceinline__ int warp_erster(bool hat, double zeit, uint64_t ord) {
  const unsigned voll = 0xffffffffu;
  double zm = hat ? zeit : INFINITY;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) zm = fmin(zm, __shfl_xor_sync(voll, zm, o));
  uint64_t om = hat && zeit == zm ? ord : ~0ull;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const uint64_t x = __shfl_xor_sync(voll, om, o);
    om = x < om ? x : om;
  }
  const unsigned wer = __ballot_sync(voll, hat && zeit == zm && ord == om);
  return wer ? __ffs(wer) - 1 : -1;
}

// the earliest point through triangle t (selbstkollision.rs:1215-1251)
__global__ void __launch_bounds__(kT, 4) stoss_pd_kernel(const __grid_constant__ SelbstArgs s) {
  const double z = zelle_aus(&s.lmax[1]);
  SC_FOR(t, s.nd) {
    s.st_art[t] = 0u;
    const uint4 dq = s.d_idx[t];
    const uint32_t d[3] = {dq.x, dq.y, dq.z};
    if (d[0] == d[1] || d[1] == d[2] || d[0] == d[2]) continue;
    const Box qt = box_of(s.qt2_lo, s.qt2_hi, t);
    if (kandidaten(qt, z, s.hp2) > kSchwer) {
      s.schwer_pd[atomicAdd(&s.zahl[SZ_SCHWER_PD], 1u)] = uint32_t(t);
      continue;
    }
    bool hat = false;
    StossPD best{};
    je_eintrag(qt, z, s.hp2.eimer, s.hp2.anf, s.hp2.ein, s.hp2.elo, s.hp2.ehi,
               [&](uint32_t v, int64_t ci, int64_t cj, int64_t ck, uint32_t) {
                 StossPD o;
                 if (stoss_pd_kandidat(s, d, qt, z, v, ci, cj, ck, hat, best.zeit, o)) {
                   hat = true;
                   best = o;
                 }
               });
    if (hat) stoss_pd_schreiben(s, t, d, best);
  }
}
// the earliest partner edge of edge i (selbstkollision.rs:1253-1283)
__global__ void __launch_bounds__(kT, 4) stoss_kk_kernel(const __grid_constant__ SelbstArgs s) {
  const double z = zelle_aus(&s.lmax[1]);
  SC_FOR(i, s.ne) {
    const uint32_t slot = uint32_t(s.nd + i);
    s.st_art[slot] = 0u;
    const uint2 ki = s.k_idx[i];
    const uint32_t i0 = ki.x, i1 = ki.y;
    if (i0 == i1) continue;
    const Box qi = box_of(s.hk2.lo, s.hk2.hi, i);
    if (kandidaten(qi, z, s.hk2) > kSchwer) {
      s.schwer_kk[atomicAdd(&s.zahl[SZ_SCHWER_KK], 1u)] = uint32_t(i);
      continue;
    }
    bool hat = false;
    StossKK best{};
    const Box32 qi32 = box32(qi);
    je_eintrag(qi, z, s.hk2.eimer, s.hk2.anf, s.hk2.ein, nullptr, nullptr,
               [&](uint32_t j, int64_t ci, int64_t cj, int64_t ck, uint32_t sq) {
                 StossKK o;
                 if (stoss_kk_kandidat(s, i, i0, i1, qi, qi32, z, j, ci, cj, ck, sq, hat, best.zeit, o)) {
                   hat = true;
                   best = o;
                 }
               });
    if (hat) stoss_kk_schreiben(s, slot, i0, i1, best);
  }
}
// The listed heavy queries, one warp each: the lanes take a cell's entries in
// turn (entry position lane, lane + 32, ...), each keeps its first hit by
// time (its own visits are in the reference's order), and the warp's first
// by (time, cell, position) writes the result.
__global__ void __launch_bounds__(kT, 4) stoss_pd_schwer_kernel(const __grid_constant__ SelbstArgs s) {
  const double z = zelle_aus(&s.lmax[1]);
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t m = s.zahl[SZ_SCHWER_PD];
  je_gezogen(0xffffffffu, 0, &s.zahl[SZ_ARBEIT_PD], m, [&](uint32_t w) {
    const uint32_t t = s.schwer_pd[w];
    const uint4 dq = s.d_idx[t];
    const uint32_t d[3] = {dq.x, dq.y, dq.z};
    const Box qt = box_of(s.qt2_lo, s.qt2_hi, t);
    const Cells c = cells_of(qt, z);  // zellbereich_ok held: the query had candidates
    const Box32 q32 = box32(qt);
    bool hat = false;
    StossPD best{};
    uint64_t ord = 0;
    for (uint32_t a = 0; a < c.total; ++a) {
      int64_t i, j, k;
      cell_at(c, a, i, j, k);
      const uint32_t h = streue(i, j, k, s.hp2.eimer);
      const uint32_t lo = s.hp2.anf[h], hi = s.hp2.anf[h + 1];
      const auto treffer = [&](uint32_t v, uint32_t e) {
        StossPD o;
        if (stoss_pd_kandidat(s, d, qt, z, v, i, j, k, hat, best.zeit, o)) {
          hat = true;
          best = o;
          ord = (uint64_t(a) << 32) | e;
        }
      };
      je_ueberlappend<8>(lo + lane, hi, 32u, q32, s.hp2.elo, s.hp2.ehi, s.hp2.ein, [](uint32_t) { return true; },
                      treffer);
    }
    const int wer = warp_erster(hat, best.zeit, ord);
    if (wer >= 0 && int(lane) == wer) stoss_pd_schreiben(s, t, d, best);
  });
}
__global__ void __launch_bounds__(kT, 4) stoss_kk_schwer_kernel(const __grid_constant__ SelbstArgs s) {
  const double z = zelle_aus(&s.lmax[1]);
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t m = s.zahl[SZ_SCHWER_KK];
  je_gezogen(0xffffffffu, 0, &s.zahl[SZ_ARBEIT_KK], m, [&](uint32_t w) {
    const int64_t ie = s.schwer_kk[w];
    const uint32_t slot = uint32_t(s.nd + ie);
    const uint2 ki = s.k_idx[ie];
    const uint32_t i0 = ki.x, i1 = ki.y;
    const Box qi = box_of(s.hk2.lo, s.hk2.hi, ie);
    const Cells c = cells_of(qi, z);
    const Box32 qi32 = box32(qi);
    bool hat = false;
    StossKK best{};
    uint64_t ord = 0;
    for (uint32_t a = 0; a < c.total; ++a) {
      int64_t i, j, k;
      cell_at(c, a, i, j, k);
      const uint32_t h = streue(i, j, k, s.hk2.eimer);
      const uint32_t lo = s.hk2.anf[h], hi = s.hk2.anf[h + 1];
      const auto treffer = [&](uint32_t jj, uint32_t e) {
        StossKK o;
        if (stoss_kk_kandidat(s, ie, i0, i1, qi, qi32, z, jj, i, j, k, e, hat, best.zeit, o)) {
          hat = true;
          best = o;
          ord = (uint64_t(a) << 32) | e;
        }
      };
      // the index test (partner edges after this one) before the box loads
      je_ueberlappend<8>(lo + lane, hi, 32u, qi32, s.hk2.elo, s.hk2.ehi, s.hk2.ein,
                      [&](uint32_t jj) { return int64_t(jj) > ie; }, treffer);
    }
    const int wer = warp_erster(hat, best.zeit, ord);
    if (wer >= 0 && int(lane) == wer) stoss_kk_schreiben(s, slot, i0, i1, best);
  });
}
// ohne_durchdrungene (selbstkollision.rs:1063-1084): keep flags per slot
__device__ bool trifft(const SelbstArgs& s, uint32_t a, uint32_t b) {
  const uint2 kd = s.k_dr[b];
  const uint32_t ts[2] = {kd.x, kd.y};
  for (int q = 0; q < 2; ++q) {
    if (ts[q] == kKein) continue;
    if (finde_schnitt(s, a, ts[q]) == kKein) continue;
    const uint4 dk = s.d_kan[ts[q]];
    if (dk.x == b || dk.y == b || dk.z == b) return true;
  }
  return false;
}
__global__ void __launch_bounds__(kT) stoss_filter_kernel(const __grid_constant__ SelbstArgs s) {
  const int64_t m = s.nd + s.ne;
  const uint32_t nsn = s.zahl[SZ_SCHNITTE] < s.cap_s ? s.zahl[SZ_SCHNITTE] : s.cap_s;
  if (blockIdx.x == 0 && threadIdx.x == 0) s.st_off[m] = 0u;
  SC_FOR(q, m) {
    const uint32_t art = s.st_art[q];
    bool keep = art != 0u;
    if (keep && nsn > 0) {
      const uint4 p = s.st_idx[q];
      if (art == 1u) {
        // dreieck_von(p1, p2, p3): the triangle of edge p1-p2 that holds p3 -
        // the searching triangle's own edge 0
        const uint32_t t = uint32_t(q);
        const uint32_t ke = s.d_kan[t].x;
        const uint2 kd = s.k_dr[ke];
        uint32_t tt = 0;
        const uint32_t cand[2] = {kd.x, kd.y};
        for (int c = 0; c < 2; ++c) {
          if (cand[c] == kKein) continue;
          const uint4 d = s.d_idx[cand[c]];
          if (d.x == p.w || d.y == p.w || d.z == p.w) {
            tt = cand[c];
            break;
          }
        }
        for (uint32_t r = s.t_off[tt]; r < s.t_off[tt + 1] && keep; ++r) {
          const uint2 k = s.k_idx[s.sn_ke[s.t_ent[r]].x];
          if (k.x == p.x || k.y == p.x) keep = false;
        }
      } else {
        // kante_von of both point pairs: the searching edge and its partner
        const uint32_t i = uint32_t(q - s.nd), j = uint32_t(s.st_n[q].w);
        keep = !(trifft(s, i, j) || trifft(s, j, i));
      }
    }
    s.st_off[q] = keep ? 1u : 0u;
  }
}

// the kept impacts in order: point-triangle by triangle, then edge-edge by edge
__global__ void __launch_bounds__(kT) stoss_list_kernel(const __grid_constant__ SelbstArgs s) {
  const int64_t m = s.nd + s.ne;
  SC_FOR(q, m)
  if (s.st_off[q + 1] != s.st_off[q]) s.im[s.st_off[q]] = uint32_t(q);
}
__device__ __forceinline__ uint32_t stoesse(const SelbstArgs& s) { return s.zahl[SZ_STOSS]; }
// per point (w > 0) its impact slots (impact << 2 | slot), in impact order
__global__ void __launch_bounds__(kT) im_count_kernel(const __grid_constant__ SelbstArgs s) {
  SC_FOR(j, stoesse(s)) {
    const uint4 p = s.st_idx[s.im[j]];
    const uint32_t pts[4] = {p.x, p.y, p.z, p.w};
    for (int k = 0; k < 4; ++k)
      if (s.w[pts[k]] > 0.0) atomicAdd(&s.im_off[pts[k]], 1u);
  }
}
__global__ void __launch_bounds__(kT) im_fill_kernel(const __grid_constant__ SelbstArgs s) {
  SC_FOR(j, stoesse(s)) {
    const uint4 p = s.st_idx[s.im[j]];
    const uint32_t pts[4] = {p.x, p.y, p.z, p.w};
    for (int k = 0; k < 4; ++k)
      if (s.w[pts[k]] > 0.0)
        s.im_ent[s.im_off[pts[k]] + atomicAdd(&s.im_cur[pts[k]], 1u)] = (uint32_t(j) << 2) | uint32_t(k);
  }
}
__global__ void __launch_bounds__(kT) im_sort_kernel(const __grid_constant__ SelbstArgs s) {
  SC_FOR(i, s.n) sort_range(s.im_ent, s.im_off[i], s.im_off[i + 1]);
}
// one response pass, per impact (selbstkollision.rs:1292-1328): the
// correction of each of its points with w > 0 into im_c
__global__ void __launch_bounds__(kT) antwort_a_kernel(const __grid_constant__ SelbstArgs s) {
  if (s.zahl[SZ_HALT]) return;
  uint32_t zahl = 0;
  SC_FOR(j, stoesse(s)) {
    const uint32_t q = s.im[j];
    const uint4 p = s.st_idx[q];
    const uint32_t pts[4] = {p.x, p.y, p.z, p.w};
    const double4 lzs = s.st_lzs[q];
    D3 n;
    double d, g[4];
    bool erste[4];
    if (s.st_art[q] == 1u) {
      const D3 x1 = ld3(s.xs, p.y), x2 = ld3(s.xs, p.z), x3 = ld3(s.xs, p.w);
      n = einheit(cross(x2 - x1, x3 - x1)) * lzs.w;
      g[0] = 1.0;
      g[1] = 1.0 - lzs.x - lzs.y;
      g[2] = lzs.x;
      g[3] = lzs.y;
      erste[0] = true;
      erste[1] = erste[2] = erste[3] = false;
      d = dot(n, ld3(s.xs, p.x) - x1);
    } else {
      const double4 n4 = s.st_n[q];
      n = d3(n4.x, n4.y, n4.z);
      const D3 a = lerp3(ld3(s.xs, p.x), ld3(s.xs, p.y), lzs.x), b = lerp3(ld3(s.xs, p.z), ld3(s.xs, p.w), lzs.y);
      g[0] = 1.0 - lzs.x;
      g[1] = lzs.x;
      g[2] = 1.0 - lzs.y;
      g[3] = lzs.y;
      erste[0] = erste[1] = true;
      erste[2] = erste[3] = false;
      d = dot(n, a - b);
    }
    const double tief = kStossAbstand - d;
    if (tief <= 0.0) {
      for (int k = 0; k < 4; ++k) s.im_c[4 * j + k] = make_double4(0, 0, 0, 0);
      continue;
    }
    double m1 = 0.0, m2 = 0.0;
    bool fest1 = true, fest2 = true;
    for (int k = 0; k < 4; ++k) {
      const uint32_t i = pts[k];
      const double4 nf = make_double4(s.nrm_fest[3 * i], s.nrm_fest[3 * i + 1], s.nrm_fest[3 * i + 2], 0.0);
      const double me = (nf.x != 0.0 || nf.y != 0.0 || nf.z != 0.0) ? s.masse[i] * 1e9 : s.masse[i];
      if (erste[k]) {
        m1 += g[k] * me;
        fest1 = fest1 && s.w[i] <= 0.0;
      } else {
        m2 += g[k] * me;
        fest2 = fest2 && s.w[i] <= 0.0;
      }
    }
    const double alpha = fest2 ? 1.0 : (fest1 ? 0.0 : m2 / (m1 + m2));
    for (int k = 0; k < 4; ++k) {
      if (!(s.w[pts[k]] > 0.0)) {
        s.im_c[4 * j + k] = make_double4(0, 0, 0, 0);
        continue;
      }
      const D3 c = erste[k] ? n * (tief * alpha) : n * (-(tief * (1.0 - alpha)));
      s.im_c[4 * j + k] = make_double4(c.x, c.y, c.z, 1.0);
    }
    ++zahl;
  }
  if (zahl) atomicAdd(&s.zahl[SZ_ANTWORT], zahl);
}
// per point: the mean of its corrections (selbstkollision.rs:1329-1336)
__global__ void __launch_bounds__(kT) antwort_b_kernel(const __grid_constant__ SelbstArgs s) {
  if (s.zahl[SZ_HALT]) return;
  uint32_t bewegt = 0;
  SC_FOR(i, s.n) {
    D3 dx = d3(0, 0, 0);
    uint32_t cnt = 0;
    for (uint32_t e = s.im_off[i]; e < s.im_off[i + 1]; ++e) {
      const double4 c = s.im_c[s.im_ent[e]];
      if (c.w == 0.0) continue;
      dx = dx + d3(c.x, c.y, c.z);
      ++cnt;
    }
    if (cnt) {
      st3(s.xs, uint32_t(i), ld3(s.xs, uint32_t(i)) + dx * (1.0 / double(cnt)));
      ++bewegt;
    }
  }
  if (bewegt) atomicAdd(&s.zahl[SZ_BEWEGT], bewegt);
}
__global__ void antwort_c_kernel(const __grid_constant__ SelbstArgs s) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    if (s.zahl[SZ_BEWEGT] == 0u) s.zahl[SZ_HALT] = 1u;
    s.zahl[SZ_BEWEGT] = 0u;
  }
}
// running sums of the statistics (impact corrections, intersections, regions)
__global__ void stat_kernel(const __grid_constant__ SelbstArgs s, unsigned long long* acc) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    acc[0] += s.zahl[SZ_ANTWORT];
    acc[1] += s.zahl[SZ_SCHNITTE];
    acc[2] += s.zahl[SZ_GEBIETE];
  }
}
}  // namespace

size_t selbst_scan_tmp_words(int64_t n) { return size_t((n + kScanChunk - 1) / kScanChunk) + 1; }
cudaError_t exclusive_scan_u32(uint32_t* data, int64_t n, uint32_t* tmp, uint32_t* total, cudaStream_t st) {
  return scan(data, n, tmp, total, st);
}
// normals, boxes; 2 scans, fill, sort, count, 2 scans; fill, springs, damping,
// count, scan, fill, sort
// (+3 and +2: the entry boxes of the point, edge and triangle hashes and of
// the two path hashes)
int selbst_launches_per_run() { return 2 + (6 + 3 + 6 + 10) + (4 + 12 + 3 + 3) + 6 + 4 + 3; }
int selbst_stoss_launches(int iterationen) { return 8 + 6 + 4 + 3 + 3 + 3 * iterationen + 1 + 3 + 2 + 2; }

// Impacts, part 1 (selbstkollision.rs:1196-1203): the longest edge at x1, the
// path boxes, the bucket counts of the point and edge path hashes. The host
// has zeroed lmax[1] and both hashes' bucket arrays.
cudaError_t selbst_stoss_zaehlen(const SelbstArgs& s, cudaStream_t st) {
  cudaError_t e;
  kante_max_kernel<<<grid_for(s.ne), kT, 0, st>>>(s, s.xs, &s.lmax[1]);
  weg_boxen_kernel<<<grid_for(s.n > s.ne ? (s.n > s.nd ? s.n : s.nd) : (s.ne > s.nd ? s.ne : s.nd)), kT, 0, st>>>(s);
  hg_count_kernel<<<grid_for(s.n), kT, 0, st>>>(s.hp2, &s.lmax[1], &s.zahl[SZ_HASH_P2]);
  hg_count_kernel<<<grid_for(s.ne), kT, 0, st>>>(s.hk2, &s.lmax[1], &s.zahl[SZ_HASH_K2]);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = scan(s.hp2.anf, int64_t(s.hp2.eimer) + 1, s.scan_tmp, nullptr, st)) != cudaSuccess) return e;
  return scan(s.hk2.anf, int64_t(s.hk2.eimer) + 1, s.scan_tmp, nullptr, st);
}

// Impacts, part 2: the hashes filled, the earliest impact per triangle and
// per edge, those between parts that already interpenetrate dropped, the
// response passes (selbstkollision.rs:1063-1343), and the statistics' sums.
// The host has checked the hash capacities and zeroed im_off and im_cur.
cudaError_t selbst_stoss_antwort(const SelbstArgs& s, int iterationen, unsigned long long* acc, cudaStream_t st) {
  cudaError_t e;
  hg_fill_kernel<<<grid_for(s.n), kT, 0, st>>>(s.hp2, &s.lmax[1]);
  hg_fill_kernel<<<grid_for(s.ne), kT, 0, st>>>(s.hk2, &s.lmax[1]);
  hg_sort_kernel<<<grid_for(s.hp2.eimer), kT, 0, st>>>(s.hp2);
  if ((e = lang_sort(s.hp2.anf, s.hp2.ein, s.hp2.eimer, st)) != cudaSuccess) return e;
  hg_sort_kernel<<<grid_for(s.hk2.eimer), kT, 0, st>>>(s.hk2);
  if ((e = lang_sort(s.hk2.anf, s.hk2.ein, s.hk2.eimer, st)) != cudaSuccess) return e;
  eintrag_boxen_kernel<<<kEintragGrid, kT, 0, st>>>(s.hp2.anf, s.hp2.eimer, s.hp2.cap, s.hp2.ein, s.hp2.lo, s.hp2.hi,
                                                    s.hp2.elo, s.hp2.ehi);
  eintrag_boxen_kernel<<<kEintragGrid, kT, 0, st>>>(s.hk2.anf, s.hk2.eimer, s.hk2.cap, s.hk2.ein, s.hk2.lo, s.hk2.hi,
                                                    s.hk2.elo, s.hk2.ehi);
  stoss_pd_kernel<<<grid_for(s.nd), kT, 0, st>>>(s);
  stoss_kk_kernel<<<grid_for(s.ne), kT, 0, st>>>(s);
  stoss_pd_schwer_kernel<<<148 * 4, kT, 0, st>>>(s);
  stoss_kk_schwer_kernel<<<148 * 4, kT, 0, st>>>(s);
  stoss_filter_kernel<<<grid_for(s.nd + s.ne), kT, 0, st>>>(s);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = scan(s.st_off, s.nd + s.ne + 1, s.scan_tmp, &s.zahl[SZ_STOSS], st)) != cudaSuccess) return e;
  stoss_list_kernel<<<grid_for(s.nd + s.ne), kT, 0, st>>>(s);
  im_count_kernel<<<grid_for(s.nd + s.ne), kT, 0, st>>>(s);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = scan(s.im_off, s.n + 1, s.scan_tmp, nullptr, st)) != cudaSuccess) return e;
  im_fill_kernel<<<grid_for(s.nd + s.ne), kT, 0, st>>>(s);
  im_sort_kernel<<<grid_for(s.n), kT, 0, st>>>(s);
  if ((e = lang_sort(s.im_off, s.im_ent, s.n, st)) != cudaSuccess) return e;
  for (int it = 0; it < iterationen; ++it) {
    antwort_a_kernel<<<grid_for(s.nd + s.ne), kT, 0, st>>>(s);
    antwort_b_kernel<<<grid_for(s.n), kT, 0, st>>>(s);
    antwort_c_kernel<<<1, 32, 0, st>>>(s);
  }
  stat_kernel<<<1, 32, 0, st>>>(s, acc);
  return cudaGetLastError();
}

// Part 1: normals, planes, boxes, bucket counts. The host has zeroed the
// bucket-count arrays (anf_p, anf_k: eimer + 1 each) and the counters.
cudaError_t selbst_hash_zaehlen(const SelbstArgs& s, cudaStream_t st) {
  tri_normals_kernel<<<grid_for(s.nd), kT, 0, st>>>(s);
  boxes_kernel<<<grid_for(s.n > s.ne ? s.n : s.ne), kT, 0, st>>>(s);
  return cudaGetLastError();
}

// Part 2: bucket starts, fill, per-bucket order; pair counts and their
// starts (the totals land in the counters). The host has checked the hash
// capacities and zeroed the fill cursors.
cudaError_t selbst_hash_fuellen_und_paare_zaehlen(const SelbstArgs& s, cudaStream_t st) {
  cudaError_t e;
  if ((e = scan(s.anf_p, int64_t(s.eimer_p) + 1, s.scan_tmp, nullptr, st)) != cudaSuccess) return e;
  if ((e = scan(s.anf_k, int64_t(s.eimer_k) + 1, s.scan_tmp, nullptr, st)) != cudaSuccess) return e;
  hash_fill_kernel<<<grid_for(s.n > s.ne ? s.n : s.ne), kT, 0, st>>>(s);
  bucket_sort_kernel<<<grid_for(s.eimer_p > s.eimer_k ? s.eimer_p : s.eimer_k), kT, 0, st>>>(s);
  if ((e = lang_sort(s.anf_p, s.ein_p, s.eimer_p, st)) != cudaSuccess) return e;
  if ((e = lang_sort(s.anf_k, s.ein_k, s.eimer_k, st)) != cudaSuccess) return e;
  eintrag_boxen_kernel<<<kEintragGrid, kT, 0, st>>>(s.anf_p, s.eimer_p, s.cap_ep, s.ein_p, s.qp_lo, s.qp_hi, s.ebp_lo,
                                                    s.ebp_hi);
  eintrag_boxen_kernel<<<kEintragGrid, kT, 0, st>>>(s.anf_k, s.eimer_k, s.cap_ek, s.ein_k, s.qk_lo, s.qk_hi, s.ebk_lo,
                                                    s.ebk_hi);
  pairs_count_kernel<<<148 * 4, kT, 0, st>>>(s);  // resident blocks; the groups take items from a counter
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = scan(s.off_t, s.nd + 1, s.scan_tmp, &s.zahl[SZ_PAARE_PT], st)) != cudaSuccess) return e;
  if ((e = scan(s.off_e, s.ne + 1, s.scan_tmp, &s.zahl[SZ_PAARE_KK], st)) != cudaSuccess) return e;
  // edges through triangles (selbstkollision.rs:858-907): the longest edge,
  // the triangle hash, the count per edge. The host has zeroed lmax and the
  // triangle hash's bucket arrays.
  kante_max_kernel<<<grid_for(s.ne), kT, 0, st>>>(s, s.x, &s.lmax[0]);
  schnitt_boxen_kernel<<<grid_for(s.nd), kT, 0, st>>>(s);
  hg_count_kernel<<<grid_for(s.nd), kT, 0, st>>>(s.hs, &s.lmax[0], &s.zahl[SZ_HASH_S]);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = scan(s.hs.anf, int64_t(s.hs.eimer) + 1, s.scan_tmp, nullptr, st)) != cudaSuccess) return e;
  hg_fill_kernel<<<grid_for(s.nd), kT, 0, st>>>(s.hs, &s.lmax[0]);
  hg_sort_kernel<<<grid_for(s.hs.eimer), kT, 0, st>>>(s.hs);
  if ((e = lang_sort(s.hs.anf, s.hs.ein, s.hs.eimer, st)) != cudaSuccess) return e;
  eintrag_boxen_kernel<<<kEintragGrid, kT, 0, st>>>(s.hs.anf, s.hs.eimer, s.hs.cap, s.hs.ein, s.hs.lo, s.hs.hi, s.hs.elo,
                                                    s.hs.ehi);
  schnitt_count_kernel<<<148 * 4, kT, 0, st>>>(s);  // resident blocks; the groups take edges from a counter
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return scan(s.off_s, s.ne + 1, s.scan_tmp, &s.zahl[SZ_SCHNITTE], st);
}

// Part 3: pairs, springs, damping, incidence lists. The host has checked the
// pair capacity and zeroed inc_off (n + 1) and inc_cur (n).
cudaError_t selbst_paare_und_federn(const SelbstArgs& s, uint32_t n_aktiv_p, uint32_t n_aktiv_s, uint32_t n_s,
                                    cudaStream_t st) {
  cudaError_t e;
  pairs_fill_kernel<<<grid_for(kG * int64_t(n_aktiv_p)), kT, 0, st>>>(s, n_aktiv_p);
  const int64_t pmax = int64_t(s.cap_pairs);
  if (s.rsize == 4)
    federn_kernel<float><<<grid_for(pmax), kT, 0, st>>>(s);
  else
    federn_kernel<double><<<grid_for(pmax), kT, 0, st>>>(s);
  static bool smem_set = false;
  if (!smem_set) {
    if ((e = cudaFuncSetAttribute(daempfung_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kDampSmem))) !=
        cudaSuccess)
      return e;
    smem_set = true;
  }
  daempfung_kernel<<<1, kDB, kDampSmem, st>>>(s);
  // penetration regions and their push springs (selbstkollision.rs:858-1058);
  // the host has zeroed hat, klemm, t_off and t_cur
  const int64_t ns = int64_t(s.cap_s);
  schnitt_fill_kernel<<<grid_for(kG * int64_t(n_aktiv_s)), kT, 0, st>>>(s, n_aktiv_s);
  {
    static bool gebiete_smem = false;
    if (!gebiete_smem) {
      if ((e = cudaFuncSetAttribute(gebiete_runden_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(kGebietSmemBytes))) != cudaSuccess)
        return e;
      gebiete_smem = true;
    }
  }
  gebiete_init_kernel<<<grid_for(n_s), kT, 0, st>>>(s);
  gebiete_vereinigen_kernel<<<grid_for(n_s), kT, 0, st>>>(s);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = scan(s.sn_toff, int64_t(n_s) + 1, s.sn_scan_tmp, nullptr, st)) != cudaSuccess) return e;
  gebiete_tausch_kernel<<<grid_for(n_s), kT, 0, st>>>(s);
  gebiete_runden_kernel<<<1, 1024, kGebietSmemBytes, st>>>(s);
  klemm_kernel<<<grid_for(ns), kT, 0, st>>>(s);
  folge_kernel<<<grid_for(s.nd), kT, 0, st>>>(s);
  if (s.rsize == 4)
    schub_kernel<float><<<grid_for(ns), kT, 0, st>>>(s);
  else
    schub_kernel<double><<<grid_for(ns), kT, 0, st>>>(s);
  t_count_kernel<<<grid_for(ns), kT, 0, st>>>(s);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = scan(s.t_off, s.nd + 1, s.scan_tmp, nullptr, st)) != cudaSuccess) return e;
  t_fill_kernel<<<grid_for(ns), kT, 0, st>>>(s);
  inc_count_kernel<<<grid_for(pmax), kT, 0, st>>>(s);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = scan(s.inc_off, s.n + 1, s.scan_tmp, &s.zahl[SZ_INZIDENZ], st)) != cudaSuccess) return e;
  inc_fill_kernel<<<grid_for(pmax), kT, 0, st>>>(s);
  inc_sort_kernel<<<grid_for(s.n), kT, 0, st>>>(s);
  if ((e = lang_sort(s.inc_off, s.inc_ent, s.n, st)) != cudaSuccess) return e;
  inc_pos_kernel<<<grid_for(int64_t(s.cap_inc)), kT, 0, st>>>(s);
  return cudaGetLastError();
}

}  // namespace k3d
