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

// selbstkollision.rs:328-344: f(entry, i, j, k) over the entries of the box's cells
template <typename F>
__device__ void je_eintrag(const Box& q, double zelle, uint32_t eimer, const uint32_t* anf, const uint32_t* ein,
                           F&& f) {
  if (!zellbereich_ok(q, zelle)) return;
  const Cells c = cells_of(q, zelle);
  for (uint32_t a = 0; a < c.total; ++a) {
    int64_t i, j, k;
    cell_at(c, a, i, j, k);
    const uint32_t h = streue(i, j, k, eimer);
    const uint32_t e1 = anf[h + 1];
    for (uint32_t s = anf[h]; s < e1; ++s) f(ein[s], i, j, k);
  }
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
// entry order (selbstkollision.rs:316-322).
__device__ __forceinline__ void sort_range(uint32_t* a, uint32_t lo, uint32_t hi) {
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
__global__ void __launch_bounds__(kT) bucket_sort_kernel(const __grid_constant__ SelbstArgs s) {
  SC_FOR(b, s.eimer_p) sort_range(s.ein_p, s.anf_p[b], s.anf_p[b + 1]);
  SC_FOR(b, s.eimer_k) sort_range(s.ein_k, s.anf_k[b], s.anf_k[b + 1]);
}

// Point-triangle search for triangle t (selbstkollision.rs:400-466): counts,
// or writes its pairs from `pos` on, in the reference's order.
template <bool FILL>
__device__ uint32_t punkt_dreieck(const SelbstArgs& s, int64_t t, uint32_t pos) {
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
  uint32_t cnt = 0;
  je_eintrag(qt, s.zelle, s.eimer_p, s.anf_p, s.ein_p, [&](uint32_t v, int64_t ci, int64_t cj, int64_t ck) {
    for (int k = 0; k < 3; ++k)
      if (gleich_oder_partner(s, v, d[k])) return;
    if (s.w[v] <= 0.0 && alle_fest) return;
    const Box qv = box_of(s.qp_lo, s.qp_hi, v);
    if (!ueberlappt(qv, qt) || !erste_zelle(qt, qv, s.zelle, ci, cj, ck)) return;
    const D3 xv = ld3(s.x, v);
    double ruhe = rt + s.r_punkt[v];
    double eine;
    if (band_abstand(s, v, d, 3, eine)) ruhe = eine;
    const double soll = ruhe + kZuschlagPaar;
    const double sd = dot(nt, xv - p[0]);
    if (fabs(sd) > soll) return;
    for (int k = 0; k < 3; ++k)
      if (dot(xv - p[k], en[k]) * sg[k] < 0.0) return;
    double g[3];
    naechster_dreieck(p[0], p[1], p[2], xv, g);
    const D3 cp = (p[0] * g[0] + p[1] * g[1]) + p[2] * g[2];
    const D3 r = xv - cp;
    const double abstand = norm(r);
    if (abstand > soll) return;
    if (FILL) {
      const uint32_t q = pos + cnt;
      if (q < s.cap_pairs) {
        const D3 n = abstand > 1e-12 ? r * (1.0 / abstand) : nt;
        s.pr_idx[q] = make_uint4(v, i0, i1, i2);
        s.pr_src[q] = make_uint2(uint32_t(t), kKein);
        s.pr_w[q] = make_double4(1.0, -g[0], -g[1], -g[2]);
        s.pr_nab[q] = make_double4(n.x, n.y, n.z, abstand);
        s.pr_ruhe[q] = ruhe;
      }
    }
    ++cnt;
  });
  return cnt;
}

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

// Edge-edge search for edge e (selbstkollision.rs:506-598).
template <bool FILL>
__device__ uint32_t kante_kante(const SelbstArgs& s, int64_t e, uint32_t pos) {
  const uint2 ka = s.k_idx[e];
  const uint32_t a0 = ka.x, a1 = ka.y;
  if (a0 == a1) return 0;
  const D3 pa0 = ld3(s.x, a0), pa1 = ld3(s.x, a1);
  const Box qe = box_of(s.qk_lo, s.qk_hi, e);
  uint32_t cnt = 0;
  je_eintrag(qe, s.zelle, s.eimer_k, s.anf_k, s.ein_k, [&](uint32_t f, int64_t ci, int64_t cj, int64_t ck) {
    if (int64_t(f) <= e) return;
    const Box qf = box_of(s.qk_lo, s.qk_hi, f);
    if (!ueberlappt(qe, qf) || !erste_zelle(qe, qf, s.zelle, ci, cj, ck)) return;
    const uint2 kb = s.k_idx[f];
    const uint32_t b0 = kb.x, b1 = kb.y;
    if (gleich_oder_partner(s, a0, b0) || gleich_oder_partner(s, a1, b0) || gleich_oder_partner(s, a0, b1) ||
        gleich_oder_partner(s, a1, b1))
      return;
    const uint32_t bb[2] = {b0, b1}, aa[2] = {a0, a1};
    double band = 0.0;
    const bool hat_band = band_abstand(s, a0, bb, 2, band) || band_abstand(s, a1, bb, 2, band) ||
                          band_abstand(s, b0, aa, 2, band) || band_abstand(s, b1, aa, 2, band);
    if (s.w[a0] <= 0.0 && s.w[a1] <= 0.0 && s.w[b0] <= 0.0 && s.w[b1] <= 0.0) return;
    const D3 pb0 = ld3(s.x, b0), pb1 = ld3(s.x, b1);
    const D3 da = pa1 - pa0, db = pb1 - pb0;
    const double la = norm(da), lb = norm(db);
    if (la < kKanteMin || lb < kKanteMin) return;
    const D3 ua = da * (1.0 / la), ub = db * (1.0 / lb);
    const double cw = dot(ua, ub);
    if (fabs(cw) > 0.99999) return;
    const D3 r = pb0 - pa0;
    const double p = dot(r, ua), q = -dot(r, ub);
    const double nen = 1.0 - cw * cw;
    const double sa = (p + cw * q) / nen;
    const double sb = (q + cw * p) / nen;
    if (!(0.0 <= sa && sa <= la) || !(0.0 <= sb && sb <= lb)) return;
    const D3 pa = pa0 + ua * sa;
    const D3 pb = pb0 + ub * sb;
    const D3 dv = pa - pb;
    const double abstand = norm(dv);
    const double ruhe = hat_band ? band : s.r_kante[e] + s.r_kante[f];
    if (abstand > ruhe + kZuschlagPaar) return;
    const D3 n = einheit(dv);
    if (!ist_kuerzeste(s, f, ub, n) || !ist_kuerzeste(s, uint32_t(e), ua, n * -1.0)) return;
    if (FILL) {
      const uint32_t w = pos + cnt;
      if (w < s.cap_pairs) {
        const double sp = sa / la, tp = sb / lb;
        s.pr_idx[w] = make_uint4(a0, a1, b0, b1);
        s.pr_src[w] = make_uint2(uint32_t(e), f);
        s.pr_w[w] = make_double4(1.0 - sp, sp, -(1.0 - tp), -tp);
        s.pr_nab[w] = make_double4(n.x, n.y, n.z, abstand);
        s.pr_ruhe[w] = ruhe;
      }
    }
    ++cnt;
  });
  return cnt;
}

// count pass: pair count per triangle and per edge (off_t[t], off_e[e])
__global__ void __launch_bounds__(kT) pairs_count_kernel(const __grid_constant__ SelbstArgs s) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {  // the scans run over n + 1 values
    s.off_t[s.nd] = 0u;
    s.off_e[s.ne] = 0u;
  }
  SC_FOR(t, s.nd) s.off_t[t] = punkt_dreieck<false>(s, t, 0);
  SC_FOR(e, s.ne) s.off_e[e] = kante_kante<false>(s, e, 0);
}

// fill pass: point-triangle pairs first (triangle order), then edge-edge
__global__ void __launch_bounds__(kT) pairs_fill_kernel(const __grid_constant__ SelbstArgs s) {
  const uint32_t npt = s.zahl[SZ_PAARE_PT];
  SC_FOR(t, s.nd) punkt_dreieck<true>(s, t, s.off_t[t]);
  SC_FOR(e, s.ne) kante_kante<true>(s, e, npt + s.off_e[e]);
}

__device__ __forceinline__ uint32_t paare(const SelbstArgs& s) {
  const uint64_t p = uint64_t(s.zahl[SZ_PAARE_PT]) + s.zahl[SZ_PAARE_KK];
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

// Per-point incidence lists of the pairs' nonzero slots, ascending.
__global__ void __launch_bounds__(kT) inc_count_kernel(const __grid_constant__ SelbstArgs s) {
  const uint32_t P = paare(s);
  SC_FOR(q, P) {
    const uint4 id = s.pr_idx[q];
    const double4 g = s.pr_w[q];
    if (g.x != 0.0) atomicAdd(&s.inc_off[id.x], 1u);
    if (g.y != 0.0) atomicAdd(&s.inc_off[id.y], 1u);
    if (g.z != 0.0) atomicAdd(&s.inc_off[id.z], 1u);
    if (g.w != 0.0) atomicAdd(&s.inc_off[id.w], 1u);
  }
}
__global__ void __launch_bounds__(kT) inc_fill_kernel(const __grid_constant__ SelbstArgs s) {
  const uint32_t P = paare(s);
  SC_FOR(q, P) {
    const uint4 id = s.pr_idx[q];
    const double4 g = s.pr_w[q];
    const uint32_t pts[4] = {id.x, id.y, id.z, id.w};
    const double gw[4] = {g.x, g.y, g.z, g.w};
    for (int k = 0; k < 4; ++k) {
      if (gw[k] == 0.0) continue;
      const uint32_t pos = s.inc_off[pts[k]] + atomicAdd(&s.inc_cur[pts[k]], 1u);
      if (pos < s.cap_inc) s.inc_ent[pos] = (uint32_t(q) << 2) | uint32_t(k);
    }
  }
}
__global__ void __launch_bounds__(kT) inc_sort_kernel(const __grid_constant__ SelbstArgs s) {
  SC_FOR(i, s.n) sort_range(s.inc_ent, s.inc_off[i], s.inc_off[i + 1]);
}
// The inverse of the lists: each nonzero slot's entry index (the PCG writes a
// pair's slot products there and sums them per point in list order).
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

}  // namespace

size_t selbst_scan_tmp_words(int64_t n) { return size_t((n + kScanChunk - 1) / kScanChunk) + 1; }
// normals, boxes; 2 scans, fill, sort, count, 2 scans; fill, springs, damping,
// count, scan, fill, sort
int selbst_launches_per_run() { return 2 + (6 + 3 + 6) + (4 + 3 + 3); }

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
  pairs_count_kernel<<<grid_for(s.nd > s.ne ? s.nd : s.ne), kT, 0, st>>>(s);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = scan(s.off_t, s.nd + 1, s.scan_tmp, &s.zahl[SZ_PAARE_PT], st)) != cudaSuccess) return e;
  return scan(s.off_e, s.ne + 1, s.scan_tmp, &s.zahl[SZ_PAARE_KK], st);
}

// Part 3: pairs, springs, damping, incidence lists. The host has checked the
// pair capacity and zeroed inc_off (n + 1) and inc_cur (n).
cudaError_t selbst_paare_und_federn(const SelbstArgs& s, cudaStream_t st) {
  cudaError_t e;
  pairs_fill_kernel<<<grid_for(s.nd > s.ne ? s.nd : s.ne), kT, 0, st>>>(s);
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
  inc_count_kernel<<<grid_for(pmax), kT, 0, st>>>(s);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = scan(s.inc_off, s.n + 1, s.scan_tmp, &s.zahl[SZ_INZIDENZ], st)) != cudaSuccess) return e;
  inc_fill_kernel<<<grid_for(pmax), kT, 0, st>>>(s);
  inc_sort_kernel<<<grid_for(s.n), kT, 0, st>>>(s);
  inc_pos_kernel<<<grid_for(int64_t(s.cap_inc)), kT, 0, st>>>(s);
  return cudaGetLastError();
}

}  // namespace k3d
