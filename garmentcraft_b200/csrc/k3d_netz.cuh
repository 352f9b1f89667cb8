// Device side of the body mesh as a signed-distance collider
// (sim/src/netzkoerper.rs): the table layout one mesh keeps in HBM, the exact
// nearest point on a triangle, the pseudonormals, the nearest query over the
// triangle grid and the segment penetration test. Shared by the mesh's own
// kernels and the step's contact query and integration (every includer that
// calls them is compiled without fused multiply-add, so the regions and
// distances round as the reference's arithmetic does).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "k3d_vec.cuh"

namespace k3d {
namespace netz {

struct Dev {
  int64_t n, nd;
  double suchtiefe;
  const double* p;  // 3 per point
  const uint4* d;   // triangle points (w unused)
  double4* fn;      // face normal
  const uint4* nb;  // neighbour across edge k (the triangle itself at an open edge)
  double4* pn;      // angle-weighted point normal
  double4* kg;      // bounding sphere: centre, radius
  double* wk;       // corner angles, 3 per triangle
  double* vt;       // volume term per triangle
  const uint32_t *pi_off, *pi_ent;
  const double* pv;  // velocity per point (3 per point), null: the body moves rigidly
  // grid
  double u0, u1, u2, zelle;
  int32_t zx, zy, zz;
  uint32_t *anf, *ein, *cur;
  uint32_t cap;
  uint32_t *pg_anf, *pg_ein;  // point grid on the same cells (Z + 1 starts; N entries, ascending per cell)
};

__device__ __forceinline__ D3 ld4(const double4& v) { return d3(v.x, v.y, v.z); }
__device__ __forceinline__ D3 punkt(const Dev& g, uint32_t i) { return ld3(g.p, i); }

// netzkoerper.rs:220-227
__device__ __forceinline__ D3 normiert(D3 a) {
  const double l = norm(a);
  if (l > 0.0) return a * (1.0 / l);
  return d3(0.0, 0.0, 0.0);
}

// `f64 as i64` (saturating, NaN to 0), then the cell index of netzkoerper.rs:87-92
__device__ __forceinline__ int64_t als_i64(double v) {
  if (isnan(v)) return 0;
  if (v >= 9.2233720368547758e18) return INT64_MAX;
  if (v <= -9.2233720368547758e18) return INT64_MIN;
  return int64_t(v);
}
__device__ __forceinline__ void zell_index(const Dev& g, D3 x, int64_t k[3]) {
  k[0] = als_i64(floor((x.x - g.u0) / g.zelle));
  k[1] = als_i64(floor((x.y - g.u1) / g.zelle));
  k[2] = als_i64(floor((x.z - g.u2) / g.zelle));
}
// netzkoerper.rs:117-128: the clamped cell range of the box [lo, hi]
__device__ __forceinline__ bool bereich(const Dev& g, D3 lo, D3 hi, int r0[3], int r1[3]) {
  int64_t a[3], b[3];
  zell_index(g, lo, a);
  zell_index(g, hi, b);
  const int64_t z[3] = {g.zx, g.zy, g.zz};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    if (b[q] < 0 || a[q] >= z[q]) return false;
    r0[q] = int(a[q] < 0 ? 0 : a[q]);
    r1[q] = int(b[q] > z[q] - 1 ? z[q] - 1 : b[q]);
  }
  return true;
}

// netzkoerper.rs:185-216 (Ericson 2005, 5.1.5); regions 0-2 corner, 3-5 edge, 6 face
__device__ __forceinline__ D3 naechster_auf_dreieck(D3 p, D3 a, D3 b, D3 c, int& reg) {
  auto quot = [](double z, double n) { return n > 0.0 ? z / n : 0.0; };
  const D3 ab = b - a, ac = c - a, ap = p - a;
  const double d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) {
    reg = 0;
    return a;
  }
  const D3 bp = p - b;
  const double d3_ = dot(ab, bp), d4 = dot(ac, bp);
  if (d3_ >= 0.0 && d4 <= d3_) {
    reg = 1;
    return b;
  }
  const double vc = d1 * d4 - d3_ * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3_ <= 0.0) {
    reg = 3;
    return a + ab * quot(d1, d1 - d3_);
  }
  const D3 cp = p - c;
  const double d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) {
    reg = 2;
    return c;
  }
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
    reg = 5;
    return a + ac * quot(d2, d2 - d6);
  }
  const double va = d3_ * d6 - d5 * d4;
  if (va <= 0.0 && d4 - d3_ >= 0.0 && d5 - d6 >= 0.0) {
    const double w = quot(d4 - d3_, (d4 - d3_) + (d5 - d6));
    reg = 4;
    return b + (c - b) * w;
  }
  const double s = va + vb + vc;
  const double v = quot(vb, s), w = quot(vc, s);
  reg = 6;
  return a + (ab * v + ac * w);
}

// netzkoerper.rs:431-447
__device__ __forceinline__ D3 pseudonormale(const Dev& g, uint32_t t, int r) {
  if (r == 6) return ld4(g.fn[t]);
  if (r >= 3) {
    const uint4 o4 = g.nb[t];
    const uint32_t o = (r == 3) ? o4.x : (r == 4 ? o4.y : o4.z);
    if (o == t) return ld4(g.fn[t]);
    return normiert(ld4(g.fn[t]) + ld4(g.fn[o]));
  }
  const uint4 d = g.d[t];
  return ld4(g.pn[r == 0 ? d.x : (r == 1 ? d.y : d.z)]);
}

struct Treffer {
  double abstand;
  D3 punkt, normale;
  uint32_t dreieck;
  int region;
};
// netzkoerper.rs:492-499
__device__ __forceinline__ Treffer ergebnis(const Dev& g, D3 x, uint32_t t, D3 c, int r) {
  const D3 pn = pseudonormale(g, t, r);
  const D3 d = x - c;
  const double l = norm(d);
  const bool aussen = dot(d, pn) >= 0.0;
  const D3 nrm = l > 1e-12 ? d * (aussen ? 1.0 / l : -1.0 / l) : pn;
  return Treffer{aussen ? l : -l, c, nrm, t, r};
}

// A conservative sphere test: the triangle may hold a point no farther than
// `best` (the slack keeps ties and rounding on the safe side).
__device__ __forceinline__ bool kugel_nah(D3 x, double4 k, double best) {
  const D3 d = x - d3(k.x, k.y, k.z);
  const double b = best + k.w;  // |x - m| <= best + r, squared (no square root)
  return dot(d, d) <= b * b * (1.0 + 1e-9) + 1e-300;
}

// netzkoerper.rs:503-539: cells in z, y, x order, each cell's triangles in
// ascending order (the reference's fill order), the sphere test and the
// strict comparison as there, so that among equal distances the same
// triangle wins as in the reference
__device__ inline bool naechster(const Dev& g, D3 x, double radius, Treffer& out) {
  int r0[3], r1[3];
  if (!bereich(g, x - d3(radius, radius, radius), x + d3(radius, radius, radius), r0, r1)) return false;
  double best = radius;
  bool hit = false;
  uint32_t bt = 0xffffffffu;
  D3 bq = d3(0, 0, 0);
  int br = 6;
  for (int kz = r0[2]; kz <= r1[2]; ++kz)
    for (int ky = r0[1]; ky <= r1[1]; ++ky)
      for (int kx = r0[0]; kx <= r1[0]; ++kx) {
        const int64_t z = (int64_t(kz) * g.zy + ky) * g.zx + kx;
        const uint32_t e1 = g.anf[z + 1];
        for (uint32_t e = g.anf[z]; e < e1; ++e) {
          const uint32_t t = g.ein[e];
          const double4 k = g.kg[t];
          if (norm(x - d3(k.x, k.y, k.z)) - k.w >= best) continue;
          const uint4 d = g.d[t];
          int reg;
          const D3 q = naechster_auf_dreieck(x, punkt(g, d.x), punkt(g, d.y), punkt(g, d.z), reg);
          const double l = norm(x - q);
          if (l < best) {
            best = l;
            hit = true;
            bt = t;
            bq = q;
            br = reg;
          }
        }
      }
  if (!hit) return false;
  out = ergebnis(g, x, bt, bq, br);
  return true;
}

// netzkoerper.rs:474-489 with the barycentric weights of :229-243: the
// surface velocity at p on triangle t, the rigid one without a field
__device__ inline D3 geschwindigkeit_an(const Dev& g, uint32_t t, D3 p, D3 starr) {
  if (!g.pv) return starr;
  const uint4 d = g.d[t];
  const D3 a = punkt(g, d.x), b = punkt(g, d.y), c = punkt(g, d.z);
  const D3 e1 = b - a, e2 = c - a, e3 = p - a;
  const double d00 = dot(e1, e1), d01 = dot(e1, e2), d11 = dot(e2, e2);
  const double d20 = dot(e3, e1), d21 = dot(e3, e2);
  const double nenner = d00 * d11 - d01 * d01;
  double w[3] = {1.0, 0.0, 0.0};
  if (nenner != 0.0) {
    const double u = (d11 * d20 - d01 * d21) / nenner;
    const double v = (d00 * d21 - d01 * d20) / nenner;
    w[0] = 1.0 - u - v, w[1] = u, w[2] = v;
  }
  const uint32_t ix[3] = {d.x, d.y, d.z};
  D3 q = d3(0.0, 0.0, 0.0);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const D3 vj = ld3(g.pv, ix[j]);
    q.x += w[j] * vj.x;
    q.y += w[j] * vj.y;
    q.z += w[j] * vj.z;
  }
  return q;
}

// netzkoerper.rs:541-593 for one segment a -> b: the first entry from
// outside; among equal segment parameters the first in the reference's cell
// order
__device__ inline bool durchstoss(const Dev& g, D3 a, D3 b, D3& p, D3& n, uint32_t& tb) {
  const D3 d = b - a;
  if (dot(d, d) < 1e-24) return false;
  int r0[3], r1[3];
  if (!bereich(g, d3(fmin(a.x, b.x), fmin(a.y, b.y), fmin(a.z, b.z)), d3(fmax(a.x, b.x), fmax(a.y, b.y), fmax(a.z, b.z)),
               r0, r1))
    return false;
  const double eps = 1e-12;
  bool hit = false;
  double sb = 0.0;
  for (int kz = r0[2]; kz <= r1[2]; ++kz)
    for (int ky = r0[1]; ky <= r1[1]; ++ky)
      for (int kx = r0[0]; kx <= r1[0]; ++kx) {
        const int64_t z = (int64_t(kz) * g.zy + ky) * g.zx + kx;
        for (uint32_t e = g.anf[z]; e < g.anf[z + 1]; ++e) {
          const uint32_t t = g.ein[e];
          if (dot(d, ld4(g.fn[t])) >= 0.0) continue;
          const uint4 tri = g.d[t];
          const D3 p0 = punkt(g, tri.x), p1 = punkt(g, tri.y), p2 = punkt(g, tri.z);
          const D3 e1 = p1 - p0, e2 = p2 - p0;
          const D3 pv = cross(d, e2);
          const double det = dot(e1, pv);
          if (fabs(det) < 1e-30) continue;
          const D3 tv = a - p0;
          const double u = dot(tv, pv) / det;
          if (u < -eps || u > 1.0 + eps) continue;
          const D3 qv = cross(tv, e1);
          const double v = dot(d, qv) / det;
          if (v < -eps || u + v > 1.0 + eps) continue;
          const double s = dot(e2, qv) / det;
          if (s >= -eps && s <= 1.0 + eps && (!hit || s < sb)) {
            hit = true;
            sb = s;
            tb = t;
          }
        }
      }
  if (!hit) return false;
  p = a + d * fmin(fmax(sb, 0.0), 1.0);
  n = ld4(g.fn[tb]);
  return true;
}

}  // namespace netz
}  // namespace k3d
