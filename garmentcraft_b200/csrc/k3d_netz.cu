// The body mesh as a signed-distance collider on the device
// (sim/src/netzkoerper.rs, Koerpernetz), and its voxelisation into the
// sampled grid of a K3D_BODY_SDF_GRID body.
//
// Layout in HBM (N points, T triangles, Z grid cells):
//   per point     positions double[3N], point normals double4[N], and a CSR
//                 of its (triangle << 2 | corner) in triangle order
//   per triangle  points uint4, face normal double4, neighbours uint4,
//                 bounding sphere double4 (centre, radius), corner angles
//                 double[3T], volume term double[T]
//   grid          cell starts uint32[Z + 1], entries (triangles, ascending
//                 per cell) uint32
// The topology checks and the neighbour table are host work done once
// (Koerpernetz::neu); everything that depends on the positions runs here, so
// a deforming body (nachfuehren) costs one host read of its hull and volume
// and one of the grid's entry count.
//
// Queries run one thread per point (or segment, or grid node). The nearest
// query walks the cells the search box touches in the reference's order,
// skips triangles whose bounding sphere is no nearer than the best so far,
// and keeps the first of the smallest distances, as the reference does; the
// query over every triangle keeps the first in triangle order. Compiled
// without fused multiply-add: the Ericson regions and distances round as the
// reference's arithmetic does, so the step sees the same contact normals.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/klon3d_mesh.h"
#include "k3d_device.cuh"
#include "k3d_selbst.h"

namespace k3d {
namespace netz {

constexpr int kT = 256;
constexpr int kTile = 128;  // triangles per shared-memory tile of the all-triangle query

// ---------------------------------------------------------------- point-dependent tables
// netzkoerper.rs:257-290, per triangle: face normal, corner angles, sphere, volume term
__global__ void __launch_bounds__(kT) flaechen_kernel(const __grid_constant__ Dev g) {
  for (int64_t t = int64_t(blockIdx.x) * kT + threadIdx.x; t < g.nd; t += int64_t(gridDim.x) * kT) {
    const uint4 d = g.d[t];
    const D3 q[3] = {punkt(g, d.x), punkt(g, d.y), punkt(g, d.z)};
    const D3 n = normiert(cross(q[1] - q[0], q[2] - q[0]));
    g.fn[t] = make_double4(n.x, n.y, n.z, 0.0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const D3 u = q[(k + 1) % 3] - q[k], v = q[(k + 2) % 3] - q[k];
      g.wk[3 * t + k] = atan2(norm(cross(u, v)), dot(u, v));  // netzkoerper.rs:246-248
    }
    g.vt[t] = dot(q[0], cross(q[1], q[2])) / 6.0;
    const D3 m = ((q[0] + q[1]) + q[2]) * (1.0 / 3.0);
    double r = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) r = fmax(r, norm(q[k] - m));
    g.kg[t] = make_double4(m.x, m.y, m.z, r);
  }
}
// per point: the angle-weighted sum of the face normals in triangle order, normalised
__global__ void __launch_bounds__(kT) punktnormalen_kernel(const __grid_constant__ Dev g) {
  for (int64_t i = int64_t(blockIdx.x) * kT + threadIdx.x; i < g.n; i += int64_t(gridDim.x) * kT) {
    D3 s = d3(0.0, 0.0, 0.0);
    for (uint32_t e = g.pi_off[i]; e < g.pi_off[i + 1]; ++e) {
      const uint32_t c = g.pi_ent[e], t = c >> 2, k = c & 3u;
      s = s + ld4(g.fn[t]) * g.wk[3 * t + k];
    }
    const D3 nn = normiert(s);
    g.pn[i] = make_double4(nn.x, nn.y, nn.z, 0.0);
  }
}
// one block: point hull (huelle_punkte, :785-797) and the volume (tree sum)
__global__ void __launch_bounds__(1024) huelle_kernel(const __grid_constant__ Dev g, double* out7) {
  __shared__ double sh[7][32];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY}, v = 0.0;
  for (int64_t i = threadIdx.x; i < g.n; i += blockDim.x) {
    const D3 q = punkt(g, uint32_t(i));
    lo[0] = fmin(lo[0], q.x), lo[1] = fmin(lo[1], q.y), lo[2] = fmin(lo[2], q.z);
    hi[0] = fmax(hi[0], q.x), hi[1] = fmax(hi[1], q.y), hi[2] = fmax(hi[2], q.z);
  }
  for (int64_t t = threadIdx.x; t < g.nd; t += blockDim.x) v += g.vt[t];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
      hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
    }
    v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  if (lane == 0) {
    for (int a = 0; a < 3; ++a) sh[a][wid] = lo[a], sh[3 + a][wid] = hi[a];
    sh[6][wid] = v;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    double l[3], h[3], s;
    for (int a = 0; a < 3; ++a) {
      l[a] = lane < nw ? sh[a][lane] : INFINITY;
      h[a] = lane < nw ? sh[3 + a][lane] : -INFINITY;
    }
    s = lane < nw ? sh[6][lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      for (int a = 0; a < 3; ++a) {
        l[a] = fmin(l[a], __shfl_xor_sync(0xffffffffu, l[a], o));
        h[a] = fmax(h[a], __shfl_xor_sync(0xffffffffu, h[a], o));
      }
      s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    if (lane == 0) {
      for (int a = 0; a < 3; ++a) out7[a] = l[a], out7[3 + a] = h[a];
      out7[6] = s;
    }
  }
}

// ---------------------------------------------------------------- triangle grid (:881-910)
// the clamped cell range of triangle t (dreieck_klammer + klammer, :800-818, :131-140)
__device__ __forceinline__ void dreieck_zellen(const Dev& g, int64_t t, int r0[3], int r1[3]) {
  const uint4 d = g.d[t];
  int64_t a[3], b[3], k[3];
  zell_index(g, punkt(g, d.x), a);
  b[0] = a[0], b[1] = a[1], b[2] = a[2];
  const uint32_t rest[2] = {d.y, d.z};
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    zell_index(g, punkt(g, rest[j]), k);
#pragma unroll
    for (int q = 0; q < 3; ++q) a[q] = a[q] < k[q] ? a[q] : k[q], b[q] = b[q] > k[q] ? b[q] : k[q];
  }
  // clamped into [0, zahl] first: a range wholly outside the grid comes out empty
  const int64_t z[3] = {g.zx, g.zy, g.zz};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    r0[q] = int(a[q] < 0 ? 0 : (a[q] > z[q] ? z[q] : a[q]));
    r1[q] = int(b[q] > z[q] - 1 ? z[q] - 1 : (b[q] < -1 ? -1 : b[q]));
  }
}
// the point grid (gitter_punkte, :863-879): each point in its clamped cell
__device__ __forceinline__ int64_t punkt_zelle(const Dev& g, uint32_t i) {
  int64_t k[3];
  zell_index(g, punkt(g, i), k);
  const int64_t z[3] = {g.zx, g.zy, g.zz};
#pragma unroll
  for (int q = 0; q < 3; ++q) k[q] = k[q] < 0 ? 0 : (k[q] > z[q] - 1 ? z[q] - 1 : k[q]);
  return (k[2] * g.zy + k[1]) * g.zx + k[0];
}
__global__ void __launch_bounds__(kT) punkte_zaehlen_kernel(const __grid_constant__ Dev g) {
  for (int64_t i = int64_t(blockIdx.x) * kT + threadIdx.x; i < g.n; i += int64_t(gridDim.x) * kT)
    atomicAdd(&g.pg_anf[punkt_zelle(g, uint32_t(i))], 1u);
}
__global__ void __launch_bounds__(kT) punkte_fuellen_kernel(const __grid_constant__ Dev g, uint32_t* cur) {
  for (int64_t i = int64_t(blockIdx.x) * kT + threadIdx.x; i < g.n; i += int64_t(gridDim.x) * kT)
    g.pg_ein[atomicAdd(&cur[punkt_zelle(g, uint32_t(i))], 1u)] = uint32_t(i);
}
__global__ void __launch_bounds__(kT) zellen_zaehlen_kernel(const __grid_constant__ Dev g) {
  for (int64_t t = int64_t(blockIdx.x) * kT + threadIdx.x; t < g.nd; t += int64_t(gridDim.x) * kT) {
    int r0[3], r1[3];
    dreieck_zellen(g, t, r0, r1);
    for (int kz = r0[2]; kz <= r1[2]; ++kz)
      for (int ky = r0[1]; ky <= r1[1]; ++ky)
        for (int kx = r0[0]; kx <= r1[0]; ++kx) atomicAdd(&g.anf[(int64_t(kz) * g.zy + ky) * g.zx + kx], 1u);
  }
}
__global__ void __launch_bounds__(kT) zellen_fuellen_kernel(const __grid_constant__ Dev g) {
  for (int64_t t = int64_t(blockIdx.x) * kT + threadIdx.x; t < g.nd; t += int64_t(gridDim.x) * kT) {
    int r0[3], r1[3];
    dreieck_zellen(g, t, r0, r1);
    for (int kz = r0[2]; kz <= r1[2]; ++kz)
      for (int ky = r0[1]; ky <= r1[1]; ++ky)
        for (int kx = r0[0]; kx <= r1[0]; ++kx) {
          const uint32_t pos = atomicAdd(&g.cur[(int64_t(kz) * g.zy + ky) * g.zx + kx], 1u);
          if (pos < g.cap) g.ein[pos] = uint32_t(t);
        }
  }
}
// Entries of a cell in ascending triangle order, the reference's fill order.
// Short cells (up to kKurz entries) are sorted by one thread each; longer ones
// (the cells round a pole of a latitude-longitude mesh hold hundreds) by a
// block in shared memory (bitonic), the longest by a Shell sort of one thread.
constexpr uint32_t kKurz = 32, kLang = 4096;
__global__ void __launch_bounds__(kT) zellen_sortieren_kernel(const uint32_t* anf, uint32_t* ein, int64_t nz) {
  for (int64_t z = int64_t(blockIdx.x) * kT + threadIdx.x; z < nz; z += int64_t(gridDim.x) * kT) {
    const uint32_t lo = anf[z], hi = anf[z + 1];
    if (hi - lo > kKurz) continue;
    for (uint32_t i = lo + 1; i < hi; ++i) {
      const uint32_t v = ein[i];
      uint32_t j = i;
      while (j > lo && ein[j - 1] > v) {
        ein[j] = ein[j - 1];
        --j;
      }
      ein[j] = v;
    }
  }
}
__global__ void __launch_bounds__(kT) zellen_lang_kernel(const uint32_t* anf, uint32_t* ein, int64_t nz) {
  __shared__ uint32_t sh[kLang];
  for (int64_t z = blockIdx.x; z < nz; z += gridDim.x) {
    const uint32_t lo = anf[z], hi = anf[z + 1], n = hi - lo;
    if (n <= kKurz) continue;
    if (n > kLang) {  // Shell sort with Ciura's gaps, one thread
      if (threadIdx.x == 0) {
        const uint32_t gaps[8] = {701u, 301u, 132u, 57u, 23u, 10u, 4u, 1u};
        for (int k = 0; k < 8; ++k) {
          const uint32_t gap = gaps[k];
          for (uint32_t i = lo + gap; i < hi; ++i) {
            const uint32_t key = ein[i];
            uint32_t j = i;
            while (j >= lo + gap && ein[j - gap] > key) {
              ein[j] = ein[j - gap];
              j -= gap;
            }
            ein[j] = key;
          }
        }
      }
      __syncthreads();
      continue;
    }
    uint32_t m = 1;
    while (m < n) m <<= 1;
    for (uint32_t i = threadIdx.x; i < m; i += kT) sh[i] = i < n ? ein[lo + i] : 0xffffffffu;
    __syncthreads();
    for (uint32_t k = 2; k <= m; k <<= 1)
      for (uint32_t j = k >> 1; j > 0; j >>= 1) {
        for (uint32_t i = threadIdx.x; i < m; i += kT) {
          const uint32_t p = i ^ j;
          if (p > i) {
            const bool auf = (i & k) == 0;
            const uint32_t a = sh[i], b = sh[p];
            if ((a > b) == auf) sh[i] = b, sh[p] = a;
          }
        }
        __syncthreads();
      }
    for (uint32_t i = threadIdx.x; i < n; i += kT) ein[lo + i] = sh[i];
    __syncthreads();
  }
}

// ---------------------------------------------------------------- queries
__device__ __forceinline__ void schreibe(const Treffer& r, int64_t q, double* ab, double* pu, double* no, int32_t* dr,
                                         int32_t* rg) {
  ab[q] = r.abstand;
  st3(pu, uint32_t(q), r.punkt);
  st3(no, uint32_t(q), r.normale);
  dr[q] = int32_t(r.dreieck);
  rg[q] = r.region;
}
__global__ void __launch_bounds__(kT) naechster_kernel(const __grid_constant__ Dev g, const double* x, int64_t n,
                                                       double radius, double* ab, double* pu, double* no, int32_t* dr,
                                                       int32_t* rg) {
  for (int64_t q = int64_t(blockIdx.x) * kT + threadIdx.x; q < n; q += int64_t(gridDim.x) * kT) {
    Treffer r;
    if (naechster(g, ld3(x, uint32_t(q)), radius, r)) {
      schreibe(r, q, ab, pu, no, dr, rg);
    } else {
      ab[q] = 0.0;
      st3(pu, uint32_t(q), d3(0, 0, 0));
      st3(no, uint32_t(q), d3(0, 0, 0));
      dr[q] = -1;
      rg[q] = -1;
    }
  }
}

// Nearest over every triangle (naechster_alle, :770-782) for points given as
// a list (x) or as grid nodes (dims > 0; only nodes whose value is NaN when
// `nur_offen`). Triangles pass through shared memory in tiles; each thread
// keeps its own best and skips a triangle by its bounding sphere.
struct Knoten {
  int32_t nx, ny, nz;
  double o0, o1, o2, s;
  float* sdf;
  double band;
  int nur_offen;
};
__device__ __forceinline__ D3 knoten_lage(const Knoten& k, int64_t q) {
  const int64_t i = q % k.nx, j = (q / k.nx) % k.ny, l = q / (int64_t(k.nx) * k.ny);
  return d3(k.o0 + k.s * double(i), k.o1 + k.s * double(j), k.o2 + k.s * double(l));
}
__global__ void __launch_bounds__(kTile) alle_kernel(const __grid_constant__ Dev g, const double* x, int64_t n,
                                                     const __grid_constant__ Knoten kn, double* ab, double* pu,
                                                     double* no, int32_t* dr, int32_t* rg) {
  __shared__ double4 sa[kTile], sb[kTile], sc[kTile], sk[kTile];
  const int64_t nblocks = (n + kTile - 1) / kTile;
  for (int64_t blk = blockIdx.x; blk < nblocks; blk += gridDim.x) {
    const int64_t q = blk * kTile + threadIdx.x;
    bool aktiv = q < n;
    D3 p = d3(0, 0, 0);
    if (aktiv) {
      if (kn.sdf) {
        p = knoten_lage(kn, q);
        if (kn.nur_offen && !isnan(kn.sdf[q])) aktiv = false;
      } else {
        p = ld3(x, uint32_t(q));
      }
    }
    // the whole block leaves when none of its threads has work
    if (__syncthreads_or(aktiv) == 0) continue;
    double best = INFINITY;
    uint32_t bt = 0;
    D3 bq = d3(0, 0, 0);
    int br = 6;
    for (int64_t t0 = 0; t0 < g.nd; t0 += kTile) {
      __syncthreads();
      const int64_t tl = t0 + threadIdx.x;
      if (tl < g.nd) {
        const uint4 d = g.d[tl];
        const D3 a = punkt(g, d.x), b = punkt(g, d.y), c = punkt(g, d.z);
        sa[threadIdx.x] = make_double4(a.x, a.y, a.z, 0.0);
        sb[threadIdx.x] = make_double4(b.x, b.y, b.z, 0.0);
        sc[threadIdx.x] = make_double4(c.x, c.y, c.z, 0.0);
        sk[threadIdx.x] = g.kg[tl];
      }
      __syncthreads();
      const int m = int(g.nd - t0 < kTile ? g.nd - t0 : kTile);
      if (aktiv) {
        for (int j = 0; j < m; ++j) {
          if (!kugel_nah(p, sk[j], best)) continue;
          int reg;
          const D3 qq = naechster_auf_dreieck(p, ld4(sa[j]), ld4(sb[j]), ld4(sc[j]), reg);
          const double l = norm(p - qq);
          const uint32_t t = uint32_t(t0 + j);
          if (l < best) {  // ascending t: the first of equal distances stays
            best = l;
            bt = t;
            bq = qq;
            br = reg;
          }
        }
      }
    }
    if (!aktiv) continue;
    const Treffer r = ergebnis(g, p, bt, bq, br);
    if (kn.sdf) {
      const double v = kn.band > 0.0 ? fmin(fmax(r.abstand, -kn.band), kn.band) : r.abstand;
      kn.sdf[q] = float(v);
    } else {
      schreibe(r, q, ab, pu, no, dr, rg);
    }
  }
}

// netzkoerper.rs:541-593 per segment
__global__ void __launch_bounds__(kT) durchstoss_kernel(const __grid_constant__ Dev g, const double* pa,
                                                        const double* pb, int64_t n, int32_t* dr, double* pu,
                                                        double* no) {
  for (int64_t q = int64_t(blockIdx.x) * kT + threadIdx.x; q < n; q += int64_t(gridDim.x) * kT) {
    D3 p, nn;
    uint32_t t = 0;
    if (durchstoss(g, ld3(pa, uint32_t(q)), ld3(pb, uint32_t(q)), p, nn, t)) {
      dr[q] = int32_t(t);
      st3(pu, uint32_t(q), p);
      st3(no, uint32_t(q), nn);
    } else {
      dr[q] = -1;
      st3(pu, uint32_t(q), d3(0, 0, 0));
      st3(no, uint32_t(q), d3(0, 0, 0));
    }
  }
}

// the surface velocity at given (triangle, point) pairs
__global__ void __launch_bounds__(kT) geschwindigkeit_kernel(const __grid_constant__ Dev g, const int32_t* dr,
                                                             const double* p, int64_t n, double sx, double sy,
                                                             double sz, double* out) {
  for (int64_t q = int64_t(blockIdx.x) * kT + threadIdx.x; q < n; q += int64_t(gridDim.x) * kT)
    st3(out, uint32_t(q), geschwindigkeit_an(g, uint32_t(dr[q]), ld3(p, uint32_t(q)), d3(sx, sy, sz)));
}

// ---------------------------------------------------------------- voxelisation
// The nearest query for the voxeliser: the same result distance as
// naechster (the value does not depend on the visiting order), found faster:
// cells in shells of growing Chebyshev distance around x's cell, a cell
// skipped when its box is no nearer than the best so far, the search ended
// when a whole shell is farther. Ties go to the smallest triangle index.
__device__ bool naechster_schalen(const Dev& g, D3 x, double radius, Treffer& out) {
  int r0[3], r1[3];
  if (!bereich(g, x - d3(radius, radius, radius), x + d3(radius, radius, radius), r0, r1)) return false;
  int64_t k0[3];
  zell_index(g, x, k0);
  int64_t smax = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int64_t lo = k0[a] - r0[a], hi = r1[a] - k0[a];
    smax = lo > smax ? lo : smax;
    smax = hi > smax ? hi : smax;
  }
  const double xs[3] = {x.x, x.y, x.z}, us[3] = {g.u0, g.u1, g.u2};
  double best = radius;
  bool hit = false;
  uint32_t bt = 0xffffffffu;
  D3 bq = d3(0, 0, 0);
  int br = 6;
  for (int64_t s = 0; s <= smax; ++s) {
    if (s >= 1 && double(s - 1) * g.zelle >= best) break;
    for (int64_t dz = -s; dz <= s; ++dz) {
      const int64_t kz = k0[2] + dz;
      if (kz < r0[2] || kz > r1[2]) continue;
      for (int64_t dy = -s; dy <= s; ++dy) {
        const int64_t ky = k0[1] + dy;
        if (ky < r0[1] || ky > r1[1]) continue;
        const bool rand = (dz == -s || dz == s || dy == -s || dy == s);
        const int64_t step = rand ? 1 : (s > 0 ? 2 * s : 1);
        for (int64_t dx = -s; dx <= s; dx += step) {
          const int64_t kx = k0[0] + dx;
          if (kx < r0[0] || kx > r1[0]) continue;
          const int64_t kk[3] = {kx, ky, kz};
          double q2 = 0.0;
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const double lo = us[a] + g.zelle * double(kk[a]), hi = lo + g.zelle;
            const double e = xs[a] < lo ? lo - xs[a] : (xs[a] > hi ? xs[a] - hi : 0.0);
            q2 += e * e;
          }
          if (q2 > best * best * (1.0 + 1e-9)) continue;
          const int64_t z = (kz * g.zy + ky) * g.zx + kx;
          const uint32_t e1 = g.anf[z + 1];
          for (uint32_t e = g.anf[z]; e < e1; ++e) {
            const uint32_t t = g.ein[e];
            if (!kugel_nah(x, g.kg[t], best)) continue;
            const uint4 d = g.d[t];
            int reg;
            const D3 q = naechster_auf_dreieck(x, punkt(g, d.x), punkt(g, d.y), punkt(g, d.z), reg);
            const double l = norm(x - q);
            if (l < best || (hit && l == best && t < bt)) {
              best = l;
              hit = true;
              bt = t;
              bq = q;
              br = reg;
            }
          }
        }
      }
    }
  }
  if (!hit) return false;
  out = ergebnis(g, x, bt, bq, br);
  return true;
}

// Bricks of 8 x 4 x 4 nodes, one block each. The block first gathers into
// shared memory every triangle that may lie within the band of one of its
// nodes: the triangles of the grid cells the brick's box grown by the band
// touches, each taken once (from the first of its cells in that range), kept
// when its bounding sphere comes within the band of the brick's box. Every
// node then tests only those, with the same values as the nearest query
// within the band (the set holds every triangle nearer than the band; ties go
// to the smallest index). A brick whose list overflows queries cell by cell.
constexpr int kZx = 8, kZy = 4, kZz = 4, kZiegel = kZx * kZy * kZz, kKand = 2048;
__global__ void __launch_bounds__(kZiegel) sdf_ziegel_kernel(const __grid_constant__ Dev g,
                                                             const __grid_constant__ Knoten kn) {
  __shared__ uint32_t kand[kKand];
  __shared__ uint32_t zahl;
  const int64_t bx = (kn.nx + kZx - 1) / kZx, by = (kn.ny + kZy - 1) / kZy, bz = (kn.nz + kZz - 1) / kZz;
  const float offen = __int_as_float(0x7fc00000);
  const double band = kn.band;
  for (int64_t zg = blockIdx.x; zg < bx * by * bz; zg += gridDim.x) {
    const int64_t i0 = (zg % bx) * kZx, j0 = ((zg / bx) % by) * kZy, k0 = (zg / (bx * by)) * kZz;
    const int64_t i1 = min(i0 + kZx, int64_t(kn.nx)), j1 = min(j0 + kZy, int64_t(kn.ny)),
                  k1 = min(k0 + kZz, int64_t(kn.nz));
    const D3 lo = d3(kn.o0 + kn.s * double(i0), kn.o1 + kn.s * double(j0), kn.o2 + kn.s * double(k0));
    const D3 hi = d3(kn.o0 + kn.s * double(i1 - 1), kn.o1 + kn.s * double(j1 - 1), kn.o2 + kn.s * double(k1 - 1));
    if (threadIdx.x == 0) zahl = 0;
    __syncthreads();
    int r0[3], r1[3];
    const bool beruehrt = bereich(g, lo - d3(band, band, band), hi + d3(band, band, band), r0, r1);
    if (beruehrt) {
      const int64_t cx = r1[0] - r0[0] + 1, cy = r1[1] - r0[1] + 1, cz = r1[2] - r0[2] + 1;
      for (int64_t c = threadIdx.x; c < cx * cy * cz; c += kZiegel) {
        const int kx = r0[0] + int(c % cx), ky = r0[1] + int((c / cx) % cy), kz = r0[2] + int(c / (cx * cy));
        const int64_t z = (int64_t(kz) * g.zy + ky) * g.zx + kx;
        for (uint32_t e = g.anf[z]; e < g.anf[z + 1]; ++e) {
          const uint32_t t = g.ein[e];
          int t0[3], t1[3];
          dreieck_zellen(g, t, t0, t1);
          if (kx != max(t0[0], r0[0]) || ky != max(t0[1], r0[1]) || kz != max(t0[2], r0[2])) continue;
          const double4 k = g.kg[t];
          const double ex = fmax(fmax(lo.x - k.x, k.x - hi.x), 0.0), ey = fmax(fmax(lo.y - k.y, k.y - hi.y), 0.0),
                       ez = fmax(fmax(lo.z - k.z, k.z - hi.z), 0.0);
          const double dq = sqrt(ex * ex + ey * ey + ez * ez) - k.w;
          if (dq > band * (1.0 + 1e-9) + 1e-12) continue;
          const uint32_t pos = atomicAdd(&zahl, 1u);
          if (pos < kKand) kand[pos] = t;
        }
      }
    }
    __syncthreads();
    const uint32_t m = zahl;
    const int li = threadIdx.x % kZx, lj = (threadIdx.x / kZx) % kZy, lk = threadIdx.x / (kZx * kZy);
    const int64_t i = i0 + li, j = j0 + lj, kk = k0 + lk;
    if (i < i1 && j < j1 && kk < k1) {
      const int64_t q = (kk * kn.ny + j) * kn.nx + i;
      const D3 x = d3(kn.o0 + kn.s * double(i), kn.o1 + kn.s * double(j), kn.o2 + kn.s * double(kk));
      float v = offen;
      if (m > kKand) {
        Treffer t;
        if (naechster_schalen(g, x, band, t)) v = float(t.abstand);
      } else if (m > 0) {
        double best = band;
        bool hit = false;
        uint32_t bt = 0xffffffffu;
        D3 bq = d3(0, 0, 0);
        int br = 6;
        for (uint32_t c = 0; c < m; ++c) {
          const uint32_t t = kand[c];
          if (!kugel_nah(x, g.kg[t], best)) continue;
          const uint4 dd = g.d[t];
          int reg;
          const D3 qq = naechster_auf_dreieck(x, punkt(g, dd.x), punkt(g, dd.y), punkt(g, dd.z), reg);
          const double l = norm(x - qq);
          if (l < best || (hit && l == best && t < bt)) {
            best = l;
            hit = true;
            bt = t;
            bq = qq;
            br = reg;
          }
        }
        if (hit) v = float(ergebnis(g, x, bt, bq, br).abstand);
      }
      kn.sdf[q] = v;
    }
    __syncthreads();
  }
}

// One thread per grid line along axis `achse`: an open run next to a set
// node takes that node's sign (band > spacing: no surface lies between two
// neighbouring nodes when one of them is at least band from it). Counts the
// nodes left open.
__global__ void __launch_bounds__(kT) sdf_linien_kernel(const __grid_constant__ Knoten kn, int achse,
                                                        unsigned long long* offen) {
  const int64_t n[3] = {kn.nx, kn.ny, kn.nz};
  const int64_t st[3] = {1, kn.nx, int64_t(kn.nx) * kn.ny};
  const int a1 = achse == 0 ? 1 : 0, a2 = achse == 2 ? 1 : 2;
  const int64_t linien = n[a1] * n[a2], len = n[achse], schritt = st[achse];
  const float b = float(kn.band);
  unsigned long long rest = 0;
  for (int64_t l = int64_t(blockIdx.x) * kT + threadIdx.x; l < linien; l += int64_t(gridDim.x) * kT) {
    float* p = kn.sdf + (l % n[a1]) * st[a1] + (l / n[a1]) * st[a2];
    float vz = 0.0f;  // sign of the last set node, 0 = none yet
    int64_t erstes = -1;
    for (int64_t i = 0; i < len; ++i) {
      const float v = p[i * schritt];
      if (isnan(v)) {
        if (vz != 0.0f) p[i * schritt] = copysignf(b, vz);
      } else {
        vz = v < 0.0f ? -1.0f : 1.0f;
        if (erstes < 0) erstes = i;
      }
    }
    if (erstes > 0) {
      const float v0 = p[erstes * schritt];
      for (int64_t i = 0; i < erstes; ++i) p[i * schritt] = copysignf(b, v0 < 0.0f ? -1.0f : 1.0f);
    }
    if (erstes < 0) rest += uint64_t(len);
  }
  if (rest) atomicAdd(offen, rest);
}

unsigned blocks_for(int64_t work, int per = kT) {
  int64_t b = (work + per - 1) / per;
  if (b > 148 * 32) b = 148 * 32;
  return unsigned(b < 1 ? 1 : b);
}

}  // namespace netz
}  // namespace k3d


// ==================================================================== host
using namespace k3d;
using namespace k3d::netz;

struct k3d_mesh {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;
  double suchtiefe = 0.0, volumen = 0.0;
  int64_t randkanten = 0, n = 0, nd = 0, eintraege = 0;
  bool gitter_leer = true;
  double u[3] = {0, 0, 0}, zelle = 0;
  int64_t zahl[3] = {0, 0, 0};
  Dev g{};
  Dev* g_dev = nullptr;              // device copy of g, read by the step's contact query
  double* pv_buf = nullptr;          // velocity field storage (3 per point); g.pv points here when set
  std::vector<double> punkte;        // host copy of the current positions
  std::vector<void*> fest;           // allocations of fixed size
  uint32_t *anf = nullptr, *cur = nullptr;  // cell starts and fill cursors (Z + 1)
  int64_t anf_cap = 0;
  uint32_t* ein = nullptr;           // cell entries
  int64_t ein_cap = 0;
  uint32_t* scan_tmp = nullptr;
  int64_t scan_cap = 0;
  uint32_t* pg_anf = nullptr;        // point grid starts (Z + 1)
  int64_t pg_cap = 0;
  uint32_t* pg_ein = nullptr;        // point grid entries (N)
  double* hull = nullptr;            // 7 doubles
  uint32_t* total = nullptr;         // the scan's sum
  unsigned long long* offen = nullptr;
  void* io = nullptr;                // query inputs and outputs
  size_t io_cap = 0;
  double ms = 0.0;
  int64_t kernels = 0, ungeklaert = 0;
};

namespace {

k3d_status fail(k3d_mesh* m, k3d_status s, const std::string& what) {
  if (m) m->err = what;
  return s;
}
k3d_status cuda_fail(k3d_mesh* m, cudaError_t e, const char* where) {
  return fail(m, K3D_DEVICE_ERROR, std::string(where) + ": " + cudaGetErrorString(e));
}
#define NCK(call, where)                                   \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return cuda_fail(m, e_, where); \
  } while (0)

template <typename T>
cudaError_t alloc(k3d_mesh* m, T*& p, size_t count) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
  if (e == cudaSuccess) m->fest.push_back(q);
  p = static_cast<T*>(q);
  return e;
}
template <typename T>
cudaError_t grow(T*& p, int64_t& cap, int64_t need) {
  if (p && need <= cap) return cudaSuccess;
  if (p) cudaFree(p);
  p = nullptr;
  const int64_t c = std::max<int64_t>(need + need / 4, 16);
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), size_t(c) * sizeof(T));
  cap = e == cudaSuccess ? c : 0;
  return e;
}
cudaError_t io_grow(k3d_mesh* m, size_t bytes) {
  if (m->io && bytes <= m->io_cap) return cudaSuccess;
  if (m->io) cudaFree(m->io);
  m->io = nullptr;
  const size_t c = std::max<size_t>(bytes + bytes / 4, 4096);
  cudaError_t e = cudaMalloc(&m->io, c);
  m->io_cap = e == cudaSuccess ? c : 0;
  return e;
}

// gitter_beide (:820-858) for the triangle grid on the hull h (lo, hi): the
// box grows by suchtiefe and joins the previous one; cells of 2 x suchtiefe;
// entries per cell counted, scanned, filled, sorted.
k3d_status gitter(k3d_mesh* m, const double h[6]) {
  Dev& g = m->g;
  cudaStream_t st = m->stream;
  const double s = m->suchtiefe, z = 2.0 * s;
  double u[3], e[3];
  for (int a = 0; a < 3; ++a) {
    u[a] = h[a] - s;
    e[a] = h[3 + a] + s;
    if (!m->gitter_leer) {
      u[a] = std::min(u[a], m->u[a]);
      e[a] = std::max(e[a], m->u[a] + m->zelle * double(m->zahl[a]));
    }
  }
  int64_t zahl[3];
  for (int a = 0; a < 3; ++a) {
    const double c = std::ceil((e[a] - u[a]) / z);
    zahl[a] = std::max<int64_t>(c > 0.0 && c < 4e18 ? int64_t(c) : 0, 1);
  }
  if (zahl[0] > 4096 || zahl[1] > 4096 || zahl[2] > 4096 || zahl[0] * zahl[1] * zahl[2] > (int64_t(1) << 28))
    return fail(m, K3D_BAD_ARGUMENT, "triangle grid over 2^28 cells: suchtiefe is too small for the body's extent");
  const int64_t nz = zahl[0] * zahl[1] * zahl[2];
  for (int a = 0; a < 3; ++a) m->u[a] = u[a], m->zahl[a] = zahl[a];
  m->zelle = z;
  m->gitter_leer = false;
  g.u0 = u[0], g.u1 = u[1], g.u2 = u[2], g.zelle = z;
  g.zx = int32_t(zahl[0]), g.zy = int32_t(zahl[1]), g.zz = int32_t(zahl[2]);
  if (!m->anf || nz + 1 > m->anf_cap) {
    int64_t cap2 = 0;
    NCK(grow(m->anf, m->anf_cap, nz + 1), "grid alloc");
    NCK(grow(m->cur, cap2, m->anf_cap), "grid alloc");
  }
  NCK(grow(m->scan_tmp, m->scan_cap, int64_t(selbst_scan_tmp_words(nz + 1))), "grid alloc");
  g.anf = m->anf;
  g.cur = m->cur;
  NCK(cudaMemsetAsync(m->anf, 0, size_t(nz + 1) * sizeof(uint32_t), st), "grid count");
  zellen_zaehlen_kernel<<<blocks_for(g.nd), kT, 0, st>>>(g);
  NCK(cudaGetLastError(), "grid count");
  NCK(exclusive_scan_u32(m->anf, nz + 1, m->scan_tmp, m->total, st), "grid scan");
  uint32_t total = 0;
  NCK(cudaMemcpyAsync(&total, m->total, sizeof(total), cudaMemcpyDeviceToHost, st), "grid read");
  NCK(cudaStreamSynchronize(st), "grid read");
  m->eintraege = total;
  NCK(grow(m->ein, m->ein_cap, int64_t(total) + 1), "grid alloc");
  g.ein = m->ein;
  g.cap = uint32_t(std::min<int64_t>(m->ein_cap, 0xffffffffll));
  NCK(cudaMemcpyAsync(m->cur, m->anf, size_t(nz) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st), "grid fill");
  zellen_fuellen_kernel<<<blocks_for(g.nd), kT, 0, st>>>(g);
  zellen_sortieren_kernel<<<blocks_for(nz), kT, 0, st>>>(g.anf, g.ein, nz);
  zellen_lang_kernel<<<unsigned(std::min<int64_t>(nz, 148 * 4)), kT, 0, st>>>(g.anf, g.ein, nz);
  NCK(cudaGetLastError(), "grid fill");
  // the point grid on the same cells (its fill cursors reuse the triangle grid's)
  NCK(grow(m->pg_anf, m->pg_cap, nz + 1), "grid alloc");
  g.pg_anf = m->pg_anf;
  g.pg_ein = m->pg_ein;
  NCK(cudaMemsetAsync(g.pg_anf, 0, size_t(nz + 1) * sizeof(uint32_t), st), "point grid");
  punkte_zaehlen_kernel<<<blocks_for(g.n), kT, 0, st>>>(g);
  NCK(exclusive_scan_u32(g.pg_anf, nz + 1, m->scan_tmp, nullptr, st), "point grid");
  NCK(cudaMemcpyAsync(m->cur, g.pg_anf, size_t(nz) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st), "point grid");
  punkte_fuellen_kernel<<<blocks_for(g.n), kT, 0, st>>>(g, m->cur);
  zellen_sortieren_kernel<<<blocks_for(nz), kT, 0, st>>>(g.pg_anf, g.pg_ein, nz);
  zellen_lang_kernel<<<unsigned(std::min<int64_t>(nz, 148 * 4)), kT, 0, st>>>(g.pg_anf, g.pg_ein, nz);
  NCK(cudaGetLastError(), "point grid");
  NCK(cudaMemcpyAsync(m->g_dev, &m->g, sizeof(Dev), cudaMemcpyHostToDevice, st), "grid view");
  m->kernels += 1 + 3 + 3 + 1 + 3 + 1 + 2;
  return K3D_OK;
}

// punktabhaengig (:257-290) on the device positions, then the grid
k3d_status punktabhaengig_und_gitter(k3d_mesh* m) {
  Dev& g = m->g;
  cudaStream_t st = m->stream;
  flaechen_kernel<<<blocks_for(g.nd), kT, 0, st>>>(g);
  punktnormalen_kernel<<<blocks_for(g.n), kT, 0, st>>>(g);
  huelle_kernel<<<1, 1024, 0, st>>>(g, m->hull);
  NCK(cudaGetLastError(), "normals");
  double h[7];
  NCK(cudaMemcpyAsync(h, m->hull, sizeof(h), cudaMemcpyDeviceToHost, st), "hull read");
  NCK(cudaStreamSynchronize(st), "hull read");
  m->kernels += 3;
  m->volumen = h[6];
  if (!(h[6] > 0.0)) return fail(m, K3D_BAD_ARGUMENT, "volume <= 0: the normals point inwards");
  return gitter(m, h);
}

struct Uhr {
  k3d_mesh* m;
  explicit Uhr(k3d_mesh* mm) : m(mm) {
    m->kernels = 0;
    cudaEventRecord(m->ev0, m->stream);
  }
  cudaError_t stopp() {
    cudaEventRecord(m->ev1, m->stream);
    cudaError_t e = cudaEventSynchronize(m->ev1);
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, m->ev0, m->ev1);
    m->ms = ms;
    return e;
  }
};

void freigeben(k3d_mesh* m) {
  if (!m) return;
  cudaSetDevice(m->device);
  for (void* p : m->fest) cudaFree(p);
  for (void* p : {static_cast<void*>(m->anf), static_cast<void*>(m->cur), static_cast<void*>(m->ein),
                  static_cast<void*>(m->scan_tmp), static_cast<void*>(m->pg_anf), m->io})
    if (p) cudaFree(p);
  if (m->ev0) cudaEventDestroy(m->ev0);
  if (m->ev1) cudaEventDestroy(m->ev1);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

void fehler_text(const std::string& s, char* err, int64_t cap) {
  if (!err || cap <= 0) return;
  const size_t k = std::min<size_t>(s.size(), size_t(cap - 1));
  std::memcpy(err, s.data(), k);
  err[k] = 0;
}

bool endlich(const double* p, int64_t n) {
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(p[i])) return false;
  return true;
}

}  // namespace

extern "C" {

k3d_status k3d_mesh_create(const double* punkte, int64_t n, const uint32_t* dreiecke, int64_t nd, double suchtiefe,
                           int32_t device, k3d_mesh** out, char* err, int64_t err_cap) {
  if (!out) return K3D_BAD_ARGUMENT;
  *out = nullptr;
  auto refuse = [&](const std::string& s) {
    fehler_text(s, err, err_cap);
    return K3D_BAD_ARGUMENT;
  };
  // Koerpernetz::neu (:297-367): the checks, in the reference's order
  if (nd <= 0 || !dreiecke) return refuse("body mesh without triangles");
  if (!(suchtiefe > 0.0)) return refuse("search depth must be positive");
  if (n <= 0 || !punkte) return refuse("a triangle names a point out of range");
  if (nd >= (int64_t(1) << 30) || n >= (int64_t(1) << 30)) return refuse("mesh too large (2^30 points or triangles at most)");
  for (int64_t q = 0; q < 3 * nd; ++q)
    if (int64_t(dreiecke[q]) >= n) return refuse("a triangle names a point out of range");
  if (!endlich(punkte, 3 * n)) return refuse("a point is not finite");
  // edges: sorted (key, triangle, edge, direction), then one or two per key
  struct Kante {
    uint64_t key;
    uint32_t t;
    uint8_t k, dir;
  };
  std::vector<Kante> ks(size_t(3 * nd));
  for (int64_t t = 0; t < nd; ++t)
    for (int k = 0; k < 3; ++k) {
      const uint32_t i = dreiecke[3 * t + k], j = dreiecke[3 * t + (k + 1) % 3];
      ks[size_t(3 * t + k)] = {(uint64_t(std::min(i, j)) << 32) | std::max(i, j), uint32_t(t), uint8_t(k),
                               uint8_t(i < j)};
    }
  std::sort(ks.begin(), ks.end(), [](const Kante& a, const Kante& b) {
    return a.key != b.key ? a.key < b.key : (a.t != b.t ? a.t < b.t : a.k < b.k);
  });
  std::vector<uint32_t> nachbar(size_t(4 * nd), 0);
  int64_t rand = 0;
  for (size_t a = 0; a < ks.size();) {
    size_t b = a;
    while (b < ks.size() && ks[b].key == ks[a].key) ++b;
    if (b - a == 1) {
      ++rand;
      nachbar[4 * ks[a].t + ks[a].k] = ks[a].t;
    } else if (b - a == 2) {
      if (ks[a].dir == ks[a + 1].dir) return refuse("mesh orientation is inconsistent at an edge");
      nachbar[4 * ks[a].t + ks[a].k] = ks[a + 1].t;
      nachbar[4 * ks[a + 1].t + ks[a + 1].k] = ks[a].t;
    } else {
      return refuse("an edge has more than two triangles");
    }
    a = b;
  }
  // per point: its (triangle << 2 | corner) in triangle order
  std::vector<uint32_t> pi_off(size_t(n + 1), 0), pi_ent(size_t(3 * nd));
  for (int64_t q = 0; q < 3 * nd; ++q) ++pi_off[dreiecke[q] + 1];
  for (int64_t i = 0; i < n; ++i) pi_off[i + 1] += pi_off[i];
  {
    std::vector<uint32_t> f(pi_off.begin(), pi_off.end() - 1);
    for (int64_t t = 0; t < nd; ++t)
      for (int k = 0; k < 3; ++k) pi_ent[f[dreiecke[3 * t + k]]++] = (uint32_t(t) << 2) | uint32_t(k);
  }
  std::vector<uint32_t> d4(size_t(4 * nd));
  for (int64_t t = 0; t < nd; ++t)
    for (int k = 0; k < 4; ++k) d4[4 * t + k] = k < 3 ? dreiecke[3 * t + k] : 0u;

  k3d_mesh* m = new k3d_mesh();
  m->device = device;
  m->suchtiefe = suchtiefe;
  m->randkanten = rand;
  m->n = n;
  m->nd = nd;
  m->punkte.assign(punkte, punkte + 3 * n);
  auto bail = [&](k3d_status s) {
    fehler_text(m->err, err, err_cap);
    freigeben(m);
    return s;
  };
  k3d_status s = [&]() -> k3d_status {
    NCK(cudaSetDevice(device), "device");
    NCK(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking), "stream");
    NCK(cudaEventCreate(&m->ev0), "event");
    NCK(cudaEventCreate(&m->ev1), "event");
    Dev& g = m->g;
    g.n = n;
    g.nd = nd;
    g.suchtiefe = suchtiefe;
    NCK(alloc(m, m->g_dev, 1), "alloc");
    NCK(alloc(m, m->pv_buf, size_t(3 * n)), "alloc");
    NCK(alloc(m, m->pg_ein, size_t(n)), "alloc");
    g.pv = nullptr;
    double* p = nullptr;
    uint4 *d = nullptr, *nb = nullptr;
    uint32_t *po = nullptr, *pe = nullptr;
    NCK(alloc(m, p, size_t(3 * n)), "alloc");
    NCK(alloc(m, d, size_t(nd)), "alloc");
    NCK(alloc(m, nb, size_t(nd)), "alloc");
    NCK(alloc(m, g.fn, size_t(nd)), "alloc");
    NCK(alloc(m, g.pn, size_t(n)), "alloc");
    NCK(alloc(m, g.kg, size_t(nd)), "alloc");
    NCK(alloc(m, g.wk, size_t(3 * nd)), "alloc");
    NCK(alloc(m, g.vt, size_t(nd)), "alloc");
    NCK(alloc(m, po, size_t(n + 1)), "alloc");
    NCK(alloc(m, pe, size_t(3 * nd)), "alloc");
    NCK(alloc(m, m->hull, 7), "alloc");
    NCK(alloc(m, m->total, 1), "alloc");
    NCK(alloc(m, m->offen, 1), "alloc");
    g.p = p, g.d = d, g.nb = nb, g.pi_off = po, g.pi_ent = pe;
    cudaStream_t st = m->stream;
    NCK(cudaMemcpyAsync(p, punkte, size_t(3 * n) * sizeof(double), cudaMemcpyHostToDevice, st), "upload");
    NCK(cudaMemcpyAsync(d, d4.data(), d4.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st), "upload");
    NCK(cudaMemcpyAsync(nb, nachbar.data(), nachbar.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st), "upload");
    NCK(cudaMemcpyAsync(po, pi_off.data(), pi_off.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st), "upload");
    NCK(cudaMemcpyAsync(pe, pi_ent.data(), pi_ent.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st), "upload");
    Uhr uhr(m);
    k3d_status r = punktabhaengig_und_gitter(m);
    if (r != K3D_OK) return r;
    NCK(uhr.stopp(), "create");
    return K3D_OK;
  }();
  if (s != K3D_OK) return bail(s);
  *out = m;
  return K3D_OK;
}

void k3d_mesh_destroy(k3d_mesh* m) { freigeben(m); }

const char* k3d_mesh_last_error(const k3d_mesh* m) { return m ? m->err.c_str() : "null mesh"; }

k3d_status k3d_mesh_update(k3d_mesh* m, const double* punkte) {
  if (!m || !punkte) return fail(m, K3D_BAD_ARGUMENT, "null argument");
  if (!endlich(punkte, 3 * m->n)) return fail(m, K3D_BAD_ARGUMENT, "a point is not finite");
  NCK(cudaSetDevice(m->device), "device");
  cudaStream_t st = m->stream;
  double* p = const_cast<double*>(m->g.p);
  Uhr uhr(m);
  NCK(cudaMemcpyAsync(p, punkte, size_t(3 * m->n) * sizeof(double), cudaMemcpyHostToDevice, st), "upload");
  const double* pv_alt = m->g.pv;
  m->g.pv = nullptr;  // the velocity field belonged to the old positions (netzkoerper.rs:409)
  k3d_status r = punktabhaengig_und_gitter(m);
  if (r == K3D_BAD_ARGUMENT) {
    m->g.pv = pv_alt;  // refused: the mesh keeps its positions and its field
    // keep the previous positions and everything that hangs on them
    const std::string why = !(m->volumen > 0.0) ? "volume <= 0 after deforming: the mesh turned inside out" : m->err;
    NCK(cudaMemcpyAsync(p, m->punkte.data(), size_t(3 * m->n) * sizeof(double), cudaMemcpyHostToDevice, st),
        "restore");
    k3d_status r2 = punktabhaengig_und_gitter(m);
    if (r2 != K3D_OK) return r2;
    NCK(uhr.stopp(), "update");
    return fail(m, K3D_BAD_ARGUMENT, why);
  }
  if (r != K3D_OK) return r;
  NCK(uhr.stopp(), "update");
  m->punkte.assign(punkte, punkte + 3 * m->n);
  return K3D_OK;
}

k3d_status k3d_mesh_set_velocity(k3d_mesh* m, const double* v) {
  if (!m) return K3D_BAD_ARGUMENT;
  if (v && !endlich(v, 3 * m->n)) return fail(m, K3D_BAD_ARGUMENT, "a velocity is not finite");
  NCK(cudaSetDevice(m->device), "device");
  cudaStream_t st = m->stream;
  if (v) NCK(cudaMemcpyAsync(m->pv_buf, v, size_t(3 * m->n) * sizeof(double), cudaMemcpyHostToDevice, st), "upload");
  m->g.pv = v ? m->pv_buf : nullptr;
  NCK(cudaMemcpyAsync(m->g_dev, &m->g, sizeof(Dev), cudaMemcpyHostToDevice, st), "view");
  NCK(cudaStreamSynchronize(st), "velocity");
  return K3D_OK;
}

k3d_status k3d_mesh_get_info(const k3d_mesh* m, k3d_mesh_info* o) {
  if (!m || !o) return K3D_BAD_ARGUMENT;
  *o = k3d_mesh_info{};
  o->n_punkte = m->n;
  o->n_dreiecke = m->nd;
  o->randkanten = m->randkanten;
  o->volumen = m->volumen;
  o->suchtiefe = m->suchtiefe;
  for (int a = 0; a < 3; ++a) o->gitter_ursprung[a] = m->u[a], o->gitter_zahl[a] = m->zahl[a];
  o->gitter_zelle = m->zelle;
  o->gitter_eintraege = m->eintraege;
  o->ms_letzter_aufruf = m->ms;
  o->kernels_letzter_aufruf = m->kernels;
  o->ungeklaert = m->ungeklaert;
  return K3D_OK;
}

k3d_status k3d_mesh_tables(k3d_mesh* m, double* fn, double* pn, uint32_t* nachbar, double* kugel) {
  if (!m) return K3D_BAD_ARGUMENT;
  NCK(cudaSetDevice(m->device), "device");
  cudaStream_t st = m->stream;
  const size_t nd = size_t(m->nd), n = size_t(m->n);
  std::vector<double4> a(std::max(nd, n));
  if (fn) {
    NCK(cudaMemcpyAsync(a.data(), m->g.fn, nd * sizeof(double4), cudaMemcpyDeviceToHost, st), "read");
    NCK(cudaStreamSynchronize(st), "read");
    for (size_t t = 0; t < nd; ++t) fn[3 * t] = a[t].x, fn[3 * t + 1] = a[t].y, fn[3 * t + 2] = a[t].z;
  }
  if (kugel) {
    NCK(cudaMemcpyAsync(a.data(), m->g.kg, nd * sizeof(double4), cudaMemcpyDeviceToHost, st), "read");
    NCK(cudaStreamSynchronize(st), "read");
    for (size_t t = 0; t < nd; ++t)
      kugel[4 * t] = a[t].x, kugel[4 * t + 1] = a[t].y, kugel[4 * t + 2] = a[t].z, kugel[4 * t + 3] = a[t].w;
  }
  if (pn) {
    NCK(cudaMemcpyAsync(a.data(), m->g.pn, n * sizeof(double4), cudaMemcpyDeviceToHost, st), "read");
    NCK(cudaStreamSynchronize(st), "read");
    for (size_t i = 0; i < n; ++i) pn[3 * i] = a[i].x, pn[3 * i + 1] = a[i].y, pn[3 * i + 2] = a[i].z;
  }
  if (nachbar) {
    std::vector<uint4> b(nd);
    NCK(cudaMemcpyAsync(b.data(), m->g.nb, nd * sizeof(uint4), cudaMemcpyDeviceToHost, st), "read");
    NCK(cudaStreamSynchronize(st), "read");
    for (size_t t = 0; t < nd; ++t) nachbar[3 * t] = b[t].x, nachbar[3 * t + 1] = b[t].y, nachbar[3 * t + 2] = b[t].z;
  }
  return K3D_OK;
}

k3d_status k3d_mesh_nearest(k3d_mesh* m, const double* x, int64_t n, double radius, double* abstand, double* punkt,
                            double* normale, int32_t* dreieck, int32_t* region) {
  if (!m || (n > 0 && !x) || n < 0) return fail(m, K3D_BAD_ARGUMENT, "null argument or negative count");
  if (n >= (int64_t(1) << 30)) return fail(m, K3D_BAD_ARGUMENT, "over 2^30 query points");
  if (n == 0) return K3D_OK;
  if (std::isnan(radius)) return fail(m, K3D_BAD_ARGUMENT, "radius is NaN");
  NCK(cudaSetDevice(m->device), "device");
  cudaStream_t st = m->stream;
  const size_t N = size_t(n);
  NCK(io_grow(m, N * (3 + 1 + 3 + 3) * sizeof(double) + N * 2 * sizeof(int32_t)), "alloc");
  double* dx = static_cast<double*>(m->io);
  double *dab = dx + 3 * N, *dpu = dab + N, *dno = dpu + 3 * N;
  int32_t* ddr = reinterpret_cast<int32_t*>(dno + 3 * N);
  int32_t* drg = ddr + N;
  NCK(cudaMemcpyAsync(dx, x, 3 * N * sizeof(double), cudaMemcpyHostToDevice, st), "upload");
  Uhr uhr(m);
  if (radius > 0.0) {
    naechster_kernel<<<blocks_for(n), kT, 0, st>>>(m->g, dx, n, radius, dab, dpu, dno, ddr, drg);
  } else {
    Knoten kn{};
    alle_kernel<<<blocks_for(n, kTile), kTile, 0, st>>>(m->g, dx, n, kn, dab, dpu, dno, ddr, drg);
  }
  NCK(cudaGetLastError(), "nearest");
  m->kernels = 1;
  NCK(uhr.stopp(), "nearest");
  m->kernels = 1;
  if (abstand) NCK(cudaMemcpyAsync(abstand, dab, N * sizeof(double), cudaMemcpyDeviceToHost, st), "read");
  if (punkt) NCK(cudaMemcpyAsync(punkt, dpu, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, st), "read");
  if (normale) NCK(cudaMemcpyAsync(normale, dno, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, st), "read");
  if (dreieck) NCK(cudaMemcpyAsync(dreieck, ddr, N * sizeof(int32_t), cudaMemcpyDeviceToHost, st), "read");
  if (region) NCK(cudaMemcpyAsync(region, drg, N * sizeof(int32_t), cudaMemcpyDeviceToHost, st), "read");
  NCK(cudaStreamSynchronize(st), "read");
  return K3D_OK;
}

k3d_status k3d_mesh_velocity_at(k3d_mesh* m, const int32_t* dreieck, const double* punkt, int64_t n,
                                const double starr[3], double* out) {
  if (!m || n < 0 || (n > 0 && (!dreieck || !punkt || !out)) || !starr) return fail(m, K3D_BAD_ARGUMENT, "null argument");
  if (n >= (int64_t(1) << 30)) return fail(m, K3D_BAD_ARGUMENT, "over 2^30 points");
  for (int64_t q = 0; q < n; ++q)
    if (dreieck[q] < 0 || int64_t(dreieck[q]) >= m->nd) return fail(m, K3D_BAD_ARGUMENT, "triangle out of range");
  if (n == 0) return K3D_OK;
  NCK(cudaSetDevice(m->device), "device");
  cudaStream_t st = m->stream;
  const size_t N = size_t(n);
  NCK(io_grow(m, N * 6 * sizeof(double) + N * sizeof(int32_t)), "alloc");
  double* dp = static_cast<double*>(m->io);
  double* dout = dp + 3 * N;
  int32_t* ddr = reinterpret_cast<int32_t*>(dout + 3 * N);
  NCK(cudaMemcpyAsync(dp, punkt, 3 * N * sizeof(double), cudaMemcpyHostToDevice, st), "upload");
  NCK(cudaMemcpyAsync(ddr, dreieck, N * sizeof(int32_t), cudaMemcpyHostToDevice, st), "upload");
  Uhr uhr(m);
  geschwindigkeit_kernel<<<blocks_for(n), kT, 0, st>>>(m->g, ddr, dp, n, starr[0], starr[1], starr[2], dout);
  NCK(cudaGetLastError(), "velocity");
  NCK(uhr.stopp(), "velocity");
  m->kernels = 1;
  NCK(cudaMemcpyAsync(out, dout, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, st), "read");
  NCK(cudaStreamSynchronize(st), "read");
  return K3D_OK;
}

k3d_status k3d_mesh_penetration(k3d_mesh* m, const double* a, const double* b, int64_t n, int32_t* dreieck,
                                double* punkt, double* normale) {
  if (!m || (n > 0 && (!a || !b || !dreieck)) || n < 0) return fail(m, K3D_BAD_ARGUMENT, "null argument");
  if (n >= (int64_t(1) << 30)) return fail(m, K3D_BAD_ARGUMENT, "over 2^30 segments");
  if (n == 0) return K3D_OK;
  NCK(cudaSetDevice(m->device), "device");
  cudaStream_t st = m->stream;
  const size_t N = size_t(n);
  NCK(io_grow(m, N * (3 + 3 + 3 + 3) * sizeof(double) + N * sizeof(int32_t)), "alloc");
  double* da = static_cast<double*>(m->io);
  double *db = da + 3 * N, *dpu = db + 3 * N, *dno = dpu + 3 * N;
  int32_t* ddr = reinterpret_cast<int32_t*>(dno + 3 * N);
  NCK(cudaMemcpyAsync(da, a, 3 * N * sizeof(double), cudaMemcpyHostToDevice, st), "upload");
  NCK(cudaMemcpyAsync(db, b, 3 * N * sizeof(double), cudaMemcpyHostToDevice, st), "upload");
  Uhr uhr(m);
  durchstoss_kernel<<<blocks_for(n), kT, 0, st>>>(m->g, da, db, n, ddr, dpu, dno);
  NCK(cudaGetLastError(), "penetration");
  NCK(uhr.stopp(), "penetration");
  m->kernels = 1;
  NCK(cudaMemcpyAsync(dreieck, ddr, N * sizeof(int32_t), cudaMemcpyDeviceToHost, st), "read");
  if (punkt) NCK(cudaMemcpyAsync(punkt, dpu, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, st), "read");
  if (normale) NCK(cudaMemcpyAsync(normale, dno, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, st), "read");
  NCK(cudaStreamSynchronize(st), "read");
  return K3D_OK;
}

k3d_status k3d_mesh_sdf(k3d_mesh* m, const int32_t dims[3], const double ursprung[3], double spacing, double band,
                        float* sdf) {
  if (!m || !dims || !ursprung || !sdf) return fail(m, K3D_BAD_ARGUMENT, "null argument");
  if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1) return fail(m, K3D_BAD_ARGUMENT, "dims must be positive");
  const int64_t nn = int64_t(dims[0]) * dims[1] * dims[2];
  if (nn > (int64_t(1) << 31)) return fail(m, K3D_BAD_ARGUMENT, "grid over 2^31 nodes");
  if (!(spacing > 0.0) || !std::isfinite(spacing)) return fail(m, K3D_BAD_ARGUMENT, "spacing must be positive");
  if (!endlich(ursprung, 3) || std::isnan(band)) return fail(m, K3D_BAD_ARGUMENT, "origin or band not finite");
  if (band > 0.0 && !(band > spacing)) return fail(m, K3D_BAD_ARGUMENT, "band must exceed the node spacing");
  NCK(cudaSetDevice(m->device), "device");
  cudaStream_t st = m->stream;
  NCK(io_grow(m, size_t(nn) * sizeof(float)), "alloc");
  Knoten kn{dims[0], dims[1], dims[2], ursprung[0], ursprung[1], ursprung[2], spacing,
            static_cast<float*>(m->io), band > 0.0 ? band : 0.0, 0};
  Uhr uhr(m);
  m->ungeklaert = 0;
  if (band > 0.0) {
    const int64_t ziegel = ((dims[0] + kZx - 1) / kZx) * int64_t((dims[1] + kZy - 1) / kZy) * ((dims[2] + kZz - 1) / kZz);
    sdf_ziegel_kernel<<<unsigned(std::min<int64_t>(ziegel, 148 * 64)), kZiegel, 0, st>>>(m->g, kn);
    NCK(cudaGetLastError(), "sdf band");
    for (int achse = 0; achse < 3; ++achse) {
      NCK(cudaMemsetAsync(m->offen, 0, sizeof(unsigned long long), st), "sdf lines");
      const int64_t linien = nn / (achse == 0 ? dims[0] : (achse == 1 ? dims[1] : dims[2]));
      sdf_linien_kernel<<<blocks_for(linien), kT, 0, st>>>(kn, achse, m->offen);
    }
    NCK(cudaGetLastError(), "sdf lines");
    unsigned long long offen = 0;
    NCK(cudaMemcpyAsync(&offen, m->offen, sizeof(offen), cudaMemcpyDeviceToHost, st), "sdf lines");
    NCK(cudaStreamSynchronize(st), "sdf lines");
    m->kernels = 4;
    m->ungeklaert = int64_t(offen);
    if (offen) {
      kn.nur_offen = 1;
      alle_kernel<<<blocks_for(nn, kTile), kTile, 0, st>>>(m->g, nullptr, nn, kn, nullptr, nullptr, nullptr, nullptr,
                                                           nullptr);
      NCK(cudaGetLastError(), "sdf exact");
      m->kernels += 1;
    }
  } else {
    alle_kernel<<<blocks_for(nn, kTile), kTile, 0, st>>>(m->g, nullptr, nn, kn, nullptr, nullptr, nullptr, nullptr,
                                                         nullptr);
    NCK(cudaGetLastError(), "sdf exact");
    m->kernels = 1;
  }
  const int64_t k = m->kernels;
  NCK(uhr.stopp(), "sdf");
  m->kernels = k;
  NCK(cudaMemcpyAsync(sdf, m->io, size_t(nn) * sizeof(float), cudaMemcpyDeviceToHost, st), "read");
  NCK(cudaStreamSynchronize(st), "read");
  return K3D_OK;
}

}  // extern "C"

namespace k3d {
const netz::Dev* mesh_device_view(const k3d_mesh* m, int* device) {
  if (!m) return nullptr;
  if (device) *device = m->device;
  return m->g_dev;
}
}  // namespace k3d
