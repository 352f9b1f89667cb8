// The persistent PCG kernel of the implicit step (internal to the library):
// grid barrier with deterministic reductions, the CG vectors, the block-row
// product, the PCG (implizit.rs:370-426) and the release pass
// (implizit.rs:908-943). Included by two translation units with different
// arithmetic flags: k3d_step.cu instantiates the forms with FP64 vectors and
// is compiled without fused multiply-add (every product and sum rounds on its
// own, as the reference's arithmetic does), k3d_step_f32.cu the form with
// FP32 vectors, compiled with fused multiply-add (fewer iterations there).
#pragma once
#include <cfloat>
#include <cstdint>

#include "k3d_step_common.cuh"

namespace k3d {

// ------------------------------------------------------------ barrier + reductions
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed_i32(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

constexpr uint64_t kBarrierLimitNs = 4000000000ull;  // 4 s per barrier wait
// The FP32 operator resolves the relative residual (P^-1 norm) to about
// 1e-6 on stiff cloth; below that the directions lose conjugacy and a solve
// can diverge. The mixed form never asks for less.
constexpr double kMixedTolFloor = 1e-6;
// Reliable updates of the mixed form: the true residual replaces the
// recursive one once r.z has fallen by kReliable since the last update, or
// grown by kGrow (then the direction restarts).
constexpr double kReliable = 1e-2;
constexpr double kGrow = 1e2;
constexpr int kMaxRed = kRedMax;

struct Shared {
  double red[kMaxRed][32];
  double res[kMaxRed];
  unsigned epoch;  // barriers passed in this launch
  unsigned rbuf;   // reductions done in this launch (partials buffer parity)
  int err;
  Grp g;           // this block's group (instance)
  unsigned bidx;   // this block's index within the group
};

// Loops of the PCG over the group's points and element ranges, strided over
// the group's blocks (for a scene of one drape: the whole grid).
#define GRP_FOR(i, lo, hi)                                                                         \
  for (int64_t i = (lo) + int64_t(sh.bidx) * blockDim.x + threadIdx.x; i < (hi); \
       i += int64_t(sh.g.nblk) * blockDim.x)

__device__ __forceinline__ unsigned atom_add_release(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// Block sum of NV values in a fixed order (warp xor tree, then the warps in
// order); the result is in v in every thread.
template <int NV>
__device__ __forceinline__ void block_sum(Shared& sh, double (&v)[NV]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sh.red[k][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = 0.0;
      for (int w = 0; w < nw; ++w) t += sh.red[k][w];
      sh.res[k] = t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = sh.res[k];
  __syncthreads();
}

// Grid barrier: every block adds one to a counter that starts at zero in
// each launch; barrier k of the launch is passed when the counter reaches
// k * gridDim.x. With NV > 0 it also sums NV doubles over the grid: each
// block writes its partials before arriving and, once through, adds all
// blocks' partials in block order itself, so every block holds the same
// bits. Partials alternate between two buffers (a block can only reuse a
// buffer after every block has passed the barrier that follows the reads).
// The wait gives up after kBarrierLimitNs or when another block has recorded
// an error; the return value is false then and the caller leaves the kernel.
template <int NV>
__device__ bool grid_sync(const StepArgs& a, Shared& sh, double (&v)[NV > 0 ? NV : 1]) {
  SyncState* s = a.sync;
  const unsigned buf = sh.rbuf & 1u;
  const unsigned nb = sh.g.nblk;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if constexpr (NV > 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double x = v[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) sh.red[k][warp] = x;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if constexpr (NV > 0) {
      const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
      for (int k = 0; k < NV; ++k) {
        double t = 0.0;
        for (int w = 0; w < nw; ++w) t += sh.red[k][w];
        sh.g.partials[(buf * kMaxRed + k) * nb + sh.bidx] = t;
      }
      sh.rbuf += 1;  // every thread read the parity at entry, before the barrier above
    }
    const unsigned target = (sh.epoch + 1) * nb;
    atom_add_release(sh.g.count, 1u);
    const uint64_t t0 = globaltimer();
    int err = 0;
    // poll the counter alone; the error flag and the time limit every 16th
    // poll (each check is another round trip behind the acquiring load)
    for (unsigned poll = 1; int(ld_acquire_u32(sh.g.count) - target) < 0; ++poll) {
      if ((poll & 15u) != 0u) continue;
      if ((err = ld_relaxed_i32(&s->error)) != 0) break;
      if (globaltimer() - t0 > kBarrierLimitNs) {
        atomicCAS(&s->error, 0, K3D_STATUS_TIMEOUT);
        err = K3D_STATUS_TIMEOUT;
        break;
      }
    }
    sh.err = err;
    sh.epoch += 1;
  }
  __syncthreads();
  if (sh.err != 0) return false;
  if constexpr (NV > 0) {
    // warp 0 adds the block partials in block order (fixed per lane, then a
    // fixed xor tree): every block gets the same bits
    if (warp == 0) {
#pragma unroll
      for (int k = 0; k < NV; ++k) {
        double x = 0.0;
        for (unsigned b = lane; b < nb; b += 32) x += __ldcg(&sh.g.partials[(buf * kMaxRed + k) * nb + b]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sh.res[k] = x;
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = sh.res[k];
  }
  return true;
}

__device__ __forceinline__ bool barrier(const StepArgs& a, Shared& sh) {
  double none[1] = {0.0};
  return grid_sync<0>(a, sh, none);
}


static __device__ __noinline__ void apply_dv64(const StepArgs& a, const Shared& sh) {
  const R4<double>* f1w = static_cast<const R4<double>*>(a.m_f1w64);
  const R4<double>* f2w = static_cast<const R4<double>*>(a.m_f2w64);
  const R4<double>* kgB = static_cast<const R4<double>*>(a.m_kgB64);
  const R4<double>* rin = static_cast<const R4<double>*>(a.m_rin64);
  const R4<double>* kgA = static_cast<const R4<double>*>(a.m_kgA64);
  const R4<double>* grad = static_cast<const R4<double>*>(a.b_grad64);
  const R4<double>* sdq = static_cast<const R4<double>*>(a.s_dq64);
  const double* sk = static_cast<const double*>(a.s_k64);
  R4<double>* slot = static_cast<R4<double>*>(a.slot64);
  auto dvp = [&](uint32_t i) -> R4<double> {
    const D3 d = ld3(a.dv, i);
    return {d.x, d.y, d.z, 0.0};
  };
  GRP_FOR(t, sh.g.t0, sh.g.t1) {
    const uint4 id = __ldg(&a.m_idx[t]);
    const uint4 ps = __ldg(&a.m_pos[t]);
    const R4<double> d[3] = {dvp(id.x), dvp(id.y), dvp(id.z)};
    R4<double> out[3];
    membran_hv<double>(f1w[t], f2w[t], rin[t], kgA[t], kgB[t], d, out);
    slot[ps.x] = out[0];
    slot[ps.y] = out[1];
    slot[ps.z] = out[2];
  }
  GRP_FOR(b, sh.g.b0, sh.g.b1) {
    const uint4 id = __ldg(&a.b_idx[b]);
    const uint4 ps = __ldg(&a.b_pos[b]);
    const R4<double> g0 = grad[4 * b], g1 = grad[4 * b + 1], g2 = grad[4 * b + 2], g3 = grad[4 * b + 3];
    const R4<double> c0 = dvp(id.x), c1 = dvp(id.y), c2 = dvp(id.z), c3 = dvp(id.w);
    const double gp = g1.x * (c1.x - c0.x) + g1.y * (c1.y - c0.y) + g1.z * (c1.z - c0.z) + g2.x * (c2.x - c0.x) +
                      g2.y * (c2.y - c0.y) + g2.z * (c2.z - c0.z) + g3.x * (c3.x - c0.x) + g3.y * (c3.y - c0.y) +
                      g3.z * (c3.z - c0.z);
    const double sc = g0.w * gp;
    slot[ps.x] = {g0.x * sc, g0.y * sc, g0.z * sc, 0.0};
    slot[ps.y] = {g1.x * sc, g1.y * sc, g1.z * sc, 0.0};
    slot[ps.z] = {g2.x * sc, g2.y * sc, g2.z * sc, 0.0};
    slot[ps.w] = {g3.x * sc, g3.y * sc, g3.z * sc, 0.0};
  }
  GRP_FOR(s, sh.g.s0, sh.g.s1) {
    const uint4 id = __ldg(&a.s_idx[s]);
    const uint2 ps = __ldg(&a.s_pos[s]);
    const R4<double> dq = sdq[s];
    const double k = sk[s];
    const R4<double> ci = dvp(id.x), cj = dvp(id.y);
    const double dx = ci.x - cj.x, dy = ci.y - cj.y, dz = ci.z - cj.z;
    const double nd = (dq.x * dx + dq.y * dy + dq.z * dz) * (1.0 - dq.w);
    const double ox = k * (dq.x * nd + dx * dq.w), oy = k * (dq.y * nd + dy * dq.w), oz = k * (dq.z * nd + dz * dq.w);
    slot[ps.x] = {ox, oy, oz, 0.0};
    slot[ps.y] = {-ox, -oy, -oz, 0.0};
  }
}

// (A dv)_i in FP64 from the slots of apply_dv64.
template <bool SC>
__device__ __noinline__ D3 a_dv64(const StepArgs& a, int64_t i) {
  const R4<double>* sl = static_cast<const R4<double>*>(a.slot64) + i;
  double x = 0, y = 0, z = 0;
  const uint32_t cnt = __ldg(&a.cnt_v[i]);
#pragma unroll 6
  for (uint32_t k = 0; k < cnt; ++k) {
    const R4<double> o = sl[size_t(k) * a.np];
    x += o.x;
    y += o.y;
    z += o.z;
  }
  if (SC) {
    const D3 sp = feder_hp64(a, i, [&](uint32_t j) { return ld3(a.dv, j); }, nullptr);
    x += sp.x;
    y += sp.y;
    z += sp.z;
  }
  const double h2 = a.h * a.h, md = a.masse[i] * (1.0 + a.h * a.daempf);
  const D3 d = ld3(a.dv, uint32_t(i));
  return d3(md * d.x + h2 * x, md * d.y + h2 * y, md * d.z + h2 * z);
}

// ------------------------------------------------------------ PCG vectors
// The PCG's vectors in precision V: the (c, w) buffers, r and ap; the
// preconditioner (symmetric 3x3 per point) and the mass term in R, the
// operator precision. FP64 vectors filter with the FP64 contact normal.
// A (c, w) buffer of the PCG: the direction c and the filtered
// preconditioned residual w = S P^-1 r as two arrays of the points (c at the
// buffer's start, w after it), so a gather of w alone touches w's sectors only.
template <typename V>
struct Dir {
  R4<V>* c;
  R4<V>* w;
  __device__ Dir(void* base, int64_t n) : c(static_cast<R4<V>*>(base)), w(static_cast<R4<V>*>(base) + n) {}
};
// c' = w + beta c at point j (implizit.rs:421), the same helper everywhere so
// every reader holds the same bits
template <typename V>
__device__ __forceinline__ R4<V> next_dir(const Dir<V>& d, int64_t j, V beta) {
  const R4<V> c = d.c[j], w = d.w[j];
  return {fmar(beta, c.x, w.x), fmar(beta, c.y, w.y), fmar(beta, c.z, w.z), V(0)};
}

template <typename R, typename V>
struct Vec {
  Dir<V> cw;
  V *r, *ap;
  const R* pinv;
  const V* nrm;
  R* nrm_r;  // the operator-precision normal, cleared with the FP64 one on release
  const R* md;
  __device__ explicit Vec(const StepArgs& a)
      : cw(a.c, a.n), r((V*)a.r), ap((V*)a.ap), pinv((const R*)a.pinv),
        nrm(sizeof(V) == 8 ? (const V*)(const void*)a.nrm_d : (const V*)a.nrm), nrm_r((R*)a.nrm),
        md((const R*)a.md) {}
};

template <typename R, typename V>
__device__ __forceinline__ void pmulv(const R* P, int64_t i, V x, V y, V z, V& ox, V& oy, V& oz) {
  const V p0 = V(P[6 * i]), p1 = V(P[6 * i + 1]), p2 = V(P[6 * i + 2]), p3 = V(P[6 * i + 3]),
          p4 = V(P[6 * i + 4]), p5 = V(P[6 * i + 5]);
  ox = p0 * x + p3 * y + p4 * z;
  oy = p3 * x + p1 * y + p5 * z;
  oz = p4 * x + p5 * y + p2 * z;
}

// w = (V) dv, c = 0: the next row product with beta = 0 applies A to dv.
template <typename V>
__device__ void dv_to_w(const StepArgs& a, const Dir<V>& cw, const Shared& sh) {
  GRP_FOR(i, sh.g.r0, sh.g.r1) {
    const D3 d = ld3(a.dv, uint32_t(i));
    cw.w[i] = {V(d.x), V(d.y), V(d.z), V(0)};
    cw.c[i] = {V(0), V(0), V(0), V(0)};
  }
}

// a 4-wide record through the read-only data path
__device__ __forceinline__ R4<float> ldg_r4(const R4<float>* p) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(p));
  return R4<float>{v.x, v.y, v.z, v.w};
}

// (A c)_i over row i of the assembled A, c = w + beta c formed at each
// neighbour from buf; with WONLY, (A w)_i (beta is not read). Blocks in R,
// vectors and sums in V.
template <typename R, typename V, bool SC, bool WONLY = false>
__device__ __forceinline__ void bsr_row(const StepArgs& a, const Dir<V>& buf, int64_t i, V beta, V& ox, V& oy,
                                        V& oz) {
  // blocks as (m00 m01 m02 m10), (m11 m12 m20 m21), m22: three loads a block;
  // the FP32 ones through the read-only path (the assembled A is not written
  // during a solve launch), so that they may move ahead of this loop's stores
  const R4<R>* b4 = static_cast<const R4<R>*>(a.bmat);
  const R* b1 = static_cast<const R*>(a.bmat) + 8 * a.bplane;
  const int64_t P = a.bplane;
  V x = 0, y = 0, z = 0;
  const uint32_t cnt = __ldg(&a.row_cnt[i]);
#pragma unroll 2
  for (uint32_t k = 0; k < cnt; ++k) {
    const int64_t sid = int64_t(k) * a.np + i;
    const uint32_t j = __ldg(&a.col[sid]);
    const R4<V> pj = WONLY ? buf.w[j] : next_dir<V>(buf, j, beta);
    R4<R> u, v;
    R w;
    if constexpr (sizeof(R) == 4) {  // measured: faster for the FP32 blocks, slower for the FP64 ones
      u = ldg_r4(&b4[sid]), v = ldg_r4(&b4[P + sid]);
      w = __ldg(&b1[sid]);
    } else {
      u = b4[sid], v = b4[P + sid];
      w = b1[sid];
    }
    x += V(u.x) * pj.x + V(u.y) * pj.y + V(u.z) * pj.z;
    y += V(u.w) * pj.x + V(v.x) * pj.y + V(v.y) * pj.z;
    z += V(v.z) * pj.x + V(v.w) * pj.y + V(w) * pj.z;
  }
  if (SC) {  // self-collision springs, matrix-free (h^2 is in their blocks)
    const R4<R>* bR = static_cast<const R4<R>*>(a.sc_bR);
    const R4<R>* wR = static_cast<const R4<R>*>(a.sc_wR);
    const R* g5R = static_cast<const R*>(a.sc_g5R);
    const R4<V> pi = next_dir<V>(buf, i, beta);
    for (uint32_t e = a.sc_off[i]; e < a.sc_off[i + 1]; ++e) {
      const uint32_t ent = a.sc_ent[e], q = ent >> 3, k = ent & 7u;
      const uint4 id = a.sc_idx[q];
      const R4<R> w4 = wR[q];
      const V g[5] = {V(w4.x), V(w4.y), V(w4.z), V(w4.w), V(g5R[q])};
      const uint32_t ix[5] = {id.x, id.y, id.z, id.w, a.sc_x5[q]};
      const V gk = g[k];
      V sx = 0, sy = 0, sz = 0;
#pragma unroll
      for (int r = 0; r < 5; ++r)
        if ((gk > V(0) && g[r] < V(0)) || (gk < V(0) && g[r] > V(0))) {
          const V om = -gk * g[r];
          const R4<V> pr = next_dir<V>(buf, ix[r], beta);
          sx += om * (pi.x - pr.x);
          sy += om * (pi.y - pr.y);
          sz += om * (pi.z - pr.z);
        }
      const R4<R> b0 = bR[2 * q], b1 = bR[2 * q + 1];
      x += V(b0.x) * sx + V(b0.w) * sy + V(b1.x) * sz;
      y += V(b0.w) * sx + V(b0.y) * sy + V(b1.y) * sz;
      z += V(b1.x) * sx + V(b1.y) * sy + V(b0.z) * sz;
    }
  }
  ox = x;
  oy = y;
  oz = z;
}

// Rows a thread takes together in the CG iteration's two point passes; each
// round issues its rows' loads before any of their stores. Measured on the
// 66k- and 201k-point sheets: one row per round is fastest (two cost 15-25 %
// more per iteration, three more still).
constexpr int kRows = 1;

// (A c)_i (or (A w)_i with WONLY) for the rows ii[q] with on[q], in one loop
// over the block ranks; the result is zero where !on[q].
template <typename R, typename V, bool WONLY, int RW>
__device__ __forceinline__ void bsr_rows(const StepArgs& a, const Dir<V>& buf, const int64_t (&ii)[RW],
                                         const bool (&on)[RW], V beta, V (&ox)[RW], V (&oy)[RW], V (&oz)[RW]) {
  const R4<R>* b4 = static_cast<const R4<R>*>(a.bmat);
  const R* b1 = static_cast<const R*>(a.bmat) + 8 * a.bplane;
  const int64_t P = a.bplane;
  uint32_t cnt[RW];
  uint32_t cmax = 0;
#pragma unroll
  for (int q = 0; q < RW; ++q) {
    cnt[q] = on[q] ? __ldg(&a.row_cnt[ii[q]]) : 0u;
    cmax = cnt[q] > cmax ? cnt[q] : cmax;
    ox[q] = oy[q] = oz[q] = V(0);
  }
#pragma unroll 2
  for (uint32_t k = 0; k < cmax; ++k) {
#pragma unroll
    for (int q = 0; q < RW; ++q) {
      if (k < cnt[q]) {
        const int64_t sid = int64_t(k) * a.np + ii[q];
        const uint32_t j = __ldg(&a.col[sid]);
        const R4<V> pj = WONLY ? buf.w[j] : next_dir<V>(buf, j, beta);
        R4<R> u, v;
        R w;
        if constexpr (sizeof(R) == 4) {
          u = ldg_r4(&b4[sid]), v = ldg_r4(&b4[P + sid]);
          w = __ldg(&b1[sid]);
        } else {
          u = b4[sid], v = b4[P + sid];
          w = b1[sid];
        }
        ox[q] += V(u.x) * pj.x + V(u.y) * pj.y + V(u.z) * pj.z;
        oy[q] += V(u.w) * pj.x + V(v.x) * pj.y + V(v.y) * pj.z;
        oz[q] += V(v.z) * pj.x + V(v.w) * pj.y + V(w) * pj.z;
      }
    }
  }
}

// x -= n (n.x): the contact filter S with the normal given by value
template <typename V>
__device__ __forceinline__ void filt3(const V (&n)[3], V& x, V& y, V& z) {
  const V d = x * n[0] + y * n[1] + z * n[2];
  x -= n[0] * d;
  y -= n[1] * d;
  z -= n[2] * d;
}

// ------------------------------------------------------------ PCG
// implizit.rs:370-426 with the assembled A, two grid syncs per iteration:
//   points: c = w + beta c (neighbours' from one (c, w) buffer, own written to
//           the other), ap = S A c, c.ap                            -> sum
//   points: dv += alpha c, r -= alpha ap, z = P r, w = S z, r.z       -> sum
// The mixed form (FP32 vectors) takes its residuals (start, reliable
// updates) from the FP64 operator. With the FP32 operator the block part of
// A c follows A c = A w + beta A c_prev: the row product gathers w alone (half
// the bytes of c and w), and ap keeps S A c_prev between iterations. The FP64
// form applies A to c directly, as the reference does. Returns false on a
// barrier error.
template <typename R, typename V, bool SC>
__device__ bool pcg(const StepArgs& a, const Vec<R, V>& vw, Shared& sh, int64_t& iters, bool& unconverged,
                    bool& breakdown, double& rest) {
  constexpr bool kLow = sizeof(V) == 4;  // FP32 vectors: the recursion needs reliable updates
  constexpr bool kRec = sizeof(R) == 4;  // A c from A w and the previous A c
  Dir<V> cur(a.c, a.n);
  Dir<V> nxt(a.cw2, a.n);
  const bool hi = kLow && a.m_f1w64 != nullptr;
  // start: pinned points 0, held points get their normal target
  GRP_FOR(i, sh.g.r0, sh.g.r1) {
    D3 d = ld3(a.dv, uint32_t(i));
    if (!a.frei[i]) {
      d = d3(0, 0, 0);
    } else {
      const D3 n = ld3(a.nrm_d, uint32_t(i));
      if (n.x != 0.0 || n.y != 0.0 || n.z != 0.0) {
        const double soll = a.adjoint ? 0.0 : a.vn_soll[i] - dot(ld3(a.v, uint32_t(i)), n);
        d = (d - n * dot(d, n)) + n * soll;
      }
    }
    st3(a.dv, uint32_t(i), d);
    cur.w[i] = {V(d.x), V(d.y), V(d.z), V(0)};
    cur.c[i] = {V(0), V(0), V(0), V(0)};
  }
  if (!barrier(a, sh)) return false;
  if (hi) {
    apply_dv64(a, sh);
    if (!barrier(a, sh)) return false;
  }
  double red[2] = {0.0, 0.0};
  GRP_FOR(i, sh.g.r0, sh.g.r1) {
    V rx = 0, ry = 0, rz = 0, zx = 0, zy = 0, zz = 0, cx = 0, cy = 0, cz = 0;
    if (a.frei[i]) {
      const D3 b = ld3(a.b, uint32_t(i));
      D3 ad;
      if (hi) {
        ad = a_dv64<SC>(a, i);
      } else {
        V hx, hy, hz;
        bsr_row<R, V, SC, true>(a, cur, i, V(0), hx, hy, hz);
        ad = d3(double(hx), double(hy), double(hz));
      }
      const D3 n = ld3(a.nrm_d, uint32_t(i));
      D3 rd = b - ad;
      rd = rd - n * dot(rd, n);
      rx = V(rd.x);
      ry = V(rd.y);
      rz = V(rd.z);
      V fx = V(b.x), fy = V(b.y), fz = V(b.z);
      filt<V>(vw.nrm, i, fx, fy, fz);
      V px, py, pz;
      pmulv<R, V>(vw.pinv, i, fx, fy, fz, px, py, pz);
      red[1] += double(fx) * double(px) + double(fy) * double(py) + double(fz) * double(pz);
      pmulv<R, V>(vw.pinv, i, rx, ry, rz, zx, zy, zz);
      cx = zx;
      cy = zy;
      cz = zz;
      filt<V>(vw.nrm, i, cx, cy, cz);
      red[0] += double(rx) * double(cx) + double(ry) * double(cy) + double(rz) * double(cz);
    }
    vw.r[3 * i] = rx;
    vw.r[3 * i + 1] = ry;
    vw.r[3 * i + 2] = rz;
    nxt.w[i] = {cx, cy, cz, V(0)};  // the first direction: w + 0 c
    nxt.c[i] = {V(0), V(0), V(0), V(0)};
  }
  if (!grid_sync<2>(a, sh, red)) return false;
  {
    const Dir<V> t = cur;
    cur = nxt;
    nxt = t;
  }
  double delta = red[0];
  const double bb = red[1];
  const double tol = kLow ? fmax(a.tol, kMixedTolFloor) : a.tol;
  const double ziel = fmax(tol * tol * fmax(bb, delta), sh.g.boden);
  int64_t it = 0;
  double beta = 0.0, delta_ref = delta;
  breakdown = false;
  while (delta > ziel && it < a.cg_max) {
    const V rb = V(beta);
    // ca = c.Ac and, for FP32 vectors, cm = c.M(1+hc)c: the Hessian part is
    // positive semi-definite, so c.Ac >= cm holds exactly; an FP32 product
    // that falls far below it has lost the direction and the solve stops
    // there as at a breakdown (the other forms keep the reference's test only).
    double ca[2] = {0.0, 0.0};
    const int64_t gstride = int64_t(sh.g.nblk) * blockDim.x;
    for (int64_t i0 = sh.g.r0 + int64_t(sh.bidx) * blockDim.x + threadIdx.x; i0 < sh.g.r1; i0 += kRows * gstride) {
      int64_t ii[kRows];
      bool on[kRows], fr[kRows];
      R4<V> ci[kRows];
      V nr[kRows][3], pp[kRows][3], md[kRows];
#pragma unroll
      for (int q = 0; q < kRows; ++q) {
        ii[q] = i0 + q * gstride;
        on[q] = ii[q] < sh.g.r1;
        const int64_t i = on[q] ? ii[q] : i0;
        ci[q] = next_dir<V>(cur, i, rb);
        fr[q] = on[q] && a.frei[i];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          nr[q][c] = vw.nrm[3 * i + c];
          pp[q][c] = kRec ? vw.ap[3 * i + c] : V(0);
        }
        md[q] = kLow ? V(vw.md[i]) : V(0);
      }
      V ax[kRows], ay[kRows], az[kRows];
      bsr_rows<R, V, kRec, kRows>(a, cur, ii, fr, rb, ax, ay, az);
#pragma unroll
      for (int q = 0; q < kRows; ++q) {
        if (!on[q]) continue;
        const int64_t i = ii[q];
        nxt.c[i] = ci[q];
        if (fr[q]) {
          filt3<V>(nr[q], ax[q], ay[q], az[q]);
          if (kRec && beta != 0.0) {  // + beta S A c_prev (the first direction has none)
            ax[q] = fmar(rb, pp[q][0], ax[q]);
            ay[q] = fmar(rb, pp[q][1], ay[q]);
            az[q] = fmar(rb, pp[q][2], az[q]);
          }
          if (kLow)
            ca[1] += double(md[q]) * (double(ci[q].x) * double(ci[q].x) + double(ci[q].y) * double(ci[q].y) +
                                      double(ci[q].z) * double(ci[q].z));
        }
        vw.ap[3 * i] = ax[q];
        vw.ap[3 * i + 1] = ay[q];
        vw.ap[3 * i + 2] = az[q];
        ca[0] += double(ci[q].x) * double(ax[q]) + double(ci[q].y) * double(ay[q]) + double(ci[q].z) * double(az[q]);
      }
    }
    if (SC) {
      // proximity springs pair by pair (implizit.rs:214-220): each nonzero
      // slot's product goes to its entry; the update phase sums a point's
      // entries in list order. c is filtered (pinned points hold 0), so the
      // slot's share of c.A c is c_k.t_k.
      const R4<R>* bR = static_cast<const R4<R>*>(a.sc_bR);
      const R4<R>* wR = static_cast<const R4<R>*>(a.sc_wR);
      const R* g5R = static_cast<const R*>(a.sc_g5R);
      R4<V>* out = static_cast<R4<V>*>(a.sc_out);
      // spring q on thread nth - 1 - q: the springs go to the threads with the
      // fewest rows first (the rows fill the threads from the grid's start)
      const int64_t nth = int64_t(sh.g.nblk) * blockDim.x;
      for (int64_t q = nth - 1 - (int64_t(sh.bidx) * blockDim.x + threadIdx.x); q < int64_t(a.sc_np); q += nth) {
        const uint4 id = a.sc_idx[q];
        const R4<R> w4 = wR[q];
        const V g[5] = {V(w4.x), V(w4.y), V(w4.z), V(w4.w), V(g5R[q])};
        const uint32_t x5 = a.sc_x5[q];
        const uint32_t ix[5] = {id.x, id.y, id.z, id.w, x5};
        R4<V> c[5];
#pragma unroll
        for (int r = 0; r < 4; ++r) c[r] = next_dir<V>(cur, ix[r], rb);
        c[4] = x5 != 0xffffffffu ? next_dir<V>(cur, x5, rb) : R4<V>{V(0), V(0), V(0), V(0)};
        const R4<R> b0 = bR[2 * q], b1 = bR[2 * q + 1];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
          const uint32_t e = a.sc_pos[8 * q + k];
          if (e == 0xffffffffu) continue;
          V sx = 0, sy = 0, sz = 0;
#pragma unroll
          for (int r = 0; r < 5; ++r)
            if ((g[k] > V(0) && g[r] < V(0)) || (g[k] < V(0) && g[r] > V(0))) {
              const V om = -g[k] * g[r];
              sx += om * (c[k].x - c[r].x);
              sy += om * (c[k].y - c[r].y);
              sz += om * (c[k].z - c[r].z);
            }
          const V tx = V(b0.x) * sx + V(b0.w) * sy + V(b1.x) * sz;
          const V ty = V(b0.w) * sx + V(b0.y) * sy + V(b1.y) * sz;
          const V tz = V(b1.x) * sx + V(b1.y) * sy + V(b0.z) * sz;
          out[e] = {tx, ty, tz, V(0)};
          ca[0] += double(c[k].x) * double(tx) + double(c[k].y) * double(ty) + double(c[k].z) * double(tz);
        }
      }
    }
    if (kLow) {
      if (!grid_sync<2>(a, sh, ca)) return false;
    } else {
      double c1[1] = {ca[0]};
      if (!grid_sync<1>(a, sh, c1)) return false;
      ca[0] = c1[0];
    }
    if (ca[0] <= DBL_MIN || !isfinite(ca[0]) || (kLow && ca[0] < 0.5 * ca[1])) {
      breakdown = true;
      break;
    }
    const double alpha = delta / ca[0];
    double rzs[1] = {0.0};
    for (int64_t i0 = sh.g.r0 + int64_t(sh.bidx) * blockDim.x + threadIdx.x; i0 < sh.g.r1; i0 += kRows * gstride) {
      int64_t ii[kRows];
      bool on[kRows], fr[kRows];
      R4<V> ci[kRows];
      D3 d[kRows];
      V ap[kRows][3], r[kRows][3], nr[kRows][3], pv[kRows][6];
      uint32_t se[kRows][2];  // the point's proximity-spring entries (SC)
#pragma unroll
      for (int q = 0; q < kRows; ++q) {  // every load first
        ii[q] = i0 + q * gstride;
        on[q] = ii[q] < sh.g.r1;
        const int64_t i = on[q] ? ii[q] : i0;
        ci[q] = nxt.c[i];
        d[q] = ld3(a.dv, uint32_t(i));
        fr[q] = a.frei[i];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          ap[q][c] = vw.ap[3 * i + c];
          r[q][c] = vw.r[3 * i + c];
          nr[q][c] = vw.nrm[3 * i + c];
        }
#pragma unroll
        for (int c = 0; c < 6; ++c) pv[q][c] = V(vw.pinv[6 * i + c]);
        se[q][0] = SC ? a.sc_off[i] : 0u;
        se[q][1] = SC ? a.sc_off[i + 1] : 0u;
      }
#pragma unroll
      for (int q = 0; q < kRows; ++q) {
        if (!on[q]) continue;
        const int64_t i = ii[q];
        st3(a.dv, uint32_t(i), d[q] + d3(double(ci[q].x), double(ci[q].y), double(ci[q].z)) * alpha);
        V apx = ap[q][0], apy = ap[q][1], apz = ap[q][2];
        if (SC && fr[q]) {  // the point's proximity-spring entries, in list order
          const R4<V>* out = static_cast<const R4<V>*>(a.sc_out);
          V sx = 0, sy = 0, sz = 0;
          for (uint32_t e = se[q][0]; e < se[q][1]; ++e) {
            const R4<V> t = out[e];
            sx += t.x;
            sy += t.y;
            sz += t.z;
          }
          filt3<V>(nr[q], sx, sy, sz);
          apx += sx;
          apy += sy;
          apz += sz;
        }
        const V rx = V(double(r[q][0]) - alpha * double(apx));
        const V ry = V(double(r[q][1]) - alpha * double(apy));
        const V rzz = V(double(r[q][2]) - alpha * double(apz));
        vw.r[3 * i] = rx;
        vw.r[3 * i + 1] = ry;
        vw.r[3 * i + 2] = rzz;
        const V* P = pv[q];
        V zx = P[0] * rx + P[3] * ry + P[4] * rzz;
        V zy = P[3] * rx + P[1] * ry + P[5] * rzz;
        V zz = P[4] * rx + P[5] * ry + P[2] * rzz;
        if (!fr[q]) zx = zy = zz = 0;
        V wx = zx, wy = zy, wz = zz;
        filt3<V>(nr[q], wx, wy, wz);
        nxt.w[i] = {wx, wy, wz, V(0)};
        rzs[0] += double(rx) * double(zx) + double(ry) * double(zy) + double(rzz) * double(zz);
      }
    }
    if (!grid_sync<1>(a, sh, rzs)) return false;
    double beta_next = rzs[0] / delta;
    const double delta_prev = delta;
    delta = rzs[0];
    if (hi && (delta < kReliable * delta_ref || delta > kGrow * delta_ref)) {
      // reliable update: replace the recursive FP32 residual by the true one,
      // S (b - A dv) with the FP64 operator; restart the direction if the
      // residual grew
      const bool restart = delta > kGrow * delta_ref;
      apply_dv64(a, sh);
      if (!barrier(a, sh)) return false;
      double rz2[1] = {0.0};
      GRP_FOR(i, sh.g.r0, sh.g.r1) {
        V rx = 0, ry = 0, rz = 0, zx = 0, zy = 0, zz = 0, wx = 0, wy = 0, wz = 0;
        if (a.frei[i]) {
          const D3 n = ld3(a.nrm_d, uint32_t(i));
          D3 rd = ld3(a.b, uint32_t(i)) - a_dv64<SC>(a, i);
          rd = rd - n * dot(rd, n);
          rx = V(rd.x);
          ry = V(rd.y);
          rz = V(rd.z);
          pmulv<R, V>(vw.pinv, i, rx, ry, rz, zx, zy, zz);
          wx = zx;
          wy = zy;
          wz = zz;
          filt<V>(vw.nrm, i, wx, wy, wz);
          rz2[0] += double(rx) * double(zx) + double(ry) * double(zy) + double(rz) * double(zz);
        }
        vw.r[3 * i] = rx;
        vw.r[3 * i + 1] = ry;
        vw.r[3 * i + 2] = rz;
        nxt.w[i] = {wx, wy, wz, V(0)};
      }
      if (!grid_sync<1>(a, sh, rz2)) return false;
      delta = rz2[0];
      beta_next = restart ? 0.0 : delta / delta_prev;
      delta_ref = delta;
    }
    beta = beta_next;
    {
      const Dir<V> t = cur;
      cur = nxt;
      nxt = t;
    }
    ++it;
  }
  iters = it;
  unconverged = delta > ziel;
  rest = sqrt(delta / fmax(bb, sh.g.boden));
  return true;
}

// ------------------------------------------------------------ release pass
// implizit.rs:924-942: normal force from the residual A dv - b along the
// contact normal; a held point that pulls on the body is released.
template <typename R, typename V, bool SC>
__device__ bool release(const StepArgs& a, const Vec<R, V>& vw, Shared& sh, double& released, bool last) {
  const bool hi = sizeof(V) == 4 && a.m_f1w64 != nullptr;
  if (hi)
    apply_dv64(a, sh);
  else
    dv_to_w<V>(a, vw.cw, sh);
  if (!barrier(a, sh)) return false;
  double cnt[1] = {0.0};
  GRP_FOR(i, sh.g.r0, sh.g.r1) {
    const D3 n = ld3(a.nrm_d, uint32_t(i));
    if (n.x == 0.0 && n.y == 0.0 && n.z == 0.0) continue;
    const D3 b = ld3(a.b, uint32_t(i));
    D3 rest;
    if (hi) {
      rest = a_dv64<SC>(a, i) - b;
    } else {
      V hx, hy, hz;
      bsr_row<R, V, SC, true>(a, vw.cw, i, V(0), hx, hy, hz);
      rest = d3(double(hx), double(hy), double(hz)) - b;
    }
    const double fn = dot(rest, n) / a.h;
    if (fn < 0.0) {
      st3(a.nrm_d, uint32_t(i), d3(0, 0, 0));
      vw.nrm_r[3 * i] = vw.nrm_r[3 * i + 1] = vw.nrm_r[3 * i + 2] = R(0);
      cnt[0] += 1.0;
      // released after the last solve: held in dv's constraint, free in friction
      if (last && a.rec_flags) a.rec_flags[i] |= 8u;
    } else {
      a.fnk[i] = fn;
    }
  }
  if (!grid_sync<1>(a, sh, cnt)) return false;
  released = cnt[0];
  return true;
}


template <typename R, typename V, bool SC, int NT>
__global__ void __launch_bounds__(NT, NT <= 256 ? 2 : 1) solve_kernel(const __grid_constant__ StepArgs a) {
  __shared__ Shared sh;
  if (threadIdx.x == 0) {
    sh.epoch = 0;
    sh.rbuf = 0;
    sh.err = 0;
    sh.g = a.grp[a.blk_grp[blockIdx.x]];
    sh.bidx = blockIdx.x - sh.g.first_blk;
  }
  __syncthreads();
  const Vec<R, V> vw(a);
  const bool lead = sh.bidx == 0 && threadIdx.x == 0;  // one thread per group
  const bool any_held = a.stats[ST_HELD] > 0;
  int64_t iters = 0;
  bool unconv = false, brk = false;
  double rest = 0.0;
  for (int pass = 0; pass < 2; ++pass) {
    if (!pcg<R, V, SC>(a, vw, sh, iters, unconv, brk, rest)) return;
    double dvm[1] = {0.0};
    GRP_FOR(i, sh.g.r0, sh.g.r1) {
      const D3 d = ld3(a.dv, uint32_t(i));
      dvm[0] = fmax(dvm[0], fmax(fabs(d.x), fmax(fabs(d.y), fabs(d.z))));
    }
    // |dv| maximum and the counters go to the statistics by atomics (the
    // groups of a batch finish at different times)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dvm[0] = fmax(dvm[0], __shfl_xor_sync(0xffffffffu, dvm[0], o));
    if ((threadIdx.x & 31) == 0 && dvm[0] > 0.0)
      atomicMax(reinterpret_cast<unsigned long long*>(&a.stat_rest_max[1]),
                (unsigned long long)__double_as_longlong(dvm[0]));
    if (lead) {
      atomicAdd(reinterpret_cast<unsigned long long*>(&a.stats[ST_CG_ITERATIONS]), (unsigned long long)iters);
      atomicAdd(reinterpret_cast<unsigned long long*>(&a.stats[ST_SOLVES]), 1ull);
      if (unconv) atomicAdd(reinterpret_cast<unsigned long long*>(&a.stats[ST_UNCONVERGED]), 1ull);
      if (brk) atomicAdd(reinterpret_cast<unsigned long long*>(&a.stats[ST_BREAKDOWNS]), 1ull);
      if (rest > 0.0)
        atomicMax(reinterpret_cast<unsigned long long*>(&a.stat_rest_max[0]),
                  (unsigned long long)__double_as_longlong(rest));
      if (sh.g.first_blk == 0) a.stats[ST_LAST_ITERATIONS] = iters;
    }
    if (a.mode == MODE_SOLVE) return;
    if (!any_held) break;
    double rel = 0.0;
    if (!release<R, V, SC>(a, vw, sh, rel, pass == 1)) return;
    if (lead && rel > 0.0)
      atomicAdd(reinterpret_cast<unsigned long long*>(&a.stats[ST_RELEASED]), (unsigned long long)rel);
    if (rel == 0.0) break;
  }
}

}  // namespace k3d
