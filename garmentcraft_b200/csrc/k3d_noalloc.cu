// k3d_operator_noalloc: A·p for callers that cannot allocate device memory.
//
// Same result as k3d_operator (A p = M(1+hc) p + h^2 H p at the scene's
// positions, implizit.rs:185-229), but nothing is allocated: every input and
// output is a device pointer the caller owns, and the only scratch is the
// file-scope array below, which lives in the library's module on every GPU
// that loads it, until the process exits.
//
// The per-point sums of the element corner products go through 64-bit
// fixed-point accumulators with integer atomics: the total does not depend on
// the order the corners arrive in, so the result is deterministic without the
// per-point corner lists a handle builds at upload (those would need memory).
// Pass 0 finds the largest corner product component M and counts each
// point's corners (in the accumulators, zero then); a middle pass takes the
// largest count K and clears the accumulators; pass 1 adds every component
// scaled by 2^(62 - ceil(log2 K) - exponent(M)) (exact power-of-two scaling),
// so a point's sum of at most K terms below 2^(62 - ceil(log2 K)) each cannot
// overflow, and the resolution is M * 2^-(62 - ceil(log2 K)).
//
// The element products round as the handle's build kernels do (this file is
// compiled without fused multiply-add, like k3d_build.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/klon3d_step.h"
#include "k3d_device.cuh"

namespace k3d {
namespace noalloc {

constexpr int64_t kMaxPoints = 131072;
constexpr int kMaxDevices = 64;
constexpr int kBlock = 256;
// [0, 3 kMaxPoints): accumulators; [3 kMaxPoints]: bits of max |product|;
// [3 kMaxPoints + 1]: set to 1 when an element names a point out of range;
// [3 kMaxPoints + 2]: set to 1 when a product or an input is not finite;
// [3 kMaxPoints + 3]: the largest number of corners at one point.
static __device__ __align__(256) unsigned long long g_scratch[3 * kMaxPoints + 32];
constexpr int64_t kMaxSlot = 3 * kMaxPoints;
constexpr int64_t kErrSlot = 3 * kMaxPoints + 1;
constexpr int64_t kNanSlot = 3 * kMaxPoints + 2;
constexpr int64_t kCntSlot = 3 * kMaxPoints + 3;

struct Args {
  int64_t n, ne, nn, nb, nt;
  const double *x, *masse;
  const uint32_t* a_p;
  const double *a_ruhe, *a_alpha;
  const uint8_t* mkante;
  const uint32_t* n_p;
  const double* n_ruhe;
  const uint32_t* b_p;
  const double* b_alpha;
  const uint32_t* m_p;
  const double *m_fl, *m_ri, *m_k, *m_s, *m_st;
  const double* p;
  double* out;
  double h, c, naht_k;
  unsigned long long* scratch;
};

__device__ __forceinline__ D3 ldp(const double* p, uint32_t i) { return ld3(p, i); }

// 2^ex scales the largest component M below 2^(62 - ceil(log2 K)), K the
// largest corner count at one point.
__device__ __forceinline__ int scale_exp(const unsigned long long* scratch) {
  const double m = __longlong_as_double((long long)scratch[kMaxSlot]);
  if (!(m > 0.0)) return 0;
  int ex = 0;
  frexp(m, &ex);  // m < 2^ex
  int lk = 0;
  while ((1ull << lk) < scratch[kCntSlot] && lk < 62) ++lk;
  return 62 - lk - ex;
}

// pass 0: record max |component|, count the point's corners, flag a
// non-finite component; pass 1: add the fixed-point component.
__device__ __forceinline__ void emit(const Args& a, int pass, int ex, uint32_t i, double vx, double vy, double vz) {
  if (pass == 0) {
    if (!isfinite(vx) || !isfinite(vy) || !isfinite(vz)) {
      a.scratch[kNanSlot] = 1ull;
      return;
    }
    const double m = fmax(fabs(vx), fmax(fabs(vy), fabs(vz)));
    if (m > 0.0) atomicMax(&a.scratch[kMaxSlot], (unsigned long long)__double_as_longlong(m));
    atomicAdd(&a.scratch[3 * size_t(i)], 1ull);
    return;
  }
  if (a.scratch[kNanSlot] != 0ull) return;
  atomicAdd(&a.scratch[3 * size_t(i)], (unsigned long long)llrint(ldexp(vx, ex)));
  atomicAdd(&a.scratch[3 * size_t(i) + 1], (unsigned long long)llrint(ldexp(vy, ex)));
  atomicAdd(&a.scratch[3 * size_t(i) + 2], (unsigned long long)llrint(ldexp(vz, ex)));
}

__device__ __forceinline__ bool in_range(const Args& a, const uint32_t* q, int k) {
  for (int j = 0; j < k; ++j)
    if (int64_t(q[j]) >= a.n) {
      a.scratch[kErrSlot] = 1ull;
      return false;
    }
  return true;
}

__global__ void zero_kernel(Args a) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < 3 * a.n; i += int64_t(gridDim.x) * blockDim.x)
    a.scratch[i] = 0ull;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.scratch[kMaxSlot] = 0ull;
    a.scratch[kErrSlot] = 0ull;
    a.scratch[kNanSlot] = 0ull;
    a.scratch[kCntSlot] = 0ull;
  }
}

// Between the passes: the largest corner count, and the accumulators back to
// zero. A non-finite p or mass is flagged here (a non-finite position makes
// its element products non-finite, flagged in pass 0).
__global__ void middle_kernel(Args a) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < a.n; i += int64_t(gridDim.x) * blockDim.x) {
    atomicMax(&a.scratch[kCntSlot], a.scratch[3 * i]);
    a.scratch[3 * i] = 0ull;
    a.scratch[3 * i + 1] = 0ull;
    a.scratch[3 * i + 2] = 0ull;
    const D3 pi = ld3(a.p, uint32_t(i));
    if (!isfinite(pi.x) || !isfinite(pi.y) || !isfinite(pi.z) || !isfinite(a.masse[i])) a.scratch[kNanSlot] = 1ull;
  }
}

// Element corner products H_e p at the positions x, in FP64: membranes
// (kontinuum.rs:584-664), bending hinges (cpu.rs:288-307, implizit.rs:199-205),
// pattern edges with their own stiffness and seams (implizit.rs:189-198,
// 742-771).
__global__ void elements_kernel(Args a, int pass) {
  const int ex = pass == 1 ? scale_exp(a.scratch) : 0;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  const int64_t t0 = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  for (int64_t t = t0; t < a.nt; t += stride) {
    const uint32_t* q = a.m_p + 3 * t;
    if (!in_range(a, q, 3)) continue;
    MembranC m;
    for (int k = 0; k < 4; ++k) m.r[k] = a.m_ri[4 * t + k];
    m.kx = a.m_k[2 * t];
    m.ky = a.m_k[2 * t + 1];
    m.sx = a.m_s[2 * t];
    m.sy = a.m_s[2 * t + 1];
    m.fl = a.m_fl[t];
    m.ek = a.m_st[3 * t];
    m.es = a.m_st[3 * t + 1];
    m.g = a.m_st[3 * t + 2];
    const D3 p0 = ld3(a.x, q[0]), e1 = ld3(a.x, q[1]) - p0, e2 = ld3(a.x, q[2]) - p0;
    const D3 f1 = e1 * m.r[0] + e2 * m.r[2], f2 = e1 * m.r[1] + e2 * m.r[3];
    D3 ba, bb, bc;
    basis3(m, ba, bb, bc);
    const D3 g = d3(dot(f1, f1), dot(f2, f2), 2.0 * dot(f1, f2));
    const D3 e = d3(0.5 * (dot(ba, g) - 1.0), 0.5 * (dot(bb, g) - 1.0), 0.5 * dot(bc, g));
    const D3 dz = du_dg(m, ba, bb, bc, d3(fmax(e.x, 0.0), fmax(e.y, 0.0), e.z));
    const D3 w = psd2(dz.x, dz.y, dz.z);
    double kg[6];
    kg_sym(m, kg);
    const R4<double> rf1 = {f1.x, f1.y, f1.z, w.x}, rf2 = {f2.x, f2.y, f2.z, w.y};
    const R4<double> rr = {m.r[0], m.r[1], m.r[2], m.r[3]};
    const R4<double> ka = {kg[0], kg[1], kg[2], kg[3]}, kb = {kg[4], kg[5], w.z, 0.0};
    R4<double> d[3], o[3];
    for (int k = 0; k < 3; ++k) {
      const D3 v = ldp(a.p, q[k]);
      d[k] = {v.x, v.y, v.z, 0.0};
    }
    membran_hv<double>(rf1, rf2, rr, ka, kb, d, o);
    for (int k = 0; k < 3; ++k) emit(a, pass, ex, q[k], o[k].x, o[k].y, o[k].z);
  }
  for (int64_t b = t0; b < a.nb; b += stride) {
    const uint32_t* q = a.b_p + 4 * b;
    if (!in_range(a, q, 4)) continue;
    D3 gr[4];
    double theta = 0.0;
    if (!dieder(ld3(a.x, q[0]), ld3(a.x, q[1]), ld3(a.x, q[2]), ld3(a.x, q[3]), theta, gr)) continue;
    const double k = 1.0 / a.b_alpha[b];
    const D3 c0 = ldp(a.p, q[0]);
    const double gp =
        dot(gr[1], ldp(a.p, q[1]) - c0) + dot(gr[2], ldp(a.p, q[2]) - c0) + dot(gr[3], ldp(a.p, q[3]) - c0);
    const double s = k * gp;
    for (int m = 0; m < 4; ++m) emit(a, pass, ex, q[m], gr[m].x * s, gr[m].y * s, gr[m].z * s);
  }
  const int64_t ns = a.ne + a.nn;
  for (int64_t s = t0; s < ns; s += stride) {
    const bool seam = s >= a.ne;
    const int64_t e = seam ? s - a.ne : s;
    const uint32_t* q = seam ? a.n_p + 2 * e : a.a_p + 2 * e;
    if (!in_range(a, q, 2)) continue;
    double k, quer;
    D3 n;
    const D3 d = ld3(a.x, q[1]) - ld3(a.x, q[0]);
    if (!seam) {
      if (a.mkante && a.mkante[e]) continue;
      k = 1.0 / a.a_alpha[e];
      if (k == 0.0) continue;
      const double l = fmax(norm(d), 1e-12);
      n = d * (1.0 / l);
      quer = fmax(1.0 - a.a_ruhe[e] / l, 0.0);
    } else {
      k = a.naht_k;
      if (k == 0.0) continue;
      const double l = norm(d);
      const double l0 = isfinite(a.n_ruhe[e]) ? a.n_ruhe[e] : l;
      if (l0 > 0.0 && l > 1e-12) {
        n = d * (1.0 / l);
        quer = fmax(1.0 - l0 / l, 0.0);
      } else {
        n = d3(0, 0, 0);
        quer = 1.0;
      }
    }
    const D3 dp = ldp(a.p, q[0]) - ldp(a.p, q[1]);
    const D3 bd = (n * (dot(n, dp) * (1.0 - quer)) + dp * quer) * k;
    emit(a, pass, ex, q[0], bd.x, bd.y, bd.z);
    emit(a, pass, ex, q[1], -bd.x, -bd.y, -bd.z);
  }
}

__global__ void finish_kernel(Args a) {
  const int ex = scale_exp(a.scratch);
  const double h2 = a.h * a.h;
  const bool nan = a.scratch[kNanSlot] != 0ull;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < a.n; i += int64_t(gridDim.x) * blockDim.x) {
    if (nan) {  // as k3d_operator, whose sums carry the NaN through
      a.out[3 * i] = a.out[3 * i + 1] = a.out[3 * i + 2] = __longlong_as_double(0x7FF8000000000000ll);
      continue;
    }
    const double md = a.masse[i] * (1.0 + a.h * a.c);
    const D3 pi = ld3(a.p, uint32_t(i));
    double hs[3];
    for (int k = 0; k < 3; ++k) hs[k] = ldexp(double((long long)a.scratch[3 * i + k]), -ex);
    a.out[3 * i] = md * pi.x + h2 * hs[0];
    a.out[3 * i + 1] = md * pi.y + h2 * hs[1];
    a.out[3 * i + 2] = md * pi.z + h2 * hs[2];
  }
}

std::mutex g_mu;
unsigned long long* g_ptr[kMaxDevices] = {};

// The device address of g_scratch on the current device, looked up once per
// device (the array's name is only a host-side stand-in in host code).
static cudaError_t scratch_on(int dev, unsigned long long** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return e;
    g_ptr[dev] = static_cast<unsigned long long*>(p);
  }
  *out = g_ptr[dev];
  return cudaSuccess;
}

}  // namespace noalloc
}  // namespace k3d

extern "C" k3d_status k3d_operator_noalloc(const k3d_params* params, const k3d_scene* s, const double* p, double* out,
                                           void* stream) {
  using namespace k3d::noalloc;
  if (!params || !s || !p || !out) return K3D_BAD_ARGUMENT;
  // the proximity springs of self-collision belong to a handle's stage
  if (params->selbstkollision != 0) return K3D_BAD_ARGUMENT;
  if (s->n_punkte < 0 || s->n_punkte > kMaxPoints) return K3D_BAD_ARGUMENT;  // scratch holds 131072 points
  if (s->n_abstand < 0 || s->n_naht < 0 || s->n_biegung < 0 || s->n_membran < 0) return K3D_BAD_ARGUMENT;
  if (s->n_punkte > 0 && (!s->x || !s->masse)) return K3D_BAD_ARGUMENT;
  if (s->n_abstand > 0 && (!s->abstand_punkte || !s->abstand_ruhe || !s->abstand_nachgiebigkeit))
    return K3D_BAD_ARGUMENT;
  if (s->n_naht > 0 && (!s->naht_punkte || !s->naht_ruhe)) return K3D_BAD_ARGUMENT;
  if (s->n_biegung > 0 && (!s->biegung_punkte || !s->biegung_nachgiebigkeit)) return K3D_BAD_ARGUMENT;
  if (s->n_membran > 0 && (!s->membran_punkte || !s->membran_flaeche || !s->membran_ruhe_inv ||
                           !s->membran_kette || !s->membran_schuss || !s->membran_steif))
    return K3D_BAD_ARGUMENT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return K3D_DEVICE_ERROR;
  Args a;
  if (scratch_on(dev, &a.scratch) != cudaSuccess) return K3D_DEVICE_ERROR;
  a.n = s->n_punkte;
  a.ne = s->n_abstand;
  a.nn = s->n_naht;
  a.nb = s->n_biegung;
  a.nt = s->n_membran;
  a.x = s->x;
  a.masse = s->masse;
  a.a_p = s->abstand_punkte;
  a.a_ruhe = s->abstand_ruhe;
  a.a_alpha = s->abstand_nachgiebigkeit;
  a.mkante = s->membran_kante;
  a.n_p = s->naht_punkte;
  a.n_ruhe = s->naht_ruhe;
  a.b_p = s->biegung_punkte;
  a.b_alpha = s->biegung_nachgiebigkeit;
  a.m_p = s->membran_punkte;
  a.m_fl = s->membran_flaeche;
  a.m_ri = s->membran_ruhe_inv;
  a.m_k = s->membran_kette;
  a.m_s = s->membran_schuss;
  a.m_st = s->membran_steif;
  a.p = p;
  a.out = out;
  a.h = s->param.bild_dt / double(std::max(params->schritte_je_bild, 1));
  a.c = s->param.daempfung;
  a.naht_k = params->naht_k;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t work = std::max<int64_t>({a.nt, a.nb, a.ne + a.nn, 1});
  const unsigned eb = unsigned(std::min<int64_t>((work + kBlock - 1) / kBlock, 148 * 16));
  const unsigned pb = unsigned(std::min<int64_t>((3 * std::max<int64_t>(a.n, 1) + kBlock - 1) / kBlock, 148 * 16));
  // launch errors left on this thread by earlier, unrelated work are not this
  // call's: clear them before launching
  (void)cudaGetLastError();
  zero_kernel<<<pb, kBlock, 0, st>>>(a);
  elements_kernel<<<eb, kBlock, 0, st>>>(a, 0);
  middle_kernel<<<pb, kBlock, 0, st>>>(a);
  elements_kernel<<<eb, kBlock, 0, st>>>(a, 1);
  finish_kernel<<<pb, kBlock, 0, st>>>(a);
  if (cudaGetLastError() != cudaSuccess) return K3D_DEVICE_ERROR;
  if (cudaStreamSynchronize(st) != cudaSuccess) return K3D_DEVICE_ERROR;
  unsigned long long flags[2] = {0, 0};  // out of range, not finite
  if (cudaMemcpy(flags, a.scratch + kErrSlot, sizeof(flags), cudaMemcpyDeviceToHost) != cudaSuccess)
    return K3D_DEVICE_ERROR;
  if (flags[0]) return K3D_BAD_ARGUMENT;
  if (flags[1]) return K3D_NON_FINITE;
  return K3D_OK;
}
