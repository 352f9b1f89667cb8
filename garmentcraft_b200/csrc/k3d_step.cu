// The implicit backward-Euler step on the device: one persistent cooperative
// kernel per substep.
//
//   build (elements)  -> per-corner force/Hv/diag records, operator records
//   build (points)    -> rhs b, block-Jacobi inverse, contact set
//   PCG (implizit.rs:370-426), up to two passes with the release test
//   (implizit.rs:908-943), then friction and integration (:957-1014).
//
// Every phase is a grid-stride loop over elements or points, separated by a
// grid barrier. Sums are deterministic: points gather their incident element
// corners in a fixed order (no float atomics), and grid reductions add the
// per-block partials in block order. The barrier waits are bounded by a
// wall-clock limit; on expiry the kernel records K3D_TIMEOUT and every block
// returns.
#include <cfloat>
#include <cstdint>

#include "k3d_solve.cuh"

namespace k3d {

// the FP32-vector form's kernels (k3d_step_f32.cu)
const void* solve_fn_f32(bool sc, int threads);

// ------------------------------------------------------------ launch
// Precision forms: 0 FP64 (R = V = double), 1 mixed (R = V = float),
// 2 FP32 storage (R = float blocks and preconditioner, V = double vectors);
// CTA sizes 256 (two CTAs per SM), 512 and 1024 (one per SM).
template <typename R, typename V>
static const void* solve_fn_t(bool sc, int threads) {
  if (threads == 256) return sc ? (const void*)solve_kernel<R, V, true, 256> : (const void*)solve_kernel<R, V, false, 256>;
  if (threads == 1024)
    return sc ? (const void*)solve_kernel<R, V, true, 1024> : (const void*)solve_kernel<R, V, false, 1024>;
  return sc ? (const void*)solve_kernel<R, V, true, 512> : (const void*)solve_kernel<R, V, false, 512>;
}
static const void* solve_fn(int precision, bool sc, int threads) {
  return precision == 0   ? solve_fn_t<double, double>(sc, threads)
         : precision == 1 ? solve_fn_f32(sc, threads)
                          : solve_fn_t<float, double>(sc, threads);
}
template <typename R, typename V>
static const void* solve_fn_rv(bool sc, int threads) {
  if constexpr (sizeof(V) == 4)
    return solve_fn_f32(sc, threads);
  else
    return solve_fn_t<R, V>(sc, threads);
}

static int g_sms = 0;

int step_grid_blocks(int precision, int threads, int device) {
  const int idx = precision < 0 || precision > 2 ? 0 : precision;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return -1;
  g_sms = prop.multiProcessorCount;
  int per_sm = 0;
  // the launch with self-collision springs must fit as well: the smaller count of both
  int per_sm_sc = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, solve_fn(idx, false, threads), threads, 0) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_sc, solve_fn(idx, true, threads), threads, 0) !=
          cudaSuccess)
    return -1;
  per_sm = per_sm_sc < per_sm ? per_sm_sc : per_sm;
  if (per_sm < 1) return -1;
  return prop.multiProcessorCount * per_sm;
}

static cudaError_t plain(const void* fn, const StepArgs& a, int64_t work, cudaStream_t st) {
  int64_t blocks = (work + kBlock - 1) / kBlock;
  const int64_t cap = int64_t(g_sms > 0 ? g_sms : 148) * 16;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  void* args[] = {(void*)&a};
  return cudaLaunchKernel(fn, dim3(unsigned(blocks)), dim3(kBlock), args, 0, st);
}

// The persistent launch: cooperative (every block resident at once), also
// inside a stream capture, where it becomes a cooperative kernel node. The
// groups' barrier counters start at zero in each launch.
static cudaError_t cooperative(const void* fn, const StepArgs& a, int blocks, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(a.grp_cnt, 0, sizeof(unsigned) * 32 * size_t(a.n_grp), st);
  if (e != cudaSuccess) return e;
  void* args[] = {(void*)&a};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(blocks));
  cfg.blockDim = dim3(unsigned(a.solve_threads > 0 ? a.solve_threads : kSolveBlock));
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, fn, args);
}

// The caller's contact set in place of the one the build found (held points
// get the given normal and normal velocity, the others none).
template <typename R>
__global__ void __launch_bounds__(kBlock) contacts_kernel(const __grid_constant__ StepArgs a) {
  R* nrm = static_cast<R*>(a.nrm);
  K3D_FOR(i, a.n) {
    const bool on = a.fest_in[i] != 0;
    const D3 n = on ? ld3(a.fest_n, uint32_t(i)) : d3(0, 0, 0);
    st3(a.nrm_d, uint32_t(i), n);
    nrm[3 * i] = R(n.x);
    nrm[3 * i + 1] = R(n.y);
    nrm[3 * i + 2] = R(n.z);
    a.vn_soll[i] = on ? a.fest_soll[i] : 0.0;
  }
}

template <typename R, typename V>
static cudaError_t launch_t(const StepArgs& a, int blocks, cudaStream_t st, int& launched) {
  cudaError_t e;
  const BuildKernels K = build_kernels(sizeof(R) == 8 ? 0 : 1);
  const int64_t elems = a.nt > a.nb ? (a.nt > a.ns ? a.nt : a.ns) : (a.nb > a.ns ? a.nb : a.ns);
  if ((e = cudaMemsetAsync(&a.stats[ST_HELD], 0, sizeof(long long), st)) != cudaSuccess) return e;
  if ((e = plain(K.elements, a, elems, st)) != cudaSuccess) return e;
  if ((e = plain(K.points, a, a.n, st)) != cudaSuccess) return e;
  launched = 2;
  if (a.fest_in) {
    if ((e = plain((const void*)contacts_kernel<R>, a, a.n, st)) != cudaSuccess) return e;
    launched += 1;
  }
  if (a.mode == MODE_SYSTEM && !a.p_out) return cudaSuccess;
  if (a.mode == MODE_OPERATOR || a.mode == MODE_RESIDUAL || a.mode == MODE_SYSTEM) {
    if ((e = plain(K.probe_load, a, a.n, st)) != cudaSuccess) return e;
    if ((e = plain(K.probe_apply, a, elems, st)) != cudaSuccess) return e;
    if ((e = plain(K.probe_out, a, a.n, st)) != cudaSuccess) return e;
    launched += 3;
    return cudaSuccess;
  }
  if (a.ev_solve0 && (e = cudaEventRecord(a.ev_solve0, st)) != cudaSuccess) return e;
  if ((e = plain(K.assemble, a, a.bplane, st)) != cudaSuccess) return e;
  launched += 1;
  if ((e = cooperative(solve_fn_rv<R, V>(a.sc_off != nullptr, a.solve_threads), a, blocks, st)) != cudaSuccess)
    return e;
  if (a.ev_solve1 && (e = cudaEventRecord(a.ev_solve1, st)) != cudaSuccess) return e;
  launched += 1;
  if (a.mode == MODE_STEP) {
    if ((e = plain(K.integrate, a, a.n, st)) != cudaSuccess) return e;
    launched += 1;
    if ((e = launch_koerperpunkte(a, st, launched)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_pcg64(const StepArgs& a, int blocks, cudaStream_t stream) {
  StepArgs s = a;
  s.mode = MODE_SOLVE;
  return cooperative(solve_fn_t<double, double>(false, s.solve_threads), s, blocks, stream);
}

cudaError_t launch_step(const StepArgs& a, int precision, int blocks, cudaStream_t stream, int& launched) {
  launched = 0;
  switch (precision) {
    case 0: return launch_t<double, double>(a, blocks, stream, launched);
    case 1: return launch_t<float, float>(a, blocks, stream, launched);
    default: return launch_t<float, double>(a, blocks, stream, launched);
  }
}

}  // namespace k3d
