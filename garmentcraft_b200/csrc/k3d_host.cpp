// Host side of the C ABI (include/klon3d_step.h): the solver handle, the
// device layout of a scene, and the frame loop (Rechenweg::bild,
// sim/src/implizit.rs:1042-1057) around the persistent step kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/klon3d_step.h"
#include "k3d_adjoint.h"
#include "k3d_netz.h"
#include "k3d_selbst_host.h"
#include "k3d_step.h"
#include "scene_build.h"

using namespace k3d;

namespace {

// One device allocation carved into 256-byte aligned pieces.
struct Arena {
  char* base = nullptr;
  size_t size = 0, used = 0;
  template <typename T>
  T* take(size_t count) {
    size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
    if (bytes == 0) bytes = 256;
    T* p = reinterpret_cast<T*>(base + used);
    used += bytes;
    return p;
  }
};


}  // namespace

struct k3d_solver {
  k3d_params p{};
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err, name;
  int blocks = 0;
  size_t rsize = 8;  // operator records, assembled blocks, preconditioner
  size_t vsize = 8;  // the PCG's vectors
  uint8_t* d_fest = nullptr;  // device copy of a caller's contact set
  double *d_fest_n = nullptr, *d_fest_soll = nullptr;
  bool uploaded = false, first_step = true;
  int64_t n = 0, nt = 0, nb = 0, ns = 0;
  double boden = 0.0;
  k3d_simparams sim{};
  std::vector<k3d_body> bodies;         // frame-start bodies as last given
  std::vector<void*> sdf_dev;           // device copies of SDF grids
  std::vector<const netz::Dev*> netz_dev;  // mesh bodies' tables (owned by their k3d_mesh)
  std::vector<void*> kp_mem;            // body-point pass: cloth triangles and per-triangle stabs
  std::vector<int64_t> seam_slot;       // spring index of each seam, -1 if not streamed
  std::vector<double2> s_kl_host;
  int64_t launches = 0;
  double last_ms = 0.0, solve_ms = 0.0;
  std::vector<cudaEvent_t> sev;  // one pair per substep of a frame
  // a frame's launches as a CUDA graph (k3d_params.graph) and the launch
  // arguments of each substep it was captured with
  cudaGraphExec_t gexec = nullptr;
  std::vector<StepArgs> gkey;
  int64_t glaunches = 0;
  Arena arena;
  StepArgs a{};  // device pointers and constants; per-launch fields are set before each launch
  double* d_pin = nullptr;  // probe input (3N)
  double* d_pout = nullptr; // probe output (3N)
  SelbstHost sc;            // self-collision proximity stage (when enabled)
  int n_grp = 1;            // instances (independent drapes) of the uploaded scene
  // adjoint: the last k3d_adjoint_forward's checkpoints (x, v, dv every k
  // substeps) and the bodies at the start of each of its frames; one segment
  // of substep records; the backward's vectors
  struct Adj {
    bool valid = false;
    int k = 0, sub = 1;
    int64_t steps = 0;
    double ms_fwd = 0.0;
    std::vector<uint8_t> first;                 // first_step at each checkpoint
    std::vector<std::vector<k3d_body>> bodies;  // per frame
    void *ck = nullptr, *rec = nullptr, *work = nullptr;
    size_t ck_bytes = 0, rec_bytes = 0, work_bytes = 0;
  } adj;
};

static k3d_status fail(k3d_solver* h, k3d_status st, const std::string& msg) {
  if (h) h->err = msg;
  return st;
}
static k3d_status cuda_fail(k3d_solver* h, cudaError_t e, const char* what) {
  return fail(h, K3D_DEVICE_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}
#define K3D_CUDA(h, call)                                   \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return cuda_fail((h), e_, #call); \
  } while (0)

// Block pattern of A (3x3 blocks): per point its sorted columns, ELL layout
// with block (rank k, row i) at k * np + i; per block the element
// contributions in a fixed order (membranes, then bends, then springs, each in
// element order, then by corner pair). Code: type << 30 | a << 28 | b << 26 | id.
struct Pattern {
  std::vector<uint32_t> cnt, col, ctr_off, ctr;
  size_t kmax = 0;
};

static bool build_pattern(size_t n, size_t np, const uint32_t* m_p, size_t nt, const uint32_t* b_p, size_t nb,
                          const std::vector<uint4>& s_idx, Pattern& P) {
  if (nt >= (size_t(1) << 26) || nb >= (size_t(1) << 26) || s_idx.size() >= (size_t(1) << 26)) return false;
  std::vector<std::vector<uint32_t>> cols(n);
  for (size_t i = 0; i < n; ++i) cols[i].push_back(uint32_t(i));
  auto link = [&](const uint32_t* q, int k) {
    for (int a = 0; a < k; ++a)
      for (int b = 0; b < k; ++b) cols[q[a]].push_back(q[b]);
  };
  for (size_t t = 0; t < nt; ++t) link(m_p + 3 * t, 3);
  for (size_t b = 0; b < nb; ++b) link(b_p + 4 * b, 4);
  for (const uint4& q : s_idx) {
    const uint32_t ij[2] = {q.x, q.y};
    link(ij, 2);
  }
  P.cnt.assign(n, 0);
  P.kmax = 0;
  for (size_t i = 0; i < n; ++i) {
    std::sort(cols[i].begin(), cols[i].end());
    cols[i].erase(std::unique(cols[i].begin(), cols[i].end()), cols[i].end());
    P.cnt[i] = uint32_t(cols[i].size());
    P.kmax = std::max(P.kmax, cols[i].size());
  }
  if (P.kmax * np >= (size_t(1) << 32)) return false;
  const size_t ns = P.kmax * np;
  P.col.assign(ns, 0);
  for (size_t i = 0; i < n; ++i)
    for (size_t k = 0; k < cols[i].size(); ++k) P.col[k * np + i] = cols[i][k];
  auto slot = [&](uint32_t i, uint32_t j) -> size_t {
    const auto& c = cols[i];
    return size_t(std::lower_bound(c.begin(), c.end(), j) - c.begin()) * np + i;
  };
  // count, then fill (stable: element order within a block)
  P.ctr_off.assign(ns + 1, 0);
  auto each = [&](auto&& f) {
    for (size_t t = 0; t < nt; ++t)
      for (uint32_t a = 0; a < 3; ++a)
        for (uint32_t b = 0; b < 3; ++b)
          f(slot(m_p[3 * t + a], m_p[3 * t + b]), (0u << 30) | (a << 28) | (b << 26) | uint32_t(t));
    for (size_t e = 0; e < nb; ++e)
      for (uint32_t a = 0; a < 4; ++a)
        for (uint32_t b = 0; b < 4; ++b)
          f(slot(b_p[4 * e + a], b_p[4 * e + b]), (1u << 30) | (a << 28) | (b << 26) | uint32_t(e));
    for (size_t q = 0; q < s_idx.size(); ++q) {
      const uint32_t ij[2] = {s_idx[q].x, s_idx[q].y};
      for (uint32_t a = 0; a < 2; ++a)
        for (uint32_t b = 0; b < 2; ++b) f(slot(ij[a], ij[b]), (2u << 30) | (a << 28) | (b << 26) | uint32_t(q));
    }
  };
  each([&](size_t sl, uint32_t) { P.ctr_off[sl + 1]++; });
  for (size_t q = 0; q < ns; ++q) P.ctr_off[q + 1] += P.ctr_off[q];
  P.ctr.assign(P.ctr_off[ns], 0);
  std::vector<uint32_t> fill(P.ctr_off.begin(), P.ctr_off.end() - 1);
  each([&](size_t sl, uint32_t code) { P.ctr[fill[sl]++] = code; });
  return true;
}

// Writable aliases of the scene constants, for the upload.
struct Carve {
  double *masse, *w, *kabst, *reib;
  uint8_t* frei;
  uint32_t *off_t, *off_b, *off_s, *ent_t, *ent_b, *ent_s, *cnt_v;
  uint4 *m_idx, *b_idx, *s_idx, *m_pos, *b_pos;
  uint2* s_pos;
  double4 *m_r, *m_basis, *m_mat;
  void *m_rin, *m_kgA, *m_rin64, *m_kgA64;
  double2 *b_kr, *s_kl;
  uint32_t *row_cnt, *col, *ctr_off, *ctr;
  Grp* grp;
  uint32_t *blk_grp, *pinst;
};

// Assigns every device array of the handle from the arena (base may be null
// to measure the size).
static void carve(k3d_solver* h, Arena& A, size_t N, size_t T, size_t B, size_t S, size_t et, size_t eb, size_t es,
                  size_t np, size_t kmax, const Pattern& P, Carve& cv) {
  const size_t nslots = np * (kmax ? kmax : 1);
  const size_t R = h->rsize;
  StepArgs& a = h->a;
  std::memset(&a, 0, sizeof(a));
  A.used = 0;
  a.x = A.take<double>(3 * N);
  a.v = A.take<double>(3 * N);
  a.dv = A.take<double>(3 * N);
  a.b = A.take<double>(3 * N);
  a.vk = A.take<double>(3 * N);
  a.load = A.take<double>(3 * N);
  a.nrm_d = A.take<double>(3 * N);
  h->d_pin = A.take<double>(3 * N);
  h->d_pout = A.take<double>(3 * N);
  a.fnk = A.take<double>(N);
  a.vn_soll = A.take<double>(N);
  h->d_fest = A.take<uint8_t>(N);  // a caller's contact set (k3d_solve_contacts)
  h->d_fest_n = A.take<double>(3 * N);
  h->d_fest_soll = A.take<double>(N);
  a.masse = cv.masse = A.take<double>(N);
  a.w = cv.w = A.take<double>(N);
  a.kabst = cv.kabst = A.take<double>(N);
  a.reib = cv.reib = A.take<double>(N);
  a.frei = cv.frei = A.take<uint8_t>(N);
  const size_t V = h->vsize;
  a.c = A.take<char>(8 * N * V);  // c and w per point
  a.r = A.take<char>(3 * N * V);
  a.z = A.take<char>(3 * N * V);
  a.ap = A.take<char>(3 * N * V);
  a.nrm = A.take<char>(3 * N * R);
  a.pinv = A.take<char>(6 * N * R);
  a.md = A.take<char>(N * R);
  a.off_t = cv.off_t = A.take<uint32_t>(N + 1);
  a.off_b = cv.off_b = A.take<uint32_t>(N + 1);
  a.off_s = cv.off_s = A.take<uint32_t>(N + 1);
  a.ent_t = cv.ent_t = A.take<uint32_t>(et);
  a.ent_b = cv.ent_b = A.take<uint32_t>(eb);
  a.ent_s = cv.ent_s = A.take<uint32_t>(es);
  a.cnt_v = cv.cnt_v = A.take<uint32_t>(N);
  a.np = int64_t(np);
  a.m_pos = cv.m_pos = A.take<uint4>(T);
  a.b_pos = cv.b_pos = A.take<uint4>(B);
  a.s_pos = cv.s_pos = A.take<uint2>(S);
  a.slot = A.take<char>(4 * nslots * R);
  a.m_idx = cv.m_idx = A.take<uint4>(T);
  a.m_r = cv.m_r = A.take<double4>(T);
  a.m_basis = cv.m_basis = A.take<double4>(T);
  a.m_mat = cv.m_mat = A.take<double4>(T);
  a.m_bc = A.take<double4>(3 * T);
  a.m_lc = A.take<double4>(3 * T);
  a.m_dc = A.take<double>(24 * T);
  a.m_f1w = A.take<char>(4 * T * R);
  a.m_f2w = A.take<char>(4 * T * R);
  a.m_kgB = A.take<char>(4 * T * R);
  a.m_rin = cv.m_rin = A.take<char>(4 * T * R);
  a.m_kgA = cv.m_kgA = A.take<char>(4 * T * R);
  a.b_idx = cv.b_idx = A.take<uint4>(B);
  a.b_kr = cv.b_kr = A.take<double2>(B);
  a.b_bc = A.take<double4>(4 * B);
  a.b_grad = A.take<char>(16 * B * R);
  a.s_idx = cv.s_idx = A.take<uint4>(S);
  a.s_kl = cv.s_kl = A.take<double2>(S);
  a.s_bc = A.take<double4>(S);
  a.s_lc = A.take<double4>(S);
  a.s_dq = A.take<char>(4 * S * R);
  a.s_k = A.take<char>(S * R);
  a.sync = A.take<SyncState>(1);
  a.partials = A.take<double>(size_t(kPartialsPerBlock) * h->blocks);  // reduction slots
  a.n_grp = h->n_grp;
  a.solve_threads = h->p.pcg_threads;
  a.grp = cv.grp = A.take<Grp>(size_t(h->n_grp));
  a.blk_grp = cv.blk_grp = A.take<uint32_t>(size_t(h->blocks));
  a.grp_cnt = A.take<unsigned>(size_t(32) * size_t(h->n_grp));
  a.pinst = cv.pinst = h->n_grp > 1 ? A.take<uint32_t>(N) : nullptr;
  a.stats = A.take<long long>(ST_COUNT);
  a.stat_rest_max = A.take<double>(2);
  // assembled A (BSR, ELL by rank) and its contribution lists
  const size_t nbs = P.kmax * np;
  a.bplane = int64_t(nbs);
  a.row_cnt = cv.row_cnt = A.take<uint32_t>(N);
  a.col = cv.col = A.take<uint32_t>(nbs);
  a.bmat = A.take<char>(9 * nbs * R);
  a.ctr_off = cv.ctr_off = A.take<uint32_t>(nbs + 1);
  a.ctr = cv.ctr = A.take<uint32_t>(P.ctr.size());
  a.cw2 = A.take<char>(8 * N * V);  // the second buffer of (c, w)
  cv.m_rin64 = cv.m_kgA64 = nullptr;
  if (R == 4) {  // FP64 operator records: the assembly of the FP32 blocks reads them
    a.m_f1w64 = A.take<double4>(T);
    a.m_f2w64 = A.take<double4>(T);
    a.m_kgB64 = A.take<double4>(T);
    a.m_rin64 = cv.m_rin64 = A.take<double4>(T);
    a.m_kgA64 = cv.m_kgA64 = A.take<double4>(T);
    a.b_grad64 = A.take<double4>(4 * B);
    a.s_dq64 = A.take<double4>(S);
    a.s_k64 = A.take<double>(S);
  }
  if (V == 4) a.slot64 = A.take<double4>(nslots);  // the FP64 residuals of the FP32-vector form
}

extern "C" {

int32_t k3d_abi_version(void) { return K3D_ABI_VERSION; }

void k3d_params_default(k3d_params* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->schritte_je_bild = 5;
  o->cg_max = 50;
  o->cg_toleranz = 1e-5;
  o->naht_k = 500.0;
  o->kontakt_rand = 1e-4;
  o->normalkraft_aus_last = 0;
  o->durchstoss_pruefen = 1;
  o->koerperpunkt_durchgaenge = 0;
  o->koerperpunkt_tiefe = 0.01;
  o->selbstkollision = 0;
  o->precision = K3D_FP64;
  o->selbst_zusatzdicke = 2.5e-3;
  o->selbst_steifigkeit = 1e-3;
  o->selbst_stoss_iterationen = 1;
  o->selbst_schnitte_an_naehten = 0;
}

void k3d_simparams_default(k3d_simparams* o) {
  if (!o) return;
  o->bild_dt = 1.0 / 60.0;
  o->schwerkraft[0] = 0.0;
  o->schwerkraft[1] = 0.0;
  o->schwerkraft[2] = -9.81;
  o->daempfung = 0.0;
}

// ------------------------------------------------------------ scene builder
k3d_status k3d_build_scene(const k3d_pattern* pattern, k3d_built_scene** out) {
  if (!pattern || !out) return K3D_BAD_ARGUMENT;
  auto* b = new k3d_built_scene;
  k3d_status st = build_scene_impl(pattern, b->s);
  if (st != K3D_OK) {
    delete b;
    *out = nullptr;
    return st;
  }
  *out = b;
  return K3D_OK;
}
k3d_status k3d_built_scene_view(k3d_built_scene* built, k3d_scene* out) {
  if (!built || !out) return K3D_BAD_ARGUMENT;
  built_scene_view(built->s, out);
  return K3D_OK;
}
void k3d_built_scene_free(k3d_built_scene* built) { delete built; }

// ------------------------------------------------------------ solver
k3d_solver* k3d_solver_create(const k3d_params* params, int32_t device) {
  auto* h = new k3d_solver;
  if (params)
    h->p = *params;
  else
    k3d_params_default(&h->p);
  h->device = device;
  if (h->p.precision < K3D_FP64 || h->p.precision > K3D_MIXED_STORAGE) {
    h->err = "unknown precision";
    return h;  // every later call reports K3D_DEVICE_ERROR
  }
  h->rsize = h->p.precision == K3D_FP64 ? 8 : 4;
  h->vsize = h->p.precision == K3D_MIXED ? 4 : 8;
  h->name = h->p.precision == K3D_MIXED           ? "B200 (f32/f64)"
            : h->p.precision == K3D_MIXED_STORAGE ? "B200 (f32 operator/f64)"
                                                  : "B200 (f64)";
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess) {
    h->err = "no CUDA device available";
    return h;  // every later call reports K3D_DEVICE_ERROR
  }
  if (h->p.pcg_threads == 0) h->p.pcg_threads = kSolveBlock;
  if (h->p.pcg_threads != 256 && h->p.pcg_threads != 512 && h->p.pcg_threads != 1024) {
    h->err = "pcg_threads must be 256, 512 or 1024";
    return h;  // every later call reports K3D_DEVICE_ERROR
  }
  h->blocks = step_grid_blocks(h->p.precision, h->p.pcg_threads, device);
  if (h->blocks <= 0) h->err = "cannot size the cooperative grid";
  else if (h->p.pcg_bloecke > 0) h->blocks = std::min(h->blocks, h->p.pcg_bloecke);
  return h;
}

static void release_device(k3d_solver* h) {
  selbst_free(h->sc);
  for (void* q : {h->adj.ck, h->adj.rec, h->adj.work})
    if (q) cudaFree(q);
  h->adj = k3d_solver::Adj{};
  if (h->arena.base) cudaFree(h->arena.base);
  h->arena = Arena{};
  for (void* p : h->sdf_dev) cudaFree(p);
  h->sdf_dev.clear();
  h->netz_dev.clear();
  for (void* p : h->kp_mem) cudaFree(p);
  h->kp_mem.clear();
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  h->gexec = nullptr;
  h->gkey.clear();
  h->uploaded = false;
}

void k3d_solver_destroy(k3d_solver* h) {
  if (!h) return;
  if (h->stream) {
    cudaStreamSynchronize(h->stream);
    release_device(h);
    cudaStreamDestroy(h->stream);
  }
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  for (cudaEvent_t e : h->sev) cudaEventDestroy(e);
  delete h;
}

const char* k3d_last_error(const k3d_solver* h) { return h ? h->err.c_str() : "null handle"; }
const char* k3d_solver_name(const k3d_solver* h) { return h ? h->name.c_str() : ""; }
double k3d_last_frame_ms(const k3d_solver* h) { return h ? h->last_ms : 0.0; }
double k3d_last_solve_ms(const k3d_solver* h) { return h ? h->solve_ms : 0.0; }
int64_t k3d_kernel_launches(const k3d_solver* h) { return h ? h->launches : 0; }
int32_t k3d_pcg_blocks(const k3d_solver* h) { return h && h->blocks > 0 ? h->blocks : 0; }

// kg = d2U/dg2 (kontinuum.rs:391-406), symmetric (00, 11, 22, 01, 02, 12)
static void kg_host(const double* ri, double fl, double kx, double ky, double sx, double sy, double ek, double es,
                    double g, double kg[6]) {
  (void)ri;
  const double a[3] = {kx * kx, ky * ky, kx * ky}, b[3] = {sx * sx, sy * sy, sx * sy},
               c[3] = {kx * sx, ky * sy, 0.5 * (kx * sy + ky * sx)};
  const double* v[3] = {a, b, c};
  const double wt[3] = {0.25 * ek, 0.25 * es, g};
  for (int q = 0; q < 6; ++q) kg[q] = 0.0;
  for (int t = 0; t < 3; ++t) {
    double s = fl * wt[t];
    kg[0] += s * v[t][0] * v[t][0];
    kg[1] += s * v[t][1] * v[t][1];
    kg[2] += s * v[t][2] * v[t][2];
    kg[3] += s * v[t][0] * v[t][1];
    kg[4] += s * v[t][0] * v[t][2];
    kg[5] += s * v[t][1] * v[t][2];
  }
}

static k3d_status validate(const k3d_scene* s) {
  if (!s || s->n_punkte < 0 || s->n_abstand < 0 || s->n_naht < 0 || s->n_biegung < 0 || s->n_membran < 0)
    return K3D_BAD_ARGUMENT;
  const int64_t n = s->n_punkte;
  if (n > 0 && (!s->x || !s->v || !s->masse || !s->w || !s->kollisionsabstand || !s->reibung)) return K3D_BAD_ARGUMENT;
  if (n >= int64_t(1) << 31) return K3D_BAD_ARGUMENT;
  auto chk = [&](const uint32_t* p, int64_t cnt) {
    for (int64_t i = 0; i < cnt; ++i)
      if (int64_t(p[i]) >= n) return false;
    return true;
  };
  if (s->n_abstand && (!s->abstand_punkte || !s->abstand_ruhe || !s->abstand_nachgiebigkeit ||
                       !chk(s->abstand_punkte, 2 * s->n_abstand)))
    return K3D_BAD_ARGUMENT;
  if (s->n_naht && (!s->naht_punkte || !s->naht_ruhe || !chk(s->naht_punkte, 2 * s->n_naht))) return K3D_BAD_ARGUMENT;
  if (s->n_biegung && (!s->biegung_punkte || !s->biegung_ruhe || !s->biegung_nachgiebigkeit ||
                       !chk(s->biegung_punkte, 4 * s->n_biegung)))
    return K3D_BAD_ARGUMENT;
  if (s->n_membran && (!s->membran_punkte || !s->membran_flaeche || !s->membran_ruhe_inv || !s->membran_kette ||
                       !s->membran_schuss || !s->membran_steif || !chk(s->membran_punkte, 3 * s->n_membran)))
    return K3D_BAD_ARGUMENT;
  if (s->n_dreiecke < 0 ||
      (s->n_dreiecke && (!s->dreiecke || !s->ruhe_inv || !chk(s->dreiecke, 3 * s->n_dreiecke))))
    return K3D_BAD_ARGUMENT;
  if (s->n_teile < 0 || (s->n_teile && (!s->teil_bereiche || !s->teil_dehnung))) return K3D_BAD_ARGUMENT;
  if (s->n_instanzen < 0 || (s->n_instanzen > 1 && !s->instanz_punkte)) return K3D_BAD_ARGUMENT;
  if (s->n_instanzen > 1) {
    const int64_t* o = s->instanz_punkte;
    if (o[0] != 0 || o[s->n_instanzen] != n) return K3D_BAD_ARGUMENT;
    for (int64_t k = 0; k < s->n_instanzen; ++k)
      if (o[k + 1] <= o[k]) return K3D_BAD_ARGUMENT;
  }
  if (s->n_koerper < 0 || s->n_koerper > kMaxBodies || (s->n_koerper && !s->koerper)) return K3D_BAD_ARGUMENT;
  for (int b = 0; b < s->n_koerper; ++b) {
    const k3d_body& k = s->koerper[b];
    if (k.instanz < -1 || (s->n_instanzen > 1 && k.instanz >= s->n_instanzen)) return K3D_BAD_ARGUMENT;
    if (k.art == K3D_BODY_SDF_GRID) {
      if (!k.sdf || k.dims[0] < 2 || k.dims[1] < 2 || k.dims[2] < 2 || !(k.spacing > 0.0)) return K3D_BAD_ARGUMENT;
    } else if (k.art == K3D_BODY_MESH) {
      if (!k.netz) return K3D_BAD_ARGUMENT;
    } else if (k.art != K3D_BODY_CYLINDER) {
      return K3D_BAD_ARGUMENT;
    }
  }
  return K3D_OK;
}

k3d_status k3d_upload_scene(k3d_solver* h, const k3d_scene* s) {
  if (!h) return K3D_BAD_ARGUMENT;
  if (!h->stream || h->blocks <= 0) return fail(h, K3D_DEVICE_ERROR, h->err.empty() ? "no device" : h->err);
  if (validate(s) != K3D_OK) return fail(h, K3D_BAD_ARGUMENT, "invalid scene (null array, index or body)");
  K3D_CUDA(h, cudaSetDevice(h->device));
  K3D_CUDA(h, cudaStreamSynchronize(h->stream));
  release_device(h);
  const int64_t n = s->n_punkte, nt = s->n_membran, nb = s->n_biegung;
  const size_t R = h->rsize;

  // instances (independent drapes of a batch): point offsets, and every
  // element group's range per instance (the groups list instance by instance)
  const int ng = s->n_instanzen > 1 ? int(s->n_instanzen) : 1;
  if (ng > h->blocks) return fail(h, K3D_BAD_ARGUMENT, "more instances than blocks of the PCG launch");
  if (ng > 1 && h->p.selbstkollision)
    return fail(h, K3D_BAD_ARGUMENT, "self-collision is not supported in a batch scene");
  std::vector<int64_t> io(ng + 1, 0);
  for (int k = 0; k <= ng; ++k) io[k] = ng > 1 ? s->instanz_punkte[k] : (k == 0 ? 0 : n);
  std::vector<uint32_t> pinst(ng > 1 ? n : 0);
  for (int k = 0; k < ng && ng > 1; ++k)
    for (int64_t i = io[k]; i < io[k + 1]; ++i) pinst[i] = uint32_t(k);
  auto inst_of = [&](uint32_t p) -> int { return ng > 1 ? int(pinst[p]) : 0; };
  // element ranges: [lo, hi) per instance; false if an element spans two
  // instances or the group is not ordered by instance
  auto ranges = [&](const uint32_t* pts, int64_t cnt, int w, std::vector<int64_t>& lo, std::vector<int64_t>& hi) {
    lo.assign(ng, 0);
    hi.assign(ng, 0);
    int prev = 0;
    for (int64_t e = 0; e < cnt; ++e) {
      const int k = inst_of(pts[w * e]);
      for (int q = 1; q < w; ++q)
        if (inst_of(pts[w * e + q]) != k) return false;
      if (k < prev) return false;
      prev = k;
    }
    int64_t e = 0;
    for (int k = 0; k < ng; ++k) {
      lo[k] = e;
      while (e < cnt && inst_of(pts[w * e]) == k) ++e;
      hi[k] = e;
    }
    return true;
  };
  std::vector<int64_t> t_lo, t_hi, b_lo, b_hi, a_lo, a_hi, n_lo, n_hi;
  if (!ranges(s->membran_punkte, nt, 3, t_lo, t_hi) || !ranges(s->biegung_punkte, nb, 4, b_lo, b_hi) ||
      !ranges(s->abstand_punkte, s->n_abstand, 2, a_lo, a_hi) || !ranges(s->naht_punkte, s->n_naht, 2, n_lo, n_hi))
    return fail(h, K3D_BAD_ARGUMENT, "an element spans two instances, or a group is not ordered by instance");

  // springs: pattern edges that carry their own stiffness, then seams
  // (implizit.rs:725-772), instance by instance
  std::vector<uint4> s_idx;
  std::vector<double2> s_kl;
  std::vector<int64_t> s_lo(ng), s_hi(ng);
  h->seam_slot.assign(size_t(s->n_naht), -1);
  for (int k = 0; k < ng; ++k) {
    s_lo[k] = int64_t(s_idx.size());
    for (int64_t e = a_lo[k]; e < a_hi[k]; ++e) {
      const bool membran = s->membran_kante && s->membran_kante[e];
      if (membran) continue;
      double kk = 1.0 / s->abstand_nachgiebigkeit[e];
      if (kk == 0.0) continue;
      s_idx.push_back(make_uint4(s->abstand_punkte[2 * e], s->abstand_punkte[2 * e + 1], 0u, 0u));
      s_kl.push_back(make_double2(kk, s->abstand_ruhe[e]));
    }
    if (h->p.naht_k != 0.0) {
      for (int64_t e = n_lo[k]; e < n_hi[k]; ++e) {
        h->seam_slot[e] = int64_t(s_idx.size());
        s_idx.push_back(make_uint4(s->naht_punkte[2 * e], s->naht_punkte[2 * e + 1], 1u, 0u));
        s_kl.push_back(make_double2(h->p.naht_k, s->naht_ruhe[e]));
      }
    }
    s_hi[k] = int64_t(s_idx.size());
  }
  const int64_t ns = int64_t(s_idx.size());
  h->n_grp = ng;
  h->s_kl_host = s_kl;

  // point -> element corner lists, in element order
  std::vector<uint32_t> off_t(n + 1, 0), off_b(n + 1, 0), off_s(n + 1, 0);
  for (int64_t t = 0; t < nt; ++t)
    for (int k = 0; k < 3; ++k) off_t[s->membran_punkte[3 * t + k] + 1]++;
  for (int64_t b = 0; b < nb; ++b)
    for (int k = 0; k < 4; ++k) off_b[s->biegung_punkte[4 * b + k] + 1]++;
  for (int64_t q = 0; q < ns; ++q) {
    off_s[s_idx[q].x + 1]++;
    off_s[s_idx[q].y + 1]++;
  }
  for (int64_t i = 0; i < n; ++i) {
    off_t[i + 1] += off_t[i];
    off_b[i + 1] += off_b[i];
    off_s[i + 1] += off_s[i];
  }
  std::vector<uint32_t> ent_t(off_t[n]), ent_b(off_b[n]), ent_s(off_s[n]);
  {
    std::vector<uint32_t> ft(off_t.begin(), off_t.end() - 1), fb(off_b.begin(), off_b.end() - 1),
        fs(off_s.begin(), off_s.end() - 1);
    for (int64_t t = 0; t < nt; ++t)
      for (int k = 0; k < 3; ++k) ent_t[ft[s->membran_punkte[3 * t + k]]++] = uint32_t(3 * t + k);
    for (int64_t b = 0; b < nb; ++b)
      for (int k = 0; k < 4; ++k) ent_b[fb[s->biegung_punkte[4 * b + k]]++] = uint32_t(4 * b + k);
    for (int64_t q = 0; q < ns; ++q) {
      ent_s[fs[s_idx[q].x]++] = uint32_t(2 * q);
      ent_s[fs[s_idx[q].y]++] = uint32_t(2 * q + 1);
    }
  }

  // operator slots (ELL): per point its membrane corners, then bend corners,
  // then spring ends; the corner of rank k at point i owns slot k * np + i
  const size_t np = (size_t(n) + 63) & ~size_t(63);
  std::vector<uint32_t> cnt_v(n, 0);
  size_t kmax = 0;
  for (int64_t i = 0; i < n; ++i) {
    cnt_v[i] = (off_t[i + 1] - off_t[i]) + (off_b[i + 1] - off_b[i]) + (off_s[i + 1] - off_s[i]);
    kmax = std::max(kmax, size_t(cnt_v[i]));
  }
  if (kmax * np >= (size_t(1) << 32)) return fail(h, K3D_BAD_ARGUMENT, "scene too large for 32-bit slots");
  std::vector<uint4> m_pos(nt), b_pos(nb);
  std::vector<uint2> s_pos(ns);
  for (int64_t i = 0; i < n; ++i) {
    uint32_t k = 0;
    for (uint32_t e = off_t[i]; e < off_t[i + 1]; ++e, ++k) {
      const uint32_t c = ent_t[e];
      (&m_pos[c / 3].x)[c % 3] = uint32_t(k * np + size_t(i));
    }
    for (uint32_t e = off_b[i]; e < off_b[i + 1]; ++e, ++k) {
      const uint32_t c = ent_b[e];
      (&b_pos[c / 4].x)[c % 4] = uint32_t(k * np + size_t(i));
    }
    for (uint32_t e = off_s[i]; e < off_s[i + 1]; ++e, ++k) {
      const uint32_t c = ent_s[e];
      (&s_pos[c / 2].x)[c % 2] = uint32_t(k * np + size_t(i));
    }
  }

  Pattern pat;
  if (!build_pattern(size_t(n), np, s->membran_punkte, size_t(nt), s->biegung_punkte, size_t(nb), s_idx, pat))
    return fail(h, K3D_BAD_ARGUMENT, "scene too large for the block pattern");

  // element constants
  std::vector<uint4> m_idx(nt), b_idx(nb);
  std::vector<double4> m_r(nt), m_basis(nt), m_mat(nt);
  std::vector<double2> b_kr(nb);
  std::vector<char> m_rin(size_t(nt) * 4 * R), m_kgA(size_t(nt) * 4 * R);
  std::vector<double4> m_rin64(R == 4 ? nt : 0), m_kgA64(R == 4 ? nt : 0);
  for (int64_t t = 0; t < nt; ++t) {
    const uint32_t* p = s->membran_punkte + 3 * t;
    m_idx[t] = make_uint4(p[0], p[1], p[2], 0u);
    const double* ri = s->membran_ruhe_inv + 4 * t;
    m_r[t] = make_double4(ri[0], ri[1], ri[2], ri[3]);
    const double* kt = s->membran_kette + 2 * t;
    const double* sc = s->membran_schuss + 2 * t;
    m_basis[t] = make_double4(kt[0], kt[1], sc[0], sc[1]);
    const double* st = s->membran_steif + 3 * t;
    m_mat[t] = make_double4(s->membran_flaeche[t], st[0], st[1], st[2]);
    double kg[6];
    kg_host(ri, s->membran_flaeche[t], kt[0], kt[1], sc[0], sc[1], st[0], st[1], st[2], kg);
    const double rin[4] = {ri[0], ri[1], ri[2], ri[3]}, kga[4] = {kg[0], kg[1], kg[2], kg[3]};
    if (R == 8) {
      std::memcpy(&m_rin[size_t(t) * 32], rin, 32);
      std::memcpy(&m_kgA[size_t(t) * 32], kga, 32);
    } else {
      m_rin64[t] = make_double4(rin[0], rin[1], rin[2], rin[3]);
      m_kgA64[t] = make_double4(kga[0], kga[1], kga[2], kga[3]);
      float fr[4], fk[4];
      for (int q = 0; q < 4; ++q) {
        fr[q] = float(rin[q]);
        fk[q] = float(kga[q]);
      }
      std::memcpy(&m_rin[size_t(t) * 16], fr, 16);
      std::memcpy(&m_kgA[size_t(t) * 16], fk, 16);
    }
  }
  for (int64_t b = 0; b < nb; ++b) {
    const uint32_t* p = s->biegung_punkte + 4 * b;
    b_idx[b] = make_uint4(p[0], p[1], p[2], p[3]);
    b_kr[b] = make_double2(1.0 / s->biegung_nachgiebigkeit[b], s->biegung_ruhe[b]);
  }
  std::vector<uint8_t> frei(n);
  double msum = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    frei[i] = s->w[i] > 0.0 ? 1 : 0;
    msum += s->masse[i];
  }
  h->boden = msum * 1e-18;

  // one allocation: measure the layout with a null base, then carve it
  const size_t N = size_t(n), T = size_t(nt), B = size_t(nb), S = size_t(ns);
  Carve cv;
  Arena probe;
  carve(h, probe, N, T, B, S, ent_t.size(), ent_b.size(), ent_s.size(), np, kmax, pat, cv);
  void* base = nullptr;
  K3D_CUDA(h, cudaMalloc(&base, probe.used));
  h->arena.base = static_cast<char*>(base);
  h->arena.size = probe.used;
  carve(h, h->arena, N, T, B, S, ent_t.size(), ent_b.size(), ent_s.size(), np, kmax, pat, cv);
  Arena& A = h->arena;
  StepArgs& a = h->a;
  if (A.used > A.size) return fail(h, K3D_DEVICE_ERROR, "arena overflow");
  K3D_CUDA(h, cudaMemsetAsync(A.base, 0, A.used, h->stream));

  cudaStream_t st = h->stream;
  auto up = [&](void* dst, const void* src, size_t b) -> cudaError_t {
    if (b == 0) return cudaSuccess;
    return cudaMemcpyAsync(dst, src, b, cudaMemcpyHostToDevice, st);
  };
  K3D_CUDA(h, up(a.x, s->x, 24 * N));
  K3D_CUDA(h, up(a.v, s->v, 24 * N));
  K3D_CUDA(h, up(cv.masse, s->masse, 8 * N));
  K3D_CUDA(h, up(cv.w, s->w, 8 * N));
  K3D_CUDA(h, up(cv.kabst, s->kollisionsabstand, 8 * N));
  K3D_CUDA(h, up(cv.reib, s->reibung, 8 * N));
  K3D_CUDA(h, up(cv.frei, frei.data(), N));
  K3D_CUDA(h, up(cv.off_t, off_t.data(), 4 * (N + 1)));
  K3D_CUDA(h, up(cv.off_b, off_b.data(), 4 * (N + 1)));
  K3D_CUDA(h, up(cv.off_s, off_s.data(), 4 * (N + 1)));
  K3D_CUDA(h, up(cv.ent_t, ent_t.data(), 4 * ent_t.size()));
  K3D_CUDA(h, up(cv.ent_b, ent_b.data(), 4 * ent_b.size()));
  K3D_CUDA(h, up(cv.ent_s, ent_s.data(), 4 * ent_s.size()));
  K3D_CUDA(h, up(cv.cnt_v, cnt_v.data(), 4 * N));
  K3D_CUDA(h, up(cv.row_cnt, pat.cnt.data(), 4 * N));
  K3D_CUDA(h, up(cv.col, pat.col.data(), 4 * pat.col.size()));
  K3D_CUDA(h, up(cv.ctr_off, pat.ctr_off.data(), 4 * pat.ctr_off.size()));
  K3D_CUDA(h, up(cv.ctr, pat.ctr.data(), 4 * pat.ctr.size()));
  K3D_CUDA(h, up(cv.m_pos, m_pos.data(), 16 * T));
  K3D_CUDA(h, up(cv.b_pos, b_pos.data(), 16 * B));
  K3D_CUDA(h, up(cv.s_pos, s_pos.data(), 8 * S));
  K3D_CUDA(h, up(cv.m_idx, m_idx.data(), 16 * T));
  K3D_CUDA(h, up(cv.m_r, m_r.data(), 32 * T));
  K3D_CUDA(h, up(cv.m_basis, m_basis.data(), 32 * T));
  K3D_CUDA(h, up(cv.m_mat, m_mat.data(), 32 * T));
  K3D_CUDA(h, up(cv.m_rin, m_rin.data(), m_rin.size()));
  K3D_CUDA(h, up(cv.m_kgA, m_kgA.data(), m_kgA.size()));
  if (cv.m_rin64) {
    K3D_CUDA(h, up(cv.m_rin64, m_rin64.data(), 32 * T));
    K3D_CUDA(h, up(cv.m_kgA64, m_kgA64.data(), 32 * T));
  }
  K3D_CUDA(h, up(cv.b_idx, b_idx.data(), 16 * B));
  K3D_CUDA(h, up(cv.b_kr, b_kr.data(), 16 * B));
  K3D_CUDA(h, up(cv.s_idx, s_idx.data(), 16 * S));
  K3D_CUDA(h, up(cv.s_kl, s_kl.data(), 16 * S));

  // groups of the PCG launch: blocks in proportion to the instances' work
  // (at least one each, largest remainders), points and elements per group.
  // An instance's PCG work per step grows as its points times its iteration
  // count, and the iteration count of a 2D mesh grows as the square root of
  // its points (the condition number grows as the mesh width squared), so
  // the weight is points^1.5.
  {
    const int B = h->blocks;
    std::vector<int> nbk(ng, 1);
    int left = B - ng;
    std::vector<std::pair<double, int>> rem;
    std::vector<double> wk(ng);
    double wsum = 0.0;
    for (int k = 0; k < ng; ++k) {
      const double pts = double(io[k + 1] - io[k]);
      wk[k] = pts * std::sqrt(pts);
      wsum += wk[k];
    }
    for (int k = 0; k < ng; ++k) {
      const double share = double(left) * wk[k] / std::max(wsum, 1e-300);
      const int whole = int(share);
      nbk[k] += whole;
      rem.push_back({share - double(whole), k});
    }
    int used = 0;
    for (int k = 0; k < ng; ++k) used += nbk[k];
    std::sort(rem.begin(), rem.end(), [](const auto& x, const auto& y) { return x.first > y.first || (x.first == y.first && x.second < y.second); });
    for (size_t q = 0; used < B; ++q, ++used) nbk[rem[q % rem.size()].second] += 1;
    std::vector<Grp> grp(ng);
    std::vector<uint32_t> blk(B);
    unsigned first = 0;
    for (int k = 0; k < ng; ++k) {
      Grp& g = grp[k];
      g.r0 = io[k];
      g.r1 = io[k + 1];
      g.t0 = t_lo[k];
      g.t1 = t_hi[k];
      g.b0 = b_lo[k];
      g.b1 = b_hi[k];
      g.s0 = s_lo[k];
      g.s1 = s_hi[k];
      g.first_blk = first;
      g.nblk = unsigned(nbk[k]);
      double msum = 0.0;
      for (int64_t i = io[k]; i < io[k + 1]; ++i) msum += s->masse[i];
      g.boden = msum * 1e-18;
      g.count = a.grp_cnt + 32 * size_t(k);
      g.partials = a.partials + size_t(kPartialsPerBlock) * size_t(first);
      for (int q = 0; q < nbk[k]; ++q) blk[first + q] = uint32_t(k);
      first += unsigned(nbk[k]);
    }
    K3D_CUDA(h, up(cv.grp, grp.data(), sizeof(Grp) * grp.size()));
    K3D_CUDA(h, up(cv.blk_grp, blk.data(), 4 * blk.size()));
    if (cv.pinst) K3D_CUDA(h, up(cv.pinst, pinst.data(), 4 * pinst.size()));
  }

  // bodies; SDF grids go to the device once here
  h->bodies.assign(s->koerper, s->koerper + s->n_koerper);
  for (int b = 0; b < s->n_koerper; ++b) {
    const k3d_body& k = s->koerper[b];
    void* d = nullptr;
    if (k.instanz < -1 || (s->n_instanzen > 1 && k.instanz >= s->n_instanzen)) return K3D_BAD_ARGUMENT;
    if (k.art == K3D_BODY_SDF_GRID) {
      size_t cnt = size_t(k.dims[0]) * k.dims[1] * k.dims[2];
      K3D_CUDA(h, cudaMalloc(&d, 4 * cnt));
      K3D_CUDA(h, up(d, k.sdf, 4 * cnt));
    }
    h->sdf_dev.push_back(d);
    const netz::Dev* nv = nullptr;
    if (k.art == K3D_BODY_MESH) {
      int dev = -1;
      nv = mesh_device_view(k.netz, &dev);
      if (!nv || dev != h->device) return fail(h, K3D_BAD_ARGUMENT, "a mesh body lives on another device");
    }
    h->netz_dev.push_back(nv);
  }
  // body points against cloth triangles (implizit.rs:1015-1025): the cloth
  // triangles on the device whenever a mesh body is present, so that the
  // pass count can change between frames
  {
    bool netz = false;
    for (const k3d_body& k : h->bodies) netz = netz || k.art == K3D_BODY_MESH;
    a.kp_passes = 0;
    a.kp_nt = 0;
    if (netz && s->n_dreiecke > 0) {
      const int64_t nt = s->n_dreiecke;
      std::vector<uint4> tri(static_cast<size_t>(nt));
      for (int64_t t = 0; t < nt; ++t)
        tri[size_t(t)] = make_uint4(s->dreiecke[3 * t], s->dreiecke[3 * t + 1], s->dreiecke[3 * t + 2], 0u);
      void *pt = nullptr, *pa = nullptr, *pb = nullptr, *pl = nullptr, *pc = nullptr;
      K3D_CUDA(h, cudaMalloc(&pt, size_t(nt) * sizeof(uint4)));
      h->kp_mem.push_back(pt);
      K3D_CUDA(h, cudaMalloc(&pa, size_t(nt) * sizeof(double4)));
      h->kp_mem.push_back(pa);
      K3D_CUDA(h, cudaMalloc(&pb, size_t(nt) * sizeof(double4)));
      h->kp_mem.push_back(pb);
      K3D_CUDA(h, cudaMalloc(&pl, size_t(nt) * sizeof(uint32_t)));
      h->kp_mem.push_back(pl);
      K3D_CUDA(h, cudaMalloc(&pc, 4 * sizeof(unsigned)));
      h->kp_mem.push_back(pc);
      K3D_CUDA(h, up(pt, tri.data(), tri.size() * sizeof(uint4)));
      a.kp_tri = static_cast<const uint4*>(pt);
      a.kp_a = static_cast<double4*>(pa);
      a.kp_b = static_cast<double4*>(pb);
      a.kp_list = static_cast<uint32_t*>(pl);
      a.kp_ctl = static_cast<unsigned*>(pc);
      a.kp_nt = nt;
    }
  }
  K3D_CUDA(h, cudaStreamSynchronize(st));
  if (h->p.selbstkollision) {
    if (n >= (int64_t(1) << 30) || s->n_dreiecke >= (int64_t(1) << 31))
      return fail(h, K3D_BAD_ARGUMENT, "scene too large for the self-collision stage");
    K3D_CUDA(h, selbst_upload(h->sc, s, h->p.selbst_zusatzdicke, h->p.selbst_steifigkeit, int(R), a.x, a.v, cv.masse,
                              cv.w, cv.reib, st));
  }

  a.n = n;
  a.nt = nt;
  a.nb = nb;
  a.ns = ns;
  h->n = n;
  h->nt = nt;
  h->nb = nb;
  h->ns = ns;
  h->sim = s->param;
  h->uploaded = true;
  h->first_step = true;
  h->err.clear();
  return K3D_OK;
}

}  // extern "C"

// Fills the per-launch fields and launches one step kernel.
// The per-launch fields of the handle's StepArgs: step constants and the
// bodies moved by t_bodies from their frame-start positions.
static void step_args(k3d_solver* h, int mode, double t_bodies, bool need_load) {
  StepArgs& a = h->a;
  const int sub = std::max(h->p.schritte_je_bild, 1);
  a.mode = mode;
  a.h = h->sim.bild_dt / double(sub);
  a.daempf = h->sim.daempfung;
  for (int k = 0; k < 3; ++k) a.g[k] = h->sim.schwerkraft[k];
  a.tol = h->p.cg_toleranz;
  a.cg_max = h->p.cg_max;
  a.kontakt_rand = h->p.kontakt_rand;
  a.boden = h->boden;
  a.normal_aus_last = h->p.normalkraft_aus_last;
  a.need_load = (need_load || h->p.normalkraft_aus_last) ? 1 : 0;
  a.first_step = (mode == MODE_STEP && h->first_step) ? 1 : 0;
  a.n_bodies = int(h->bodies.size());
  a.durchstoss_pruefen = h->p.durchstoss_pruefen ? 1 : 0;
  a.kp_passes = a.kp_nt > 0 ? std::max(h->p.koerperpunkt_durchgaenge, 0) : 0;
  a.kp_tief = h->p.koerperpunkt_tiefe;
  for (int b = 0; b < a.n_bodies; ++b) {
    const k3d_body& k = h->bodies[b];
    Body& d = a.bodies[b];
    d.art = k.art;
    for (int q = 0; q < 3; ++q) {
      d.dims[q] = k.dims[q];
      d.punkt[q] = k.punkt[q] + k.geschwindigkeit[q] * t_bodies;  // Koerper::verschoben (koerper.rs:122-133)
      d.achse[q] = k.achse[q];
      d.vel[q] = k.geschwindigkeit[q];
      d.ursprung[q] = k.ursprung[q];
    }
    d.radius = k.radius;
    d.spacing = k.spacing;
    d.sdf = static_cast<const float*>(h->sdf_dev[b]);
    d.netz = h->netz_dev[b];
    d.inst = h->n_grp > 1 ? k.instanz : -1;
  }
}

static k3d_status launch(k3d_solver* h, int mode, double t_bodies, bool need_load) {
  StepArgs& a = h->a;
  step_args(h, mode, t_bodies, need_load);
  int launched = 0;
  if (h->sc.on) {  // proximity pairs, regions and springs before the system (implizit.rs:668-707)
    SelbstArgs& ss = h->sc.s;
    ss.n_bodies = a.n_bodies;
    ss.kabst = a.kabst;
    ss.rand = a.kontakt_rand;
    ss.an_naehten = h->p.selbst_schnitte_an_naehten;
    if (a.n_bodies > 0)
      K3D_CUDA(h, cudaMemcpyAsync(h->sc.bodies_dev, a.bodies, sizeof(Body) * size_t(a.n_bodies),
                                  cudaMemcpyHostToDevice, h->stream));
    if (mode == MODE_STEP)  // the way the impact stage checks starts here (implizit.rs:903)
      K3D_CUDA(h, cudaMemcpyAsync(h->sc.x0, a.x, 24 * size_t(h->n), cudaMemcpyDeviceToDevice, h->stream));
    cudaError_t es = selbst_run(h->sc, a.h, h->stream, launched);
    if (es != cudaSuccess) return cuda_fail(h, es, "self-collision stage");
  }
  selbst_step_args(h->sc, a);
  cudaError_t e = launch_step(a, h->p.precision, h->blocks, h->stream, launched);
  h->launches += launched;
  if (e != cudaSuccess) return cuda_fail(h, e, "step kernel launch");
  if (h->sc.on && mode == MODE_STEP) {  // cloth against cloth on the way (implizit.rs:1027-1037)
    int ls = 0;
    cudaError_t es = selbst_stoss_run(h->sc, a.x, a.nrm_d, std::max(h->p.selbst_stoss_iterationen, 0), h->stream, ls);
    h->launches += ls;
    if (es != cudaSuccess) return cuda_fail(h, es, "self-collision impact stage");
  }
  if (mode == MODE_STEP) h->first_step = false;
  return K3D_OK;
}

// Sum of the PCG launch times recorded by the last frame(s).
static void sum_solve_ms(k3d_solver* h, size_t ev_used) {
  double t = 0.0;
  for (size_t q = 0; q + 1 < ev_used; q += 2) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, h->sev[q], h->sev[q + 1]) == cudaSuccess) t += ms;
  }
  h->solve_ms = t;
}

static k3d_status check_sync(k3d_solver* h) {
  K3D_CUDA(h, cudaStreamSynchronize(h->stream));
  SyncState ss;
  K3D_CUDA(h, cudaMemcpy(&ss, h->a.sync, sizeof(ss), cudaMemcpyDeviceToHost));
  if (ss.error != 0) {
    cudaMemset(&h->a.sync->error, 0, sizeof(int));
    return fail(h, K3D_TIMEOUT, "a device barrier wait ran out of time");
  }
  return K3D_OK;
}

static k3d_status read_stats(k3d_solver* h, k3d_stats* out) {
  long long st[ST_COUNT];
  double rm[2];
  K3D_CUDA(h, cudaMemcpy(st, h->a.stats, sizeof(st), cudaMemcpyDeviceToHost));
  K3D_CUDA(h, cudaMemcpy(rm, h->a.stat_rest_max, sizeof(rm), cudaMemcpyDeviceToHost));
  if (out) {
    std::memset(out, 0, sizeof(*out));
    out->cg_iterationen = st[ST_CG_ITERATIONS];
    out->loesungen = st[ST_SOLVES];
    out->nicht_konvergiert = st[ST_UNCONVERGED];
    out->kontakte = st[ST_CONTACTS];
    out->haftend = st[ST_STICKING];
    out->freigegeben = st[ST_RELEASED];
    out->durchstoesse = st[ST_PENETRATIONS];
    out->koerperpunkte = st[ST_BODY_POINTS];
    out->rest_max = rm[0];
    out->zusammenbrueche = st[ST_BREAKDOWNS];
    out->dv_max = rm[1];
    out->naehe_punkt_dreieck = int64_t(h->sc.naehe_pt);
    out->naehe_kante_kante = int64_t(h->sc.naehe_kk);
    if (h->sc.on) {
      unsigned long long acc[3];
      K3D_CUDA(h, cudaMemcpy(acc, h->sc.acc, sizeof(acc), cudaMemcpyDeviceToHost));
      out->selbst_stoesse = int64_t(acc[0]);
      out->durchdringungen = int64_t(acc[1]);
      out->durchdringungsgebiete = int64_t(acc[2]);
    }
  }
  if (st[ST_NONFINITE] > 0) return fail(h, K3D_NON_FINITE, "non-finite position or velocity after the step");
  return K3D_OK;
}

static k3d_status reset_stats(k3d_solver* h) {
  h->sc.naehe_pt = h->sc.naehe_kk = 0;
  if (h->sc.on) K3D_CUDA(h, cudaMemsetAsync(h->sc.acc, 0, 3 * sizeof(unsigned long long), h->stream));
  K3D_CUDA(h, cudaMemsetAsync(h->a.stats, 0, sizeof(long long) * ST_COUNT, h->stream));
  K3D_CUDA(h, cudaMemsetAsync(h->a.stat_rest_max, 0, sizeof(double) * 2, h->stream));
  return K3D_OK;
}

static k3d_status ready(k3d_solver* h) {
  if (!h) return K3D_BAD_ARGUMENT;
  if (!h->uploaded) return fail(h, K3D_BAD_ARGUMENT, "no scene uploaded");
  K3D_CUDA(h, cudaSetDevice(h->device));
  return K3D_OK;
}

// One frame of substeps as one CUDA graph: the substeps' launch arguments
// are formed first (step_args writes host fields only); when they equal
// those of the captured graph it is replayed, else the frame is captured
// again and the executable graph updated (or instantiated anew).
static k3d_status frame_graph(k3d_solver* h) {
  const int sub = std::max(h->p.schritte_je_bild, 1);
  const double hs = h->sim.bild_dt / double(sub);
  const bool first0 = h->first_step;
  std::vector<StepArgs> key(static_cast<size_t>(sub));
  h->a.ev_solve0 = h->a.ev_solve1 = nullptr;
  for (int k = 0; k < sub; ++k) {
    step_args(h, MODE_STEP, double(k + 1) * hs, false);
    key[size_t(k)] = h->a;
    h->first_step = false;
  }
  h->first_step = first0;
  bool same = h->gexec && h->gkey.size() == key.size();
  for (size_t k = 0; same && k < key.size(); ++k)
    same = std::memcmp(&key[k], &h->gkey[k], sizeof(StepArgs)) == 0;
  if (!same) {
    K3D_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int64_t l0 = h->launches;
    k3d_status st = K3D_OK;
    for (int k = 0; k < sub && st == K3D_OK; ++k) st = launch(h, MODE_STEP, double(k + 1) * hs, false);
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(h->stream, &g);
    if (st != K3D_OK || ec != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      h->first_step = first0;
      h->launches = l0;
      if (st != K3D_OK) return st;
      return cuda_fail(h, ec, "frame capture");
    }
    h->glaunches = h->launches - l0;
    h->launches = l0;
    if (h->gexec) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(h->gexec, g, &info) != cudaSuccess) {
        (void)cudaGetLastError();
        cudaGraphExecDestroy(h->gexec);
        h->gexec = nullptr;
      }
    }
    cudaError_t ei = cudaSuccess;
    if (!h->gexec) ei = cudaGraphInstantiate(&h->gexec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
      h->gexec = nullptr;
      h->gkey.clear();
      return cuda_fail(h, ei, "frame graph instantiate");
    }
    h->gkey = std::move(key);
  }
  K3D_CUDA(h, cudaGraphLaunch(h->gexec, h->stream));
  h->launches += h->glaunches;
  h->first_step = false;
  return K3D_OK;
}

// One frame of substeps on the resident state.
static k3d_status frame_device(k3d_solver* h, size_t& ev_used) {
  const int sub = std::max(h->p.schritte_je_bild, 1);
  const double hs = h->sim.bild_dt / double(sub);
  if (h->p.graph && !h->sc.on) {
    k3d_status st = frame_graph(h);
    if (st != K3D_OK) return st;
    for (auto& b : h->bodies)
      for (int q = 0; q < 3; ++q) b.punkt[q] += b.geschwindigkeit[q] * h->sim.bild_dt;
    return K3D_OK;
  }
  for (int k = 0; k < sub; ++k) {
    while (h->sev.size() < ev_used + 2) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return fail(h, K3D_DEVICE_ERROR, "event create");
      h->sev.push_back(e);
    }
    h->a.ev_solve0 = h->sev[ev_used];
    h->a.ev_solve1 = h->sev[ev_used + 1];
    ev_used += 2;
    k3d_status st = launch(h, MODE_STEP, double(k + 1) * hs, false);
    h->a.ev_solve0 = h->a.ev_solve1 = nullptr;
    if (st != K3D_OK) return st;
  }
  // the bodies end the frame moved by v * bild_dt (implizit.rs:1047-1054)
  for (auto& b : h->bodies)
    for (int q = 0; q < 3; ++q) b.punkt[q] += b.geschwindigkeit[q] * h->sim.bild_dt;
  return K3D_OK;
}

extern "C" {

k3d_status k3d_upload_state(k3d_solver* h, const double* x, const double* v) {
  k3d_status st = ready(h);
  if (st != K3D_OK) return st;
  if (x) K3D_CUDA(h, cudaMemcpyAsync(h->a.x, x, 24 * size_t(h->n), cudaMemcpyHostToDevice, h->stream));
  if (v) K3D_CUDA(h, cudaMemcpyAsync(h->a.v, v, 24 * size_t(h->n), cudaMemcpyHostToDevice, h->stream));
  K3D_CUDA(h, cudaStreamSynchronize(h->stream));
  return K3D_OK;
}

k3d_status k3d_download_state(k3d_solver* h, double* x, double* v) {
  k3d_status st = ready(h);
  if (st != K3D_OK) return st;
  if (x) K3D_CUDA(h, cudaMemcpyAsync(x, h->a.x, 24 * size_t(h->n), cudaMemcpyDeviceToHost, h->stream));
  if (v) K3D_CUDA(h, cudaMemcpyAsync(v, h->a.v, 24 * size_t(h->n), cudaMemcpyDeviceToHost, h->stream));
  K3D_CUDA(h, cudaStreamSynchronize(h->stream));
  return K3D_OK;
}

k3d_status k3d_frame(k3d_solver* h, k3d_scene* s, k3d_stats* stats) {
  k3d_status st = ready(h);
  if (st != K3D_OK) return st;
  if (!s || s->n_punkte != h->n || !s->x || !s->v) return fail(h, K3D_BAD_ARGUMENT, "scene does not match the upload");
  if (s->n_koerper != int32_t(h->bodies.size())) return fail(h, K3D_BAD_ARGUMENT, "body count changed; upload again");
  // state, seam rest lengths and body positions as the caller holds them now
  K3D_CUDA(h, cudaMemcpyAsync(h->a.x, s->x, 24 * size_t(h->n), cudaMemcpyHostToDevice, h->stream));
  K3D_CUDA(h, cudaMemcpyAsync(h->a.v, s->v, 24 * size_t(h->n), cudaMemcpyHostToDevice, h->stream));
  bool seams = false;
  for (size_t e = 0; e < h->seam_slot.size() && s->naht_ruhe; ++e)
    if (h->seam_slot[e] >= 0 && h->s_kl_host[h->seam_slot[e]].y != s->naht_ruhe[e] &&
        !(std::isnan(s->naht_ruhe[e]))) {
      h->s_kl_host[h->seam_slot[e]].y = s->naht_ruhe[e];
      seams = true;
    }
  if (seams)
    K3D_CUDA(h, cudaMemcpyAsync(const_cast<double2*>(h->a.s_kl), h->s_kl_host.data(), 16 * h->s_kl_host.size(),
                                cudaMemcpyHostToDevice, h->stream));
  K3D_CUDA(h, selbst_set_naht_ruhe(h->sc, s->naht_ruhe, s->n_naht, h->stream));
  for (int b = 0; b < s->n_koerper; ++b)
    for (int q = 0; q < 3; ++q) {
      h->bodies[b].punkt[q] = s->koerper[b].punkt[q];
      h->bodies[b].geschwindigkeit[q] = s->koerper[b].geschwindigkeit[q];
    }
  h->sim = s->param;
  st = reset_stats(h);
  if (st != K3D_OK) return st;
  K3D_CUDA(h, cudaEventRecord(h->ev0, h->stream));
  size_t ev_used = 0;
  st = frame_device(h, ev_used);
  if (st != K3D_OK) return st;
  K3D_CUDA(h, cudaEventRecord(h->ev1, h->stream));
  K3D_CUDA(h, cudaMemcpyAsync(s->x, h->a.x, 24 * size_t(h->n), cudaMemcpyDeviceToHost, h->stream));
  K3D_CUDA(h, cudaMemcpyAsync(s->v, h->a.v, 24 * size_t(h->n), cudaMemcpyDeviceToHost, h->stream));
  st = check_sync(h);
  if (st != K3D_OK) return st;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  h->last_ms = ms;
  sum_solve_ms(h, ev_used);
  s->zeit += s->param.bild_dt;
  return read_stats(h, stats);
}

k3d_status k3d_frames_resident(k3d_solver* h, int32_t n_frames, k3d_stats* stats) {
  k3d_status st = ready(h);
  if (st != K3D_OK) return st;
  if (n_frames < 0) return fail(h, K3D_BAD_ARGUMENT, "negative frame count");
  st = reset_stats(h);
  if (st != K3D_OK) return st;
  K3D_CUDA(h, cudaEventRecord(h->ev0, h->stream));
  size_t ev_used = 0;
  for (int f = 0; f < n_frames; ++f) {
    st = frame_device(h, ev_used);
    if (st != K3D_OK) return st;
  }
  K3D_CUDA(h, cudaEventRecord(h->ev1, h->stream));
  st = check_sync(h);
  if (st != K3D_OK) return st;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  h->last_ms = ms;
  sum_solve_ms(h, ev_used);
  return read_stats(h, stats);
}

k3d_status k3d_operator(k3d_solver* h, const double* p, double* out) {
  k3d_status st = ready(h);
  if (st != K3D_OK) return st;
  if (!p || !out) return fail(h, K3D_BAD_ARGUMENT, "null vector");
  K3D_CUDA(h, cudaMemcpyAsync(h->d_pin, p, 24 * size_t(h->n), cudaMemcpyHostToDevice, h->stream));
  h->a.p_in = h->d_pin;
  h->a.p_out = h->d_pout;
  st = launch(h, MODE_OPERATOR, 0.0, false);
  if (st != K3D_OK) return st;
  K3D_CUDA(h, cudaMemcpyAsync(out, h->d_pout, 24 * size_t(h->n), cudaMemcpyDeviceToHost, h->stream));
  return check_sync(h);
}

k3d_status k3d_system_for(k3d_solver* h, k3d_system_readback* rb) {
  k3d_status st = ready(h);
  if (st != K3D_OK) return st;
  if (!rb) return fail(h, K3D_BAD_ARGUMENT, "null readback");
  h->a.p_out = rb->f ? h->d_pout : nullptr;
  st = launch(h, MODE_SYSTEM, 0.0, true);
  if (st != K3D_OK) return st;
  st = check_sync(h);
  if (st != K3D_OK) return st;
  const size_t N = size_t(h->n);
  auto down = [&](void* dst, const void* src, size_t b) { return cudaMemcpy(dst, src, b, cudaMemcpyDeviceToHost); };
  if (rb->rhs) K3D_CUDA(h, down(rb->rhs, h->a.b, 24 * N));
  if (rb->f) K3D_CUDA(h, down(rb->f, h->d_pout, 24 * N));
  if (rb->last) K3D_CUDA(h, down(rb->last, h->a.load, 24 * N));
  std::vector<double> nrm(3 * N);
  K3D_CUDA(h, down(nrm.data(), h->a.nrm_d, 24 * N));
  if (rb->normale) std::memcpy(rb->normale, nrm.data(), 24 * N);
  if (rb->vn_soll) K3D_CUDA(h, down(rb->vn_soll, h->a.vn_soll, 8 * N));
  if (rb->fest)
    for (size_t i = 0; i < N; ++i)
      rb->fest[i] = (nrm[3 * i] != 0.0 || nrm[3 * i + 1] != 0.0 || nrm[3 * i + 2] != 0.0) ? 1 : 0;
  if (rb->pinv) {
    std::vector<double> P(6 * N);
    if (h->rsize == 8) {
      K3D_CUDA(h, down(P.data(), h->a.pinv, 48 * N));
    } else {
      std::vector<float> Pf(6 * N);
      K3D_CUDA(h, down(Pf.data(), h->a.pinv, 24 * N));
      for (size_t q = 0; q < 6 * N; ++q) P[q] = Pf[q];
    }
    for (size_t i = 0; i < N; ++i) {
      const double* p = &P[6 * i];
      double* o = rb->pinv + 9 * i;
      o[0] = p[0]; o[1] = p[3]; o[2] = p[4];
      o[3] = p[3]; o[4] = p[1]; o[5] = p[5];
      o[6] = p[4]; o[7] = p[5]; o[8] = p[2];
    }
  }
  return K3D_OK;
}

k3d_status k3d_solve(k3d_solver* h, double* dv_inout, k3d_cg_result* out) {
  k3d_status st = ready(h);
  if (st != K3D_OK) return st;
  if (!dv_inout) return fail(h, K3D_BAD_ARGUMENT, "null dv");
  K3D_CUDA(h, cudaMemcpyAsync(h->a.dv, dv_inout, 24 * size_t(h->n), cudaMemcpyHostToDevice, h->stream));
  st = reset_stats(h);
  if (st != K3D_OK) return st;
  st = launch(h, MODE_SOLVE, 0.0, false);
  if (st != K3D_OK) return st;
  K3D_CUDA(h, cudaMemcpyAsync(dv_inout, h->a.dv, 24 * size_t(h->n), cudaMemcpyDeviceToHost, h->stream));
  st = check_sync(h);
  if (st != K3D_OK) return st;
  long long sv[ST_COUNT];
  double rm[2];
  K3D_CUDA(h, cudaMemcpy(sv, h->a.stats, sizeof(sv), cudaMemcpyDeviceToHost));
  K3D_CUDA(h, cudaMemcpy(rm, h->a.stat_rest_max, sizeof(rm), cudaMemcpyDeviceToHost));
  if (out) {
    out->iterationen = sv[ST_LAST_ITERATIONS];
    out->nicht_konvergiert = sv[ST_UNCONVERGED] ? 1 : 0;
    out->breakdown = sv[ST_BREAKDOWNS] ? 1 : 0;
    out->rest = rm[0];
  }
  return sv[ST_UNCONVERGED] ? K3D_NOT_CONVERGED : K3D_OK;
}

k3d_status k3d_solve_contacts(k3d_solver* h, const k3d_contact_set* fest, double* dv_inout, k3d_cg_result* out) {
  k3d_status st = ready(h);
  if (st != K3D_OK) return st;
  if (!fest || !fest->fest || !fest->normale || !fest->vn_soll) return fail(h, K3D_BAD_ARGUMENT, "null contact set");
  if (h->sc.on) return fail(h, K3D_BAD_ARGUMENT, "a caller's contact set with self-collision on");
  const size_t N = size_t(h->n);
  K3D_CUDA(h, cudaMemcpyAsync(h->d_fest, fest->fest, N, cudaMemcpyHostToDevice, h->stream));
  K3D_CUDA(h, cudaMemcpyAsync(h->d_fest_n, fest->normale, 24 * N, cudaMemcpyHostToDevice, h->stream));
  K3D_CUDA(h, cudaMemcpyAsync(h->d_fest_soll, fest->vn_soll, 8 * N, cudaMemcpyHostToDevice, h->stream));
  h->a.fest_in = h->d_fest;
  h->a.fest_n = h->d_fest_n;
  h->a.fest_soll = h->d_fest_soll;
  st = k3d_solve(h, dv_inout, out);
  h->a.fest_in = nullptr;
  h->a.fest_n = h->a.fest_soll = nullptr;
  return st;
}

k3d_status k3d_residual(k3d_solver* h, const double* dv, double* out) {
  k3d_status st = ready(h);
  if (st != K3D_OK) return st;
  if (!dv || !out) return fail(h, K3D_BAD_ARGUMENT, "null vector");
  K3D_CUDA(h, cudaMemcpyAsync(h->d_pin, dv, 24 * size_t(h->n), cudaMemcpyHostToDevice, h->stream));
  h->a.p_in = h->d_pin;
  h->a.p_out = h->d_pout;
  st = launch(h, MODE_RESIDUAL, 0.0, false);
  if (st != K3D_OK) return st;
  K3D_CUDA(h, cudaMemcpyAsync(out, h->d_pout, 24 * size_t(h->n), cudaMemcpyDeviceToHost, h->stream));
  return check_sync(h);
}

k3d_status k3d_read_warm_start(k3d_solver* h, double* dv) {
  k3d_status st = ready(h);
  if (st != K3D_OK) return st;
  if (!dv) return fail(h, K3D_BAD_ARGUMENT, "null vector");
  K3D_CUDA(h, cudaStreamSynchronize(h->stream));
  K3D_CUDA(h, cudaMemcpy(dv, h->a.dv, 24 * size_t(h->n), cudaMemcpyDeviceToHost));
  return K3D_OK;
}

k3d_status k3d_read_load(k3d_solver* h, double* out) {
  k3d_status st = ready(h);
  if (st != K3D_OK) return st;
  if (!out) return fail(h, K3D_BAD_ARGUMENT, "null vector");
  K3D_CUDA(h, cudaMemcpy(out, h->a.load, 24 * size_t(h->n), cudaMemcpyDeviceToHost));
  return K3D_OK;
}

// ------------------------------------------------------------ self-collision probes
static bool selbst_ready(k3d_solver* h) {
  if (ready(h) != K3D_OK) return false;
  if (!h->sc.on || !h->sc.ran) {
    fail(h, K3D_BAD_ARGUMENT, "self-collision is off or has not run");
    return false;
  }
  return cudaStreamSynchronize(h->stream) == cudaSuccess;
}

int64_t k3d_selfcollision_pairs(k3d_solver* h, int64_t cap, int32_t* art, uint32_t* punkte, double* gewichte,
                                double* normale, double* abstand, double* ruhe) {
  if (!selbst_ready(h)) return -1;
  const SelbstArgs& s = h->sc.s;
  const int64_t np = int64_t(h->sc.n_pt) + h->sc.n_kk;
  const int64_t m = std::min(np, cap);
  if (m <= 0) return np;
  std::vector<uint4> idx(m);
  std::vector<double4> w(m), nab(m);
  std::vector<double> ru(m);
  if (cudaMemcpy(idx.data(), s.pr_idx, 16 * m, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(w.data(), s.pr_w, 32 * m, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(nab.data(), s.pr_nab, 32 * m, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(ru.data(), s.pr_ruhe, 8 * m, cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  for (int64_t q = 0; q < m; ++q) {
    if (art) art[q] = q < int64_t(h->sc.n_pt) ? 0 : 1;
    if (punkte) {
      punkte[4 * q] = idx[q].x;
      punkte[4 * q + 1] = idx[q].y;
      punkte[4 * q + 2] = idx[q].z;
      punkte[4 * q + 3] = idx[q].w;
    }
    if (gewichte) {
      gewichte[4 * q] = w[q].x;
      gewichte[4 * q + 1] = w[q].y;
      gewichte[4 * q + 2] = w[q].z;
      gewichte[4 * q + 3] = w[q].w;
    }
    if (normale) {
      normale[3 * q] = nab[q].x;
      normale[3 * q + 1] = nab[q].y;
      normale[3 * q + 2] = nab[q].z;
    }
    if (abstand) abstand[q] = nab[q].w;
    if (ruhe) ruhe[q] = ru[q];
  }
  return np;
}

int64_t k3d_selfcollision_hash(k3d_solver* h, int32_t kanten, int64_t cap_anfang, uint32_t* anfang,
                               int64_t cap_eintraege, uint32_t* eintraege, int64_t* n_eintraege) {
  if (!selbst_ready(h)) return -1;
  const SelbstArgs& s = h->sc.s;
  const uint32_t eimer = kanten ? s.eimer_k : s.eimer_p;
  const uint32_t* anf = kanten ? s.anf_k : s.anf_p;
  const uint32_t* ein = kanten ? s.ein_k : s.ein_p;
  uint32_t total = 0;
  if (cudaMemcpy(&total, anf + eimer, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  if (n_eintraege) *n_eintraege = total;
  if (anfang && cap_anfang > 0 &&
      cudaMemcpy(anfang, anf, 4 * size_t(std::min<int64_t>(cap_anfang, int64_t(eimer) + 1)),
                 cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  if (eintraege && cap_eintraege > 0 && total > 0 &&
      cudaMemcpy(eintraege, ein, 4 * size_t(std::min<int64_t>(cap_eintraege, total)), cudaMemcpyDeviceToHost) !=
          cudaSuccess)
    return -1;
  return int64_t(eimer);
}

int64_t k3d_selfcollision_springs(k3d_solver* h, int64_t cap, double* kraft, double* block) {
  if (!selbst_ready(h)) return -1;
  const SelbstArgs& s = h->sc.s;
  const int64_t np = int64_t(h->sc.n_pt) + h->sc.n_kk;
  const int64_t m = std::min(np, cap);
  if (m <= 0) return np;
  std::vector<double4> kf(m), b0(m), b1(m);
  if (cudaMemcpy(kf.data(), s.pr_kf, 32 * m, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(b0.data(), s.pr_b0, 32 * m, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(b1.data(), s.pr_b1, 32 * m, cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  for (int64_t q = 0; q < m; ++q) {
    if (kraft) {
      kraft[3 * q] = kf[q].x;
      kraft[3 * q + 1] = kf[q].y;
      kraft[3 * q + 2] = kf[q].z;
    }
    if (block) {
      const double B[9] = {b0[q].x, b0[q].w, b1[q].x, b0[q].w, b0[q].y, b1[q].y, b1[q].x, b1[q].y, b0[q].z};
      for (int k = 0; k < 9; ++k) block[9 * q + k] = B[k];
    }
  }
  return np;
}


// ------------------------------------------------------------ adjoint
static k3d_status adj_check(k3d_solver* h) {
  if (h->p.precision != K3D_FP64) return fail(h, K3D_BAD_ARGUMENT, "the adjoint needs K3D_FP64");
  if (h->p.selbstkollision) return fail(h, K3D_BAD_ARGUMENT, "the adjoint needs self-collision off");
  if (h->p.normalkraft_aus_last) return fail(h, K3D_BAD_ARGUMENT, "the adjoint needs normalkraft_aus_last off");
  if (h->bodies.size() > size_t(kMaxAdjointBodies))
    return fail(h, K3D_BAD_ARGUMENT, "the adjoint takes at most 14 bodies");
  for (const k3d_body& k : h->bodies)
    if (k.art == K3D_BODY_MESH) return fail(h, K3D_BAD_ARGUMENT, "the adjoint takes cylinder and grid bodies only");
  return K3D_OK;
}

static bool grow(void*& p, size_t& have, size_t need) {
  if (need <= have) return true;
  if (p) cudaFree(p);
  p = nullptr;
  have = 0;
  if (cudaMalloc(&p, need) != cudaSuccess) return false;
  have = need;
  return true;
}

k3d_status k3d_adjoint_forward(k3d_solver* h, int32_t n_frames, int32_t k, k3d_stats* stats) {
  k3d_status st = ready(h);
  if (st != K3D_OK) return st;
  if ((st = adj_check(h)) != K3D_OK) return st;
  if (n_frames < 1 || k < 1) return fail(h, K3D_BAD_ARGUMENT, "frames and checkpoint spacing must be positive");
  auto& A = h->adj;
  const int sub = std::max(h->p.schritte_je_bild, 1);
  const int64_t steps = int64_t(n_frames) * sub, nck = (steps + k - 1) / k;
  const size_t N3 = 3 * size_t(h->n);
  if (!grow(A.ck, A.ck_bytes, size_t(nck) * 3 * N3 * sizeof(double)))
    return fail(h, K3D_DEVICE_ERROR, "out of device memory for the adjoint checkpoints");
  A.valid = false;
  A.k = k;
  A.sub = sub;
  A.steps = steps;
  A.first.assign(size_t(nck), 0);
  A.bodies.clear();
  st = reset_stats(h);
  if (st != K3D_OK) return st;
  const double hs = h->sim.bild_dt / double(sub);
  double* ck = static_cast<double*>(A.ck);
  K3D_CUDA(h, cudaEventRecord(h->ev0, h->stream));
  for (int f = 0; f < n_frames; ++f) {
    A.bodies.push_back(h->bodies);
    for (int q = 0; q < sub; ++q) {
      const int64_t j = int64_t(f) * sub + q;
      if (j % k == 0) {
        double* c = ck + size_t(j / k) * 3 * N3;
        K3D_CUDA(h, cudaMemcpyAsync(c, h->a.x, N3 * 8, cudaMemcpyDeviceToDevice, h->stream));
        K3D_CUDA(h, cudaMemcpyAsync(c + N3, h->a.v, N3 * 8, cudaMemcpyDeviceToDevice, h->stream));
        K3D_CUDA(h, cudaMemcpyAsync(c + 2 * N3, h->a.dv, N3 * 8, cudaMemcpyDeviceToDevice, h->stream));
        A.first[size_t(j / k)] = h->first_step ? 1 : 0;
      }
      st = launch(h, MODE_STEP, double(q + 1) * hs, false);
      if (st != K3D_OK) return st;
    }
    for (auto& b : h->bodies)
      for (int q = 0; q < 3; ++q) b.punkt[q] += b.geschwindigkeit[q] * h->sim.bild_dt;
  }
  K3D_CUDA(h, cudaEventRecord(h->ev1, h->stream));
  st = check_sync(h);
  if (st != K3D_OK) return st;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  h->last_ms = ms;
  A.ms_fwd = ms;
  st = read_stats(h, stats);
  if (st == K3D_OK) A.valid = true;
  return st;
}

k3d_status k3d_adjoint_backward(k3d_solver* h, const double* gx, const double* gv, double* gx0, double* gv0,
                                double* g_membran, double* g_biegung, k3d_adjoint_stats* out) {
  k3d_status st = ready(h);
  if (st != K3D_OK) return st;
  if ((st = adj_check(h)) != K3D_OK) return st;
  auto& A = h->adj;
  if (!A.valid) return fail(h, K3D_BAD_ARGUMENT, "no adjoint forward to go back through");
  if (!gx || !gv) return fail(h, K3D_BAD_ARGUMENT, "null cotangent");
  const size_t N = size_t(h->n), N3 = 3 * N, T = size_t(h->nt), B = size_t(h->nb), S = size_t(h->ns);
  const size_t k = size_t(A.k);
  // one record: x, v, dv (3N each), fn (N) in doubles, then flags (N)
  const size_t rec_d = 10 * N, rec_stride = ((rec_d * 8 + 4 * N) + 255) & ~size_t(255);
  if (!grow(A.rec, A.rec_bytes, k * rec_stride)) return fail(h, K3D_DEVICE_ERROR, "out of device memory (records)");
  const size_t n_vec = 16;  // final state (3) and the backward's 13 vectors
  const size_t work_d = n_vec * N3 + 10 * T + 13 * B + 6 * S + 4 * T + B + 2 + ST_COUNT;
  if (!grow(A.work, A.work_bytes, work_d * 8)) return fail(h, K3D_DEVICE_ERROR, "out of device memory (adjoint)");
  double* w = static_cast<double*>(A.work);
  double* fin = w;
  double* vec = w + 3 * N3;
  AdjArgs J{};
  double** vs[13] = {&J.xq, &J.vq, &J.adv, &J.gq, &J.rq, &J.nq, &J.xa, &J.va, &J.gg, &J.arq, &J.lam, &J.alam, &J.mu};
  for (int q = 0; q < 13; ++q) *vs[q] = vec + size_t(q) * N3;
  double* tail = w + n_vec * N3;
  J.om = tail;
  J.ob = J.om + 10 * T;
  J.os = J.ob + 13 * B;
  J.acc_m = J.os + 6 * S;
  J.acc_b = J.acc_m + 4 * T;
  J.rest = J.acc_b + B;
  J.stats = reinterpret_cast<long long*>(J.rest + 2);
  // keep the forward's final state; the segments overwrite the resident one
  K3D_CUDA(h, cudaMemcpyAsync(fin, h->a.x, N3 * 8, cudaMemcpyDeviceToDevice, h->stream));
  K3D_CUDA(h, cudaMemcpyAsync(fin + N3, h->a.v, N3 * 8, cudaMemcpyDeviceToDevice, h->stream));
  K3D_CUDA(h, cudaMemcpyAsync(fin + 2 * N3, h->a.dv, N3 * 8, cudaMemcpyDeviceToDevice, h->stream));
  const std::vector<k3d_body> bodies_end = h->bodies;
  const bool first_end = h->first_step;
  K3D_CUDA(h, cudaMemcpyAsync(J.xq, gx, N3 * 8, cudaMemcpyHostToDevice, h->stream));
  K3D_CUDA(h, cudaMemcpyAsync(J.vq, gv, N3 * 8, cudaMemcpyHostToDevice, h->stream));
  K3D_CUDA(h, cudaMemsetAsync(J.lam, 0, N3 * 8, h->stream));
  K3D_CUDA(h, cudaMemsetAsync(J.acc_m, 0, (4 * T + B + 2 + ST_COUNT) * 8, h->stream));
  const double hs = h->sim.bild_dt / double(A.sub);
  const double* ck = static_cast<const double*>(A.ck);
  char* rec = static_cast<char*>(A.rec);
  const int64_t nck = (A.steps + A.k - 1) / A.k;
  cudaEvent_t e_r0 = nullptr, e_r1 = nullptr;
  K3D_CUDA(h, cudaEventCreate(&e_r0));
  K3D_CUDA(h, cudaEventCreate(&e_r1));
  double ms_re = 0.0;
  K3D_CUDA(h, cudaEventRecord(h->ev0, h->stream));
  for (int64_t seg = nck - 1; seg >= 0 && st == K3D_OK; --seg) {
    const int64_t j0 = seg * A.k, j1 = std::min<int64_t>(j0 + A.k, A.steps);
    const double* c = ck + size_t(seg) * 3 * N3;
    K3D_CUDA(h, cudaEventRecord(e_r0, h->stream));
    K3D_CUDA(h, cudaMemcpyAsync(h->a.x, c, N3 * 8, cudaMemcpyDeviceToDevice, h->stream));
    K3D_CUDA(h, cudaMemcpyAsync(h->a.v, c + N3, N3 * 8, cudaMemcpyDeviceToDevice, h->stream));
    K3D_CUDA(h, cudaMemcpyAsync(h->a.dv, c + 2 * N3, N3 * 8, cudaMemcpyDeviceToDevice, h->stream));
    h->first_step = A.first[size_t(seg)] != 0;
    // the segment again, recording each substep
    for (int64_t j = j0; j < j1 && st == K3D_OK; ++j) {
      double* r = reinterpret_cast<double*>(rec + size_t(j - j0) * rec_stride);
      h->bodies = A.bodies[size_t(j / A.sub)];
      K3D_CUDA(h, cudaMemcpyAsync(r, h->a.x, N3 * 8, cudaMemcpyDeviceToDevice, h->stream));
      K3D_CUDA(h, cudaMemcpyAsync(r + N3, h->a.v, N3 * 8, cudaMemcpyDeviceToDevice, h->stream));
      h->a.rec_flags = reinterpret_cast<uint32_t*>(r + rec_d);
      K3D_CUDA(h, cudaMemsetAsync(h->a.rec_flags, 0, N * sizeof(uint32_t), h->stream));
      st = launch(h, MODE_STEP, double(j % A.sub + 1) * hs, false);
      h->a.rec_flags = nullptr;
      if (st != K3D_OK) break;
      K3D_CUDA(h, cudaMemcpyAsync(r + 2 * N3, h->a.dv, N3 * 8, cudaMemcpyDeviceToDevice, h->stream));
      K3D_CUDA(h, cudaMemcpyAsync(r + 3 * N3, h->a.fnk, N * 8, cudaMemcpyDeviceToDevice, h->stream));
    }
    if (st != K3D_OK) break;
    K3D_CUDA(h, cudaEventRecord(e_r1, h->stream));
    // back through it
    for (int64_t j = j1 - 1; j >= j0; --j) {
      const double* r = reinterpret_cast<const double*>(rec + size_t(j - j0) * rec_stride);
      h->bodies = A.bodies[size_t(j / A.sub)];
      step_args(h, MODE_STEP, double(j % A.sub + 1) * hs, false);
      StepArgs a = h->a;
      a.x = const_cast<double*>(r);
      a.v = const_cast<double*>(r + N3);
      J.x = r;
      J.v = r + N3;
      J.dv = r + 2 * N3;
      J.fn = r + 3 * N3;
      J.flags = reinterpret_cast<const uint32_t*>(r + rec_d);
      int launched = 0;
      cudaError_t e = launch_adjoint_step(a, J, h->blocks, h->stream, launched);
      h->launches += launched;
      if (e != cudaSuccess) {
        st = cuda_fail(h, e, "adjoint step launch");
        break;
      }
    }
    K3D_CUDA(h, cudaStreamSynchronize(h->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e_r0, e_r1);
    ms_re += ms;
  }
  K3D_CUDA(h, cudaEventRecord(h->ev1, h->stream));
  cudaEventDestroy(e_r0);
  cudaEventDestroy(e_r1);
  // the forward's final state again
  K3D_CUDA(h, cudaMemcpyAsync(h->a.x, fin, N3 * 8, cudaMemcpyDeviceToDevice, h->stream));
  K3D_CUDA(h, cudaMemcpyAsync(h->a.v, fin + N3, N3 * 8, cudaMemcpyDeviceToDevice, h->stream));
  K3D_CUDA(h, cudaMemcpyAsync(h->a.dv, fin + 2 * N3, N3 * 8, cudaMemcpyDeviceToDevice, h->stream));
  h->bodies = bodies_end;
  h->first_step = first_end;
  k3d_status sy = check_sync(h);
  if (st != K3D_OK) return st;
  if (sy != K3D_OK) return sy;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  if (gx0) K3D_CUDA(h, cudaMemcpy(gx0, J.xq, N3 * 8, cudaMemcpyDeviceToHost));
  if (gv0) K3D_CUDA(h, cudaMemcpy(gv0, J.vq, N3 * 8, cudaMemcpyDeviceToHost));
  if (g_membran && T > 0) {
    std::vector<double> gm(4 * T);
    K3D_CUDA(h, cudaMemcpy(gm.data(), J.acc_m, 4 * T * 8, cudaMemcpyDeviceToHost));
    for (size_t t = 0; t < T; ++t)
      for (size_t q = 0; q < 4; ++q) g_membran[4 * t + q] = gm[q * T + t];
  }
  if (g_biegung && B > 0) K3D_CUDA(h, cudaMemcpy(g_biegung, J.acc_b, B * 8, cudaMemcpyDeviceToHost));
  long long sts[ST_COUNT];
  K3D_CUDA(h, cudaMemcpy(sts, J.stats, sizeof(sts), cudaMemcpyDeviceToHost));
  if (out) {
    std::memset(out, 0, sizeof(*out));
    out->cg_iterationen = sts[ST_CG_ITERATIONS];
    out->loesungen = sts[ST_SOLVES];
    out->nicht_konvergiert = sts[ST_UNCONVERGED];
    out->zusammenbrueche = sts[ST_BREAKDOWNS];
    out->ms_vorwaerts = A.ms_fwd;
    out->ms_rueckwaerts = ms;
    out->ms_neuberechnung = ms_re;
  }
  return K3D_OK;
}

}  // extern "C"
