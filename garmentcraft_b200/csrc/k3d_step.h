// Kernel arguments of the persistent step kernel (internal to the library).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "k3d_device.cuh"

namespace k3d {

constexpr int kBlock = 256;       // ordinary launches
constexpr int kSolveBlock = 512;  // the persistent PCG launch's default CTA size (256 and 1024 also built)

enum Mode : int { MODE_STEP = 0, MODE_SYSTEM = 1, MODE_OPERATOR = 2, MODE_SOLVE = 3, MODE_RESIDUAL = 4 };

// device statistics slots (int64)
enum StatSlot : int {
  ST_CG_ITERATIONS = 0,
  ST_SOLVES = 1,
  ST_UNCONVERGED = 2,
  ST_CONTACTS = 3,
  ST_STICKING = 4,
  ST_RELEASED = 5,
  ST_BREAKDOWNS = 6,
  ST_NONFINITE = 7,
  ST_LAST_ITERATIONS = 8,
  ST_HELD = 9,
  ST_PENETRATIONS = 10,  // segment entries through a mesh body (ImplizitStatistik::durchstoesse)
  ST_BODY_POINTS = 11,   // triangles lifted over a body point (ImplizitStatistik::koerperpunkte)
  ST_COUNT = 16
};

constexpr int K3D_STATUS_TIMEOUT = 6;

// Grid reductions of the PCG launch: up to kRedMax doubles per barrier, the
// block partials double-buffered (k3d_step.cu).
constexpr int kRedMax = 4;
constexpr int kPartialsPerBlock = 2 * kRedMax;

struct SyncState {
  unsigned count;  // barrier arrivals in this launch (zeroed before each launch)
  unsigned pad0[31];
  int error;       // K3D_STATUS_TIMEOUT after a wait gave up
  int pad1[31];
};

// One instance of a batch (an independent drape) and the group of blocks of
// the PCG launch that solves it: its points, elements, barrier counter and
// reduction partials. A scene of one drape is one group over all blocks.
struct Grp {
  int64_t r0, r1;                  // points
  int64_t t0, t1, b0, b1, s0, s1;  // membranes, bends, springs
  unsigned first_blk, nblk;
  double boden;       // convergence floor: 1e-18 of the instance's mass (implizit.rs:390-391)
  unsigned* count;    // barrier arrivals (zeroed before each launch)
  double* partials;   // kPartialsPerBlock per block of the group
};

struct StepArgs {
  int64_t n, nt, nb, ns;
  int mode, first_step, need_load, normal_aus_last;
  int cg_max, n_bodies;
  int durchstoss_pruefen, pad0;  // segment check against mesh bodies (implizit.rs:988-1002)
  // body points against cloth triangles after integration (implizit.rs:1015-1025)
  int kp_passes, kp_pad;
  double kp_tief;
  int64_t kp_nt;            // cloth triangles
  const uint4* kp_tri;      // their points
  double4 *kp_a, *kp_b;     // per triangle its deepest stab: (depth, normal), (weights, body point)
  uint32_t* kp_list;        // triangles with a stab
  unsigned* kp_ctl;         // listed stabs, corrections in this pass, stop
  double h, daempf, g[3], tol, kontakt_rand, boden;
  Body bodies[kMaxBodies];
  // points (double)
  double *x, *v, *dv, *b, *vk, *fnk, *load, *vn_soll, *nrm_d;
  const double *masse, *w, *kabst, *reib;
  const uint8_t* frei;
  // points (operator precision)
  void *c, *r, *z, *ap, *pinv, *nrm, *md;
  // point -> element corner lists (per-step build)
  const uint32_t *off_t, *ent_t, *off_b, *ent_b, *off_s, *ent_s;
  // operator: element corner (rank k at point i) owns slot k * np + i; point
  // i sums its cnt_v[i] slots
  const uint32_t* cnt_v;
  int64_t np;
  const uint4 *m_pos, *b_pos;
  const uint2* s_pos;
  void* slot;
  // membranes
  const uint4* m_idx;
  const double4 *m_r, *m_basis, *m_mat;
  double4 *m_bc, *m_lc;
  double* m_dc;  // 8 per corner (6 used)
  void *m_f1w, *m_f2w, *m_kgB;
  const void *m_rin, *m_kgA;
  // bends
  const uint4* b_idx;
  const double2* b_kr;
  double4* b_bc;
  void* b_grad;
  // springs
  const uint4* s_idx;
  const double2* s_kl;
  double4 *s_bc, *s_lc;
  void *s_dq, *s_k;
  // assembled A: block (rank k, row i) at k * np + i of `bplane` blocks, 9
  // planes of R (row-major 3x3); per block the contribution list ctr_off/ctr
  const uint32_t *row_cnt, *col, *ctr_off, *ctr;
  void* bmat;
  int64_t bplane;
  void* cw2;  // second (c, w) buffer: the row product reads one, writes the other
  // FP64 copies of the operator records for the residuals of the mixed form
  // (start residual, reliable updates, release test); null in the FP64 form
  void *m_f1w64, *m_f2w64, *m_kgB64, *b_grad64, *s_dq64, *s_k64, *slot64;
  const void *m_rin64, *m_kgA64;
  // proximity springs of cloth self-collision (the stage's last run), null
  // when off: per point its (pair << 2 | slot) entries; per pair its points,
  // weights, force and k, block k[(1-mu) n n^T + mu I] as (xx, yy, zz, xy),
  // (xz, yz, mu, 0), and the operator copies (h^2 block as 2 R4, weights R4)
  const uint32_t *sc_off, *sc_ent;
  const uint4* sc_idx;
  const double4 *sc_w, *sc_kf, *sc_b0, *sc_b1;
  const void *sc_bR, *sc_wR;
  // the fifth point and weight of each spring (kKein / 0 for proximity pairs;
  // the push springs of penetration regions join an edge to a triangle)
  const uint32_t* sc_x5;
  const double* sc_g5;
  const void* sc_g5R;
  // the PCG iteration's spring product spring by spring: each nonzero slot's
  // entry index (sc_pos, per spring << 3 | slot) and the per-entry products
  // (sc_out, R4), summed per point in list order; sc_np springs
  const uint32_t* sc_pos;
  void* sc_out;
  uint32_t sc_np;
  // probes
  const double* p_in;
  double* p_out;
  // the caller's contact set of a solve (k3d_solve_contacts), null otherwise:
  // held flag, unit normal (3 per point) and required normal velocity; it
  // replaces the set the build found against the bodies
  const uint8_t* fest_in;
  const double *fest_n, *fest_soll;
  // instances (independent drapes): per point its instance (null for one),
  // the groups of the PCG launch and each block's group
  const uint32_t* pinst;
  const Grp* grp;
  const uint32_t* blk_grp;
  unsigned* grp_cnt;  // the groups' counters, 32 words apart
  int n_grp;
  // adjoint: the PCG solves S A S lam = S b with a zero target on held points
  // (adjoint != 0); the step records each point's branches in rec_flags
  // (null: no record; zeroed before the step): bit 0 held after the release
  // pass, bit 1 stick, bit 2 slip, bit 3 released after the last solve (the
  // second release pass), body k: bit 4 + 2k pushed out, bit 5 + 2k inward
  // normal velocity removed
  int adjoint;
  uint32_t* rec_flags;
  int solve_threads;  // threads per CTA of the persistent PCG launch (256, 512 or 1024)
  int pad_st;
  // bookkeeping
  cudaEvent_t ev_solve0, ev_solve1;  // around the PCG launch (host-side handles)
  SyncState* sync;
  double* partials;  // kPartialsPerBlock * blocks
  long long* stats;
  double* stat_rest_max;
};

// The build, probe and integration kernels (compiled apart from the PCG).
struct BuildKernels {
  const void *elements, *points, *assemble, *probe_load, *probe_apply, *probe_out, *integrate;
};
BuildKernels build_kernels(int precision);

// CTAs of the persistent PCG launch that fit at once (SMs x CTAs per SM) for
// the form and CTA size (256, 512 or 1024 threads); -1 on error.
int step_grid_blocks(int precision, int threads, int device);
// Enqueues one substep (or probe) on `stream`; `launched` = kernels enqueued.
cudaError_t launch_step(const StepArgs& a, int precision, int blocks, cudaStream_t stream, int& launched);
// The FP64 PCG launch alone on the system built before (one pass, no release
// test): dv (start and result), b, normals and the assembled A as in `a`.
cudaError_t launch_pcg64(const StepArgs& a, int blocks, cudaStream_t stream);
// The body-point passes after integration (none when kp_passes or kp_nt is 0).
cudaError_t launch_koerperpunkte(const StepArgs& a, cudaStream_t stream, int& launched);
constexpr int kMaxAdjointBodies = 14;  // bodies whose push-outs fit in rec_flags

}  // namespace k3d
