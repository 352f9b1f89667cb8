// Adjoint of one implicit substep on the device (internal to the library).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "k3d_step.h"

namespace k3d {

// Buffers of one backward substep. The record holds the substep's input
// state, its final solution and each point's normal force and branch flags
// (StepArgs::rec_flags). xq, vq enter as the cotangents of the substep's
// output x, v and leave as those of its input x, v. All vectors are 3 per
// point (double) unless noted.
struct AdjArgs {
  const double *x, *v, *dv, *fn;  // record (fn: 1 per point)
  const uint32_t* flags;          // record (1 per point)
  double *xq, *vq;
  double *adv, *gq, *rq, *nq, *xa, *va, *gg, *arq, *lam, *alam, *mu;
  // element derivatives of mu.Phi, direction-major: membranes [10][nt]
  // (f1, f2 components, E_warp, E_weft, G, grain rotation), hinges [13][nb]
  // (12 coordinates, k), springs [6][ns] (both ends' coordinates)
  double *om, *ob, *os;
  // parameter cotangents summed over the substeps: [4][nt], [nb]
  double *acc_m, *acc_b;
  long long* stats;  // the adjoint PCG's statistics (ST_COUNT)
  double* rest;      // 2
};

// Enqueues the backward of one substep: the build at the recorded input
// state (StepArgs x, v point at the record; dv at lam, the adjoint solve's
// warm start and result), then the point, solve and element stages.
cudaError_t launch_adjoint_step(const StepArgs& a, const AdjArgs& j, int blocks, cudaStream_t stream, int& launched);

}  // namespace k3d
