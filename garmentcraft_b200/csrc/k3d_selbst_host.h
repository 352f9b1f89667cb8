// Host side of the self-collision proximity stage (internal to the library).
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/klon3d_step.h"
#include "k3d_selbst.h"
#include "k3d_step.h"

namespace k3d {

struct SelbstHost {
  bool on = false;   // tables uploaded (ImplizitParameter::selbstkollision)
  bool ran = false;  // a run has filled the pair buffers
  SelbstArgs s{};
  std::vector<void*> fest, pairs, hashk;  // device allocations: fixed, pair-sized, edge-hash
  std::vector<double> naht_ruhe;          // host copy of the seam rest lengths on the device
  double* naht_ruhe_dev = nullptr;
  uint32_t n_pt = 0, n_kk = 0;          // pairs of the last run
  uint64_t naehe_pt = 0, naehe_kk = 0;  // pairs since the last statistics reset
};

// Builds the mesh tables from the scene and allocates the device buffers.
cudaError_t selbst_upload(SelbstHost& H, const k3d_scene* sc, double zusatzdicke, double steifigkeit, int rsize,
                          const double* x, double* v, const double* masse, const double* w, const double* reib,
                          cudaStream_t st);
void selbst_free(SelbstHost& H);
cudaError_t selbst_grow_edge_hash(SelbstHost& H, uint32_t cap);
cudaError_t selbst_grow_pairs(SelbstHost& H, uint32_t cap);
cudaError_t selbst_set_naht_ruhe(SelbstHost& H, const double* ruhe, int64_t n_naht, cudaStream_t st);
// One run on the current state with substep h (two host reads of the counts).
cudaError_t selbst_run(SelbstHost& H, double h, cudaStream_t st, int& launches);
// The springs of the last run into the step kernel's arguments (null when off).
void selbst_step_args(const SelbstHost& H, StepArgs& a);

}  // namespace k3d
