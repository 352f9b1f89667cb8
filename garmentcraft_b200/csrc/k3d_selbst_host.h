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
  std::vector<void*> schn, wege;          // intersection-sized; path-hash entries
  double* x0 = nullptr;                   // positions at the start of the substep
  Body* bodies_dev = nullptr;             // the substep's bodies (pinch test)
  unsigned long long* acc = nullptr;      // impact corrections, intersections, regions since the reset
  uint32_t n_s = 0;                       // intersections of the last run
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
cudaError_t selbst_grow_schnitte(SelbstHost& H, uint32_t cap);
cudaError_t selbst_grow_wege(SelbstHost& H, uint32_t cap_p, uint32_t cap_k);
cudaError_t selbst_grow_pairs(SelbstHost& H, uint32_t cap);
cudaError_t selbst_set_naht_ruhe(SelbstHost& H, const double* ruhe, int64_t n_naht, cudaStream_t st);
// One run on the current state with substep h (two host reads of the counts).
cudaError_t selbst_run(SelbstHost& H, double h, cudaStream_t st, int& launches);
// Impacts on the way from the substep's start to x (the step's positions,
// changed in place) and their response; held points (nonzero nrm_fest) weigh
// 1e9 times their mass (one host read of the path hashes' sizes).
cudaError_t selbst_stoss_run(SelbstHost& H, double* x, const double* nrm_fest, int iterationen, cudaStream_t st,
                            int& launches);
// The springs of the last run into the step kernel's arguments (null when off).
void selbst_step_args(const SelbstHost& H, StepArgs& a);

}  // namespace k3d
