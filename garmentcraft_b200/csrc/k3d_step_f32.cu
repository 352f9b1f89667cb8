// The PCG kernels of the FP32-vector form (K3D_MIXED), compiled with fused
// multiply-add: its FP32 recursion loses fewer iterations with the fused
// products (measured on the 66k- and 201k-point sheets). The kernel itself
// is k3d_solve.cuh.
#include "k3d_solve.cuh"

namespace k3d {

const void* solve_fn_f32(bool sc, int threads) {
  if (threads == 256)
    return sc ? (const void*)solve_kernel<float, float, true, 256> : (const void*)solve_kernel<float, float, false, 256>;
  if (threads == 1024)
    return sc ? (const void*)solve_kernel<float, float, true, 1024>
              : (const void*)solve_kernel<float, float, false, 1024>;
  return sc ? (const void*)solve_kernel<float, float, true, 512> : (const void*)solve_kernel<float, float, false, 512>;
}

}  // namespace k3d
