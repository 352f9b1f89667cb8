// Host side of the body mesh for the rest of the library (internal).
#pragma once
#include "../../include/klon3d_mesh.h"
#include "k3d_netz.cuh"

namespace k3d {
// The mesh's tables as the device reads them (a device pointer, valid until
// the mesh is destroyed; refreshed in place by k3d_mesh_update) and the
// device the mesh lives on.
const netz::Dev* mesh_device_view(const k3d_mesh* m, int* device);
}  // namespace k3d
