// Packed dipole records shared by the dA/dt kernels (coil.cu, coil_table.cu).
#pragma once

#include <cuda_runtime.h>

namespace cunibs {

// One placement's dipoles in the head frame, centred on the coil origin, each component stored
// twice so a shared-memory load yields a ready float2 broadcast: {s,s}, {m,m} per axis.
struct __align__(16) DipolePacked {
    float2 sx, sy, sz, mx, my, mz;
};

// A coil whose moments all lie along its own z axis, in the coil frame: position and the z moment,
// each stored twice as for DipolePacked. Shared by every placement.
struct __align__(16) ZDipolePacked {
    float2 sx, sy, sz, m;
};

}  // namespace cunibs
