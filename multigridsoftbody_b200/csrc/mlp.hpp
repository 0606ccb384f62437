// Internal interface between the network (mlp.cu) and the solver (solver.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

struct mgsb_mlp;

namespace mgsb {
// BF16 tensor-core image of the current parameters (device pointer).
const uint8_t* mlp_device_image(const mgsb_mlp* h);
int mlp_device(const mgsb_mlp* h);
}  // namespace mgsb
