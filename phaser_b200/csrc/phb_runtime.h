// Host-side helpers shared by the translation units of libphaser_b200.
#pragma once

#include <cuda_runtime.h>
#include "../../include/phaser_b200.h"

namespace phb {

// Record and map the last CUDA error of a launch to a status code.
int check_launch();
int record_cuda(cudaError_t err);
// count a kernel launch issued without check_launch() (e.g. cudaLaunchKernelEx)
void count_launch();

}  // namespace phb
