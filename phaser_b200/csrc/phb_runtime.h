// Host-side helpers shared by the translation units of libphaser_b200.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include "../../include/phaser_b200.h"

namespace phb {

// NVTX range over one host entry point: a timeline profiler (or ncu --nvtx
// --nvtx-include "phb_solver_group/") shows the launches it issues under its name.
// NVTX v3 is header-only; with no tool attached a push / pop is a null check.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// Record and map the last CUDA error of a launch to a status code.
int check_launch();
int record_cuda(cudaError_t err);
// count a kernel launch issued without check_launch() (e.g. cudaLaunchKernelEx)
void count_launch();

// launch `kernel` over `blocks` CTAs of `threads` threads in thread-block clusters
// of `cluster` CTAs (1 = no cluster attribute)
template <typename... P, typename... A>
inline int launch_clustered(void (*kernel)(P...), unsigned blocks, unsigned threads, unsigned cluster, size_t smem,
                            cudaStream_t st, A &&...args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(blocks, 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = cluster > 1 ? 1 : 0;
    const int rc = record_cuda(cudaLaunchKernelEx(&cfg, kernel, static_cast<A &&>(args)...));
    if (rc == PHB_OK) count_launch();
    return rc;
}

}  // namespace phb
