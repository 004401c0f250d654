// Status codes, CUDA error capture and version of libphaser_b200.
#include <atomic>
#include <cstring>
#include "phb_runtime.h"

namespace phb {

static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

static thread_local char g_last_cuda[256] = "";

int record_cuda(cudaError_t err) {
    if (err == cudaSuccess) return PHB_OK;
    std::strncpy(g_last_cuda, cudaGetErrorString(err), sizeof(g_last_cuda) - 1);
    g_last_cuda[sizeof(g_last_cuda) - 1] = '\0';
    return PHB_ERR_CUDA;
}

int check_launch() {
    const int rc = record_cuda(cudaGetLastError());
    if (rc == PHB_OK) count_launch();
    return rc;
}

}  // namespace phb

extern "C" {

const char *phb_status_string(int status) {
    switch (status) {
        case PHB_OK: return "ok";
        case PHB_ERR_INVALID_ARG: return "invalid argument";
        case PHB_ERR_UNSUPPORTED: return "unsupported shape or option";
        case PHB_ERR_CUDA: return "CUDA error";
        case PHB_ERR_NONFINITE: return "NaN or inf encountered";
        case PHB_ERR_OUTSIDE: return "probe positions completely outside object";
        case PHB_ERR_SCRATCH_LIMIT: return "problem too large for the 64 MiB static scratch of phb_solver_group_static";
        default: return "unknown status";
    }
}

int phb_version(void) { return 100; }

const char *phb_last_cuda_error(void) { return phb::g_last_cuda; }

int64_t phb_kernel_launches(void) { return (int64_t)phb::g_launches.load(); }

int phb_event_create(void **event) {
    if (!event) return PHB_ERR_INVALID_ARG;
    cudaEvent_t ev = nullptr;
    const int rc = phb::record_cuda(cudaEventCreate(&ev));
    *event = (void *)ev;
    return rc;
}

int phb_event_destroy(void *event) {
    if (!event) return PHB_ERR_INVALID_ARG;
    return phb::record_cuda(cudaEventDestroy((cudaEvent_t)event));
}

int phb_event_record(void *event, void *stream) {
    if (!event) return PHB_ERR_INVALID_ARG;
    return phb::record_cuda(cudaEventRecord((cudaEvent_t)event, (cudaStream_t)stream));
}

int phb_event_elapsed_ms(void *start, void *end, float *ms) {
    if (!start || !end || !ms) return PHB_ERR_INVALID_ARG;
    int rc = phb::record_cuda(cudaEventSynchronize((cudaEvent_t)end));
    if (rc) return rc;
    return phb::record_cuda(cudaEventElapsedTime(ms, (cudaEvent_t)start, (cudaEvent_t)end));
}

}  // extern "C"
