// Status codes, CUDA error capture and version of libphaser_b200.
#include <atomic>
#include <cstring>
#include "phb_runtime.h"

namespace phb {

// FP32 FMA throughput probe: eight independent fmaf chains per thread (enough to cover
// the FMA latency at full occupancy), 2 FLOP per fmaf.  The result is written only if it
// equals a value it never takes, so the chains are not removed.
__global__ void __launch_bounds__(512) k_fma_peak(float *sink, int iters) {
    float a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = 1.0f + 1e-3f * (float)(threadIdx.x + j);
    const float b = 0.999999f, c = 1e-6f;
#pragma unroll 4
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = fmaf(a[j], b, c);
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += a[j];
    if (s == -1.0f) sink[blockIdx.x] = s;
}

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

int phb_fp32_peak(int32_t iters, double *tflops, float *ms, void *stream) {
    if (iters < 1 || !tflops) return PHB_ERR_INVALID_ARG;
    int dev = 0, sms = 0;
    int rc = phb::record_cuda(cudaGetDevice(&dev));
    if (!rc) rc = phb::record_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (rc) return rc;
    const int blocks = sms * 4, threads = 512;   // 64 warps per SM
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if ((rc = phb::record_cuda(cudaEventCreate(&e0)))) return rc;
    if ((rc = phb::record_cuda(cudaEventCreate(&e1)))) {
        cudaEventDestroy(e0);
        return rc;
    }
    phb::k_fma_peak<<<blocks, threads, 0, st>>>(nullptr, iters);   // warm-up (clocks, module load)
    rc = phb::check_launch();
    if (!rc) rc = phb::record_cuda(cudaEventRecord(e0, st));
    if (!rc) {
        phb::k_fma_peak<<<blocks, threads, 0, st>>>(nullptr, iters);
        rc = phb::check_launch();
    }
    if (!rc) rc = phb::record_cuda(cudaEventRecord(e1, st));
    if (!rc) rc = phb::record_cuda(cudaEventSynchronize(e1));
    float t = 0.f;
    if (!rc) rc = phb::record_cuda(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    const double flop = 2.0 * 8.0 * (double)iters * (double)blocks * (double)threads;
    *tflops = flop / ((double)t * 1e-3) / 1e12;
    if (ms) *ms = t;
    return PHB_OK;
}

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
