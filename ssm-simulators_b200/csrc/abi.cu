// Library-wide C ABI helpers: version, thread-local error text, device status.
#include <stdarg.h>
#include <stdio.h>

#include "common.cuh"

namespace ssm {

static thread_local char g_last_error[512] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

int cuda_fail(cudaError_t e, const char *where) {
    set_error("%s: %s", where, cudaGetErrorString(e));
    return SSM_ERR_CUDA;
}

int sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
    return n > 0 ? n : 148;
}

}  // namespace ssm

extern "C" {

int ssm_version(void) { return 100; }

const char *ssm_last_error(void) { return ssm::g_last_error; }

int ssm_check_status(const void *workspace, void *stream) {
    if (!workspace) {
        ssm::set_error("ssm_check_status: workspace is NULL");
        return SSM_ERR_ARG;
    }
    ssm::WorkspaceHeader h;
    cudaStream_t st = (cudaStream_t)stream;
    SSM_CUDA(cudaMemcpyAsync(&h, workspace, sizeof(h), cudaMemcpyDeviceToHost, st));
    SSM_CUDA(cudaStreamSynchronize(st));
    if (h.err == SSM_ERR_NOISE_RANGE) {
        ssm::set_error("trajectory %d needed more injected increments than its noise row holds",
                       h.err_detail);
        return SSM_ERR_NOISE_RANGE;
    }
    if (h.err != 0) {
        ssm::set_error("device error code %d (detail %d)", h.err, h.err_detail);
        return SSM_ERR_DEVICE;
    }
    return SSM_OK;
}

}  // extern "C"
