// Library-wide helpers: error capture, device queries, scratch buffers.
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <cstdio>
#include <string>

#include "sg_common.cuh"

namespace sg {

static thread_local std::string g_last_error;
static std::atomic<int64_t> g_launches{0};
static std::atomic<int64_t> g_device_allocs{0};

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

cudaError_t device_alloc_raw(void **p, size_t bytes) {
    g_device_allocs.fetch_add(1, std::memory_order_relaxed);
    return cudaMalloc(p, bytes);
}

static int32_t *g_status[64] = {};

int32_t *device_status_word() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (!g_status[dev]) {
        int32_t *p = nullptr;
        if (device_alloc(&p, sizeof(int32_t)) != cudaSuccess) return nullptr;
        if (cudaMemset(p, 0, sizeof(int32_t)) != cudaSuccess) {
            cudaFree(p);
            return nullptr;
        }
        g_status[dev] = p;
    }
    return g_status[dev];
}

int set_error(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int cuda_error(cudaError_t e, const char *what) {
    char buf[512];
    snprintf(buf, sizeof buf, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    if (e == cudaErrorMemoryAllocation) return set_error(SG_ERR_NOMEM, buf);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return set_error(SG_ERR_NODEVICE, buf);
    return set_error(SG_ERR_CUDA, buf);
}

int sm_count() {
    static thread_local int dev_cached = -1, sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return sms;
    if (dev != dev_cached) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0) sms = v;
        dev_cached = dev;
    }
    return sms;
}

int Scratch::reserve(size_t want) {
    int dev = 0;
    SG_CUDA(cudaGetDevice(&dev));
    if (ptr && bytes >= want && dev == device) return SG_OK;
    if (ptr) {
        int cur = dev;
        cudaSetDevice(device);
        cudaFree(ptr);
        cudaSetDevice(cur);
        ptr = nullptr;
        bytes = 0;
    }
    cudaError_t e = device_alloc(&ptr, want);
    if (e != cudaSuccess) {
        ptr = nullptr;
        return cuda_error(e, "scratch allocation");
    }
    bytes = want;
    device = dev;
    return SG_OK;
}

Scratch::~Scratch() {
    // Process teardown: the context may already be gone; ignore errors.
    if (ptr) cudaFree(ptr);
}

}  // namespace sg

extern "C" int sg_abi_version(void) { return 1; }

// Kernel launches issued by the library since the last reset.
extern "C" int64_t sg_launch_count(int reset) {
    const int64_t v = sg::g_launches.load();
    if (reset) sg::g_launches.store(0);
    return v;
}

extern "C" int64_t sg_device_alloc_count(int reset) {
    const int64_t v = sg::g_device_allocs.load();
    if (reset) sg::g_device_allocs.store(0);
    return v;
}

extern "C" int sg_device_status(int32_t reset, int32_t *status) {
    SG_CHECK_ARG(status, "status is null");
    int32_t *w = sg::device_status_word();
    if (!w) return sg::set_error(SG_ERR_CUDA, "device status word unavailable");
    SG_CUDA(cudaDeviceSynchronize());
    SG_CUDA(cudaMemcpy(status, w, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (reset) SG_CUDA(cudaMemset(w, 0, sizeof(int32_t)));
    return SG_OK;
}

extern "C" const char *sg_last_error(void) { return sg::g_last_error.c_str(); }

extern "C" int sg_device_count(void) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        sg::cuda_error(e, "cudaGetDeviceCount");
        return 0;
    }
    return n;
}
