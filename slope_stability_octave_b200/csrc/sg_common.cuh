// Shared helpers for the slopegpu library: status codes, error capture, launch shapes.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/slopegpu.h"

namespace sg {

// Records a message for sg_last_error() (thread-local) and returns the code.
int set_error(int code, const std::string &msg);
int cuda_error(cudaError_t e, const char *what);

#define SG_CUDA(call)                                          \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return sg::cuda_error(_e, #call); \
    } while (0)

#define SG_CHECK_ARG(cond, msg)                                \
    do {                                                       \
        if (!(cond)) return sg::set_error(SG_ERR_ARG, msg);    \
    } while (0)

// Number of kernel launches issued by the library (every launch computes its grid through
// grid_for or calls count_launch), read by sg_launch_count for benchmark reporting.
void count_launch(int n = 1);

// Every device allocation of the library goes through device_alloc (counted, read by
// sg_device_alloc_count), so a caller can check that a timed region allocated nothing.
cudaError_t device_alloc_raw(void **p, size_t bytes);
template <typename T>
inline cudaError_t device_alloc(T **p, size_t bytes) {
    return device_alloc_raw(reinterpret_cast<void **>(p), bytes);
}

// The library's device status word on the current device (allocated and zeroed on first
// use; null if that fails): kernels with bounded waits record there that a wait gave up.
int32_t *device_status_word();

// Launch shape: grid sized in multiples of the SM count (148 on B200) for
// grid-stride kernels, capped by the work.
int sm_count();
inline unsigned grid_for(int64_t work, int block, int per_sm = 8) {
    count_launch();
    int64_t need = (work + block - 1) / block;
    int64_t cap = (int64_t)sm_count() * per_sm;
    if (need < 1) need = 1;
    return (unsigned)(need < cap ? need : cap);
}

// Launch shape for kernels that give each CTA a run of `chunk` consecutive items (rows or
// output blocks) and walk it in order: ceil(n / chunk) CTAs.
inline unsigned grid_chunks(int64_t n, int64_t chunk) {
    count_launch();
    const int64_t g = (n + chunk - 1) / chunk;
    return (unsigned)(g < 1 ? 1 : g);
}
// Chunk length for that mapping: a multiple of `unit`, at most `most`, and short enough to
// give every SM eight CTAs when n is small.
inline int64_t chunk_len(int64_t n, int64_t unit, int64_t most) {
    const int64_t slots = (int64_t)sm_count() * 8;
    const int64_t want = (n + slots - 1) / slots;
    const int64_t c = ((want + unit - 1) / unit) * unit;
    return c < unit ? unit : (c > most ? most : c);
}

// Growable device scratch owned by the library (host-buffer entry points only).
struct Scratch {
    void *ptr = nullptr;
    size_t bytes = 0;
    int device = -1;
    int reserve(size_t want);
    ~Scratch();
};

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace sg
