// Allocation-free variant of the host-buffer 3D return mapping (sg_constitutive3d).
//
// sg_constitutive3d reserves a device staging buffer with cudaMalloc on its first call (and
// again whenever a larger call arrives) and creates two streams per call.  Some callers cannot
// have that: a MEX/oct-file running under a fixed device-memory budget that was sized when
// the session started, or a host loop that must not pay the device-wide synchronisation that
// cudaMalloc/cudaFree imply while other streams are busy.  This entry point stages through a
// statically sized array that is part of the library's device image instead, issues its
// copies and its kernel on the legacy default stream, and never allocates device memory.
//
// Limits and contract:
//   * at most SG_NOALLOC_MAX_POINTS points per call (larger calls are rejected with
//     SG_ERR_ARG before anything is launched; split them on the host);
//   * the first call on each device looks up the array's device address (the library's
//     module is loaded then, which is when the array itself gets its memory); make that first
//     call before starting any stream capture;
//   * nothing in the array needs to start at zero: every byte a call reads was written by the
//     same call (inputs copied in, then every output point written by the kernel);
//   * there is one array per device and process, so calls that overlap in time on the same
//     device -- from two host threads, say -- race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "sg_common.cuh"

namespace sg {
int launch_constitutive(int dim, bool fused, const double *E, const double *m0, const double *m1,
                        const double *psi, const double *shear, const double *lame, double lambda, char davis,
                        int64_t n, double *S, double *DS, uint8_t *branch, cudaStream_t st);
}

namespace {

// the capacity is the one the public header states; the array below is sized from it
constexpr int64_t kMaxPoints = SG_NOALLOC_MAX_POINTS;
static_assert(kMaxPoints > 0, "SG_NOALLOC_MAX_POINTS must be positive");
constexpr size_t kAlign = 256;
// per point: E 6 + c_bar, sin_phi, shear, lame 4 + S 6 + DS 36 doubles + 1 branch byte;
// each of the 8 carved arrays is rounded up to kAlign
constexpr size_t kScratchBytes = (size_t)kMaxPoints * (sizeof(double) * (6 + 4 + 6 + 36) + 1) + 8 * kAlign;

__device__ __align__(256) unsigned char g_constitutive_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char *g_scratch_ptr[kMaxDevices] = {};

// Device address of this device's copy of the array (looked up once per device).
int scratch_for_current_device(unsigned char **out) {
    int dev = 0;
    SG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return sg::set_error(SG_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_constitutive_scratch);
        if (e != cudaSuccess || !p) return sg::cuda_error(e, "no-allocation scratch address");
        g_scratch_ptr[dev] = (unsigned char *)p;
    }
    *out = g_scratch_ptr[dev];
    return SG_OK;
}

}  // namespace

using namespace sg;

extern "C" int sg_constitutive3d_noalloc(const double *E, const double *c_bar, const double *sin_phi,
                                         const double *shear, const double *bulk, const double *lame,
                                         int64_t n_int, double *S, double *DS, uint8_t *branch) {
    (void)bulk;  // unused by the return mapping, as in the reference kernel
    SG_CHECK_ARG(n_int >= 0, "n_int must be >= 0");
    if (n_int > kMaxPoints)
        return set_error(SG_ERR_ARG, "n_int exceeds the no-allocation scratch (" + std::to_string(kMaxPoints) +
                                         " points per call)");
    if (n_int == 0) return SG_OK;
    SG_CHECK_ARG(E && c_bar && sin_phi && shear && lame && S, "null input/output pointer");
    unsigned char *base = nullptr;
    int rc = scratch_for_current_device(&base);
    if (rc) return rc;
    const int64_t n = n_int;
    auto carve = [&](size_t bytes) {
        unsigned char *p = base;
        base += (bytes + kAlign - 1) & ~(kAlign - 1);
        return p;
    };
    double *dE = (double *)carve(sizeof(double) * 6 * n);
    double *dcb = (double *)carve(sizeof(double) * n);
    double *dsp = (double *)carve(sizeof(double) * n);
    double *dG = (double *)carve(sizeof(double) * n);
    double *dL = (double *)carve(sizeof(double) * n);
    double *dS = (double *)carve(sizeof(double) * 6 * n);
    double *dDS = DS ? (double *)carve(sizeof(double) * 36 * n) : nullptr;
    uint8_t *dbr = branch ? (uint8_t *)carve(n) : nullptr;
    const cudaStream_t st = 0;
    SG_CUDA(cudaMemcpyAsync(dE, E, sizeof(double) * 6 * n, cudaMemcpyHostToDevice, st));
    SG_CUDA(cudaMemcpyAsync(dcb, c_bar, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    SG_CUDA(cudaMemcpyAsync(dsp, sin_phi, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    SG_CUDA(cudaMemcpyAsync(dG, shear, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    SG_CUDA(cudaMemcpyAsync(dL, lame, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    rc = launch_constitutive(3, false, dE, dcb, dsp, nullptr, dG, dL, 1.0, 'B', n, dS, dDS, dbr, st);
    if (rc) return rc;
    SG_CUDA(cudaMemcpyAsync(S, dS, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, st));
    if (DS) SG_CUDA(cudaMemcpyAsync(DS, dDS, sizeof(double) * 36 * n, cudaMemcpyDeviceToHost, st));
    if (branch) SG_CUDA(cudaMemcpyAsync(branch, dbr, n, cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    return SG_OK;
}
