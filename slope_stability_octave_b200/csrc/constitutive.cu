// (a1-a4) Constitutive kernels and their C-ABI entry points.
//
// Layout: the reference MEX layout, i.e. per-point AoS (Octave column-major n_s x n_int):
// E[6p + c], S[6p + c], DS[36p + k].  One thread per point; each warp stages its 32 points'
// outputs in shared memory and writes them back as contiguous 256-byte runs, so stores stay
// fully coalesced although every point owns a 288-byte tangent.
#include <cuda_runtime.h>

#include <algorithm>

#include "instr.cuh"
#include "mc_point.cuh"
#include "sg_common.cuh"

namespace sg {

constexpr int MC_BLOCK = 128;
constexpr int MC_WARPS = MC_BLOCK / 32;

// Tangent staging pitch in doubles (36 -> 37 keeps 8-byte smem accesses conflict-free).
constexpr int DS3_PITCH = 37;
constexpr int S3_PITCH = 7;

template <bool WANT_DS, bool FUSED_REDUCTION>
__global__ void __launch_bounds__(MC_BLOCK) k_mc3d(const double *__restrict__ E, const double *__restrict__ m0,
                                                    const double *__restrict__ m1, const double *__restrict__ psi,
                                                    const double *__restrict__ shear, const double *__restrict__ lame,
                                                    double lambda, char davis, int64_t n, double *__restrict__ S,
                                                    double *__restrict__ DS, uint8_t *__restrict__ branch) {
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *sds = smem + warp * (32 * DS3_PITCH);
    double *ss = smem + MC_WARPS * 32 * DS3_PITCH + warp * (32 * S3_PITCH);
    const int64_t stride = (int64_t)gridDim.x * MC_BLOCK;
    for (int64_t base = ((int64_t)blockIdx.x * MC_WARPS + warp) * 32; base < n; base += stride) {
        const int64_t p = base + lane;
        const int cnt = (int)(n - base < 32 ? n - base : 32);
        // the warp's strains (6 consecutive doubles per point) arrive as one contiguous run,
        // staged through the S buffer instead of six loads with a 48-byte lane stride
        for (int idx = lane; idx < cnt * 6; idx += 32) {
            const int q = idx / 6, c = idx - q * 6;
            ss[q * S3_PITCH + c] = __ldcs(E + 6 * base + idx);
        }
        __syncwarp();
        double e[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) e[c] = ss[lane * S3_PITCH + c];
        __syncwarp();
        if (p < n) {
            double cb, sp;
            if (FUSED_REDUCTION) {
                davis_reduce(m0[p], m1[p], psi[p], lambda, davis, cb, sp);
            } else {
                cb = m0[p];
                sp = m1[p];
            }
            double s[6];
            const int b = mc3d_point<WANT_DS>(e, cb, sp, shear[p], lame[p], s, sds + lane * DS3_PITCH);
#pragma unroll
            for (int c = 0; c < 6; ++c) ss[lane * S3_PITCH + c] = s[c];
            if (branch) branch[p] = (uint8_t)b;
        }
        __syncwarp();
        for (int idx = lane; idx < cnt * 6; idx += 32) {
            const int q = idx / 6, c = idx - q * 6;
            S[6 * base + idx] = ss[q * S3_PITCH + c];
        }
        if (WANT_DS) {
            for (int idx = lane; idx < cnt * 36; idx += 32) {
                const int q = idx / 36, k = idx - q * 36;
                DS[36 * base + idx] = sds[q * DS3_PITCH + k];
            }
        }
        __syncwarp();
    }
}

constexpr int DS2_PITCH = 9;
constexpr int S2_PITCH = 5;

template <bool WANT_DS, bool FUSED_REDUCTION>
__global__ void __launch_bounds__(MC_BLOCK) k_mc2d(const double *__restrict__ E, const double *__restrict__ m0,
                                                    const double *__restrict__ m1, const double *__restrict__ psi,
                                                    const double *__restrict__ shear, const double *__restrict__ lame,
                                                    double lambda, char davis, int64_t n, double *__restrict__ S,
                                                    double *__restrict__ DS, uint8_t *__restrict__ branch) {
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *sds = smem + warp * (32 * DS2_PITCH);
    double *ss = smem + MC_WARPS * 32 * DS2_PITCH + warp * (32 * S2_PITCH);
    const int64_t stride = (int64_t)gridDim.x * MC_BLOCK;
    for (int64_t base = ((int64_t)blockIdx.x * MC_WARPS + warp) * 32; base < n; base += stride) {
        const int64_t p = base + lane;
        const int cnt = (int)(n - base < 32 ? n - base : 32);
        if (p < n) {
            const double e[3] = {E[3 * p], E[3 * p + 1], E[3 * p + 2]};
            double cb, sp;
            if (FUSED_REDUCTION) {
                davis_reduce(m0[p], m1[p], psi[p], lambda, davis, cb, sp);
            } else {
                cb = m0[p];
                sp = m1[p];
            }
            double s[4];
            const int b = mc2d_point<WANT_DS>(e, cb, sp, shear[p], lame[p], s, sds + lane * DS2_PITCH);
#pragma unroll
            for (int c = 0; c < 4; ++c) ss[lane * S2_PITCH + c] = s[c];
            if (branch) branch[p] = (uint8_t)b;
        }
        __syncwarp();
        for (int idx = lane; idx < cnt * 4; idx += 32) {
            const int q = idx / 4, c = idx - q * 4;
            S[4 * base + idx] = ss[q * S2_PITCH + c];
        }
        if (WANT_DS) {
            for (int idx = lane; idx < cnt * 9; idx += 32) {
                const int q = idx / 9, k = idx - q * 9;
                DS[9 * base + idx] = sds[q * DS2_PITCH + k];
            }
        }
        __syncwarp();
    }
}

__global__ void k_reduction(const double *__restrict__ c0, const double *__restrict__ phi,
                            const double *__restrict__ psi, double lambda, char davis, int64_t n,
                            double *__restrict__ c_bar, double *__restrict__ sin_phi) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        double cb, sp;
        davis_reduce(c0[p], phi[p], psi[p], lambda, davis, cb, sp);
        c_bar[p] = cb;
        sin_phi[p] = sp;
    }
}

// Launches one of the constitutive kernels.  For FUSED, m0/m1/psi are c0/phi/psi and
// (lambda, davis) select the reduction; otherwise m0/m1 are c_bar/sin_phi.
int launch_constitutive(int dim, bool fused, const double *E, const double *m0, const double *m1,
                        const double *psi, const double *shear, const double *lame, double lambda, char davis,
                        int64_t n, double *S, double *DS, uint8_t *branch, cudaStream_t st) {
    if (n <= 0) return SG_OK;
    const unsigned grid = grid_for(n, MC_BLOCK, 16);
    const InstrToken tk = instr_begin(DS ? IK_CONST_SDS : IK_CONST_S, st);
    if (dim == 3) {
        const size_t sm = sizeof(double) * MC_WARPS * 32 * (DS3_PITCH + S3_PITCH);
        if (DS) {
            if (fused) k_mc3d<true, true><<<grid, MC_BLOCK, sm, st>>>(E, m0, m1, psi, shear, lame, lambda, davis, n, S, DS, branch);
            else k_mc3d<true, false><<<grid, MC_BLOCK, sm, st>>>(E, m0, m1, psi, shear, lame, lambda, davis, n, S, DS, branch);
        } else {
            if (fused) k_mc3d<false, true><<<grid, MC_BLOCK, sm, st>>>(E, m0, m1, psi, shear, lame, lambda, davis, n, S, DS, branch);
            else k_mc3d<false, false><<<grid, MC_BLOCK, sm, st>>>(E, m0, m1, psi, shear, lame, lambda, davis, n, S, DS, branch);
        }
    } else {
        const size_t sm = sizeof(double) * MC_WARPS * 32 * (DS2_PITCH + S2_PITCH);
        if (DS) {
            if (fused) k_mc2d<true, true><<<grid, MC_BLOCK, sm, st>>>(E, m0, m1, psi, shear, lame, lambda, davis, n, S, DS, branch);
            else k_mc2d<true, false><<<grid, MC_BLOCK, sm, st>>>(E, m0, m1, psi, shear, lame, lambda, davis, n, S, DS, branch);
        } else {
            if (fused) k_mc2d<false, true><<<grid, MC_BLOCK, sm, st>>>(E, m0, m1, psi, shear, lame, lambda, davis, n, S, DS, branch);
            else k_mc2d<false, false><<<grid, MC_BLOCK, sm, st>>>(E, m0, m1, psi, shear, lame, lambda, davis, n, S, DS, branch);
        }
    }
    instr_end(tk, st);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

// Host-buffer path: pipelined over chunks on two streams so that the host->device copy of
// chunk i+1 and the device->host copy of chunk i-1 overlap the kernel of chunk i.
static int constitutive_host(int dim, const double *E, const double *c_bar, const double *sin_phi,
                             const double *shear, const double *lame, int64_t n, double *S, double *DS,
                             uint8_t *branch) {
    SG_CHECK_ARG(n >= 0, "n_int must be >= 0");
    if (n == 0) return SG_OK;
    SG_CHECK_ARG(E && c_bar && sin_phi && shear && lame && S, "null input/output pointer");
    const int ns_in = dim == 3 ? 6 : 3, ns_out = dim == 3 ? 6 : 4, nds = dim == 3 ? 36 : 9;
    const size_t per_pt = sizeof(double) * (ns_in + 4 + ns_out + (DS ? nds : 0)) + (branch ? 1 : 0);
    const int64_t chunk = std::max<int64_t>(1 << 16, std::min<int64_t>(n, (int64_t)(256u << 20) / (int64_t)per_pt));
    const int nbuf = 2;
    static thread_local Scratch scratch;
    const size_t buf_bytes = (size_t)chunk * per_pt + 8 * 256;
    int rc = scratch.reserve(buf_bytes * nbuf);
    if (rc) return rc;
    cudaStream_t st[2];
    SG_CUDA(cudaStreamCreateWithFlags(&st[0], cudaStreamNonBlocking));
    SG_CUDA(cudaStreamCreateWithFlags(&st[1], cudaStreamNonBlocking));
    int status = SG_OK;
    for (int64_t off = 0, it = 0; off < n && status == SG_OK; off += chunk, ++it) {
        const int64_t m = std::min(chunk, n - off);
        const int b = (int)(it % nbuf);
        char *base = (char *)scratch.ptr + b * buf_bytes;
        auto carve = [&](size_t bytes) { char *p = base; base += (bytes + 255) & ~size_t(255); return p; };
        double *dE = (double *)carve(sizeof(double) * ns_in * m);
        double *dcb = (double *)carve(sizeof(double) * m);
        double *dsp = (double *)carve(sizeof(double) * m);
        double *dG = (double *)carve(sizeof(double) * m);
        double *dL = (double *)carve(sizeof(double) * m);
        double *dS = (double *)carve(sizeof(double) * ns_out * m);
        double *dDS = DS ? (double *)carve(sizeof(double) * nds * m) : nullptr;
        uint8_t *dbr = branch ? (uint8_t *)carve(m) : nullptr;
        cudaStream_t s = st[b];
        cudaError_t e = cudaSuccess;
        e = e ? e : cudaMemcpyAsync(dE, E + ns_in * off, sizeof(double) * ns_in * m, cudaMemcpyHostToDevice, s);
        e = e ? e : cudaMemcpyAsync(dcb, c_bar + off, sizeof(double) * m, cudaMemcpyHostToDevice, s);
        e = e ? e : cudaMemcpyAsync(dsp, sin_phi + off, sizeof(double) * m, cudaMemcpyHostToDevice, s);
        e = e ? e : cudaMemcpyAsync(dG, shear + off, sizeof(double) * m, cudaMemcpyHostToDevice, s);
        e = e ? e : cudaMemcpyAsync(dL, lame + off, sizeof(double) * m, cudaMemcpyHostToDevice, s);
        if (e) { status = cuda_error(e, "host->device copy"); break; }
        status = launch_constitutive(dim, false, dE, dcb, dsp, nullptr, dG, dL, 1.0, 'B', m, dS, dDS, dbr, s);
        if (status) break;
        e = cudaMemcpyAsync(S + ns_out * off, dS, sizeof(double) * ns_out * m, cudaMemcpyDeviceToHost, s);
        if (!e && DS) e = cudaMemcpyAsync(DS + nds * off, dDS, sizeof(double) * nds * m, cudaMemcpyDeviceToHost, s);
        if (!e && branch) e = cudaMemcpyAsync(branch + off, dbr, m, cudaMemcpyDeviceToHost, s);
        if (e) { status = cuda_error(e, "device->host copy"); break; }
    }
    cudaError_t e0 = cudaStreamSynchronize(st[0]);
    cudaError_t e1 = cudaStreamSynchronize(st[1]);
    cudaStreamDestroy(st[0]);
    cudaStreamDestroy(st[1]);
    if (status) return status;
    if (e0) return cuda_error(e0, "constitutive stream 0");
    if (e1) return cuda_error(e1, "constitutive stream 1");
    return SG_OK;
}

}  // namespace sg

using namespace sg;

extern "C" int sg_constitutive3d(const double *E, const double *c_bar, const double *sin_phi, const double *shear,
                                 const double *bulk, const double *lame, int64_t n_int, double *S, double *DS,
                                 uint8_t *branch) {
    (void)bulk;
    return constitutive_host(3, E, c_bar, sin_phi, shear, lame, n_int, S, DS, branch);
}

extern "C" int sg_constitutive2d(const double *E, const double *c_bar, const double *sin_phi, const double *shear,
                                 const double *bulk, const double *lame, int64_t n_int, double *S, double *DS,
                                 uint8_t *branch) {
    (void)bulk;
    return constitutive_host(2, E, c_bar, sin_phi, shear, lame, n_int, S, DS, branch);
}

extern "C" int sg_constitutive3d_dev(const double *E, const double *c_bar, const double *sin_phi,
                                     const double *shear, const double *bulk, const double *lame, int64_t n_int,
                                     double *S, double *DS, uint8_t *branch, void *stream) {
    (void)bulk;
    SG_CHECK_ARG(n_int >= 0, "n_int must be >= 0");
    if (n_int == 0) return SG_OK;
    SG_CHECK_ARG(E && c_bar && sin_phi && shear && lame && S, "null device pointer");
    return launch_constitutive(3, false, E, c_bar, sin_phi, nullptr, shear, lame, 1.0, 'B', n_int, S, DS, branch,
                               as_stream(stream));
}

extern "C" int sg_constitutive2d_dev(const double *E, const double *c_bar, const double *sin_phi,
                                     const double *shear, const double *bulk, const double *lame, int64_t n_int,
                                     double *S, double *DS, uint8_t *branch, void *stream) {
    (void)bulk;
    SG_CHECK_ARG(n_int >= 0, "n_int must be >= 0");
    if (n_int == 0) return SG_OK;
    SG_CHECK_ARG(E && c_bar && sin_phi && shear && lame && S, "null device pointer");
    return launch_constitutive(2, false, E, c_bar, sin_phi, nullptr, shear, lame, 1.0, 'B', n_int, S, DS, branch,
                               as_stream(stream));
}

// Per-block partial sums of weight * Psi; the host adds them in block order (deterministic).
template <int DIM>
__global__ void __launch_bounds__(256) k_potential(const double *__restrict__ E, const double *__restrict__ c_bar,
                                                   const double *__restrict__ sin_phi,
                                                   const double *__restrict__ shear, const double *__restrict__ bulk,
                                                   const double *__restrict__ lame,
                                                   const double *__restrict__ weight, int64_t n,
                                                   double *__restrict__ part) {
    constexpr int NS = DIM == 3 ? 6 : 3;
    __shared__ double sh[256 / 32];
    double acc = 0.0;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        double e[NS];
#pragma unroll
        for (int c = 0; c < NS; ++c) e[c] = E[NS * p + c];
        const double psi = DIM == 3 ? potential3d(e, c_bar[p], sin_phi[p], shear[p], bulk[p], lame[p])
                                    : potential2d(e, c_bar[p], sin_phi[p], shear[p], bulk[p], lame[p]);
        acc += weight[p] * psi;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        part[blockIdx.x] = t;
    }
}

extern "C" int sg_reduction_dev(const double *c0, const double *phi, const double *psi, double lambda,
                                char davis_type, int64_t n, double *c_bar, double *sin_phi, void *stream) {
    SG_CHECK_ARG(n >= 0, "n must be >= 0");
    SG_CHECK_ARG(davis_type == 'A' || davis_type == 'B' || davis_type == 'C', "Davis type must be 'A', 'B' or 'C'");
    SG_CHECK_ARG(lambda > 0.0, "lambda must be positive");
    if (n == 0) return SG_OK;
    SG_CHECK_ARG(c0 && phi && psi && c_bar && sin_phi, "null device pointer");
    k_reduction<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(c0, phi, psi, lambda, davis_type, n, c_bar, sin_phi);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

// Integrated potential sum_p weight[p] * Psi(E_p) (CONSTITUTIVE.m:363-387 with potential_3D.m /
// potential_2D.m).  Device arrays; the result is returned to the host (synchronises stream).
extern "C" int sg_potential_dev(int dim, const double *E, const double *c_bar, const double *sin_phi,
                                const double *shear, const double *bulk, const double *lame, const double *weight,
                                int64_t n_int, double *result, void *stream) {
    SG_CHECK_ARG(dim == 2 || dim == 3, "dim must be 2 or 3");
    SG_CHECK_ARG(n_int >= 0 && result, "bad argument");
    *result = 0.0;
    if (n_int == 0) return SG_OK;
    SG_CHECK_ARG(E && c_bar && sin_phi && shear && bulk && lame && weight, "null device pointer");
    constexpr int NBLK = 296;
    static thread_local Scratch ws;
    int rc = ws.reserve(sizeof(double) * NBLK);
    if (rc) return rc;
    const cudaStream_t st = as_stream(stream);
    const unsigned grid = (unsigned)std::min<int64_t>(NBLK, (n_int + 255) / 256);
    count_launch();
    if (dim == 3) k_potential<3><<<grid, 256, 0, st>>>(E, c_bar, sin_phi, shear, bulk, lame, weight, n_int, (double *)ws.ptr);
    else k_potential<2><<<grid, 256, 0, st>>>(E, c_bar, sin_phi, shear, bulk, lame, weight, n_int, (double *)ws.ptr);
    SG_CUDA(cudaGetLastError());
    double part[NBLK];
    SG_CUDA(cudaMemcpyAsync(part, ws.ptr, sizeof(double) * grid, cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    double t = 0.0;
    for (unsigned b = 0; b < grid; ++b) t += part[b];
    *result = t;
    return SG_OK;
}
