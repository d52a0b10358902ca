// (b3, b5) Drop-in element tangent assembly with the reference's scatter map.
//
// Same contract as +ASSEMBLY/mex/assemble_K_tangent_vals.c:38-172 (3D) and
// assemble_K_tangent_vals_2D.c:31-165 (2D): V[map-1] += (sum_q B_q'(w_q D_q)B_q)_loc, map is
// 1-based int64 with 0 = skip.  One CTA per element: the element's gradients and weighted
// tangents are staged in shared memory, D*B is formed once per point and shared by all
// local columns, and each thread owns local entries (r, c) of the element matrix, which it
// adds to V with one atomic each.  The general (non-symmetric) product is formed, so the
// result does not depend on DS being symmetric.
//
// Map entries beyond nnz_out are skipped and flagged; the call then returns SG_ERR_ARG.
#include <cuda_runtime.h>

#include <algorithm>

#include "sg_common.cuh"

namespace sg {

template <int DIM>
__device__ __forceinline__ int bcol_nz(const double *dphi_q, int np, int c, int rows[3], double vals[3]) {
    // column c = DIM*i + comp of the local strain-displacement matrix at one point;
    // dphi_q[d*np + i] holds dN_i/dx_d.
    const int i = c / DIM, comp = c - i * DIM;
    const double d1 = dphi_q[i], d2 = dphi_q[np + i];
    if (DIM == 3) {
        const double d3 = dphi_q[2 * np + i];
        if (comp == 0) { rows[0] = 0; vals[0] = d1; rows[1] = 3; vals[1] = d2; rows[2] = 5; vals[2] = d3; }
        else if (comp == 1) { rows[0] = 1; vals[0] = d2; rows[1] = 3; vals[1] = d1; rows[2] = 4; vals[2] = d3; }
        else { rows[0] = 2; vals[0] = d3; rows[1] = 4; vals[1] = d2; rows[2] = 5; vals[2] = d1; }
        return 3;
    } else {
        if (comp == 0) { rows[0] = 0; vals[0] = d1; rows[1] = 2; vals[1] = d2; }
        else { rows[0] = 1; vals[0] = d2; rows[1] = 2; vals[1] = d1; }
        return 2;
    }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_assemble_general(const double *__restrict__ DPhi1, const double *__restrict__ DPhi2,
                                                          const double *__restrict__ DPhi3, const double *__restrict__ DS,
                                                          const double *__restrict__ W, const int64_t *__restrict__ smap,
                                                          int np, int nq, int64_t ne, int64_t nnz, double *__restrict__ V,
                                                          int *__restrict__ bad_index) {
    constexpr int NS = DIM == 3 ? 6 : 3;
    extern __shared__ double sh[];
    const int nl = DIM * np;
    double *dphi = sh;                   // [q][d][i]
    double *D = dphi + nq * DIM * np;    // [q][a + NS*b], weighted
    double *DB = D + nq * NS * NS;       // [q][a + NS*c]
    for (int64_t e = blockIdx.x; e < ne; e += gridDim.x) {
        const int64_t g0 = e * nq;
        for (int idx = threadIdx.x; idx < nq * np; idx += blockDim.x) {
            const int q = idx / np, i = idx - q * np;
            dphi[(q * DIM + 0) * np + i] = DPhi1[g0 * np + idx];
            dphi[(q * DIM + 1) * np + i] = DPhi2[g0 * np + idx];
            if (DIM == 3) dphi[(q * DIM + 2) * np + i] = DPhi3[g0 * np + idx];
        }
        for (int idx = threadIdx.x; idx < nq * NS * NS; idx += blockDim.x) {
            const int q = idx / (NS * NS);
            D[idx] = W[g0 + q] * DS[g0 * NS * NS + idx];
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < nq * NS * nl; idx += blockDim.x) {
            const int q = idx / (NS * nl), rem = idx - q * NS * nl;
            const int c = rem / NS, a = rem - c * NS;
            int rows[3];
            double vals[3];
            const int k = bcol_nz<DIM>(dphi + q * DIM * np, np, c, rows, vals);
            double s = 0.0;
            for (int t = 0; t < k; ++t) s += D[q * NS * NS + a + NS * rows[t]] * vals[t];
            DB[q * NS * nl + a + NS * c] = s;
        }
        __syncthreads();
        const int64_t *m_e = smap + e * (int64_t)nl * nl;
        for (int idx = threadIdx.x; idx < nl * nl; idx += blockDim.x) {
            const int64_t m = m_e[idx];
            if (m <= 0) continue;
            if (m > nnz) {
                atomicExch(bad_index, 1);
                continue;
            }
            const int c = idx / nl, r = idx - c * nl;
            double s = 0.0;
            for (int q = 0; q < nq; ++q) {
                int rows[3];
                double vals[3];
                const int k = bcol_nz<DIM>(dphi + q * DIM * np, np, r, rows, vals);
                for (int t = 0; t < k; ++t) s += vals[t] * DB[q * NS * nl + rows[t] + NS * c];
            }
            atomicAdd(&V[m - 1], s);
        }
        __syncthreads();
    }
}

static size_t general_smem(int dim, int np, int nq) {
    const int ns = dim == 3 ? 6 : 3;
    return sizeof(double) * ((size_t)nq * dim * np + (size_t)nq * ns * ns + (size_t)nq * ns * dim * np);
}

static int launch_general(int dim, const double *D1, const double *D2, const double *D3, const double *DS,
                          const double *W, const int64_t *smap, int np, int nq, int64_t ne, int64_t nnz, double *V,
                          int *flag, cudaStream_t st) {
    if (ne <= 0) return SG_OK;
    const size_t sm = general_smem(dim, np, nq);
    const unsigned grid = (unsigned)std::min<int64_t>(ne, (int64_t)sm_count() * 16);
    count_launch();
    if (dim == 3) {
        if (sm > 48 * 1024) SG_CUDA(cudaFuncSetAttribute(k_assemble_general<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_assemble_general<3><<<grid, 256, sm, st>>>(D1, D2, D3, DS, W, smap, np, nq, ne, nnz, V, flag);
    } else {
        if (sm > 48 * 1024) SG_CUDA(cudaFuncSetAttribute(k_assemble_general<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_assemble_general<2><<<grid, 256, sm, st>>>(D1, D2, D3, DS, W, smap, np, nq, ne, nnz, V, flag);
    }
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

static int check_sizes(int dim, int np, int64_t n_int, int64_t ne, int nq, int64_t nnz) {
    SG_CHECK_ARG(np > 0 && np <= 32, "n_p must be in 1..32");
    SG_CHECK_ARG(nq > 0 && nq <= 64, "n_q must be in 1..64");
    SG_CHECK_ARG(ne >= 0 && nnz >= 0, "negative size");
    SG_CHECK_ARG(n_int == ne * (int64_t)nq, "n_int must equal n_e * n_q");
    SG_CHECK_ARG(general_smem(dim, np, nq) <= 200 * 1024, "element too large for shared-memory staging");
    return SG_OK;
}

// Host-buffer assembly: V resident on the device, inputs streamed in element chunks on two
// streams (copies of one chunk overlap the kernel of the other).
static int assemble_host(int dim, const double *D1, const double *D2, const double *D3, const double *DS,
                         const double *W, const int64_t *smap, int np, int64_t n_int, int64_t ne, int nq,
                         int64_t nnz, double *V) {
    int rc = check_sizes(dim, np, n_int, ne, nq, nnz);
    if (rc) return rc;
    SG_CHECK_ARG(V || nnz == 0, "null V_tang");
    if (nnz == 0) return SG_OK;
    SG_CHECK_ARG(ne == 0 || (D1 && D2 && DS && W && smap && (dim == 2 || D3)), "null input pointer");
    const int ns = dim == 3 ? 6 : 3, nl = dim * np;
    const size_t per_elem = sizeof(double) * ((size_t)nq * (dim * np + ns * ns + 1)) + sizeof(int64_t) * nl * nl;
    const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(std::max<int64_t>(ne, 1), (int64_t)(192u << 20) / (int64_t)per_elem));
    static thread_local Scratch scratch;
    const size_t buf_bytes = (size_t)chunk * per_elem + 8 * 256;
    const size_t v_bytes = ((sizeof(double) * nnz + 255) & ~size_t(255)) + 256;
    rc = scratch.reserve(v_bytes + 2 * buf_bytes);
    if (rc) return rc;
    double *dV = (double *)scratch.ptr;
    int *dflag = (int *)((char *)scratch.ptr + v_bytes - 256);
    cudaStream_t st[2];
    SG_CUDA(cudaStreamCreateWithFlags(&st[0], cudaStreamNonBlocking));
    SG_CUDA(cudaStreamCreateWithFlags(&st[1], cudaStreamNonBlocking));
    cudaEvent_t zeroed;
    SG_CUDA(cudaEventCreateWithFlags(&zeroed, cudaEventDisableTiming));
    int status = SG_OK;
    cudaError_t e = cudaMemsetAsync(dV, 0, v_bytes, st[0]);
    if (!e) e = cudaEventRecord(zeroed, st[0]);
    if (!e) e = cudaStreamWaitEvent(st[1], zeroed, 0);
    if (e) status = cuda_error(e, "zero V");
    for (int64_t off = 0, it = 0; off < ne && status == SG_OK; off += chunk, ++it) {
        const int64_t m = std::min(chunk, ne - off);
        const int b = (int)(it & 1);
        char *base = (char *)scratch.ptr + v_bytes + b * buf_bytes;
        auto carve = [&](size_t bytes) { char *p = base; base += (bytes + 255) & ~size_t(255); return p; };
        const size_t nd = (size_t)m * nq * np, nds = (size_t)m * nq * ns * ns;
        double *d1 = (double *)carve(sizeof(double) * nd);
        double *d2 = (double *)carve(sizeof(double) * nd);
        double *d3 = dim == 3 ? (double *)carve(sizeof(double) * nd) : nullptr;
        double *dds = (double *)carve(sizeof(double) * nds);
        double *dw = (double *)carve(sizeof(double) * m * nq);
        int64_t *dm = (int64_t *)carve(sizeof(int64_t) * (size_t)m * nl * nl);
        const size_t g0 = (size_t)off * nq;
        cudaStream_t s = st[b];
        e = cudaMemcpyAsync(d1, D1 + g0 * np, sizeof(double) * nd, cudaMemcpyHostToDevice, s);
        if (!e) e = cudaMemcpyAsync(d2, D2 + g0 * np, sizeof(double) * nd, cudaMemcpyHostToDevice, s);
        if (!e && dim == 3) e = cudaMemcpyAsync(d3, D3 + g0 * np, sizeof(double) * nd, cudaMemcpyHostToDevice, s);
        if (!e) e = cudaMemcpyAsync(dds, DS + g0 * ns * ns, sizeof(double) * nds, cudaMemcpyHostToDevice, s);
        if (!e) e = cudaMemcpyAsync(dw, W + g0, sizeof(double) * m * nq, cudaMemcpyHostToDevice, s);
        if (!e) e = cudaMemcpyAsync(dm, smap + (size_t)off * nl * nl, sizeof(int64_t) * (size_t)m * nl * nl, cudaMemcpyHostToDevice, s);
        if (e) { status = cuda_error(e, "host->device copy"); break; }
        status = launch_general(dim, d1, d2, d3, dds, dw, dm, np, nq, m, nnz, dV, dflag, s);
    }
    cudaError_t e0 = cudaStreamSynchronize(st[0]);
    cudaError_t e1 = cudaStreamSynchronize(st[1]);
    int flag = 0;
    if (status == SG_OK && !e0 && !e1) {
        e = cudaMemcpy(V, dV, sizeof(double) * nnz, cudaMemcpyDeviceToHost);
        if (!e) e = cudaMemcpy(&flag, dflag, sizeof(int), cudaMemcpyDeviceToHost);
        if (e) status = cuda_error(e, "device->host copy");
    }
    cudaEventDestroy(zeroed);
    cudaStreamDestroy(st[0]);
    cudaStreamDestroy(st[1]);
    if (status) return status;
    if (e0) return cuda_error(e0, "assembly stream 0");
    if (e1) return cuda_error(e1, "assembly stream 1");
    if (flag) return set_error(SG_ERR_ARG, "scatter_map holds an index larger than nnz_out");
    return SG_OK;
}

}  // namespace sg

using namespace sg;

extern "C" int sg_assemble_ktangent3d(const double *DPhi1, const double *DPhi2, const double *DPhi3, const double *DS,
                                      const double *WEIGHT, const int64_t *scatter_map, int32_t n_p, int64_t n_int,
                                      int64_t n_e, int32_t n_q, int64_t nnz_out, double *V_tang) {
    return assemble_host(3, DPhi1, DPhi2, DPhi3, DS, WEIGHT, scatter_map, n_p, n_int, n_e, n_q, nnz_out, V_tang);
}

extern "C" int sg_assemble_ktangent2d(const double *DPhi1, const double *DPhi2, const double *DS, const double *WEIGHT,
                                      const int64_t *scatter_map, int32_t n_p, int64_t n_int, int64_t n_e, int32_t n_q,
                                      int64_t nnz_out, double *V_tang) {
    return assemble_host(2, DPhi1, DPhi2, nullptr, DS, WEIGHT, scatter_map, n_p, n_int, n_e, n_q, nnz_out, V_tang);
}

// Device variant: V_tang is zeroed and accumulated on `stream`; an index beyond nnz_out
// is skipped (checked by the host-buffer variant only).
extern "C" int sg_assemble_ktangent_dev(int dim, const double *DPhi1, const double *DPhi2, const double *DPhi3,
                                        const double *DS, const double *WEIGHT, const int64_t *scatter_map,
                                        int32_t n_p, int64_t n_e, int32_t n_q, int64_t nnz_out, double *V_tang,
                                        void *stream) {
    SG_CHECK_ARG(dim == 2 || dim == 3, "dim must be 2 or 3");
    int rc = check_sizes(dim, n_p, n_e * (int64_t)n_q, n_e, n_q, nnz_out);
    if (rc) return rc;
    if (nnz_out == 0) return SG_OK;
    SG_CHECK_ARG(V_tang, "null V_tang");
    cudaStream_t st = as_stream(stream);
    static thread_local Scratch flag_buf;
    rc = flag_buf.reserve(256);
    if (rc) return rc;
    SG_CUDA(cudaMemsetAsync(V_tang, 0, sizeof(double) * nnz_out, st));
    return launch_general(dim, DPhi1, DPhi2, DPhi3, DS, WEIGHT, scatter_map, n_p, n_q, n_e, nnz_out, V_tang,
                          (int *)flag_buf.ptr, st);
}
