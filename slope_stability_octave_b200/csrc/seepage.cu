// Unconfined seepage (pore pressure) on the mechanical mesh: the device side of the
// reference's SEEPAGE package.
//
//   k_seepage_system     per element and local node: one row of the element tangent of the
//                        penalised Darcy problem, K_D + Bw' E C (newton_flow.m:104-118), and
//                        one entry of the residual f = -Bw'(wc .* (Bw pw + grho kappa .* q2))
//                        (newton_flow.m:120-123, seepage_problem_3D.m:42-46), scattered into
//                        the mesh's node adjacency with 1 x 1 blocks and into a node vector
//   k_point_gradient     Bw * field per integration point (q2 = Bw y, grad_p = Bw pw;
//                        seepage_problem_3D.m:43,62)
//   k_seepage_saturation element mean of the pressure at the integration points and the
//                        saturation flag pw_aver_e >= 0.1 eps (seepage_problem_3D.m:63-74)
//   k_scalar_dirichlet   identity rows and columns of the Dirichlet nodes: the Krylov solve
//                        on the full node vector then equals the reference's K(Q_w, Q_w)
//
// Relative permeability (newton_flow.m:92-99): perm_r = 1 where pw_int >= eps, pw_int / eps
// for 0 < pw_int < eps, 0 for pw_int <= 0; its derivative 1 / eps on the middle piece only.
// The per-element penalty eps (penalty_parameters_3D.m) and the conductivity per point come
// from the host set-up.  Element contributions are added with FP64 atomics (the order of
// the additions, and so the last bits of the sums, can differ between runs).

#include <cuda_runtime.h>

#include "mesh.h"
#include "sg_common.cuh"

namespace sg {

// kappa_mode: 0 -> kappa = 0 (2D initial right-hand side), 1 -> kappa = 1 (3D initial
// right-hand side), 2 -> kappa = perm_r(pw_int) with the Newton tangent's E term
template <int DIM, int NP>
__global__ void __launch_bounds__(256) k_seepage_system(int64_t n_e, int nq, const int32_t *__restrict__ elem,
                                                        const double *__restrict__ dphi,
                                                        const double *__restrict__ w,
                                                        const double *__restrict__ hat,
                                                        const double *__restrict__ pw,
                                                        const double *__restrict__ conduct,
                                                        const double *__restrict__ eps,
                                                        const double *__restrict__ gy, double grho,
                                                        int kappa_mode, const int32_t *__restrict__ pair_blk,
                                                        double *__restrict__ K, double *__restrict__ F) {
    const int64_t total = n_e * NP;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t / NP;
        const int a = (int)(t - e * NP);
        double pe[NP];
#pragma unroll
        for (int i = 0; i < NP; ++i) pe[i] = __ldg(pw + __ldg(elem + e * NP + i));
        double ka[NP];
#pragma unroll
        for (int b = 0; b < NP; ++b) ka[b] = 0.0;
        double fa = 0.0;
        const double ep = __ldg(eps + e);
        for (int q = 0; q < nq; ++q) {
            const int64_t g = e * nq + q;
            const double *D = dphi + g * DIM * NP;
            const double *H = hat + (int64_t)q * NP;   // HatP(:, q)
            double pint = 0.0;
#pragma unroll
            for (int i = 0; i < NP; ++i) pint += __ldg(H + i) * pe[i];
            double perm = 1.0, der = 0.0;
            if (pint < ep && pint > 0.0) {
                perm = pint / ep;
                der = 1.0 / ep;
            } else if (pint <= 0.0) {
                perm = 0.0;
            }
            const double kappa = kappa_mode == 0 ? 0.0 : (kappa_mode == 1 ? 1.0 : perm);
            const double cg = __ldg(conduct + g), wg = __ldg(w + g);
            const double wc = wg * cg;
            double da[DIM], q3[DIM], gyg[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                double s = 0.0;
#pragma unroll
                for (int i = 0; i < NP; ++i) s += __ldg(D + d * NP + i) * pe[i];
                gyg[d] = __ldg(gy + g * DIM + d);
                q3[d] = s + grho * kappa * gyg[d];
                da[d] = __ldg(D + d * NP + a);
            }
            double dq = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) dq += da[d] * q3[d];
            fa -= wc * dq;
            if (K) {
                // K_D: wc * grad(phi_a) . grad(phi_b)
#pragma unroll
                for (int b = 0; b < NP; ++b) {
                    double s = 0.0;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) s += da[d] * __ldg(D + d * NP + b);
                    ka[b] += wc * s;
                }
                // Bw' E C: (grad(phi_a) . vE) phi_b, vE = conduct * perm_r' * weight * grho * (Bw y)
                if (kappa_mode == 2 && der != 0.0) {
                    const double ce = cg * der * wg;
                    double s = 0.0;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) s += da[d] * (ce * (grho * gyg[d]));
#pragma unroll
                    for (int b = 0; b < NP; ++b) ka[b] += s * __ldg(H + b);
                }
            }
        }
        if (F) atomicAdd(F + __ldg(elem + e * NP + a), fa);
        if (K) {
            const int32_t *pb = pair_blk + (e * NP + a) * NP;
#pragma unroll
            for (int b = 0; b < NP; ++b) atomicAdd(K + __ldg(pb + b), ka[b]);
        }
    }
}

template <int DIM, int NP>
__global__ void k_point_gradient(int64_t n_int, int nq, const int32_t *__restrict__ elem,
                                 const double *__restrict__ dphi, const double *__restrict__ field,
                                 double *__restrict__ out) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_int;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = g / nq;
        double v[NP];
#pragma unroll
        for (int i = 0; i < NP; ++i) v[i] = __ldg(field + __ldg(elem + e * NP + i));
        const double *D = dphi + g * DIM * NP;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < NP; ++i) s += __ldg(D + d * NP + i) * v[i];
            out[g * DIM + d] = s;
        }
    }
}

template <int NP>
__global__ void k_seepage_saturation(int64_t n_e, int nq, const int32_t *__restrict__ elem,
                                     const double *__restrict__ w, const double *__restrict__ hat,
                                     const double *__restrict__ pw, const double *__restrict__ eps,
                                     double *__restrict__ mean, uint8_t *__restrict__ sat) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_e;
         e += (int64_t)gridDim.x * blockDim.x) {
        double pe[NP];
#pragma unroll
        for (int i = 0; i < NP; ++i) pe[i] = __ldg(pw + __ldg(elem + e * NP + i));
        double num = 0.0, den = 0.0, only = 0.0;
        for (int q = 0; q < nq; ++q) {
            double pint = 0.0;
#pragma unroll
            for (int i = 0; i < NP; ++i) pint += __ldg(hat + (int64_t)q * NP + i) * pe[i];
            const double wg = __ldg(w + e * nq + q);
            num += pint * wg;
            den += wg;
            only = pint;
        }
        const double m = nq > 1 ? num / den : only;
        if (mean) mean[e] = m;
        if (sat) sat[e] = m >= 0.1 * __ldg(eps + e) ? 1 : 0;
    }
}

__global__ void k_scalar_dirichlet(int64_t n_blocks, const int32_t *__restrict__ row_of,
                                   const int32_t *__restrict__ col, const double *__restrict__ mask,
                                   double *__restrict__ K) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n_blocks;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r = __ldg(row_of + p), c = __ldg(col + p);
        if (__ldg(mask + r) == 0.0 || __ldg(mask + c) == 0.0) K[p] = (r == c) ? 1.0 : 0.0;
    }
}

__global__ void k_mask_vector(int64_t n, const double *__restrict__ mask, double *__restrict__ v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (__ldg(mask + i) == 0.0) v[i] = 0.0;
}

}  // namespace sg

using namespace sg;

#define SG_NP_DISPATCH(DIMV, NPV, BODY)                                              \
    if ((DIMV) == 3 && (NPV) == 10) { [[maybe_unused]] constexpr int DD = 3, PP = 10; BODY; }         \
    else if ((DIMV) == 3 && (NPV) == 4) { [[maybe_unused]] constexpr int DD = 3, PP = 4; BODY; }      \
    else if ((DIMV) == 2 && (NPV) == 6) { [[maybe_unused]] constexpr int DD = 2, PP = 6; BODY; }      \
    else if ((DIMV) == 2 && (NPV) == 3) { [[maybe_unused]] constexpr int DD = 2, PP = 3; BODY; }      \
    else return set_error(SG_ERR_ARG, "seepage: supported elements are P1/P2 triangles and tetrahedra");

extern "C" int sg_mesh_bsr_scalar(sg_mesh *m, const sg_bsr **bsr) {
    SG_CHECK_ARG(m && bsr, "null argument");
    if (!m->bsr1_ready) {
        sg_bsr &S = m->bsr1;
        const sg_bsr &B = m->bsr;
        S.b = 1;
        S.n_rows = B.n_rows;
        S.n_blocks = B.n_blocks;
        S.row_ptr = B.row_ptr;
        S.col = B.col;
        S.d_row_ptr = B.d_row_ptr;
        S.d_col = B.d_col;
        S.d_diag = B.d_diag;
        S.d_transpose = B.d_transpose;
        S.d_row_of = B.d_row_of;
        S.owned_by_mesh = 1;
        m->bsr1_ready = true;
    }
    *bsr = &m->bsr1;
    return SG_OK;
}

extern "C" int sg_seepage_system_dev(const sg_mesh *m, const double *hat, const double *pw, const double *conduct,
                                     const double *eps, const double *gy, double grho, int32_t kappa_mode,
                                     const double *mask, double *K, double *F, void *stream) {
    SG_CHECK_ARG(m && hat && pw && conduct && eps && gy, "null input pointer");
    SG_CHECK_ARG(kappa_mode >= 0 && kappa_mode <= 2, "kappa_mode must be 0, 1 or 2");
    SG_CHECK_ARG(K || F, "nothing to compute (K and F both null)");
    cudaStream_t st = as_stream(stream);
    if (K) SG_CUDA(cudaMemsetAsync(K, 0, sizeof(double) * m->bsr.n_blocks, st));
    if (F) SG_CUDA(cudaMemsetAsync(F, 0, sizeof(double) * m->n_n, st));
    SG_NP_DISPATCH(m->dim, m->np, (k_seepage_system<DD, PP><<<grid_for(m->n_e * PP, 256), 256, 0, st>>>(
                                       m->n_e, m->nq, m->d_elem, m->d_dphi, m->d_w, hat, pw, conduct, eps, gy, grho,
                                       kappa_mode, m->d_pair_blk, K, F)));
    SG_CUDA(cudaGetLastError());
    if (mask) {
        if (K) k_scalar_dirichlet<<<grid_for(m->bsr.n_blocks, 256), 256, 0, st>>>(
                   m->bsr.n_blocks, m->bsr.d_row_of, m->bsr.d_col, mask, K);
        if (F) k_mask_vector<<<grid_for(m->n_n, 256), 256, 0, st>>>(m->n_n, mask, F);
        SG_CUDA(cudaGetLastError());
    }
    return SG_OK;
}

extern "C" int sg_point_gradient_dev(const sg_mesh *m, const double *field, double *grad, void *stream) {
    SG_CHECK_ARG(m && field && grad, "null argument");
    cudaStream_t st = as_stream(stream);
    SG_NP_DISPATCH(m->dim, m->np, (k_point_gradient<DD, PP><<<grid_for(m->n_int, 256), 256, 0, st>>>(
                                       m->n_int, m->nq, m->d_elem, m->d_dphi, field, grad)));
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

extern "C" int sg_seepage_saturation_dev(const sg_mesh *m, const double *hat, const double *pw, const double *eps,
                                         double *mean, uint8_t *sat, void *stream) {
    SG_CHECK_ARG(m && hat && pw && eps && (mean || sat), "null argument");
    cudaStream_t st = as_stream(stream);
    SG_NP_DISPATCH(m->dim, m->np, (k_seepage_saturation<PP><<<grid_for(m->n_e, 256), 256, 0, st>>>(
                                       m->n_e, m->nq, m->d_elem, m->d_w, hat, pw, eps, mean, sat)));
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}
