// (a5, a6, b1-b4) Element operators on the device-resident mesh.
//
//   strain     E = B U                        CONSTITUTIVE.m:218,251 (B of elastic_stiffness_matrix_3D.m:105-132)
//   force      F = B' (w .* S)                CONSTITUTIVE.m:268-285
//   assemble   K_t = sum_e sum_q B'(w D)B     assemble_K_tangent_vals.c:77-171, into the node-adjacency BSR
//   elastic_ds DS_elast                       CONSTITUTIVE.m:413-422 (2D IOTA quirk kept, see below)
//   kr_blend   K_r = sym(r K_el + (1-r) K_t)  CONSTITUTIVE.m:515-532, with Dirichlet rows/columns
//                                             replaced by identity so the full-DOF system has the
//                                             K(Q,Q) solution on the free DOFs
//   to_ref     K values in the reference's find() order (drop-in output of build_K_r_QQ_vals)
//
// Strain rows: 3D (e11, e22, e33, g12, g23, g13); 2D (e11, e22, g12).
#include <cuda_runtime.h>

#include <algorithm>

#include <vector>

#include "instr.cuh"
#include "mc_point.cuh"
#include "mesh.h"
#include "sg_common.cuh"

namespace sg {

template <int DIM>
__global__ void k_strain(const int32_t *__restrict__ elem, const double *__restrict__ dphi, int np, int nq,
                         int64_t n_int, const double *__restrict__ U, double *__restrict__ E) {
    constexpr int NS = DIM == 3 ? 6 : 3;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_int; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = g / nq;
        const double *d = dphi + g * DIM * np;
        double s[NS];
#pragma unroll
        for (int a = 0; a < NS; ++a) s[a] = 0.0;
        for (int i = 0; i < np; ++i) {
            const int64_t v = elem[e * np + i];
            const double d1 = d[i], d2 = d[np + i];
            if (DIM == 3) {
                const double d3 = d[2 * np + i];
                const double ux = U[3 * v], uy = U[3 * v + 1], uz = U[3 * v + 2];
                s[0] += d1 * ux;
                s[1] += d2 * uy;
                s[2] += d3 * uz;
                s[3] += d2 * ux + d1 * uy;
                s[4] += d3 * uy + d2 * uz;
                s[5] += d3 * ux + d1 * uz;
            } else {
                const double ux = U[2 * v], uy = U[2 * v + 1];
                s[0] += d1 * ux;
                s[1] += d2 * uy;
                s[2] += d2 * ux + d1 * uy;
            }
        }
#pragma unroll
        for (int a = 0; a < NS; ++a) E[g * NS + a] = s[a];
    }
}

// One thread per (element, local node): sums the element's quadrature points, then adds
// its dim force components with atomics (F must be zeroed first).
template <int DIM>
__global__ void k_force(const int32_t *__restrict__ elem, const double *__restrict__ dphi,
                        const double *__restrict__ w, int np, int nq, int64_t n_e, const double *__restrict__ S,
                        int s_rows, double *__restrict__ F) {
    const int64_t total = n_e * np;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t / np;
        const int i = (int)(t - e * np);
        double f[DIM];
#pragma unroll
        for (int c = 0; c < DIM; ++c) f[c] = 0.0;
        for (int q = 0; q < nq; ++q) {
            const int64_t g = e * nq + q;
            const double *d = dphi + g * DIM * np;
            const double *s = S + g * s_rows;
            const double wq = w[g];
            const double d1 = d[i], d2 = d[np + i];
            if (DIM == 3) {
                const double d3 = d[2 * np + i];
                f[0] += wq * (d1 * s[0] + d2 * s[3] + d3 * s[5]);
                f[1] += wq * (d2 * s[1] + d1 * s[3] + d3 * s[4]);
                f[2] += wq * (d3 * s[2] + d2 * s[4] + d1 * s[5]);
            } else {
                f[0] += wq * (d1 * s[0] + d2 * s[2]);
                f[1] += wq * (d2 * s[1] + d1 * s[2]);
            }
        }
        const int64_t v = elem[e * np + i];
#pragma unroll
        for (int c = 0; c < DIM; ++c) atomicAdd(&F[v * DIM + c], f[c]);
    }
}

// Fused stress-only residual of 3D P2 tetrahedra: F = B'(w S(B U)) with the return mapping
// in between (CONSTITUTIVE.build_F_all / build_F_reduced after the reduction: strain
// CONSTITUTIVE.m:218, stress constitutive_3D_kernel.h:101-410 without the tangent, force
// CONSTITUTIVE.m:268-285).  A CTA takes RES_ELEMS elements.  Phase 1, a thread per point:
// E = B U in registers (k_strain's summation order), S from the stress-only return mapping,
// kept in shared memory; phase 2, a thread per (element, node): the node's force over the
// element's points from the shared stresses (k_force's order), added with atomics.  E and S
// never reach global memory, and each point's gradients are read from DRAM once.  F must be
// zeroed first.
constexpr int RES_ELEMS = 16;
constexpr int RES_MAXQ = 16;
constexpr int RES_THREADS = 192;

__global__ void __launch_bounds__(RES_THREADS) k_residual3d(const int32_t *__restrict__ elem,
                                                            const double *__restrict__ dphi,
                                                            const double *__restrict__ w, int nq, int64_t n_e,
                                                            const double *__restrict__ U,
                                                            const double *__restrict__ c_bar,
                                                            const double *__restrict__ sin_phi,
                                                            const double *__restrict__ shear,
                                                            const double *__restrict__ lame,
                                                            uint8_t *__restrict__ branch, double *__restrict__ F) {
    constexpr int NP = 10;
    __shared__ double sS[RES_ELEMS * RES_MAXQ * 7];
    const int t = threadIdx.x;
    for (int64_t e0 = (int64_t)blockIdx.x * RES_ELEMS; e0 < n_e; e0 += (int64_t)gridDim.x * RES_ELEMS) {
        {
            const int le = t / nq, q = t - le * nq;
            const int64_t e = e0 + le;
            if (le < RES_ELEMS && e < n_e) {
                const int64_t g = e * nq + q;
                const double *d = dphi + g * 3 * NP;
                double E[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                for (int i = 0; i < NP; ++i) {
                    const int64_t v = elem[e * NP + i];
                    const double d1 = d[i], d2 = d[NP + i], d3 = d[2 * NP + i];
                    const double ux = U[3 * v], uy = U[3 * v + 1], uz = U[3 * v + 2];
                    E[0] += d1 * ux;
                    E[1] += d2 * uy;
                    E[2] += d3 * uz;
                    E[3] += d2 * ux + d1 * uy;
                    E[4] += d3 * uy + d2 * uz;
                    E[5] += d3 * ux + d1 * uz;
                }
                double st[6];
                const int b = mc3d_point<false>(E, c_bar[g], sin_phi[g], shear[g], lame[g], st, nullptr);
                if (branch) branch[g] = (uint8_t)b;
#pragma unroll
                for (int c = 0; c < 6; ++c) sS[(le * nq + q) * 7 + c] = st[c];
            }
        }
        __syncthreads();
        {
            const int le = t / NP, i = t - le * NP;
            const int64_t e = e0 + le;
            if (le < RES_ELEMS && e < n_e) {
                double f0 = 0.0, f1 = 0.0, f2 = 0.0;
                for (int q = 0; q < nq; ++q) {
                    const int64_t g = e * nq + q;
                    const double *d = dphi + g * 3 * NP;
                    const double *s = sS + (le * nq + q) * 7;
                    const double wq = w[g];
                    const double d1 = d[i], d2 = d[NP + i], d3 = d[2 * NP + i];
                    f0 += wq * (d1 * s[0] + d2 * s[3] + d3 * s[5]);
                    f1 += wq * (d2 * s[1] + d1 * s[3] + d3 * s[4]);
                    f2 += wq * (d3 * s[2] + d2 * s[4] + d1 * s[5]);
                }
                const int64_t v = elem[e * NP + i];
                atomicAdd(&F[3 * v], f0);
                atomicAdd(&F[3 * v + 1], f1);
                atomicAdd(&F[3 * v + 2], f2);
            }
        }
        __syncthreads();
    }
}

// Nonzeros of column (node j, comp c) of the local B at one point.
template <int DIM>
__device__ __forceinline__ void bcol(const double *d, int np, int j, int c, int r[3], double v[3]) {
    const double d1 = d[j], d2 = d[np + j];
    if (DIM == 3) {
        const double d3 = d[2 * np + j];
        if (c == 0) { r[0] = 0; v[0] = d1; r[1] = 3; v[1] = d2; r[2] = 5; v[2] = d3; }
        else if (c == 1) { r[0] = 1; v[0] = d2; r[1] = 3; v[1] = d1; r[2] = 4; v[2] = d3; }
        else { r[0] = 2; v[0] = d3; r[1] = 4; v[1] = d2; r[2] = 5; v[2] = d1; }
    } else {
        if (c == 0) { r[0] = 0; v[0] = d1; r[1] = 2; v[1] = d2; }
        else { r[0] = 1; v[0] = d2; r[1] = 2; v[1] = d1; }
        r[2] = 0; v[2] = 0.0;
    }
}

// One thread per (element, local column (node j, comp c)); accumulates the whole column of
// the element matrix over the element's points in registers, then adds it into the BSR
// blocks (node_i, node_j) with one atomic per entry.
template <int DIM, int NP>
__global__ void __launch_bounds__(128) k_assemble_bsr(const int32_t *__restrict__ pair_blk,
                                                      const double *__restrict__ dphi, const double *__restrict__ w,
                                                      int nq, int64_t n_e, const double *__restrict__ DS,
                                                      double *__restrict__ K) {
    constexpr int NS = DIM == 3 ? 6 : 3;
    constexpr int NL = DIM * NP;
    const int64_t total = n_e * NL;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t / NL;
        const int col = (int)(t - e * NL);
        const int j = col / DIM, c = col - j * DIM;
        double acc[NL];
#pragma unroll
        for (int k = 0; k < NL; ++k) acc[k] = 0.0;
        for (int q = 0; q < nq; ++q) {
            const int64_t g = e * nq + q;
            const double *d = dphi + g * DIM * NP;
            const double *D = DS + g * NS * NS;
            const double wq = w[g];
            int r[3];
            double v[3];
            bcol<DIM>(d, NP, j, c, r, v);
            double db[NS];
#pragma unroll
            for (int a = 0; a < NS; ++a) {
                double s = D[a + NS * r[0]] * v[0] + D[a + NS * r[1]] * v[1];
                if (DIM == 3) s += D[a + NS * r[2]] * v[2];
                db[a] = wq * s;
            }
#pragma unroll
            for (int i = 0; i < NP; ++i) {
                const double d1 = d[i], d2 = d[NP + i];
                if (DIM == 3) {
                    const double d3 = d[2 * NP + i];
                    acc[3 * i + 0] += d1 * db[0] + d2 * db[3] + d3 * db[5];
                    acc[3 * i + 1] += d2 * db[1] + d1 * db[3] + d3 * db[4];
                    acc[3 * i + 2] += d3 * db[2] + d2 * db[4] + d1 * db[5];
                } else {
                    acc[2 * i + 0] += d1 * db[0] + d2 * db[2];
                    acc[2 * i + 1] += d2 * db[1] + d1 * db[2];
                }
            }
        }
        const int32_t *pb = pair_blk + e * NP * NP;
#pragma unroll
        for (int i = 0; i < NP; ++i) {
            const int64_t blk = pb[i * NP + j];   // block (node_i, node_j)
#pragma unroll
            for (int cp = 0; cp < DIM; ++cp) atomicAdd(&K[blk * DIM * DIM + cp * DIM + c], acc[DIM * i + cp]);
        }
    }
}

// ------------------------------------------------------------------ deterministic P2-tet assembly
//
// Two passes instead of one pass of atomics (same arithmetic as k_assemble_bsr up to rounding,
// but every block sums its terms in a fixed order, so K is bitwise reproducible; and exactly
// symmetric):
//   k_element_blocks_p2tet  per element, its 55 upper node blocks (i <= j) of
//       sum_q w_q B_q' sym(D_q) B_q, with the element's D, gradients and weights staged in
//       shared memory once; D B is formed once per (point, column) and shared by the blocks;
//       diagonal blocks are computed on and above their diagonal and mirrored;
//   k_gather_blocks3        per BSR block, the sum of its element contributions in element
//       order (the transpose of an upper block for the lower ones), written as K_t, or
//       blended into K_r = r K_el + (1 - r) K_t with identity on Dirichlet rows/columns
//       (the k_kr_blend epilogue; K_el and K_t being exactly symmetric, its averaging with the
//       transposed block is the identity).
// sym(D) = (D + D')/2 is what the reference's symmetrisation of K_r applies to its unsymmetric
// sums (CONSTITUTIVE.m:515-532): B' sym(D) B = sym(B' D B).
constexpr int KE_EPB = 8, KE_TPE = 18;   // elements per CTA, threads per element (one per chunk)
constexpr int KE_PITCH = 10;             // doubles per stored element block (9 + 1: 16-byte aligned)

// The 18 chunks of an element's upper node blocks: node j and up to 4 row nodes i0 .. i0+3
// (i <= j); chunk c owns blocks (i, j) for i in [i0, min(i0 + 4, j + 1)).
__constant__ int8_t c_ke_j[KE_TPE] = {0, 1, 2, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 8, 9, 9, 9};
__constant__ int8_t c_ke_i0[KE_TPE] = {0, 0, 0, 0, 0, 4, 0, 4, 0, 4, 0, 4, 0, 4, 8, 0, 4, 8};

__device__ __forceinline__ int ke_slot(int i, int j) { return i * 10 - i * (i - 1) / 2 + (j - i); }

// One thread's chunk of an element (node j, row nodes i0 .. min(i0 + 3, j)): its node blocks
// summed over the element's points from sym(D) (nq x 36), the gradients (nq x [3][10]) and
// the weights in shared memory, written to the element's slots of Ke.
__device__ __forceinline__ void ke_chunk(const double *sD, const double *sPhi, const double *sW, int nq, int j,
                                         int i0, double *__restrict__ Ke_e) {
    double acc[4][9];
#pragma unroll
    for (int ii = 0; ii < 4; ++ii)
#pragma unroll
        for (int k = 0; k < 9; ++k) acc[ii][k] = 0.0;
    for (int q = 0; q < nq; ++q) {
        const double *D = sD + q * 36, *d = sPhi + q * 30;
        const double wq = sW[q];
        // w sym(D) B(:, (j, cj)) for the three components of node j
        double db[3][6];
#pragma unroll
        for (int cj = 0; cj < 3; ++cj) {
            int r[3];
            double v[3];
            bcol<3>(d, 10, j, cj, r, v);
#pragma unroll
            for (int a = 0; a < 6; ++a)
                db[cj][a] = wq * (D[a + 6 * r[0]] * v[0] + D[a + 6 * r[1]] * v[1] + D[a + 6 * r[2]] * v[2]);
        }
#pragma unroll
        for (int ii = 0; ii < 4; ++ii) {
            const int i = i0 + ii;
            if (i > j) break;
#pragma unroll
            for (int ci = 0; ci < 3; ++ci) {
                int r[3];
                double v[3];
                bcol<3>(d, 10, i, ci, r, v);
#pragma unroll
                for (int cj = 0; cj < 3; ++cj)
                    acc[ii][ci * 3 + cj] += v[0] * db[cj][r[0]] + v[1] * db[cj][r[1]] + v[2] * db[cj][r[2]];
            }
        }
    }
#pragma unroll
    for (int ii = 0; ii < 4; ++ii) {
        const int i = i0 + ii;
        if (i > j) break;
        if (i == j) {   // diagonal node block: its upper triangle, mirrored (exactly symmetric)
            acc[ii][3] = acc[ii][1];
            acc[ii][6] = acc[ii][2];
            acc[ii][7] = acc[ii][5];
        }
        double *out = Ke_e + ke_slot(i, j) * KE_PITCH;
#pragma unroll
        for (int k = 0; k < 9; ++k) out[k] = acc[ii][k];
    }
}

// Staging by plain loads (any alignment of DS, any nq).
__global__ void __launch_bounds__(KE_EPB * KE_TPE, 3) k_element_blocks_p2tet(int64_t n_e, int nq,
                                                                          const double *__restrict__ dphi,
                                                                          const double *__restrict__ w,
                                                                          const double *__restrict__ DS,
                                                                          double *__restrict__ Ke) {
    extern __shared__ double ke_smem[];
    const int per = nq * (36 + 30 + 1);
    const int le = threadIdx.x / KE_TPE, lc = threadIdx.x - le * KE_TPE;
    const int j = c_ke_j[lc], i0 = c_ke_i0[lc];
    for (int64_t e0 = (int64_t)blockIdx.x * KE_EPB; e0 < n_e; e0 += (int64_t)gridDim.x * KE_EPB) {
        // stage the CTA's elements: sym(D) per point, gradients [q][d][i], weights
        const int64_t ne_here = n_e - e0 < KE_EPB ? n_e - e0 : KE_EPB;
        __syncthreads();
        for (int t = threadIdx.x; t < ne_here * nq * 36; t += blockDim.x) {
            const int64_t ge = t / 36;                         // element-local point index (el * nq + q)
            const int k = t - (int)ge * 36, a = k % 6, b = k / 6;
            const double *D = DS + (e0 * nq + ge) * 36;
            const int el = (int)(ge / nq);
            ke_smem[el * per + (ge - (int64_t)el * nq) * 36 + k] = 0.5 * (D[a + 6 * b] + D[b + 6 * a]);
        }
        for (int t = threadIdx.x; t < ne_here * nq * 30; t += blockDim.x) {
            const int el = t / (nq * 30), r = t - el * nq * 30;
            ke_smem[el * per + nq * 36 + r] = dphi[(e0 * nq) * 30 + t];
        }
        for (int t = threadIdx.x; t < ne_here * nq; t += blockDim.x) {
            const int el = t / nq, q = t - el * nq;
            ke_smem[el * per + nq * 66 + q] = w[e0 * nq + t];
        }
        __syncthreads();
        if (le < ne_here) {
            const double *sD = ke_smem + le * per;
            ke_chunk(sD, sD + nq * 36, sD + nq * 66, nq, j, i0, Ke + (e0 + le) * 55 * KE_PITCH);
        }
    }
}

// Staging by bulk copies, two stages: a batch's DS, gradients and weights are three contiguous
// ranges of global memory (element-major), each brought into shared memory by one
// cp.async.bulk whose completion is counted on the stage's mbarrier; the copy of the next
// batch runs while the current one is computed.  sym(D) is formed in place once a batch has
// landed (each off-diagonal pair by one thread, the same rounding as the plain-load kernel),
// so both kernels write bitwise the same blocks.  Needs DS, dphi and w 16-byte aligned.
//   shared: [2 mbarriers | status | pad] then 2 stages of
//           D (KE_EPB nq 36) | gradients (KE_EPB nq 30) | weights (KE_EPB nq, rounded up to even)
constexpr long long KE_WAIT_CYCLES = 2000000000LL;   // about one second at the boost clock
__constant__ int8_t c_sym_a[15] = {0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 3, 3, 4};
__constant__ int8_t c_sym_b[15] = {1, 2, 3, 4, 5, 2, 3, 4, 5, 3, 4, 5, 4, 5, 5};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool ke_wait(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > KE_WAIT_CYCLES) return false;
    }
}

__device__ __forceinline__ void ke_bulk(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Thread 0: the copies of batch b (elements b KE_EPB ..) into the stage at shared address `stage`.
__device__ __forceinline__ void ke_issue(int64_t b, int64_t n_e, int nq, const double *dphi, const double *w,
                                         const double *DS, uint32_t stage, uint32_t bar) {
    const int64_t e0 = b * KE_EPB;
    const int64_t ne = n_e - e0 < KE_EPB ? n_e - e0 : KE_EPB;
    const uint32_t dB = (uint32_t)(ne * nq * 36 * 8), pB = (uint32_t)(ne * nq * 30 * 8);
    const uint32_t wB = (uint32_t)(ne * nq * 8) & ~15u;   // an odd last weight is loaded plainly
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(dB + pB + wB) : "memory");
    ke_bulk(stage, DS + e0 * nq * 36, dB, bar);
    ke_bulk(stage + (uint32_t)(KE_EPB * nq * 36 * 8), dphi + e0 * nq * 30, pB, bar);
    if (wB) ke_bulk(stage + (uint32_t)(KE_EPB * nq * 66 * 8), w + e0 * nq, wB, bar);
}

__global__ void __launch_bounds__(KE_EPB * KE_TPE, 2) k_element_blocks_p2tet_bulk(int64_t n_e, int nq,
                                                                               const double *__restrict__ dphi,
                                                                               const double *__restrict__ w,
                                                                               const double *__restrict__ DS,
                                                                               double *__restrict__ Ke,
                                                                               int32_t *__restrict__ status) {
    extern __shared__ __align__(16) unsigned char ke_sm[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(ke_sm);
    volatile int *s_fail = reinterpret_cast<volatile int *>(ke_sm + 16);
    const int wpad = (KE_EPB * nq + 1) & ~1;
    const int per_stage = KE_EPB * nq * 66 + wpad;   // doubles
    double *stages = reinterpret_cast<double *>(ke_sm + 32);
    const uint32_t bar0 = smem_u32(&bars[0]), bar1 = smem_u32(&bars[1]);
    const uint32_t st0 = smem_u32(stages), st1 = st0 + (uint32_t)per_stage * 8;
    const int tid = threadIdx.x;
    const int le = tid / KE_TPE, lc = tid - le * KE_TPE;
    const int j = c_ke_j[lc], i0 = c_ke_i0[lc];
    const int64_t n_batches = (n_e + KE_EPB - 1) / KE_EPB;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *s_fail = 0;
    }
    __syncthreads();
    int64_t b = blockIdx.x;
    if (tid == 0 && b < n_batches) ke_issue(b, n_e, nq, dphi, w, DS, st0, bar0);
    for (int it = 0; b < n_batches; ++it, b += gridDim.x) {
        const int s = it & 1;
        const uint32_t bar = s ? bar1 : bar0;
        const int64_t bn = b + gridDim.x;
        // the other stage was released by the barrier that ended the previous batch
        if (tid == 0 && bn < n_batches) ke_issue(bn, n_e, nq, dphi, w, DS, s ? st0 : st1, s ? bar0 : bar1);
        if (tid == 0 && !ke_wait(bar, (uint32_t)((it >> 1) & 1))) *s_fail = 1;
        __syncthreads();
        if (*s_fail) {
            if (tid == 0) {
                atomicOr(status, 1);
                if (bn < n_batches) ke_wait(s ? bar0 : bar1, (uint32_t)(((it + 1) >> 1) & 1));   // bounded drain
            }
            return;
        }
        double *sD = stages + (int64_t)s * per_stage;
        double *sPhi = sD + KE_EPB * nq * 36, *sW = sD + KE_EPB * nq * 66;
        const int64_t e0 = b * KE_EPB;
        const int ne = (int)(n_e - e0 < KE_EPB ? n_e - e0 : KE_EPB);
        for (int t = tid; t < ne * nq * 15; t += blockDim.x) {
            const int p = t / 15, k = t - p * 15;
            double *D = sD + p * 36;
            const int a = c_sym_a[k], c = c_sym_b[k];
            const double v = 0.5 * (D[a + 6 * c] + D[c + 6 * a]);
            D[a + 6 * c] = v;
            D[c + 6 * a] = v;
        }
        if (tid == 0 && ((ne * nq) & 1)) sW[ne * nq - 1] = w[e0 * nq + ne * nq - 1];
        // generic writes to the stage, ordered before the bulk copy that refills it
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (le < ne)
            ke_chunk(sD + le * nq * 36, sPhi + le * nq * 30, sW + le * nq, nq, j, i0, Ke + (e0 + le) * 55 * KE_PITCH);
        __syncthreads();
    }
}

// A warp sums the contributions of 32 consecutive blocks (a lane per block, its element
// blocks read as five 16-byte words), then writes the 32 results as one contiguous run through
// shared memory (and reads K_el for the blend the same way).
constexpr int KG_WARPS = 8;
template <bool BLEND>
__global__ void __launch_bounds__(KG_WARPS * 32) k_gather_blocks3(int64_t n_blocks, const int32_t *__restrict__ cptr,
                                                                  const uint32_t *__restrict__ contrib,
                                                                  const double *__restrict__ Ke,
                                                                  const int32_t *__restrict__ row_of,
                                                                  const int32_t *__restrict__ col,
                                                                  const double *__restrict__ mask, double r,
                                                                  const double *__restrict__ Kel,
                                                                  double *__restrict__ Kout) {
    __shared__ double sOut[KG_WARPS][32 * 9];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *so = sOut[warp];
    const int64_t stride = (int64_t)gridDim.x * KG_WARPS * 32;
    for (int64_t base = ((int64_t)blockIdx.x * KG_WARPS + warp) * 32; base < n_blocks; base += stride) {
        const int64_t p = base + lane;
        double acc[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) acc[k] = 0.0;
        if (p < n_blocks) {
            // contributions in list order, two in flight (both index and block loads issued
            // before either is added)
            auto add = [&](uint32_t src, const double *x) {
                if (src >> 31) {
#pragma unroll
                    for (int a = 0; a < 3; ++a)
#pragma unroll
                        for (int b = 0; b < 3; ++b) acc[a * 3 + b] += x[b * 3 + a];
                } else {
#pragma unroll
                    for (int k = 0; k < 9; ++k) acc[k] += x[k];
                }
            };
            auto fetch = [&](uint32_t src, double *x) {
                const double2 *v = reinterpret_cast<const double2 *>(Ke + (int64_t)(src & 0x7fffffffu) * KE_PITCH);
#pragma unroll
                for (int h = 0; h < 5; ++h) {
                    const double2 t = __ldg(v + h);
                    x[2 * h] = t.x;
                    x[2 * h + 1] = t.y;
                }
            };
            const int32_t l1 = cptr[p + 1];
            int32_t l = cptr[p];
            for (; l + 1 < l1; l += 2) {
                const uint32_t s0 = contrib[l], s1 = contrib[l + 1];
                double x0[10], x1[10];
                fetch(s0, x0);
                fetch(s1, x1);
                add(s0, x0);
                add(s1, x1);
            }
            if (l < l1) {
                const uint32_t s0 = contrib[l];
                double x0[10];
                fetch(s0, x0);
                add(s0, x0);
            }
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) so[lane * 9 + k] = acc[k];
        __syncwarp();
        const int cnt = (int)(n_blocks - base < 32 ? n_blocks - base : 32);
        for (int idx = lane; idx < cnt * 9; idx += 32) {
            const int pl = idx / 9, k = idx - pl * 9;
            const int64_t o = base * 9 + idx;
            double v = so[idx];
            if (BLEND) {
                const int64_t pb = base + pl, I = row_of[pb], J = col[pb];
                const int a = k / 3, b = k - a * 3;
                const bool free = mask[I * 3 + a] != 0.0 && mask[J * 3 + b] != 0.0;
                const double el = Kel ? Kel[o] : 0.0;
                v = free ? r * el + (1.0 - r) * v : ((I == J && a == b) ? 1.0 : 0.0);
            }
            Kout[o] = v;
        }
        __syncwarp();
    }
}

// Element blocks of the deterministic path into m->d_ke (allocated on first use): the
// bulk-staged kernel (two CTAs per SM) when DS, the gradients and the weights are 16-byte
// aligned and two stages fit in shared memory, else the plain-load kernel.
static int element_blocks(sg_mesh *m, const double *DS, cudaStream_t st) {
    if (!m->d_ke) SG_CUDA(device_alloc(&m->d_ke, sizeof(double) * (size_t)m->n_e * 55 * KE_PITCH));
    const int64_t batches = (m->n_e + KE_EPB - 1) / KE_EPB;
    const size_t stage = sizeof(double) * ((size_t)KE_EPB * m->nq * 66 + (size_t)((KE_EPB * m->nq + 1) & ~1));
    const size_t smem_bulk = 32 + 2 * stage;
    const bool aligned = ((reinterpret_cast<uintptr_t>(DS) | reinterpret_cast<uintptr_t>(m->d_dphi) |
                           reinterpret_cast<uintptr_t>(m->d_w)) & 15) == 0;
    int32_t *status = device_status_word();
    if (aligned && status && smem_bulk <= 113 * 1024) {
        static thread_local size_t configured_bulk = 0;
        if (smem_bulk > configured_bulk) {
            SG_CUDA(cudaFuncSetAttribute(k_element_blocks_p2tet_bulk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem_bulk));
            configured_bulk = smem_bulk;
        }
        count_launch();
        const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(batches, (int64_t)sm_count() * 2));
        k_element_blocks_p2tet_bulk<<<grid, KE_EPB * KE_TPE, smem_bulk, st>>>(m->n_e, m->nq, m->d_dphi, m->d_w, DS,
                                                                             m->d_ke, status);
        SG_CUDA(cudaGetLastError());
        return SG_OK;
    }
    const size_t smem = sizeof(double) * (size_t)KE_EPB * m->nq * (36 + 30 + 1);
    static thread_local size_t configured = 0;
    if (smem > configured) {
        SG_CUDA(cudaFuncSetAttribute(k_element_blocks_p2tet, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured = smem;
    }
    count_launch();
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(batches, (int64_t)sm_count() * 8));
    k_element_blocks_p2tet<<<grid, KE_EPB * KE_TPE, smem, st>>>(m->n_e, m->nq, m->d_dphi, m->d_w, DS, m->d_ke);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

static bool deterministic_path(const sg_mesh *m) { return m->d_contrib && m->dim == 3 && m->np == 10; }

// DS_elast = 2 * shear * DEV + bulk * VOL with IOTA = [1;1;1; zeros(ns-3,1)] (CONSTITUTIVE.m:413-422).
// For ns == 3 (2D) the reference's IOTA has three ones, so VOL is the all-ones 3x3 matrix;
// that arithmetic is reproduced as is.
template <int NS>
__global__ void k_elastic_ds(const double *__restrict__ shear, const double *__restrict__ bulk, int64_t n,
                             double *__restrict__ DS) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x) {
        const double G = shear[g], Kb = bulk[g];
#pragma unroll
        for (int j = 0; j < NS; ++j)
#pragma unroll
            for (int i = 0; i < NS; ++i) {
                const double vol = (i < 3 && j < 3) ? 1.0 : 0.0;
                const double id = (i == j) ? ((NS == 6) ? (i < 3 ? 1.0 : 0.5) : (i < 2 ? 1.0 : 0.5)) : 0.0;
                const double dev = id - vol / 3.0;
                DS[g * NS * NS + i + NS * j] = 2.0 * dev * G + vol * Kb;
            }
    }
}

// K_r for every BSR entry: v1 = r Kel + (1-r) Kt at (i,j), v2 the same at (j,i), K_r = (v1+v2)/2;
// Dirichlet rows/columns are zero with a unit diagonal.  Kel may be null (r is then ignored).
template <int DIM>
__global__ void k_kr_blend(int64_t n_blocks, const int32_t *__restrict__ row_of, const int32_t *__restrict__ col,
                           const int32_t *__restrict__ tr, const double *__restrict__ mask, double r,
                           const double *__restrict__ Kel, const double *__restrict__ Kt, double *__restrict__ Kr) {
    constexpr int BB = DIM * DIM;
    const int64_t total = n_blocks * BB;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = t / BB;
        const int ab = (int)(t - p * BB), a = ab / DIM, b = ab - a * DIM;
        const int64_t I = row_of[p], J = col[p];
        const int64_t pt = tr[p];
        const double ra = mask[I * DIM + a], cb = mask[J * DIM + b];
        double out;
        if (ra != 0.0 && cb != 0.0) {
            const double el1 = Kel ? Kel[p * BB + ab] : 0.0, el2 = Kel ? Kel[pt * BB + b * DIM + a] : 0.0;
            const double v1 = r * el1 + (1.0 - r) * Kt[p * BB + ab];
            const double v2 = r * el2 + (1.0 - r) * Kt[pt * BB + b * DIM + a];
            out = (v1 + v2) / 2.0;
        } else {
            out = (I == J && a == b) ? 1.0 : 0.0;
        }
        Kr[p * BB + ab] = out;
    }
}

// (K + K')/2 on the BSR pattern (used once for the elastic matrix, like CONSTITUTIVE.m:429).
template <int DIM>
__global__ void k_symmetrize(int64_t n_blocks, const int32_t *__restrict__ tr, const double *__restrict__ K,
                             double *__restrict__ Ks) {
    constexpr int BB = DIM * DIM;
    const int64_t total = n_blocks * BB;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = t / BB;
        const int ab = (int)(t - p * BB), a = ab / DIM, b = ab - a * DIM;
        Ks[p * BB + ab] = (K[p * BB + ab] + K[(int64_t)tr[p] * BB + b * DIM + a]) / 2.0;
    }
}

__global__ void k_gather(int64_t n, const int64_t *__restrict__ idx, const double *__restrict__ src,
                         double *__restrict__ dst) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        dst[k] = src[idx[k]];
}

}  // namespace sg

using namespace sg;

extern "C" int sg_strain_dev(const sg_mesh *m, const double *U, double *E, void *stream) {
    SG_CHECK_ARG(m && U && E, "null argument");
    const cudaStream_t st = as_stream(stream);
    if (m->dim == 3) k_strain<3><<<grid_for(m->n_int, 256), 256, 0, st>>>(m->d_elem, m->d_dphi, m->np, m->nq, m->n_int, U, E);
    else k_strain<2><<<grid_for(m->n_int, 256), 256, 0, st>>>(m->d_elem, m->d_dphi, m->np, m->nq, m->n_int, U, E);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

extern "C" int sg_force_dev(const sg_mesh *m, const double *S, int32_t s_rows, double *F, void *stream) {
    SG_CHECK_ARG(m && S && F, "null argument");
    SG_CHECK_ARG(s_rows >= m->ns, "s_rows smaller than the number of strain components");
    const cudaStream_t st = as_stream(stream);
    SG_CUDA(cudaMemsetAsync(F, 0, sizeof(double) * m->n_n * m->dim, st));
    const int64_t work = m->n_e * m->np;
    if (m->dim == 3) k_force<3><<<grid_for(work, 256), 256, 0, st>>>(m->d_elem, m->d_dphi, m->d_w, m->np, m->nq, m->n_e, S, s_rows, F);
    else k_force<2><<<grid_for(work, 256), 256, 0, st>>>(m->d_elem, m->d_dphi, m->d_w, m->np, m->nq, m->n_e, S, s_rows, F);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

extern "C" int sg_residual_dev(const sg_mesh *m, const double *U, const double *c_bar, const double *sin_phi,
                               const double *shear, const double *lame, uint8_t *branch, double *F, void *stream) {
    SG_CHECK_ARG(m && U && c_bar && sin_phi && shear && lame && F, "null argument");
    SG_CHECK_ARG(m->dim == 3 && m->np == 10, "the fused residual is for P2 tetrahedra");
    SG_CHECK_ARG(m->nq >= 1 && m->nq <= RES_MAXQ, "too many integration points per element");
    const cudaStream_t st = as_stream(stream);
    SG_CUDA(cudaMemsetAsync(F, 0, sizeof(double) * m->n_n * 3, st));
    if (m->n_e == 0) return SG_OK;
    const InstrToken tk = instr_begin(IK_RESIDUAL, st);
    count_launch();
    const int64_t ctas = (m->n_e + RES_ELEMS - 1) / RES_ELEMS;
    const unsigned grid = (unsigned)std::min<int64_t>(ctas, (int64_t)sm_count() * 8);
    k_residual3d<<<grid, RES_THREADS, 0, st>>>(m->d_elem, m->d_dphi, m->d_w, m->nq, m->n_e, U, c_bar, sin_phi,
                                               shear, lame, branch, F);
    instr_end(tk, st);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

extern "C" int sg_assemble_bsr_dev(const sg_mesh *m_, const double *DS, double *K, void *stream) {
    SG_CHECK_ARG(m_ && DS && K, "null argument");
    sg_mesh *m = const_cast<sg_mesh *>(m_);   // the element-block scratch is the mesh's own
    const cudaStream_t st = as_stream(stream);
    if (deterministic_path(m)) {
        const InstrToken tk = instr_begin(IK_ASSEMBLY, st);
        int rc = element_blocks(m, DS, st);
        if (!rc) {
            k_gather_blocks3<false><<<grid_for(m->bsr.n_blocks, KG_WARPS * 32, 8), KG_WARPS * 32, 0, st>>>(
                m->bsr.n_blocks, m->d_contrib_ptr, m->d_contrib, m->d_ke, nullptr, nullptr, nullptr, 0.0, nullptr, K);
            if (cudaGetLastError() != cudaSuccess) rc = set_error(SG_ERR_CUDA, "k_gather_blocks3 launch");
        }
        instr_end(tk, st);
        return rc;
    }
    SG_CUDA(cudaMemsetAsync(K, 0, sizeof(double) * m->bsr.n_blocks * m->dim * m->dim, st));
    const int64_t work = m->n_e * m->dim * m->np;
    const InstrToken tk = instr_begin(IK_ASSEMBLY, st);
    struct End {
        const InstrToken &t;
        cudaStream_t s;
        ~End() { instr_end(t, s); }
    } end_guard{tk, st};
    if (m->dim == 3 && m->np == 10)
        k_assemble_bsr<3, 10><<<grid_for(work, 128, 16), 128, 0, st>>>(m->d_pair_blk, m->d_dphi, m->d_w, m->nq, m->n_e, DS, K);
    else if (m->dim == 2 && m->np == 6)
        k_assemble_bsr<2, 6><<<grid_for(work, 128, 16), 128, 0, st>>>(m->d_pair_blk, m->d_dphi, m->d_w, m->nq, m->n_e, DS, K);
    else if (m->dim == 3 && m->np == 4)
        k_assemble_bsr<3, 4><<<grid_for(work, 128, 16), 128, 0, st>>>(m->d_pair_blk, m->d_dphi, m->d_w, m->nq, m->n_e, DS, K);
    else if (m->dim == 2 && m->np == 3)
        k_assemble_bsr<2, 3><<<grid_for(work, 128, 16), 128, 0, st>>>(m->d_pair_blk, m->d_dphi, m->d_w, m->nq, m->n_e, DS, K);
    else
        return set_error(SG_ERR_ARG, "BSR assembly supports P1/P2 triangles and tetrahedra");
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

extern "C" int sg_elastic_ds_dev(const sg_mesh *m, const double *shear, const double *bulk, double *DS, void *stream) {
    SG_CHECK_ARG(m && shear && bulk && DS, "null argument");
    const cudaStream_t st = as_stream(stream);
    if (m->dim == 3) k_elastic_ds<6><<<grid_for(m->n_int, 256), 256, 0, st>>>(shear, bulk, m->n_int, DS);
    else k_elastic_ds<3><<<grid_for(m->n_int, 256), 256, 0, st>>>(shear, bulk, m->n_int, DS);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}


extern "C" int sg_symmetrize_bsr_dev(const sg_mesh *m, const double *K, double *Ks, void *stream) {
    SG_CHECK_ARG(m && K && Ks && K != Ks, "null or aliased argument");
    const cudaStream_t st = as_stream(stream);
    const int64_t work = m->bsr.n_blocks * m->dim * m->dim;
    if (m->dim == 3) k_symmetrize<3><<<grid_for(work, 256), 256, 0, st>>>(m->bsr.n_blocks, m->bsr.d_transpose, K, Ks);
    else k_symmetrize<2><<<grid_for(work, 256), 256, 0, st>>>(m->bsr.n_blocks, m->bsr.d_transpose, K, Ks);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

extern "C" int sg_kr_blend_dev(const sg_mesh *m, double r, const double *Kel, const double *Kt, double *Kr,
                               void *stream) {
    SG_CHECK_ARG(m && Kt && Kr && Kt != Kr, "null or aliased argument");
    const cudaStream_t st = as_stream(stream);
    const int32_t *row_of = m->bsr.d_row_of;
    const int64_t work = m->bsr.n_blocks * m->dim * m->dim;
    if (m->dim == 3)
        k_kr_blend<3><<<grid_for(work, 256), 256, 0, st>>>(m->bsr.n_blocks, row_of, m->bsr.d_col, m->bsr.d_transpose, m->d_mask, r, Kel, Kt, Kr);
    else
        k_kr_blend<2><<<grid_for(work, 256), 256, 0, st>>>(m->bsr.n_blocks, row_of, m->bsr.d_col, m->bsr.d_transpose, m->d_mask, r, Kel, Kt, Kr);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

// K_r = r K_el + (1 - r) K_t from the tangent DS in one assembly (P2 tetrahedra: the
// deterministic two-pass assembly with the blend as its epilogue; other elements: assembly into
// Kt_scratch, then k_kr_blend).  Kt_scratch may be null on the P2-tetrahedron path.
extern "C" int sg_assemble_kr_dev(sg_mesh *m, const double *DS, double r, const double *Kel, double *Kt_scratch,
                                  double *Kr, void *stream) {
    SG_CHECK_ARG(m && DS && Kr && Kr != Kel, "null or aliased argument");
    const cudaStream_t st = as_stream(stream);
    if (deterministic_path(m)) {
        const InstrToken tk = instr_begin(IK_ASSEMBLY, st);
        int rc = element_blocks(m, DS, st);
        if (!rc) {
            k_gather_blocks3<true><<<grid_for(m->bsr.n_blocks, KG_WARPS * 32, 8), KG_WARPS * 32, 0, st>>>(
                m->bsr.n_blocks, m->d_contrib_ptr, m->d_contrib, m->d_ke, m->bsr.d_row_of, m->bsr.d_col, m->d_mask, r,
                Kel, Kr);
            if (cudaGetLastError() != cudaSuccess) rc = set_error(SG_ERR_CUDA, "k_gather_blocks3 launch");
        }
        instr_end(tk, st);
        return rc;
    }
    SG_CHECK_ARG(Kt_scratch && Kt_scratch != Kr, "this element type needs a separate K_t buffer");
    int rc = sg_assemble_bsr_dev(m, DS, Kt_scratch, stream);
    if (!rc) rc = sg_kr_blend_dev(m, r, Kel, Kt_scratch, Kr, stream);
    return rc;
}

extern "C" int sg_bsr_to_ref_dev(sg_mesh *m, const double *K, double *V_ref, void *stream) {
    SG_CHECK_ARG(m && K && V_ref, "null argument");
    const cudaStream_t st = as_stream(stream);
    if (!m->d_ref2bsr) {
        // value index of K(ref_I, ref_J) for every pattern entry, built once per mesh
        const int dim = m->dim;
        std::vector<int32_t> tr(m->bsr.n_blocks);
        SG_CUDA(cudaMemcpy(tr.data(), m->bsr.d_transpose, sizeof(int32_t) * tr.size(), cudaMemcpyDeviceToHost));
        std::vector<int64_t> idx(m->nnz_ref);
        int64_t k = 0;
        const sg_bsr &B = m->bsr;
        for (int64_t v = 0; v < m->n_n; ++v)
            for (int a = 0; a < dim; ++a) {
                if (m->dof2q[v * dim + a] < 0) continue;
                for (int32_t p = B.row_ptr[v]; p < B.row_ptr[v + 1]; ++p) {
                    const int64_t wn = B.col[p];
                    for (int b = 0; b < dim; ++b) {
                        if (m->dof2q[wn * dim + b] < 0) continue;
                        // entry (row q(v,a), col q(wn,b)) holds K(ref_I = q(wn,b), ref_J = q(v,a))
                        idx[k++] = (int64_t)tr[p] * dim * dim + b * dim + a;
                    }
                }
            }
        SG_CUDA(sg::device_alloc(&m->d_ref2bsr, sizeof(int64_t) * (idx.size() ? idx.size() : 1)));
        SG_CUDA(cudaMemcpy(m->d_ref2bsr, idx.data(), sizeof(int64_t) * idx.size(), cudaMemcpyHostToDevice));
    }
    k_gather<<<grid_for(m->nnz_ref, 256), 256, 0, st>>>(m->nnz_ref, m->d_ref2bsr, K, V_ref);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}
