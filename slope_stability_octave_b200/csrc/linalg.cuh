// Device linear-algebra building blocks for the Krylov solver and the AMG V-cycle.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mesh.h"

namespace sg {

// y = alpha * A x + beta * y  (BSR, b x b blocks, values of type VT, vectors of type XT)
template <typename VT, typename XT>
int bsr_spmv(const sg_bsr &A, const VT *vals, const XT *x, XT *y, double alpha, double beta, cudaStream_t st);
// r = b - A x
template <typename VT, typename XT>
int bsr_residual(const sg_bsr &A, const VT *vals, const XT *x, const XT *b, XT *r, cudaStream_t st);

// Rectangular-block row SpMV: y = alpha * M x + beta * y (mode 0) or y = bvec - M x (mode 1),
// M with br x bc blocks.  Supported shapes: 1x1 2x2 3x3 6x6 2x3 3x2 3x6 6x3.
// nblk (total blocks, -1 if unknown) selects the number of lanes per row.
template <typename VT, typename XT>
int rect_spmv(int br, int bc, int64_t nrows, const int32_t *rp, const int32_t *col, const VT *vals, const XT *x,
              XT *y, double alpha, double beta, const XT *bvec, int mode, cudaStream_t st, int64_t nblk = -1);

// Y(:, c) = A X(:, c) for c < k, FP64 3x3 blocks; X, Y column-major (leading dimensions may
// be negative).  Reads the matrix once per 8 columns; each column equals bsr_spmv's bitwise.
int bsr_spmm(const sg_bsr &A, const double *vals, const double *X, int64_t ldx, double *Y, int64_t ldy, int k,
             cudaStream_t st);

// The same product through node-interleaved copies of 16 columns at a time (Xi, Yi: 16 n
// doubles each of scratch): for many columns of long vectors, whose column-wise gathers would
// not stay in L2.
int bsr_spmm_interleaved(const sg_bsr &A, const double *vals, const double *X, int64_t ldx, double *Y, int64_t ldy,
                         int k, double *Xi, double *Yi, cudaStream_t st);

// Reduction workspace for dot products: partial sums of `nblk` blocks per column.
constexpr int DOT_BLOCKS = 296;  // 2 x 148 SMs
constexpr int DOT_THREADS = 256;

// out[i] = V(:, i)' w for i < m (V column-major, leading dimension ldv); deterministic.
int multidot(int64_t n, int m, const double *V, int64_t ldv, const double *w, double *partial, double *out,
             cudaStream_t st);
// w -= V(:, 0:m) h      (h on the device)
int gemv_sub(int64_t n, int m, const double *V, int64_t ldv, const double *h, double *w, cudaStream_t st);
// x += V(:, 0:m) y      (y on the device)
int gemv_add(int64_t n, int m, const double *V, int64_t ldv, const double *y, double *x, cudaStream_t st);
// Level-0 SpMV of the FP32 V-cycle on an FP16 copy of a 3x3-block matrix: each block is
// stored as three rows of four halves (the fourth zero), i.e. three uint2 words per block,
// holding the values divided by ``scale`` (a power of two).  mode 1: y = b - scale * (A x);
// mode 0: y = scale * (A x).
int h3_spmv(int64_t nrows, int64_t nblk, const int32_t *rp, const int32_t *col, const uint2 *vals, float scale,
            const float *x, float *y, const float *bvec, int mode, cudaStream_t st);
// A32 = (float) A and A16 = the FP16 3x4-padded rows of A / scale (block rows of 3 doubles;
// magnitudes beyond the FP16 range are clamped)
int to_float_half3(int64_t nblk, const double *A, float *A32, uint2 *A16, float scale, cudaStream_t st);

// Tall-skinny block products (blocked Gram-Schmidt): C = diag(sign) U' X (U n x m with m <= 256,
// X n x b with b <= 16; C column-major m x b, ldc; part: 296 * m * 16 doubles of scratch),
// deterministic; and Y -= U C.
constexpr int TS_PART_CTAS = 296;
int gemm_tn(int64_t n, int m, int b, const double *U, int64_t ldu, const double *X, int64_t ldx,
            const double *sign, double *C, int ldc, double *part, cudaStream_t st);
int gemm_nn_sub(int64_t n, int m, int b, const double *U, int64_t ldu, const double *C, int ldc, double *Y,
                int64_t ldy, cudaStream_t st);

// Gram-matrix A-orthogonalisation (the one-pass recurrence of A_orthogonalize.m in the
// coordinates of the input columns):
//   gram_upper       G(m, i) = S(:, m)' AS(:, i) for m <= i < k (G: k x k column-major;
//                    part: GR_CTAS * 64 * 64 doubles of scratch), deterministic;
//   gram_recurrence  T, the A-norms^2 nt, the signs sig and *kout (device) from G on one CTA;
//                    Ta (k x k, row-major [m][o]) holds the kept columns' coefficients in
//                    output order (last processed first), pmap (k ints) their processing
//                    indices; Tp: k x k scratch;
//   ts_apply         Y(:, o) = X(:, 0:k) Ta(:, o) for o < *kout (inputs past pmap[o] skipped:
//                    their coefficients are zero).
constexpr int GR_CTAS = 444;   // 3 per SM
int gram_upper(int64_t n, int k, const double *S, int64_t lds, const double *AS, int64_t ldas, double *G,
               double *part, cudaStream_t st);
int gram_recurrence(int k, const double *G, double *Tp, double eps, double *Ta, double *nt, double *sig,
                    int32_t *kout, int32_t *pmap, cudaStream_t st);
int ts_apply(int64_t n, int k, const int32_t *kout, const int32_t *pmap, const double *X, int64_t ldx,
             const double *Ta, double *Y, int64_t ldy, cudaStream_t st);

// Device-count variants for graph-replayed loops// Device-count variants for graph-replayed loops: m = min(cnt[0] + add, mmax) columns, basis
// V, or *Vp when V is null (both on the device)
int multidot_dc(int64_t n, const int32_t *cnt, int add, int mmax, const double *V, const double *const *Vp,
                int64_t ldv, const double *w, double *partial, double *out, cudaStream_t st);
// w += sign * V(:, 0:m) h
int gemv_dc(int sign, int64_t n, const int32_t *cnt, int add, int mmax, const double *V, const double *const *Vp,
            int64_t ldv, const double *h, double *w, cudaStream_t st);

// y = a x + b y
int axpby(int64_t n, double a, const double *x, double b, double *y, cudaStream_t st);
// y = x * s where s = *num / *den on the device (den may be null -> s = *num)
int scale_dev(int64_t n, const double *x, const double *num, int invert, double *y, cudaStream_t st);

}  // namespace sg
