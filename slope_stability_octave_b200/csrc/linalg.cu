// (c2) Node-block BSR SpMV and (c1, c3) Krylov vector kernels.
//
// SpMV: a group of lanes per block row of the matrix (two lane mappings, see k_spmv_blk and
// k_spmv_row); the lanes' partial sums are combined with warp shuffles.  Rows are assigned in
// warp-uniform slots so the shuffles never diverge.
// Dot products use a fixed two-stage tree (per-block partials, then one ordered pass), so
// results are bitwise reproducible from run to run.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "instr.cuh"
#include "linalg.cuh"
#include "sg_common.cuh"

namespace sg {

template <typename T> struct Acc { using type = double; };
template <> struct Acc<float> { using type = float; };

// Two lane mappings, chosen per block shape from measurements on the SSR slope hierarchy
// (fine 3x3, coarse 6x6, transfer 3x6 / 6x3):
//
// k_spmv_blk: G lanes per block row of the matrix, one block per lane per step (the lane reads
//   the block's br*bc contiguous values).  Best for 3x3 (G = 32 at ~28 blocks per row:
//   4.8 TB/s) and the short rows of P.
// k_spmv_row: LPR lanes per block row of the matrix, BR lanes per block: lane (slot, a) reads
//   row a of the group's slot-th block, so a warp's loads walk one contiguous run of SLOTS
//   blocks; U steps are loaded before the first product.  Best for wide blocks (6x6: 2.3x
//   the lane-per-block mapping, whose 288-byte lane stride spreads each load over 32 lines).
// Both sum in a fixed order (reproducible bitwise from run to run).
template <int BR, int BC, int G, typename VT, typename XT>
__global__ void __launch_bounds__(256) k_spmv_blk(int64_t nrows, const int32_t *__restrict__ rp,
                                                  const int32_t *__restrict__ col, const VT *__restrict__ vals,
                                                  const XT *__restrict__ x, XT *__restrict__ y, double alpha,
                                                  double beta, const XT *__restrict__ bvec, int mode,
                                                  int64_t rows_per_cta) {
    using A = typename Acc<XT>::type;
    constexpr int GPW = 32 / G;  // rows per warp
    const int lane = threadIdx.x & 31, g = lane / G, gl = lane - g * G;
    // a CTA owns rows_per_cta consecutive rows and its warps walk them in order, so the x
    // entries of neighbouring rows are still in L1 when the next rows gather them
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_cta;
    const int64_t rend = r0 + rows_per_cta < nrows ? r0 + rows_per_cta : nrows;
    const int64_t wstep = (int64_t)(blockDim.x >> 5) * GPW;
    for (int64_t base = r0 + (int64_t)(threadIdx.x >> 5) * GPW; base < rend; base += wstep) {
        const int64_t row = base + g;
        A acc[BR];
#pragma unroll
        for (int a = 0; a < BR; ++a) acc[a] = 0;
        if (row < rend) {
            const int32_t p1 = rp[row + 1];
            for (int32_t p = rp[row] + gl; p < p1; p += G) {
                const int64_t j = col[p];
                A xj[BC];
#pragma unroll
                for (int b = 0; b < BC; ++b) xj[b] = (A)x[j * BC + b];
                const VT *v = vals + (int64_t)p * BR * BC;
#pragma unroll
                for (int a = 0; a < BR; ++a)
#pragma unroll
                    for (int b = 0; b < BC; ++b) acc[a] += (A)v[a * BC + b] * xj[b];
            }
        }
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1)
#pragma unroll
            for (int a = 0; a < BR; ++a) acc[a] += __shfl_xor_sync(0xffffffffu, acc[a], off);
        if (row < rend && gl == 0) {
#pragma unroll
            for (int a = 0; a < BR; ++a) {
                const int64_t k = row * BR + a;
                if (mode == 1) y[k] = (XT)((A)bvec[k] - acc[a]);
                else if (beta == 0.0) y[k] = (XT)(alpha * acc[a]);
                else y[k] = (XT)(alpha * acc[a] + beta * (A)y[k]);
            }
        }
    }
}

template <int BR, int BC, int LPR, int U, typename VT, typename XT>
__global__ void __launch_bounds__(256) k_spmv_row(int64_t nrows, const int32_t *__restrict__ rp,
                                                  const int32_t *__restrict__ col, const VT *__restrict__ vals,
                                                  const XT *__restrict__ x, XT *__restrict__ y, double alpha,
                                                  double beta, const XT *__restrict__ bvec, int mode) {
    using A = typename Acc<XT>::type;
    constexpr int BB = BR * BC, SLOTS = LPR / BR, RPW = 32 / LPR;  // rows per warp
    const int lane = threadIdx.x & 31, rg = lane / LPR, li = lane - rg * LPR;
    const int slot = li / BR, a = li - slot * BR;
    const bool active = slot < SLOTS;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * RPW; base < nrows; base += nwarps * RPW) {
        const int64_t row = base + rg;
        A acc = 0;
        if (row < nrows && active) {
            const int32_t p0 = rp[row] + slot, p1 = rp[row + 1];
            for (int32_t p = p0; p < p1; p += U * SLOTS) {
                int64_t c[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int32_t q = p + u * SLOTS;
                    c[u] = q < p1 ? col[q] : -1;
                }
                A vv[U][BC], xv[U][BC];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const VT *v = vals + (int64_t)(p + u * SLOTS) * BB + a * BC;
                    const XT *xc = x + (c[u] < 0 ? 0 : c[u]) * BC;
                    if (c[u] >= 0) {
#pragma unroll
                        for (int b = 0; b < BC; ++b) {
                            vv[u][b] = (A)__ldg(v + b);
                            xv[u][b] = (A)__ldg(xc + b);
                        }
                    } else {
#pragma unroll
                        for (int b = 0; b < BC; ++b) vv[u][b] = xv[u][b] = 0;
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int b = 0; b < BC; ++b) acc += vv[u][b] * xv[u][b];
            }
        }
        // sum over the group's slots for component a (all lanes take part in the shuffles)
        A tot = 0;
        const int g0 = rg * LPR;
#pragma unroll
        for (int sl = 0; sl < SLOTS; ++sl) tot += __shfl_sync(0xffffffffu, acc, g0 + sl * BR + (active ? a : 0));
        if (row < nrows && active && slot == 0) {
            const int64_t k = row * BR + a;
            if (mode == 1) y[k] = (XT)((A)bvec[k] - tot);
            else if (beta == 0.0) y[k] = (XT)(alpha * tot);
            else y[k] = (XT)(alpha * tot + beta * (A)y[k]);
        }
    }
}

// k_spmv_cta: a CTA of 32 * W threads per block row, for coarse levels whose few rows each
// hold hundreds of blocks (there a warp per row occupies a fraction of the SMs and each warp
// walks its row serially).  Each warp uses k_spmv_row's (slot, a) lane mapping over its share
// of the row (warp w starts at slot w * SLOTS and steps by W * SLOTS); the warps' partial sums
// meet in shared memory and are added in warp order (reproducible bitwise).
template <int BR, int BC, int W, typename VT, typename XT>
__global__ void __launch_bounds__(32 * W) k_spmv_cta(int64_t nrows, const int32_t *__restrict__ rp,
                                                     const int32_t *__restrict__ col, const VT *__restrict__ vals,
                                                     const XT *__restrict__ x, XT *__restrict__ y, double alpha,
                                                     double beta, const XT *__restrict__ bvec, int mode) {
    using A = typename Acc<XT>::type;
    constexpr int BB = BR * BC, SLOTS = 32 / BR;
    __shared__ A part[W][BR];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int slot = lane / BR, a = lane - slot * BR;
    const bool active = slot < SLOTS;
    for (int64_t row = blockIdx.x; row < nrows; row += gridDim.x) {
        A acc = 0;
        if (active) {
            const int32_t p1 = rp[row + 1];
            for (int32_t p = rp[row] + w * SLOTS + slot; p < p1; p += W * SLOTS) {
                const int64_t c = col[p];
                const VT *v = vals + (int64_t)p * BB + a * BC;
                const XT *xc = x + c * BC;
#pragma unroll
                for (int b = 0; b < BC; ++b) acc += (A)__ldg(v + b) * (A)__ldg(xc + b);
            }
        }
        A tot = 0;
#pragma unroll
        for (int sl = 0; sl < SLOTS; ++sl) tot += __shfl_sync(0xffffffffu, acc, sl * BR + (active ? a : 0));
        if (lane < BR) part[w][lane] = tot;
        __syncthreads();
        if (w == 0 && lane < BR) {
            A sum = 0;
#pragma unroll
            for (int q = 0; q < W; ++q) sum += part[q][lane];
            const int64_t k = row * BR + lane;
            if (mode == 1) y[k] = (XT)((A)bvec[k] - sum);
            else if (beta == 0.0) y[k] = (XT)(alpha * sum);
            else y[k] = (XT)(alpha * sum + beta * (A)y[k]);
        }
        __syncthreads();
    }
}

// rows below which a coarse 6x6 level with long rows takes a CTA per row (k_spmv_cta)
constexpr int64_t CTA_ROW_LIMIT = 1184;

template <int BR, int BC, typename VT, typename XT>
static void spmv_launch(int64_t nrows, int64_t nblk, const int32_t *rp, const int32_t *col, const VT *vals,
                        const XT *x, XT *y, double alpha, double beta, const XT *bvec, int mode, cudaStream_t st) {
    const double avg = nblk > 0 && nrows > 0 ? (double)nblk / (double)nrows : 8.0;
    // the node-block shapes of the fine level are the ones timed for the roofline report
    constexpr bool fine = (BR == BC) && (BR == 3 || BR == 2);
    InstrToken tk;
    if (fine) tk = instr_begin(sizeof(VT) == 8 ? IK_SPMV3_F64 : IK_SPMV3_F32, st);
    constexpr bool wide = BR == 6 && BC == 6;
    constexpr bool tall_f64 = BR == 6 && BC == 3 && sizeof(VT) == 8;
    if constexpr (wide) {
        if (nrows < CTA_ROW_LIMIT && avg >= 48.0) {
            count_launch();
            k_spmv_cta<BR, BC, 8, VT, XT><<<(unsigned)nrows, 256, 0, st>>>(nrows, rp, col, vals, x, y, alpha, beta,
                                                                           bvec, mode);
            return;
        }
    }
    if (wide || tall_f64) {
        const int lpr = avg >= 48.0 ? 32 : 16;
        const unsigned grid = grid_for(nrows * lpr, 256, 16);
        if (lpr == 32) {
            if (wide) k_spmv_row<BR, BC, 32, 1, VT, XT><<<grid, 256, 0, st>>>(nrows, rp, col, vals, x, y, alpha, beta, bvec, mode);
            else k_spmv_row<BR, BC, 32, 3, VT, XT><<<grid, 256, 0, st>>>(nrows, rp, col, vals, x, y, alpha, beta, bvec, mode);
        } else {
            k_spmv_row<BR, BC, 16, 2, VT, XT><<<grid, 256, 0, st>>>(nrows, rp, col, vals, x, y, alpha, beta, bvec, mode);
        }
    } else {
        const int G = avg >= 16.0 ? 32 : (avg >= 8.0 ? 16 : 8);
        // up to four rows (G = 32) or 16 rows (G = 8) per warp
        const int64_t rpc = chunk_len(nrows, 8 * (32 / G), 32 * (32 / G));
        const unsigned grid = grid_chunks(nrows, rpc);
        switch (G) {
            case 32: k_spmv_blk<BR, BC, 32, VT, XT><<<grid, 256, 0, st>>>(nrows, rp, col, vals, x, y, alpha, beta, bvec, mode, rpc); break;
            case 16: k_spmv_blk<BR, BC, 16, VT, XT><<<grid, 256, 0, st>>>(nrows, rp, col, vals, x, y, alpha, beta, bvec, mode, rpc); break;
            default: k_spmv_blk<BR, BC, 8, VT, XT><<<grid, 256, 0, st>>>(nrows, rp, col, vals, x, y, alpha, beta, bvec, mode, rpc); break;
        }
    }
    if (fine) instr_end(tk, st);
}

template <typename VT, typename XT>
int rect_spmv(int br, int bc, int64_t nrows, const int32_t *rp, const int32_t *col, const VT *vals, const XT *x,
              XT *y, double alpha, double beta, const XT *bvec, int mode, cudaStream_t st, int64_t nblk) {
#define SG_SPMV_CASE(R, Cc) \
    if (br == R && bc == Cc) { spmv_launch<R, Cc>(nrows, nblk, rp, col, vals, x, y, alpha, beta, bvec, mode, st); SG_CUDA(cudaGetLastError()); return SG_OK; }
    SG_SPMV_CASE(1, 1) SG_SPMV_CASE(2, 2) SG_SPMV_CASE(3, 3) SG_SPMV_CASE(6, 6)
    SG_SPMV_CASE(2, 3) SG_SPMV_CASE(3, 2) SG_SPMV_CASE(3, 6) SG_SPMV_CASE(6, 3)
#undef SG_SPMV_CASE
    return set_error(SG_ERR_ARG, "unsupported BSR block shape");
}
template int rect_spmv<double, double>(int, int, int64_t, const int32_t *, const int32_t *, const double *, const double *,
                                       double *, double, double, const double *, int, cudaStream_t, int64_t);
template int rect_spmv<float, float>(int, int, int64_t, const int32_t *, const int32_t *, const float *, const float *,
                                     float *, double, double, const float *, int, cudaStream_t, int64_t);
template int rect_spmv<float, double>(int, int, int64_t, const int32_t *, const int32_t *, const float *,
                                      const double *, double *, double, double, const double *, int, cudaStream_t,
                                      int64_t);

template <typename VT, typename XT>
int bsr_spmv(const sg_bsr &A, const VT *vals, const XT *x, XT *y, double alpha, double beta, cudaStream_t st) {
    return rect_spmv<VT, XT>(A.b, A.b, A.n_rows, A.d_row_ptr, A.d_col, vals, x, y, alpha, beta, nullptr, 0, st,
                             A.n_blocks);
}
template <typename VT, typename XT>
int bsr_residual(const sg_bsr &A, const VT *vals, const XT *x, const XT *b, XT *r, cudaStream_t st) {
    return rect_spmv<VT, XT>(A.b, A.b, A.n_rows, A.d_row_ptr, A.d_col, vals, x, r, 1.0, 0.0, b, 1, st, A.n_blocks);
}
template int bsr_spmv<double, double>(const sg_bsr &, const double *, const double *, double *, double, double, cudaStream_t);
template int bsr_spmv<float, float>(const sg_bsr &, const float *, const float *, float *, double, double, cudaStream_t);
template int bsr_residual<double, double>(const sg_bsr &, const double *, const double *, const double *, double *, cudaStream_t);
template int bsr_residual<float, float>(const sg_bsr &, const float *, const float *, const float *, float *, cudaStream_t);

// ------------------------------------------------------------------ multi-vector SpMM

// Y(:, c) = A X(:, c) for c < kc (FP64 3x3 blocks; X, Y column-major with leading dimensions
// ldx, ldy, which may be negative to walk the columns backwards).  k_spmv_blk's lane mapping
// (G lanes per block row, one block per lane per step) with KC columns per pass: each block's
// values are read once per pass and multiplied into every column, where KC SpMVs would read
// the matrix KC times.  Partial sums are combined by the same fixed shuffle tree, so every
// column equals the single-vector SpMV of that column bitwise.
template <int G, int KC>
__global__ void __launch_bounds__(256) k_spmm3(int64_t nrows, const int32_t *__restrict__ rp,
                                               const int32_t *__restrict__ col, const double *__restrict__ vals,
                                               const double *__restrict__ X, int64_t ldx, double *__restrict__ Y,
                                               int64_t ldy, int kc) {
    constexpr int GPW = 32 / G;
    const int lane = threadIdx.x & 31, g = lane / G, gl = lane - g * G;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * GPW; base < nrows; base += nwarps * GPW) {
        const int64_t row = base + g;
        double acc[KC][3];
#pragma unroll
        for (int c = 0; c < KC; ++c) acc[c][0] = acc[c][1] = acc[c][2] = 0.0;
        if (row < nrows) {
            const int32_t p1 = rp[row + 1];
            for (int32_t p = rp[row] + gl; p < p1; p += G) {
                const int64_t j = col[p];
                double v[9];
#pragma unroll
                for (int t = 0; t < 9; ++t) v[t] = __ldg(vals + (int64_t)p * 9 + t);
#pragma unroll
                for (int c = 0; c < KC; ++c) {
                    if (c < kc) {
                        const double *xc = X + c * ldx + j * 3;
                        const double x0 = __ldg(xc), x1 = __ldg(xc + 1), x2 = __ldg(xc + 2);
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            acc[c][a] += v[a * 3] * x0;
                            acc[c][a] += v[a * 3 + 1] * x1;
                            acc[c][a] += v[a * 3 + 2] * x2;
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1)
#pragma unroll
            for (int c = 0; c < KC; ++c)
                if (c < kc)
#pragma unroll
                    for (int a = 0; a < 3; ++a) acc[c][a] += __shfl_xor_sync(0xffffffffu, acc[c][a], off);
        if (row < nrows && gl == 0) {
#pragma unroll
            for (int c = 0; c < KC; ++c)
                if (c < kc)
#pragma unroll
                    for (int a = 0; a < 3; ++a) Y[c * ldy + row * 3 + a] = acc[c][a];
        }
    }
}

template <int KC>
static void spmm_pass(const sg_bsr &A, int G, const double *vals, const double *X, int64_t ldx, double *Y,
                      int64_t ldy, int kc, cudaStream_t st) {
    const unsigned grid = grid_for(A.n_rows * G, 256, 16);
    switch (G) {
        case 32: k_spmm3<32, KC><<<grid, 256, 0, st>>>(A.n_rows, A.d_row_ptr, A.d_col, vals, X, ldx, Y, ldy, kc); break;
        case 16: k_spmm3<16, KC><<<grid, 256, 0, st>>>(A.n_rows, A.d_row_ptr, A.d_col, vals, X, ldx, Y, ldy, kc); break;
        default: k_spmm3<8, KC><<<grid, 256, 0, st>>>(A.n_rows, A.d_row_ptr, A.d_col, vals, X, ldx, Y, ldy, kc); break;
    }
}

// Node-interleaved SpMM for many vectors: the KC (8 or 16) columns of a pass are packed so that
// node j's three components of all KC columns are one contiguous run of 3 KC doubles
// ([component][column]); a block's x gather is then 24 KC contiguous bytes however far apart
// the original columns lie.  A warp computes one block row (the lane mapping is described at
// the kernel); the sums are combined in a fixed order, so the result is reproducible.
template <int KC>
__global__ void __launch_bounds__(256) k_spmm3i(int64_t nrows, int64_t rows_per_cta, const int32_t *__restrict__ rp,
                                                const int32_t *__restrict__ col, const double *__restrict__ vals,
                                                const double *__restrict__ Xi, double *__restrict__ Yi) {
    // a warp per block row; lane = (block slot bs in 0 .. 32/KC - 1, column c in 0 .. KC - 1):
    // the warp takes the row's blocks 32/KC at a time, the lanes of a slot load their block's
    // nine values together (coalesced requests) and hand them round by shuffles, each lane
    // reads column c of x_j; the slots' sums are combined by a fixed tree at the end
    constexpr int NS = 32 / KC;
    const int lane = threadIdx.x & 31, c = lane & (KC - 1), bs = lane / KC, base = lane & ~(KC - 1);
    // a CTA owns rows_per_cta consecutive rows, walked in order by its warps
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_cta;
    const int64_t rend = r0 + rows_per_cta < nrows ? r0 + rows_per_cta : nrows;
    for (int64_t row = r0 + (threadIdx.x >> 5); row < rend; row += blockDim.x >> 5) {
        double y0 = 0.0, y1 = 0.0, y2 = 0.0;
        const int32_t p1 = rp[row + 1];
        for (int32_t p0 = rp[row]; p0 < p1; p0 += NS) {
            const int32_t p = p0 + bs;
            const bool live = p < p1;
            int64_t j = 0;
            double av = 0.0, a8 = 0.0;
            if (live) {
                j = col[p];
                if (c < 9) av = __ldg(vals + (int64_t)p * 9 + c);
                if (KC == 8 && c == 0) a8 = __ldg(vals + (int64_t)p * 9 + 8);
            }
            double u0 = 0.0, u1 = 0.0, u2 = 0.0;
            if (live) {
                const double *x = Xi + j * 3 * KC + c;
                u0 = __ldg(x);
                u1 = __ldg(x + KC);
                u2 = __ldg(x + 2 * KC);
            }
            double a[9];
#pragma unroll
            for (int t = 0; t < 8; ++t) a[t] = __shfl_sync(0xffffffffu, av, base + t);
            a[8] = KC == 8 ? __shfl_sync(0xffffffffu, a8, base) : __shfl_sync(0xffffffffu, av, base + 8);
            y0 += a[0] * u0 + a[1] * u1 + a[2] * u2;
            y1 += a[3] * u0 + a[4] * u1 + a[5] * u2;
            y2 += a[6] * u0 + a[7] * u1 + a[8] * u2;
        }
#pragma unroll
        for (int off = KC; off < 32; off <<= 1) {
            y0 += __shfl_xor_sync(0xffffffffu, y0, off);
            y1 += __shfl_xor_sync(0xffffffffu, y1, off);
            y2 += __shfl_xor_sync(0xffffffffu, y2, off);
        }
        if (bs == 0) {
            double *yr = Yi + row * 3 * KC + c;
            yr[0] = y0;
            yr[KC] = y1;
            yr[2 * KC] = y2;
        }
    }
}

// Column-major <-> node-interleaved copies through shared-memory tiles of 64 rows x KC
// columns: every global access runs along a column (read) or along the interleaved rows
// (write) of the tile, so both sides are coalesced.
constexpr int PK_ROWS = 64;
template <int KC>
__global__ void __launch_bounds__(256) k_pack_tiles(int64_t n, int kc, const double *__restrict__ X, int64_t ldx,
                                                    double *__restrict__ Xi) {
    __shared__ double t[PK_ROWS][KC + 1];
    const int64_t ntiles = (n + PK_ROWS - 1) / PK_ROWS;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t r0 = tile * PK_ROWS;
        __syncthreads();
        for (int e = threadIdx.x; e < PK_ROWS * KC; e += blockDim.x) {
            const int c = e / PK_ROWS, r = e - c * PK_ROWS;
            const int64_t rr = r0 + r;
            t[r][c] = (c < kc && rr < n) ? X[(int64_t)c * ldx + rr] : 0.0;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < PK_ROWS * KC; e += blockDim.x) {
            const int r = e / KC, c = e - r * KC;
            const int64_t rr = r0 + r;
            if (rr < n) Xi[rr * KC + c] = t[r][c];
        }
    }
}
template <int KC>
__global__ void __launch_bounds__(256) k_unpack_tiles(int64_t n, int kc, const double *__restrict__ Yi,
                                                      double *__restrict__ Y, int64_t ldy) {
    __shared__ double t[PK_ROWS][KC + 1];
    const int64_t ntiles = (n + PK_ROWS - 1) / PK_ROWS;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t r0 = tile * PK_ROWS;
        __syncthreads();
        for (int e = threadIdx.x; e < PK_ROWS * KC; e += blockDim.x) {
            const int r = e / KC, c = e - r * KC;
            const int64_t rr = r0 + r;
            t[r][c] = rr < n ? Yi[rr * KC + c] : 0.0;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < PK_ROWS * KC; e += blockDim.x) {
            const int c = e / PK_ROWS, r = e - c * PK_ROWS;
            const int64_t rr = r0 + r;
            if (c < kc && rr < n) Y[(int64_t)c * ldy + rr] = t[r][c];
        }
    }
}

// k_spmm3i for 16 columns with a column pair per lane: lane = (block slot bs in 0..3,
// pair s in 0..7) takes columns 2s and 2s + 1, loading them as one 16-byte word per component
// from the node-interleaved copy.  The nine values of a slot's block are loaded by its eight
// lanes together and handed round by shuffles (the ninth by lane 0), as in k_spmm3i, but one
// set of shuffles now serves 16 columns instead of 8, as does each warp-wide gather of x.
// Each step issues the loads of two groups of four blocks before either group's products
// (eight x gathers in flight per warp), and a CTA owns rows_per_cta consecutive rows that its
// warps walk in order, so the x runs of neighbouring rows are reused from L1.
__global__ void __launch_bounds__(256, 4) k_spmm3p(int64_t nrows, int64_t rows_per_cta,
                                                const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                                                const double *__restrict__ vals, const double *__restrict__ Xi,
                                                double *__restrict__ Yi) {
    constexpr int KC = 16, NS = 4, UNR = 2;
    const int lane = threadIdx.x & 31, s = lane & 7, bs = lane >> 3, base = lane & ~7;
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_cta;
    const int64_t rend = r0 + rows_per_cta < nrows ? r0 + rows_per_cta : nrows;
    for (int64_t row = r0 + (threadIdx.x >> 5); row < rend; row += blockDim.x >> 5) {
        double y[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
        const int32_t p1 = rp[row + 1];
        for (int32_t p0 = rp[row]; p0 < p1; p0 += NS * UNR) {
            int64_t j[UNR];
            double av[UNR], a8[UNR];
            bool live[UNR];
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                const int32_t p = p0 + q * NS + bs;
                live[q] = p < p1;
                j[q] = 0;
                av[q] = 0.0;
                a8[q] = 0.0;
                if (live[q]) {
                    j[q] = col[p];
                    av[q] = __ldg(vals + (int64_t)p * 9 + s);
                    if (s == 0) a8[q] = __ldg(vals + (int64_t)p * 9 + 8);
                }
            }
            double2 u[UNR][3];
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                u[q][0] = u[q][1] = u[q][2] = make_double2(0.0, 0.0);
                if (live[q]) {
                    const double2 *x = reinterpret_cast<const double2 *>(Xi + j[q] * 3 * KC) + s;
                    u[q][0] = __ldg(x);
                    u[q][1] = __ldg(x + KC / 2);
                    u[q][2] = __ldg(x + KC);
                }
            }
#pragma unroll
            for (int q = 0; q < UNR; ++q) {
                double a[9];
#pragma unroll
                for (int t = 0; t < 8; ++t) a[t] = __shfl_sync(0xffffffffu, av[q], base + t);
                a[8] = __shfl_sync(0xffffffffu, a8[q], base);
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    y[r][0] += a[3 * r] * u[q][0].x + a[3 * r + 1] * u[q][1].x + a[3 * r + 2] * u[q][2].x;
                    y[r][1] += a[3 * r] * u[q][0].y + a[3 * r + 1] * u[q][1].y + a[3 * r + 2] * u[q][2].y;
                }
            }
        }
#pragma unroll
        for (int off = 8; off < 32; off <<= 1)
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                y[r][0] += __shfl_xor_sync(0xffffffffu, y[r][0], off);
                y[r][1] += __shfl_xor_sync(0xffffffffu, y[r][1], off);
            }
        if (bs == 0) {
            double2 *yr = reinterpret_cast<double2 *>(Yi + row * 3 * KC) + s;
#pragma unroll
            for (int r = 0; r < 3; ++r) yr[r * KC / 2] = make_double2(y[r][0], y[r][1]);
        }
    }
}

int bsr_spmm_interleaved(const sg_bsr &A, const double *vals, const double *X, int64_t ldx, double *Y, int64_t ldy,
                         int k, double *Xi, double *Yi, cudaStream_t st) {
    if (A.b != 3) return set_error(SG_ERR_ARG, "bsr_spmm: 3x3 blocks only");
    const int64_t n = A.n_rows * 3;
    // 16 columns per pass with a column pair per lane (k_spmm3p, about 10 % less per column
    // than the 8-column k_spmm3i at 32-64 columns); a last pass of at most 8 columns takes
    // k_spmm3i, which reads half the gathered bytes of a half-empty 16-column pass
    for (int c0 = 0; c0 < k;) {
        const int rest = k - c0;
        const int KC = rest > 8 ? 16 : 8;
        const int kc = std::min(KC, rest);
        const InstrToken tk = instr_begin(IK_SPMM_AORTH, st);
        instr_units(IK_SPMM_AORTH, kc);
        const int64_t tiles = (n + PK_ROWS - 1) / PK_ROWS;
        const unsigned gt = grid_for(tiles * 256, 256, 8);
        const int64_t rpc = chunk_len(A.n_rows, 8, 64);
        if (KC == 16) {
            k_pack_tiles<16><<<gt, 256, 0, st>>>(n, kc, X + c0 * ldx, ldx, Xi);
            k_spmm3p<<<grid_chunks(A.n_rows, rpc), 256, 0, st>>>(A.n_rows, rpc, A.d_row_ptr, A.d_col, vals, Xi, Yi);
            k_unpack_tiles<16><<<gt, 256, 0, st>>>(n, kc, Yi, Y + c0 * ldy, ldy);
        } else {
            k_pack_tiles<8><<<gt, 256, 0, st>>>(n, kc, X + c0 * ldx, ldx, Xi);
            k_spmm3i<8><<<grid_chunks(A.n_rows, rpc), 256, 0, st>>>(A.n_rows, rpc, A.d_row_ptr, A.d_col, vals, Xi, Yi);
            k_unpack_tiles<8><<<gt, 256, 0, st>>>(n, kc, Yi, Y + c0 * ldy, ldy);
        }
        instr_end(tk, st);
        SG_CUDA(cudaGetLastError());
        c0 += kc;
    }
    return SG_OK;
}

int bsr_spmm(const sg_bsr &A, const double *vals, const double *X, int64_t ldx, double *Y, int64_t ldy, int k,
             cudaStream_t st) {
    if (A.b != 3) return set_error(SG_ERR_ARG, "bsr_spmm: 3x3 blocks only");
    const double avg = A.n_rows > 0 ? (double)A.n_blocks / (double)A.n_rows : 8.0;
    // the same lanes per row as the single-vector SpMV (bitwise-equal columns)
    const int G = avg >= 16.0 ? 32 : (avg >= 8.0 ? 16 : 8);
    // Columns per pass: every block row gathers x entries of its ~28 neighbours from each
    // column, so the pass's input vectors must stay resident in L2 (126 MB) to be read from
    // DRAM about once; keep them within ~48 MB (8 columns on meshes up to 0.6M nodes, 2 on the
    // 3M-DOF slope) and read the matrix once per pass.
    const double vec_bytes = 8.0 * (double)A.n_rows * 3;
    const int kcmax = vec_bytes * 8 <= 48e6 ? 8 : (vec_bytes * 4 <= 48e6 ? 4 : (vec_bytes * 2 <= 48e6 ? 2 : 1));
    for (int c0 = 0; c0 < k; c0 += kcmax) {
        const int kc = std::min(kcmax, k - c0);
        const InstrToken tk = instr_begin(IK_SPMM_AORTH, st);
        instr_units(IK_SPMM_AORTH, kc);
        const double *Xc = X + c0 * ldx;
        double *Yc = Y + c0 * ldy;
        if (kcmax == 8) spmm_pass<8>(A, G, vals, Xc, ldx, Yc, ldy, kc, st);
        else if (kcmax == 4) spmm_pass<4>(A, G, vals, Xc, ldx, Yc, ldy, kc, st);
        else spmm_pass<2>(A, G, vals, Xc, ldx, Yc, ldy, kc, st);
        instr_end(tk, st);
        SG_CUDA(cudaGetLastError());
    }
    return SG_OK;
}

// ------------------------------------------------------------------ FP16 level-0 SpMV

// Lane mapping of k_spmv_blk (G lanes per block row, one block per lane per step); a lane reads
// its block as three 8-byte words (one padded block row each) and accumulates in FP32.
template <int G>
__global__ void __launch_bounds__(256) k_spmv_h3(int64_t nrows, const int32_t *__restrict__ rp,
                                                 const int32_t *__restrict__ col, const uint2 *__restrict__ vals,
                                                 float scale, const float *__restrict__ x, float *__restrict__ y,
                                                 const float *__restrict__ bvec, int mode) {
    constexpr int GPW = 32 / G;
    const int lane = threadIdx.x & 31, g = lane / G, gl = lane - g * G;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * GPW; base < nrows; base += nwarps * GPW) {
        const int64_t row = base + g;
        float acc[3] = {0.f, 0.f, 0.f};
        if (row < nrows) {
            const int32_t p1 = rp[row + 1];
            for (int32_t p = rp[row] + gl; p < p1; p += G) {
                const int64_t j = col[p];
                const float x0 = x[j * 3], x1 = x[j * 3 + 1], x2 = x[j * 3 + 2];
                const uint2 *v = vals + (int64_t)p * 3;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const uint2 w = __ldg(v + a);
                    const float2 lo = __half22float2(*reinterpret_cast<const __half2 *>(&w.x));
                    const float2 hi = __half22float2(*reinterpret_cast<const __half2 *>(&w.y));
                    acc[a] += lo.x * x0 + lo.y * x1 + hi.x * x2;
                }
            }
        }
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1)
#pragma unroll
            for (int a = 0; a < 3; ++a) acc[a] += __shfl_xor_sync(0xffffffffu, acc[a], off);
        if (row < nrows && gl == 0) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const int64_t k = row * 3 + a;
                y[k] = mode == 1 ? bvec[k] - scale * acc[a] : scale * acc[a];
            }
        }
    }
}

int h3_spmv(int64_t nrows, int64_t nblk, const int32_t *rp, const int32_t *col, const uint2 *vals, float scale,
            const float *x, float *y, const float *bvec, int mode, cudaStream_t st) {
    const double avg = nblk > 0 && nrows > 0 ? (double)nblk / (double)nrows : 8.0;
    const InstrToken tk = instr_begin(IK_SPMV3_F16, st);
    const int G = avg >= 16.0 ? 32 : (avg >= 8.0 ? 16 : 8);
    const unsigned grid = grid_for(nrows * G, 256, 16);
    switch (G) {
        case 32: k_spmv_h3<32><<<grid, 256, 0, st>>>(nrows, rp, col, vals, scale, x, y, bvec, mode); break;
        case 16: k_spmv_h3<16><<<grid, 256, 0, st>>>(nrows, rp, col, vals, scale, x, y, bvec, mode); break;
        default: k_spmv_h3<8><<<grid, 256, 0, st>>>(nrows, rp, col, vals, scale, x, y, bvec, mode); break;
    }
    instr_end(tk, st);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

__global__ void k_to_float_half3(int64_t nrows3, const double *__restrict__ A, float *__restrict__ A32,
                                 uint2 *__restrict__ A16, float inv_scale) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrows3; r += (int64_t)gridDim.x * blockDim.x) {
        float f[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            f[c] = (float)A[r * 3 + c];
            A32[r * 3 + c] = f[c];
        }
        __half h[4];
#pragma unroll
        for (int c = 0; c < 3; ++c) h[c] = __float2half_rn(fminf(fmaxf(f[c] * inv_scale, -65504.f), 65504.f));
        h[3] = __float2half_rn(0.f);
        const __half2 lo = __halves2half2(h[0], h[1]), hi = __halves2half2(h[2], h[3]);
        uint2 w;
        w.x = *reinterpret_cast<const unsigned *>(&lo);
        w.y = *reinterpret_cast<const unsigned *>(&hi);
        A16[r] = w;
    }
}

int to_float_half3(int64_t nblk, const double *A, float *A32, uint2 *A16, float scale, cudaStream_t st) {
    const int64_t n = nblk * 3;
    k_to_float_half3<<<grid_for(n, 256), 256, 0, st>>>(n, A, A32, A16, 1.0f / scale);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

// ------------------------------------------------------------------ dots and GEMV

__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x < 32) {
        t = (l < (int)(blockDim.x >> 5)) ? sh[l] : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
    }
    return t;  // valid in thread 0
}

// partial[i * gridDim.x + block] = sum over this block's row chunk of V(r, i) * w(r)
__global__ void __launch_bounds__(DOT_THREADS) k_multidot(int64_t n, int m, const double *__restrict__ V, int64_t ldv,
                                                          const double *__restrict__ w, double *__restrict__ partial) {
    __shared__ double sh[32];
    const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = blockIdx.x * chunk, r1 = min(n, r0 + chunk);
    int i = 0;
    for (; i + 4 <= m; i += 4) {
        double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
            const double wr = w[r];
            s0 += V[(i + 0) * ldv + r] * wr;
            s1 += V[(i + 1) * ldv + r] * wr;
            s2 += V[(i + 2) * ldv + r] * wr;
            s3 += V[(i + 3) * ldv + r] * wr;
        }
        s0 = block_sum(s0, sh);
        if (threadIdx.x == 0) partial[(i + 0) * gridDim.x + blockIdx.x] = s0;
        s1 = block_sum(s1, sh);
        if (threadIdx.x == 0) partial[(i + 1) * gridDim.x + blockIdx.x] = s1;
        s2 = block_sum(s2, sh);
        if (threadIdx.x == 0) partial[(i + 2) * gridDim.x + blockIdx.x] = s2;
        s3 = block_sum(s3, sh);
        if (threadIdx.x == 0) partial[(i + 3) * gridDim.x + blockIdx.x] = s3;
    }
    for (; i < m; ++i) {
        double s = 0;
        for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) s += V[i * ldv + r] * w[r];
        s = block_sum(s, sh);
        if (threadIdx.x == 0) partial[i * gridDim.x + blockIdx.x] = s;
    }
}

// out[i] = sum_b partial[i * nb + b]   (one block per column, fixed order)
__global__ void k_reduce_partials(int m, int nb, const double *__restrict__ partial, double *__restrict__ out) {
    __shared__ double sh[32];
    for (int i = blockIdx.x; i < m; i += gridDim.x) {
        double s = 0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[(int64_t)i * nb + b];
        s = block_sum(s, sh);
        if (threadIdx.x == 0) out[i] = s;
    }
}

int multidot(int64_t n, int m, const double *V, int64_t ldv, const double *w, double *partial, double *out,
             cudaStream_t st) {
    if (m <= 0) return SG_OK;
    count_launch(2);
    k_multidot<<<DOT_BLOCKS, DOT_THREADS, 0, st>>>(n, m, V, ldv, w, partial);
    k_reduce_partials<<<std::min(m, 1024), 256, 0, st>>>(m, DOT_BLOCKS, partial, out);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

template <int SIGN>
__global__ void k_gemv(int64_t n, int m, const double *__restrict__ V, int64_t ldv, const double *__restrict__ h,
                       double *__restrict__ w) {
    extern __shared__ double hs[];
    for (int i = threadIdx.x; i < m; i += blockDim.x) hs[i] = h[i];
    __syncthreads();
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        double s = 0;
        for (int i = 0; i < m; ++i) s += hs[i] * V[i * ldv + r];
        w[r] = SIGN > 0 ? w[r] + s : w[r] - s;
    }
}

int gemv_sub(int64_t n, int m, const double *V, int64_t ldv, const double *h, double *w, cudaStream_t st) {
    if (m <= 0) return SG_OK;
    k_gemv<-1><<<grid_for(n, 256, 8), 256, sizeof(double) * m, st>>>(n, m, V, ldv, h, w);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

int gemv_add(int64_t n, int m, const double *V, int64_t ldv, const double *y, double *x, cudaStream_t st) {
    if (m <= 0) return SG_OK;
    k_gemv<1><<<grid_for(n, 256, 8), 256, sizeof(double) * m, st>>>(n, m, V, ldv, y, x);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

// ------------------------------------------------------------------ tall-skinny block products
//
// For the blocked Gram-Schmidt of the A-orthogonalisation: C = U' X with U an n x m basis and
// X an n x b block (b <= TS_B), and Y -= U C.  Each of TS_CTAS CTAs owns a contiguous row range
// and runs over it in tiles of TS_ROWS rows: the tile's X rows and, 16 columns at a time, its
// U rows are staged in shared memory and thread (j, l) adds U(r, j) X(r, l) over the tile's rows;
// the CTAs' partial sums are then added in CTA order (bitwise reproducible).  U is read once
// for the whole block instead of once per column of X.
constexpr int TS_B = 16, TS_ROWS = 32, TS_CTAS = 296, TS_MAXM = 256;

__global__ void __launch_bounds__(256) k_gemm_tn_partial(int64_t n, int m, int b, const double *__restrict__ U,
                                                         int64_t ldu, const double *__restrict__ X, int64_t ldx,
                                                         double *__restrict__ part) {
    __shared__ double sX[TS_ROWS][TS_B];
    __shared__ double sU[TS_ROWS][17];
    const int t = threadIdx.x, jj = t >> 4, ll = t & 15;
    const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = blockIdx.x * chunk, r1 = min(n, r0 + chunk);
    constexpr int MAXG = TS_MAXM / 16;
    double acc[MAXG];
#pragma unroll
    for (int g = 0; g < MAXG; ++g) acc[g] = 0.0;
    const int ng = (m + 15) / 16;
    for (int64_t rt = r0; rt < r1; rt += TS_ROWS) {
        const int nr = (int)min((int64_t)TS_ROWS, r1 - rt);
        __syncthreads();
        for (int e = t; e < TS_ROWS * TS_B; e += 256) {
            const int r = e % TS_ROWS, l = e / TS_ROWS;
            sX[r][l] = (r < nr && l < b) ? X[l * ldx + rt + r] : 0.0;
        }
#pragma unroll
        for (int g = 0; g < MAXG; ++g) {
            if (g < ng) {
                __syncthreads();
                for (int e = t; e < TS_ROWS * 16; e += 256) {
                    const int r = e % TS_ROWS, j = e / TS_ROWS, jc = g * 16 + j;
                    sU[r][j] = (r < nr && jc < m) ? U[jc * ldu + rt + r] : 0.0;
                }
                __syncthreads();
                double a = acc[g];
#pragma unroll 8
                for (int r = 0; r < TS_ROWS; ++r) a += sU[r][jj] * sX[r][ll];
                acc[g] = a;
            }
        }
    }
#pragma unroll
    for (int g = 0; g < MAXG; ++g) {
        const int j = g * 16 + jj;
        if (g < ng && j < m && ll < b) part[((int64_t)blockIdx.x * m + j) * TS_B + ll] = acc[g];
    }
}

// C(j, l) = sign(j) * sum over CTAs of the partials (sign may be null)
__global__ void k_gemm_tn_reduce(int m, int b, int nparts, const double *__restrict__ part,
                                 const double *__restrict__ sign, double *__restrict__ C, int ldc) {
    for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < m * b; o += gridDim.x * blockDim.x) {
        const int j = o / b, l = o - j * b;
        double s = 0.0;
        for (int p = 0; p < nparts; ++p) s += part[((int64_t)p * m + j) * TS_B + l];
        C[j + (int64_t)l * ldc] = sign ? s * sign[j] : s;
    }
}

// Y(:, l) -= U(:, 0:m) C(:, l) for l < b; C is m x b column-major (ldc), staged in shared memory
__global__ void __launch_bounds__(256) k_gemm_nn_sub(int64_t n, int m, int b, const double *__restrict__ U,
                                                     int64_t ldu, const double *__restrict__ C, int ldc,
                                                     double *__restrict__ Y, int64_t ldy) {
    extern __shared__ double sC[];   // [j][l], m x TS_B
    for (int e = threadIdx.x; e < m * TS_B; e += blockDim.x) {
        const int j = e / TS_B, l = e - j * TS_B;
        sC[e] = l < b ? C[j + (int64_t)l * ldc] : 0.0;
    }
    __syncthreads();
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        double y[TS_B];
#pragma unroll
        for (int l = 0; l < TS_B; ++l) y[l] = 0.0;
        for (int j = 0; j < m; ++j) {
            const double u = U[j * ldu + r];
#pragma unroll
            for (int l = 0; l < TS_B; ++l) y[l] += u * sC[j * TS_B + l];
        }
        for (int l = 0; l < b; ++l) Y[l * ldy + r] -= y[l];
    }
}

int gemm_tn(int64_t n, int m, int b, const double *U, int64_t ldu, const double *X, int64_t ldx,
            const double *sign, double *C, int ldc, double *part, cudaStream_t st) {
    if (m <= 0 || b <= 0) return SG_OK;
    if (m > TS_MAXM || b > TS_B) return set_error(SG_ERR_ARG, "gemm_tn: block too large");
    count_launch(2);
    k_gemm_tn_partial<<<TS_CTAS, 256, 0, st>>>(n, m, b, U, ldu, X, ldx, part);
    k_gemm_tn_reduce<<<(m * b + 255) / 256, 256, 0, st>>>(m, b, TS_CTAS, part, sign, C, ldc);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

int gemm_nn_sub(int64_t n, int m, int b, const double *U, int64_t ldu, const double *C, int ldc, double *Y,
                int64_t ldy, cudaStream_t st) {
    if (m <= 0 || b <= 0) return SG_OK;
    if (m > TS_MAXM || b > TS_B) return set_error(SG_ERR_ARG, "gemm_nn_sub: block too large");
    k_gemm_nn_sub<<<grid_for(n, 256, 8), 256, sizeof(double) * m * TS_B, st>>>(n, m, b, U, ldu, C, ldc, Y, ldy);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

// ------------------------------------------------------------------ Gram-matrix A-orthogonalisation
//
// The one-pass recurrence of A_orthogonalize.m expressed in the coordinates of the input
// columns S (processing order): with G = S' (A S), the kept columns are U = S T for an upper
// triangular T, every coefficient (A s_i)' u_j = (T' G)(j, i) and every A-norm temp' (A s_i)
// comes from G, so the n-long work is one Gram product and two tall-skinny products
// (U = S T, A U = (A S) T) instead of a sequence of vector passes per column.

__device__ __forceinline__ uint32_t sh_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sh_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// One FP64 MMA of the tensor cores: the 8 x 8 tile (c0, c1) += A (8 x 4, a) B (4 x 8, b),
// fragments as in the PTX m8n8k4 .f64 layout.
__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// Partial sums of one 16 NA x 16 NA tile of G (rows m0 + [0, 16 NA), columns i0 + [0, 16 NA))
// over this CTA's row range, in tiles of GR_R rows staged in shared memory ([column][row],
// padded) by 8-byte cp.async, two stages; thread (mb, ib) owns the entries
// (m0 + mb + 16 a, i0 + ib + 16 b).  part: gridDim.x x (16 NA)^2.  On a diagonal tile
// (DIAG, m0 == i0) the products with a > b, all below the diagonal, are not formed.
constexpr int GR_R = 32, GR_LD = GR_R + 1;
template <int NA, bool DIAG>
__global__ void __launch_bounds__(256) k_gram_partial(int64_t n, int k, const double *__restrict__ S, int64_t lds,
                                                      const double *__restrict__ AS, int64_t ldas, int m0, int i0,
                                                      double *__restrict__ part) {
    constexpr int TW = 16 * NA;
    extern __shared__ double gsm[];   // [2 stages][S tile, AS tile][TW][GR_LD]
    const int t = threadIdx.x, ib = t & 15, mb = t >> 4;
    const int64_t chunk = ((n + gridDim.x - 1) / gridDim.x + GR_R - 1) / GR_R * GR_R;
    const int64_t r0 = blockIdx.x * chunk, r1 = min(n, r0 + chunk);
    double acc[NA][NA];
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NA; ++b) acc[a][b] = 0.0;
    auto stage = [&](int st, int64_t rt) {
        double *sS = gsm + st * 2 * TW * GR_LD, *sA = sS + TW * GR_LD;
        for (int e = t; e < TW * GR_R; e += 256) {
            const int c = e / GR_R, r = e - c * GR_R;
            const int64_t row = rt + r;
            const int cm = m0 + c, ci = i0 + c;
            if (row < r1 && cm < k) cp_async8(sS + c * GR_LD + r, S + cm * lds + row);
            else sS[c * GR_LD + r] = 0.0;
            if (row < r1 && ci < k) cp_async8(sA + c * GR_LD + r, AS + ci * ldas + row);
            else sA[c * GR_LD + r] = 0.0;
        }
    };
    if (r0 < r1) stage(0, r0);
    cp_async_commit();
    int it = 0;
    for (int64_t rt = r0; rt < r1; rt += GR_R, ++it) {
        if (rt + GR_R < r1) stage((it + 1) & 1, rt + GR_R);
        cp_async_commit();
        cp_async_wait1();
        __syncthreads();
        const double *sS = gsm + (it & 1) * 2 * TW * GR_LD, *sA = sS + TW * GR_LD;
#pragma unroll 4
        for (int r = 0; r < GR_R; ++r) {
            double sv[NA], xv[NA];
#pragma unroll
            for (int a = 0; a < NA; ++a) sv[a] = sS[(mb + 16 * a) * GR_LD + r];
#pragma unroll
            for (int b = 0; b < NA; ++b) xv[b] = sA[(ib + 16 * b) * GR_LD + r];
#pragma unroll
            for (int a = 0; a < NA; ++a)
#pragma unroll
                for (int b = 0; b < NA; ++b)
                    if (!DIAG || a <= b) acc[a][b] += sv[a] * xv[b];   // (a > b): m > i, unused
        }
        __syncthreads();
    }
    double *out = part + (int64_t)blockIdx.x * TW * TW;
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NA; ++b) out[(mb + 16 * a) * TW + ib + 16 * b] = acc[a][b];
}

// k_gram_partial for 64 x 64 tiles on the FP64 tensor cores (mma.sync m8n8k4 .f64): the
// same row tiles and stages (pitch padded to GR_R + 4 for conflict-free fragment reads);
// warp w owns G rows m0 + 32 (w & 1) .. + 32 and columns i0 + 16 (w >> 1) .. + 16 as 4 x 2
// tiles of 8 x 8; A = S' (a = S[row t][column m0 + g]), B = AS (b = AS[row t][column g]).
constexpr int GM_TW = 64, GM_LD = GR_R + 4;
constexpr size_t GM_SMEM = sizeof(double) * 2 * 2 * GM_TW * GM_LD;
__global__ void __launch_bounds__(256) k_gram_partial_mma(int64_t n, int k, const double *__restrict__ S,
                                                          int64_t lds, const double *__restrict__ AS, int64_t ldas,
                                                          int m0, int i0, double *__restrict__ part) {
    extern __shared__ double gmsm[];   // [2 stages][S tile, AS tile][GM_TW][GM_LD]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp & 1) * 32, wi = (warp >> 1) * 16;
    const int64_t chunk = ((n + gridDim.x - 1) / gridDim.x + GR_R - 1) / GR_R * GR_R;
    const int64_t r0 = blockIdx.x * chunk, r1 = min(n, r0 + chunk);
    double acc[4][2][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    auto stage = [&](int st, int64_t rt) {
        double *sS = gmsm + st * 2 * GM_TW * GM_LD, *sA = sS + GM_TW * GM_LD;
        for (int e = tid; e < GM_TW * GR_R; e += 256) {
            const int c = e / GR_R, r = e - c * GR_R;
            const int64_t row = rt + r;
            const int cm = m0 + c, ci = i0 + c;
            if (row < r1 && cm < k) cp_async8(sS + c * GM_LD + r, S + cm * lds + row);
            else sS[c * GM_LD + r] = 0.0;
            if (row < r1 && ci < k) cp_async8(sA + c * GM_LD + r, AS + ci * ldas + row);
            else sA[c * GM_LD + r] = 0.0;
        }
    };
    if (r0 < r1) stage(0, r0);
    cp_async_commit();
    int it = 0;
    for (int64_t rt = r0; rt < r1; rt += GR_R, ++it) {
        if (rt + GR_R < r1) stage((it + 1) & 1, rt + GR_R);
        cp_async_commit();
        cp_async_wait1();
        __syncthreads();
        const double *sS = gmsm + (it & 1) * 2 * GM_TW * GM_LD, *sA = sS + GM_TW * GM_LD;
#pragma unroll
        for (int k4 = 0; k4 < GR_R; k4 += 4) {
            double a[4], b[2];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = sS[(wm + 8 * i + g) * GM_LD + k4 + t];
#pragma unroll
            for (int j = 0; j < 2; ++j) b[j] = sA[(wi + 8 * j + g) * GM_LD + k4 + t];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
        __syncthreads();
    }
    double *out = part + (int64_t)blockIdx.x * GM_TW * GM_TW;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) out[(wm + 8 * i + g) * GM_TW + wi + 8 * j + 2 * t + h] = acc[i][j][h];
}

// G(m0 + ml, i0 + il) = the sum of the CTAs' partials: a warp per entry, lane l adding the
// partials l, l + 32, ... and a fixed shuffle tree combining the lanes (ldg: G's leading
// dimension)
__global__ void k_gram_reduce(int k, int TW, int nparts, const double *__restrict__ part, int m0, int i0,
                              double *__restrict__ G, int ldg) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int o = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; o < TW * TW; o += nw) {
        const int ml = o / TW, il = o - ml * TW;
        if (m0 + ml >= k || i0 + il >= k) continue;   // uniform over the warp
        double s = 0.0;
        for (int p = lane; p < nparts; p += 32) s += part[(int64_t)p * TW * TW + o];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) G[(m0 + ml) + (int64_t)(i0 + il) * ldg] = s;
    }
}

// The recurrence on one CTA.  G: k x k column-major (entries m <= i used); Tp: k x k scratch
// (column p = the coefficients of kept column p in S, zero when dropped); out: Ta k x k,
// row-major [m][o], the columns of T in output order (kept columns, last processed first);
// nt[i] = the A-norm^2 of column i, sig[i] its sign; *kout = the number kept and pmap[o] the
// processing index of output column o (decreasing in o).  G and Tp are staged in shared
// memory when 2 k^2 doubles fit (smem_k2 != 0).
__global__ void __launch_bounds__(256) k_gram_recurrence(int k, const double *__restrict__ Gg, double *__restrict__ Tpg,
                                                         double eps, double *__restrict__ Ta,
                                                         double *__restrict__ nt, double *__restrict__ sig,
                                                         int32_t *__restrict__ kout, int32_t *__restrict__ pmap,
                                                         int smem_k2) {
    extern __shared__ double rsm[];   // [c: k][t: k][red: 256][map: k ints] (+ G, Tp when staged)
    double *c = rsm, *tv = c + k, *red = tv + k;
    int *map = reinterpret_cast<int *>(red + 256);
    const double *G = Gg;
    double *Tp = Tpg;
    const int tid = threadIdx.x;
    if (smem_k2) {
        double *sG = red + 256 + (k + 1) / 2;
        double *sT = sG + (int64_t)k * k;
        for (int e = tid; e < k * k; e += 256) {
            const int i = e / k, m = e - i * k;
            sG[e] = m <= i ? Gg[e] : 0.0;
        }
        G = sG;
        Tp = sT;
    }
    __syncthreads();
    for (int i = 0; i < k; ++i) {
        const double *Gi = G + (int64_t)i * k;
        // c_j = sig_j (A s_i)' u_j for the columns processed before
        for (int j = tid; j < i; j += 256) {
            const double *Tj = Tp + (int64_t)j * k;
            double s = 0.0;
            for (int m = 0; m <= j; ++m) s += Tj[m] * Gi[m];
            c[j] = sig[j] * s;
        }
        __syncthreads();
        // temp = s_i - sum_j c_j u_j in S coordinates (entries m <= i)
        for (int m = tid; m <= i; m += 256) {
            double v = m == i ? 1.0 : 0.0;
            for (int j = m; j < i; ++j) v -= c[j] * Tp[m + (int64_t)j * k];
            tv[m] = v;
        }
        __syncthreads();
        // temp' (A s_i), a fixed-order tree
        double p = 0.0;
        for (int m = tid; m <= i; m += 256) p += tv[m] * Gi[m];
        red[tid] = p;
        __syncthreads();
        for (int h = 128; h > 0; h >>= 1) {
            if (tid < h) red[tid] += red[tid + h];
            __syncthreads();
        }
        const double nrm = red[0];
        const bool keep = fabs(nrm) > eps;
        const double sc = keep ? 1.0 / sqrt(fabs(nrm)) : 0.0;
        double *Ti = Tp + (int64_t)i * k;
        for (int m = tid; m < k; m += 256) Ti[m] = m <= i ? tv[m] * sc : 0.0;
        if (tid == 0) {
            nt[i] = nrm;
            sig[i] = (keep && nrm < 0.0) ? -1.0 : 1.0;
        }
        __syncthreads();
    }
    if (tid == 0) {
        int o = 0;
        for (int i = k - 1; i >= 0; --i)
            if (fabs(nt[i]) > eps) map[o++] = i;
        *kout = o;
        red[0] = (double)o;
    }
    __syncthreads();
    const int ko = (int)red[0];
    for (int o = tid; o < ko; o += 256) pmap[o] = map[o];
    for (int e = tid; e < k * k; e += 256) {
        const int m = e / k, o = e - m * k;
        Ta[e] = o < ko ? Tp[m + (int64_t)map[o] * k] : 0.0;
    }
}

// Y(:, o) = X(:, 0:k) Ta(:, o) for o < *kout, output columns in chunks of 8 NJ (blockIdx.y):
// X rows in tiles of TA_R, columns of X (and rows of Ta) in stages of TA_MC through shared
// memory (8-byte cp.async, two stages); thread (lane, warp) owns rows lane + 32 q and output
// columns o0 + warp NJ + j.
constexpr int TA_R = 128, TA_MC = 16;
template <int NJ>
__global__ void __launch_bounds__(256, (NJ > 4 ? 2 : 3)) k_ts_apply(int64_t n, int k, const int32_t *__restrict__ kout,
                                                  const int32_t *__restrict__ pmap, const double *__restrict__ X,
                                                  int64_t ldx, const double *__restrict__ Ta, double *__restrict__ Y,
                                                  int64_t ldy) {
    constexpr int OC = 8 * NJ;
    __shared__ double sX[2][TA_MC][TA_R];
    __shared__ __align__(16) double sT[2][TA_MC][OC];
    const int ko = *kout;
    const int o0 = blockIdx.y * OC;
    if (o0 >= ko) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // the chunk's columns depend on inputs 0 .. pmap[o0] only (Ta is zero below)
    const int kk = min(k, pmap[o0] + 1);
    const int nmc = (kk + TA_MC - 1) / TA_MC;
    const int64_t ntiles = (n + TA_R - 1) / TA_R;
    const int64_t nsteps = ((ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x) * nmc;   // (tile, chunk) pairs
    if (blockIdx.x >= ntiles) return;
    auto stage = [&](int st, int64_t s) {
        const int64_t rt = (blockIdx.x + (s / nmc) * gridDim.x) * TA_R;
        const int mc = (int)(s % nmc) * TA_MC;
        for (int e = tid; e < TA_MC * TA_R; e += 256) {
            const int cc = e / TA_R, r = e - cc * TA_R;
            const int64_t row = rt + r;
            const int col = mc + cc;
            if (row < n && col < kk) cp_async8(&sX[st][cc][r], X + col * ldx + row);
            else sX[st][cc][r] = 0.0;
        }
        for (int e = tid; e < TA_MC * OC; e += 256) {
            const int cc = e / OC, oo = e - cc * OC;
            const int m = mc + cc, o = o0 + oo;
            sT[st][cc][oo] = (m < kk && o < ko) ? Ta[(int64_t)m * k + o] : 0.0;
        }
    };
    double acc[4][NJ];
    stage(0, 0);
    cp_async_commit();
    for (int64_t s = 0; s < nsteps; ++s) {
        if (s % nmc == 0) {
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int j = 0; j < NJ; ++j) acc[q][j] = 0.0;
        }
        if (s + 1 < nsteps) stage((int)((s + 1) & 1), s + 1);
        cp_async_commit();
        cp_async_wait1();
        __syncthreads();
        const int st = (int)(s & 1);
#pragma unroll 4
        for (int cc = 0; cc < TA_MC; ++cc) {
            double xv[4], tw[NJ];
#pragma unroll
            for (int q = 0; q < 4; ++q) xv[q] = sX[st][cc][lane + 32 * q];
            if constexpr (NJ % 2 == 0) {   // the warp's NJ coefficients as NJ/2 16-byte broadcasts
                const double2 *t2 = reinterpret_cast<const double2 *>(&sT[st][cc][warp * NJ]);
#pragma unroll
                for (int j = 0; j < NJ / 2; ++j) {
                    const double2 v = t2[j];
                    tw[2 * j] = v.x;
                    tw[2 * j + 1] = v.y;
                }
            } else {
#pragma unroll
                for (int j = 0; j < NJ; ++j) tw[j] = sT[st][cc][warp * NJ + j];
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int j = 0; j < NJ; ++j) acc[q][j] += xv[q] * tw[j];
        }
        __syncthreads();
        if (s % nmc == nmc - 1) {
            const int64_t rt = (blockIdx.x + (s / nmc) * gridDim.x) * TA_R;
#pragma unroll
            for (int j = 0; j < NJ; ++j) {
                const int o = o0 + warp * NJ + j;
                if (o >= ko) continue;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int64_t row = rt + lane + 32 * q;
                    if (row < n) Y[o * ldy + row] = acc[q][j];
                }
            }
        }
    }
}

int gram_upper(int64_t n, int k, const double *S, int64_t lds, const double *AS, int64_t ldas, double *G,
               double *part, cudaStream_t st) {
    if (k <= 0) return SG_OK;
    const int NA = k <= 16 ? 1 : (k <= 32 ? 2 : (k <= 48 ? 3 : 4));
    const int TW = 16 * NA;
    const size_t smem = sizeof(double) * 2 * 2 * TW * GR_LD;
    static thread_local bool configured = false;
    if (!configured) {   // stages of 48- and 64-wide tiles exceed the default 48 KB
        SG_CUDA(cudaFuncSetAttribute(k_gram_partial<3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(sizeof(double) * 2 * 2 * 48 * GR_LD)));
        SG_CUDA(cudaFuncSetAttribute(k_gram_partial_mma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)GM_SMEM));
        configured = true;
    }
    const int nt = (k + TW - 1) / TW;
    for (int p = 0; p < nt; ++p)
        for (int q = 0; q <= p; ++q) {
            count_launch(2);
            const int m0 = q * TW, i0 = p * TW;
            switch (NA) {
                case 1: k_gram_partial<1, true><<<GR_CTAS, 256, smem, st>>>(n, k, S, lds, AS, ldas, m0, i0, part); break;
                case 2: k_gram_partial<2, true><<<GR_CTAS, 256, smem, st>>>(n, k, S, lds, AS, ldas, m0, i0, part); break;
                case 3: k_gram_partial<3, true><<<GR_CTAS, 256, smem, st>>>(n, k, S, lds, AS, ldas, m0, i0, part); break;
                default:   // 64-wide tiles on the FP64 tensor cores
                    k_gram_partial_mma<<<GR_CTAS, 256, GM_SMEM, st>>>(n, k, S, lds, AS, ldas, m0, i0, part);
                    break;
            }
            k_gram_reduce<<<(TW * TW * 32 + 255) / 256, 256, 0, st>>>(k, TW, GR_CTAS, part, m0, i0, G, k);
            SG_CUDA(cudaGetLastError());
        }
    return SG_OK;
}

int gram_recurrence(int k, const double *G, double *Tp, double eps, double *Ta, double *nt, double *sig,
                    int32_t *kout, int32_t *pmap, cudaStream_t st) {
    if (k <= 0) return SG_OK;
    const size_t base = sizeof(double) * (2 * (size_t)k + 256 + (k + 1) / 2);
    const size_t full = base + sizeof(double) * 2 * (size_t)k * k;
    const bool staged = full <= 200 * 1024;
    const size_t smem = staged ? full : base;
    static thread_local size_t configured = 0;
    if (smem > 48 * 1024 && smem > configured) {
        SG_CUDA(cudaFuncSetAttribute(k_gram_recurrence, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured = smem;
    }
    count_launch();
    k_gram_recurrence<<<1, 256, smem, st>>>(k, G, Tp, eps, Ta, nt, sig, kout, pmap, staged ? 1 : 0);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

// The 64-column variant of k_ts_apply on the FP64 tensor cores (mma.sync m8n8k4 .f64, the
// FP64 MMA of sm_100a): CTA tile 128 rows x 64 output columns, inputs in stages of TM_MC
// columns of X / rows of Ta staged by 8-byte cp.async (two stages, pitches padded by 4
// doubles so the fragment reads are free of bank conflicts); warp w owns rows 32 (w & 3) ..
// + 32 and columns 32 (w >> 2) .. + 32 as 4 x 4 tiles of 8 x 8, an MMA per tile and step of 4
// inputs.  Fragments (PTX m8n8k4 f64): A (8 x 4) a = X[row g][input t], B (4 x 8)
// b = Ta[input t][column g], C (8 x 8) c0, c1 = [row g][columns 2 t, 2 t + 1], with
// g = lane / 4, t = lane % 4.
constexpr int TM_MC = 16, TM_OC = 64, TM_XP = TA_R + 4, TM_TP = TM_OC + 4;
constexpr size_t TM_SMEM = sizeof(double) * 2 * TM_MC * (TM_XP + TM_TP);

__global__ void __launch_bounds__(256) k_ts_apply_mma(int64_t n, int k, const int32_t *__restrict__ kout,
                                                      const int32_t *__restrict__ pmap, const double *__restrict__ X,
                                                      int64_t ldx, const double *__restrict__ Ta, double *__restrict__ Y,
                                                      int64_t ldy) {
    extern __shared__ double tmsm[];
    double *sXb = tmsm, *sTb = tmsm + 2 * TM_MC * TM_XP;   // [stage][input][row] / [stage][input][column]
    const int ko = *kout;
    const int o0 = blockIdx.y * TM_OC;
    if (o0 >= ko) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wr = (warp & 3) * 32, wc = (warp >> 2) * 32;
    const int kk = min(k, pmap[o0] + 1);
    const int nmc = (kk + TM_MC - 1) / TM_MC;
    const int64_t ntiles = (n + TA_R - 1) / TA_R;
    if (blockIdx.x >= ntiles) return;
    const int64_t nsteps = ((ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x) * nmc;
    auto stage = [&](int stg, int64_t s) {
        const int64_t rt = (blockIdx.x + (s / nmc) * gridDim.x) * TA_R;
        const int mc = (int)(s % nmc) * TM_MC;
        double *sX = sXb + stg * TM_MC * TM_XP, *sT = sTb + stg * TM_MC * TM_TP;
        for (int e = tid; e < TM_MC * TA_R; e += 256) {
            const int cc = e / TA_R, r = e - cc * TA_R;
            const int64_t row = rt + r;
            const int col = mc + cc;
            if (row < n && col < kk) cp_async8(sX + cc * TM_XP + r, X + col * ldx + row);
            else sX[cc * TM_XP + r] = 0.0;
        }
        for (int e = tid; e < TM_MC * TM_OC; e += 256) {
            const int cc = e / TM_OC, oo = e - cc * TM_OC;
            const int m = mc + cc, o = o0 + oo;
            sT[cc * TM_TP + oo] = (m < kk && o < ko) ? Ta[(int64_t)m * k + o] : 0.0;
        }
    };
    double acc[4][4][2];
    stage(0, 0);
    cp_async_commit();
    for (int64_t s = 0; s < nsteps; ++s) {
        if (s % nmc == 0) {
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
        }
        if (s + 1 < nsteps) stage((int)((s + 1) & 1), s + 1);
        cp_async_commit();
        cp_async_wait1();
        __syncthreads();
        const double *sX = sXb + (int)(s & 1) * TM_MC * TM_XP, *sT = sTb + (int)(s & 1) * TM_MC * TM_TP;
#pragma unroll
        for (int k4 = 0; k4 < TM_MC; k4 += 4) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = sX[(k4 + t) * TM_XP + wr + 8 * i + g];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = sT[(k4 + t) * TM_TP + wc + 8 * j + g];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
        __syncthreads();
        if (s % nmc == nmc - 1) {
            const int64_t rt = (blockIdx.x + (s / nmc) * gridDim.x) * TA_R;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int64_t row = rt + wr + 8 * i + g;
                if (row >= n) continue;
#pragma unroll
                for (int j = 0; j < 4; ++j)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int o = o0 + wc + 8 * j + 2 * t + h;
                        if (o < ko) Y[o * ldy + row] = acc[i][j][h];
                    }
            }
        }
    }
}

int ts_apply(int64_t n, int k, const int32_t *kout, const int32_t *pmap, const double *X, int64_t ldx,
             const double *Ta, double *Y, int64_t ldy, cudaStream_t st) {
    if (k <= 0 || n <= 0) return SG_OK;
    const int64_t ntiles = (n + TA_R - 1) / TA_R;
    if (k >= 64) {   // 64-column chunks on the FP64 tensor cores
        static thread_local int resident_mma = 0;
        if (!resident_mma) {
            SG_CUDA(cudaFuncSetAttribute(k_ts_apply_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TM_SMEM));
            int r = 0;
            SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_ts_apply_mma, 256, TM_SMEM));
            resident_mma = std::max(1, r);
        }
        const dim3 grid((unsigned)std::min<int64_t>(ntiles, (int64_t)sm_count() * resident_mma),
                        (unsigned)((k + TM_OC - 1) / TM_OC));
        count_launch();
        k_ts_apply_mma<<<grid, 256, TM_SMEM, st>>>(n, k, kout, pmap, X, ldx, Ta, Y, ldy);
        SG_CUDA(cudaGetLastError());
        return SG_OK;
    }
    const int nj = (k + 7) / 8;
    const int oc = 8 * nj;
    // CTAs resident per SM for this variant (registers and shared memory), once per variant
    static thread_local int resident[9] = {};
    if (!resident[nj]) {
        const void *fn = nj == 1 ? (const void *)k_ts_apply<1> : nj == 2 ? (const void *)k_ts_apply<2>
                       : nj == 3 ? (const void *)k_ts_apply<3> : nj == 4 ? (const void *)k_ts_apply<4>
                       : nj == 5 ? (const void *)k_ts_apply<5> : nj == 6 ? (const void *)k_ts_apply<6>
                       : nj == 7 ? (const void *)k_ts_apply<7> : (const void *)k_ts_apply<8>;
        int r = 0;
        SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, fn, 256, 0));
        resident[nj] = std::max(1, r);
    }
    const dim3 grid((unsigned)std::min<int64_t>(ntiles, (int64_t)sm_count() * resident[nj]),
                    (unsigned)((k + oc - 1) / oc));
    count_launch();
    switch (nj) {
        case 1: k_ts_apply<1><<<grid, 256, 0, st>>>(n, k, kout, pmap, X, ldx, Ta, Y, ldy); break;
        case 2: k_ts_apply<2><<<grid, 256, 0, st>>>(n, k, kout, pmap, X, ldx, Ta, Y, ldy); break;
        case 3: k_ts_apply<3><<<grid, 256, 0, st>>>(n, k, kout, pmap, X, ldx, Ta, Y, ldy); break;
        case 4: k_ts_apply<4><<<grid, 256, 0, st>>>(n, k, kout, pmap, X, ldx, Ta, Y, ldy); break;
        case 5: k_ts_apply<5><<<grid, 256, 0, st>>>(n, k, kout, pmap, X, ldx, Ta, Y, ldy); break;
        case 6: k_ts_apply<6><<<grid, 256, 0, st>>>(n, k, kout, pmap, X, ldx, Ta, Y, ldy); break;
        case 7: k_ts_apply<7><<<grid, 256, 0, st>>>(n, k, kout, pmap, X, ldx, Ta, Y, ldy); break;
        default: k_ts_apply<8><<<grid, 256, 0, st>>>(n, k, kout, pmap, X, ldx, Ta, Y, ldy); break;
    }
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

// ------------------------------------------------------------------ device-count variants
//
// The number of columns is read from device memory (cnt[0] + add, at most mmax) and the basis
// pointer may be too (Vp[0] when V is null), so that one captured sequence of launches serves
// every iteration of a graph-replayed loop.  Same arithmetic and summation order as the
// host-count kernels above.

__global__ void __launch_bounds__(DOT_THREADS) k_multidot_dc(int64_t n, const int32_t *__restrict__ cnt, int add,
                                                             int mmax, const double *V, const double *const *Vp,
                                                             int64_t ldv, const double *__restrict__ w,
                                                             double *__restrict__ partial) {
    __shared__ double sh[32];
    const int m = min(cnt[0] + add, mmax);
    const double *__restrict__ B = V ? V : Vp[0];
    const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = blockIdx.x * chunk, r1 = min(n, r0 + chunk);
    int i = 0;
    for (; i + 4 <= m; i += 4) {
        double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
            const double wr = w[r];
            s0 += B[(i + 0) * ldv + r] * wr;
            s1 += B[(i + 1) * ldv + r] * wr;
            s2 += B[(i + 2) * ldv + r] * wr;
            s3 += B[(i + 3) * ldv + r] * wr;
        }
        s0 = block_sum(s0, sh);
        if (threadIdx.x == 0) partial[(i + 0) * gridDim.x + blockIdx.x] = s0;
        s1 = block_sum(s1, sh);
        if (threadIdx.x == 0) partial[(i + 1) * gridDim.x + blockIdx.x] = s1;
        s2 = block_sum(s2, sh);
        if (threadIdx.x == 0) partial[(i + 2) * gridDim.x + blockIdx.x] = s2;
        s3 = block_sum(s3, sh);
        if (threadIdx.x == 0) partial[(i + 3) * gridDim.x + blockIdx.x] = s3;
    }
    for (; i < m; ++i) {
        double s = 0;
        for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) s += B[i * ldv + r] * w[r];
        s = block_sum(s, sh);
        if (threadIdx.x == 0) partial[i * gridDim.x + blockIdx.x] = s;
    }
}

__global__ void k_reduce_partials_dc(const int32_t *__restrict__ cnt, int add, int mmax, int nb,
                                     const double *__restrict__ partial, double *__restrict__ out) {
    __shared__ double sh[32];
    const int m = min(cnt[0] + add, mmax);
    for (int i = blockIdx.x; i < m; i += gridDim.x) {
        double s = 0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[(int64_t)i * nb + b];
        s = block_sum(s, sh);
        if (threadIdx.x == 0) out[i] = s;
    }
}

template <int SIGN>
__global__ void k_gemv_dc(int64_t n, const int32_t *__restrict__ cnt, int add, int mmax, const double *V,
                          const double *const *Vp, int64_t ldv, const double *__restrict__ h,
                          double *__restrict__ w) {
    extern __shared__ double hs[];
    const int m = min(cnt[0] + add, mmax);
    const double *__restrict__ B = V ? V : Vp[0];
    for (int i = threadIdx.x; i < m; i += blockDim.x) hs[i] = h[i];
    __syncthreads();
    if (m <= 0) return;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        double s = 0;
        for (int i = 0; i < m; ++i) s += hs[i] * B[i * ldv + r];
        w[r] = SIGN > 0 ? w[r] + s : w[r] - s;
    }
}

int multidot_dc(int64_t n, const int32_t *cnt, int add, int mmax, const double *V, const double *const *Vp,
                int64_t ldv, const double *w, double *partial, double *out, cudaStream_t st) {
    if (mmax <= 0) return SG_OK;
    count_launch(2);
    k_multidot_dc<<<DOT_BLOCKS, DOT_THREADS, 0, st>>>(n, cnt, add, mmax, V, Vp, ldv, w, partial);
    k_reduce_partials_dc<<<std::min(mmax, 1024), 256, 0, st>>>(cnt, add, mmax, DOT_BLOCKS, partial, out);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

int gemv_dc(int sign, int64_t n, const int32_t *cnt, int add, int mmax, const double *V, const double *const *Vp,
            int64_t ldv, const double *h, double *w, cudaStream_t st) {
    if (mmax <= 0) return SG_OK;
    const unsigned grid = grid_for(n, 256, 8);
    if (sign > 0) k_gemv_dc<1><<<grid, 256, sizeof(double) * mmax, st>>>(n, cnt, add, mmax, V, Vp, ldv, h, w);
    else k_gemv_dc<-1><<<grid, 256, sizeof(double) * mmax, st>>>(n, cnt, add, mmax, V, Vp, ldv, h, w);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

__global__ void k_axpby(int64_t n, double a, const double *__restrict__ x, double b, double *__restrict__ y) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        y[r] = (b == 0.0) ? a * x[r] : a * x[r] + b * y[r];
}

int axpby(int64_t n, double a, const double *x, double b, double *y, cudaStream_t st) {
    k_axpby<<<grid_for(n, 256, 8), 256, 0, st>>>(n, a, x, b, y);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

// y = x * s, s = num[0] (invert: 1 / num[0])
__global__ void k_scale(int64_t n, const double *__restrict__ x, const double *__restrict__ num, int invert,
                        double *__restrict__ y) {
    const double s = invert ? 1.0 / num[0] : num[0];
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        y[r] = x[r] * s;
}

int scale_dev(int64_t n, const double *x, const double *num, int invert, double *y, cudaStream_t st) {
    k_scale<<<grid_for(n, 256, 8), 256, 0, st>>>(n, x, num, invert, y);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

// sum mask * (a - b)^2 partials (Newton residual over the free DOFs)
__global__ void __launch_bounds__(DOT_THREADS) k_masked_diff2(int64_t n, const double *__restrict__ a,
                                                              const double *__restrict__ b,
                                                              const double *__restrict__ mask,
                                                              double *__restrict__ partial) {
    __shared__ double sh[32];
    const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = blockIdx.x * chunk, r1 = min(n, r0 + chunk);
    double s = 0;
    for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
        const double d = (a[r] - (b ? b[r] : 0.0)) * (mask ? mask[r] : 1.0);
        s += d * d;
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

}  // namespace sg

using namespace sg;

extern "C" int sg_bsr_spmv_dev(const sg_bsr *A, const double *vals, const double *x, double *y, void *stream) {
    SG_CHECK_ARG(A && vals && x && y, "null argument");
    return bsr_spmv<double, double>(*A, vals, x, y, 1.0, 0.0, as_stream(stream));
}

extern "C" int sg_bsr_info(const sg_bsr *A, int64_t *info) {
    SG_CHECK_ARG(A && info, "null argument");
    info[0] = A->b;
    info[1] = A->n_rows;
    info[2] = A->n_blocks;
    return SG_OK;
}

// Host-visible reductions (synchronise `stream`).
extern "C" int sg_dot_dev(int64_t n, const double *x, const double *y, double *result, void *stream) {
    SG_CHECK_ARG(x && y && result && n >= 0, "bad argument");
    static thread_local Scratch ws;
    int rc = ws.reserve(sizeof(double) * (DOT_BLOCKS + 8));
    if (rc) return rc;
    double *part = (double *)ws.ptr, *out = part + DOT_BLOCKS;
    const cudaStream_t st = as_stream(stream);
    rc = multidot(n, 1, x, n, y, part, out, st);
    if (rc) return rc;
    SG_CUDA(cudaMemcpyAsync(result, out, sizeof(double), cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    return SG_OK;
}

// result = sum_r mask[r] * (a[r] - b[r])^2   (b, mask nullable)
extern "C" int sg_masked_diff_norm2_dev(int64_t n, const double *a, const double *b, const double *mask,
                                        double *result, void *stream) {
    SG_CHECK_ARG(a && result && n >= 0, "bad argument");
    static thread_local Scratch ws;
    int rc = ws.reserve(sizeof(double) * (DOT_BLOCKS + 8));
    if (rc) return rc;
    double *part = (double *)ws.ptr, *out = part + DOT_BLOCKS;
    const cudaStream_t st = as_stream(stream);
    count_launch(2);
    k_masked_diff2<<<DOT_BLOCKS, DOT_THREADS, 0, st>>>(n, a, b, mask, part);
    k_reduce_partials<<<1, 256, 0, st>>>(1, DOT_BLOCKS, part, out);
    SG_CUDA(cudaGetLastError());
    SG_CUDA(cudaMemcpyAsync(result, out, sizeof(double), cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    return SG_OK;
}

extern "C" int sg_axpby_dev(int64_t n, double a, const double *x, double b, double *y, void *stream) {
    SG_CHECK_ARG(x && y && n >= 0, "bad argument");
    return axpby(n, a, x, b, y, as_stream(stream));
}
